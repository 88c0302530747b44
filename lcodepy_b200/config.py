"""Flat string-keyed configuration, with the same keys, defaults, accessors
and 3D adjustments as the reference's ``lcode.config`` package.

Reference: lcode/config/config.py:13-258, lcode/config/default_config_values.py.
Keys and default values are an interface (a user's config dict must mean the
same thing here), so they are kept identical.
"""
from __future__ import annotations

import copy as _copy
import pprint
from typing import Any

import numpy as np

#: Default values (lcode/config/default_config_values.py:3-103).
default_config_values = {
    'geometry': 'circ',
    'processing-unit-type': 'cpu',
    'window-width': 5.0,
    'transverse-step': 0.05,
    'window-length': 15.0,
    'xi-step': 0.05,
    'time-limit': 200.5,
    'time-step': 25,
    'plasma-particles-per-cell': 10,
    'ion-model': 'mobile',
    'ion-mass': 1836,
    'plasma-shape': 'legacy',
    'plasma-rshape': 'uniform',
    'plasma-width': 1,
    'plasma-width-2': 0,
    'plasma-density-2': 0.5,
    'plasma-zshape': '''
        ''',
    'declustering-enabled': False,
    'declustering-averaging': 3,
    'declustering-force': 0.3,
    'declustering-damping': 0.1,
    'declustering-limit': 1e-3,
    'beam-substepping-energy': 2,
    'magnetic-field': 0,
    'substepping-depth': 3,
    'substepping-sensitivity': 0.2,
    'bound-padding-steps': 10,
    'plasma-padding-steps': 15,
    'dual-plasma-approach': False,
    'plasma-coarseness': 5,
    'rigid-beam': False,
    'field-solver-subtraction-coefficient': 1,
    'trapped-path-limit': 0,
    'correctotransverse-steps': 2,
}

# Extra keys understood by this package only (the reference ignores unknown
# keys, so adding them keeps configs interchangeable).
#   'precision': 'fp64' (default; the reference's arithmetic) or 'mixed'
#                (FP32 deposition and FP32 transforms, FP64 particles).
#   'deposit-precision', 'field-precision': 'fp64' or 'fp32', overriding
#                'precision' for the deposition or the field solve alone.
#   'print-every': xi steps between the on-axis Ez lines (reference: 10).


def _factorize(n: int) -> list[int]:
    """Prime factors of n (with repeats)."""
    out, d = [], 2
    while n > 1:
        while n % d == 0:
            out.append(d)
            n //= d
        d += 1
    return out


def good_size(number: int) -> bool:
    """True for odd sizes whose (size - 1) factors into 2,3,5,7 and at most one
    11 or 13 -- FFTW's fast real-to-real sizes (config.py:250-258)."""
    fs = _factorize(number - 1)
    return bool(all(f in (2, 3, 4, 5, 7, 11, 13) for f in fs)
                and fs.count(11) + fs.count(13) < 2 and number % 2)


class Config:
    """Dict-backed config with typed getters (config.py:13-163)."""

    def __init__(self, new_config_values: dict | None = None,
                 default_config: bool = True):
        self.config_values: dict[str, Any] = {}
        # The array module the reference exposes for user callbacks.  This
        # package always computes on the GPU; user callbacks (rigid-beam
        # density, plasma shape) are evaluated with numpy on the host.
        self.xp = np
        if default_config:
            self.update(default_config_values)
        if new_config_values is not None:
            self.update(new_config_values)

    # -- accessors (same coercions as config.py:35-64) --
    def get(self, option_name: str, fallback: str = '') -> str:
        if option_name in self.config_values:
            return str(self.config_values.get(option_name))
        return fallback

    def getraw(self, option_name: str):
        return self.config_values.get(option_name)

    def getbool(self, option_name: str, fallback: bool = False) -> bool:
        s = self.get(option_name).lower()
        if s == 'true':
            return True
        if s == 'false':
            return False
        return fallback

    def getint(self, option_name: str, fallback: int = 0) -> int:
        try:
            return int(float(self.get(option_name)))
        except ValueError:
            return fallback

    def getfloat(self, option_name: str, fallback: float = 0.0) -> float:
        try:
            return float(self.get(option_name))
        except ValueError:
            return fallback

    def set(self, option_name: str, option_value: Any):
        self.config_values[option_name] = option_value
        if option_name == 'geometry' and self.config_values['geometry'] == 'circ':
            self.config_values['geometry'] = '2d'

    def update(self, new_config_values: dict | None = None):
        if new_config_values is not None:
            for key in new_config_values:
                self.set(key, new_config_values[key])

    def __copy__(self) -> 'Config':
        ret = Config()
        ret.config_values = _copy.copy(self.config_values)
        return ret

    def dump(self, runas_name: str):
        """Write the effective config as an importable Python file
        (the reference writes ``runas.py`` the same way, config.py:86-148;
        in 3D the stored window-width is the half-width again)."""
        vals = dict(self.config_values)
        if str(vals.get('geometry', '')).lower() == '3d':
            vals['window-width'] = float(vals['window-width']) / 2
        for k, v in list(vals.items()):
            if callable(v):
                vals[k] = f'external function {v!r}'
        with open(runas_name, 'w') as f:
            f.write('"""\nSimulation performed with the following settings.\n"""\n\n')
            f.write('config = ' + pprint.pformat(vals, sort_dicts=False) + '\n')

    # -- 3D adjustments (config.py:185-236) --
    def _adjust_config_values_3d(self):
        if self.get('geometry') == '3d':
            self.set('window-width', 2 * self.getfloat('window-width'))
            self.adjust_window_width_and_steps_3d()
            self.adjust_plasma_fineness()
            if self.get('field-solver-subtraction-coefficient') == '1':
                self.set('field-solver-subtraction-coefficient',
                         1 + self.getfloat('xi-step'))

    def adjust_window_width_and_steps_3d(self):
        estim = int(self.getfloat('window-width') / self.getfloat('transverse-step'))
        lower = max(estim - 100, 0)
        good = np.array([a for a in range(lower, estim + 100) if good_size(a)])
        steps = int(good[np.abs(good - estim).argmin()])
        self.set('window-width', steps * self.getfloat('transverse-step'))
        self.set('window-width-steps', steps)

    def adjust_plasma_fineness(self):
        s = np.sqrt(self.getfloat('plasma-particles-per-cell'))
        self.set('plasma-fineness', round(s))
        self.set('plasma-particles-per-cell', round(s) ** 2)
        if 0. < s < 1.:
            self.set('plasma-fineness', 1 / round(1 / s))
            self.set('plasma-particles-per-cell', 1 / round(1 / s) ** 2)
