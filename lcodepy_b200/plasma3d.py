"""Plasma: initial state, solver operators and the predictor-corrector xi step
on the device.

Initial state and matrices follow lcode/plasma3d/initialization.py:15-414 and
lcode/plasma3d/profile.py:111-145 (host numpy, then uploaded once); the xi
step follows lcode/plasma3d/solver.py:25-78 and runs entirely through
liblcb.so.

Device layout (HBM, FP64, C order):
  particles  SoA, sorts concatenated: x_init y_init x_offt y_offt px py pz q m,
             each (n_sorts * Ns * Ns,), two copies (prev / full) that swap
             roles every xi step;
  fields     7 planes N x N (Ex Ey Ez Bx By Bz Phi) for prev, full and two
             half-step scratch sets;
  currents   ro jx jy jz, each (2, N, N) (plane = sort; background ions put
             ro_initial in plane 1), prev and full;
  operators  folded DST-I / DCT-I blocks and the solver matrices, FP64 (or
             FP32 in mixed precision), built by lcb_field_operators_build.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .config import Config
from .data import Arrays

ELECTRON_CHARGE = -1
ELECTRON_MASS = 1
FIELD_NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")
CURRENT_NAMES = ("ro", "jx", "jy", "jz")
PARTICLE_NAMES = ("x_init", "y_init", "x_offt", "y_offt", "px", "py", "pz", "q", "m")


# ---------------------------------------------------------------------------
# Field solver operators (initialization.py:15-67 and the DST-I / DCT-I
# matrices of fields.py:16-31), built on the device.
# ---------------------------------------------------------------------------

class FieldOperators:
    """The field solver's constant operators, built on the device by
    liblcb (folded DST-I / DCT-I blocks and the solver matrices)."""

    def __init__(self, N, h, sub_coeff, device, mixed_precision):
        L = _lib.load()
        self.precision = _lib.LCB_PREC_MIXED if mixed_precision else _lib.LCB_PREC_FP64
        nbytes = L.lcb_field_operators_bytes(N, self.precision)
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        _lib.check(L.lcb_field_operators_build(N, h, sub_coeff, self.precision,
                                               self.buf.data_ptr(), nbytes,
                                               _lib.stream_handle()),
                   "lcb_field_operators_build")

    @property
    def ptr(self):
        return self.buf.data_ptr()


# ---------------------------------------------------------------------------
# Initial plasma (initialization.py:72-135, profile.py)
# ---------------------------------------------------------------------------

def make_plasma_grid(steps, step_size, fineness):
    """Particle lattice coordinates (one axis), initialization.py:72-104."""
    plasma_step = step_size / fineness
    if fineness % 2:
        right = np.arange(steps // 2 * fineness) * plasma_step
        left = -right[:0:-1]
    elif 0. < fineness < 1.:
        right = np.arange(steps // (2 / fineness)) * plasma_step
        left = -right[:0:-1]
    else:
        right = (.5 + np.arange(steps // 2 * fineness)) * plasma_step
        left = -right[::-1]
    grid = np.concatenate([left, right])
    assert np.array_equal(grid, -grid[::-1])
    return grid


def _radial_coef(profile, width, width2, density2, r):
    """Transverse density profiles, profile.py:3-47."""
    coef = np.ones_like(r)
    if profile in ('1', 'uniform'):
        pass
    elif profile in ('2', 'stepwise'):
        dr = width2 - width
        if dr > 0:
            mask = (width < r) & (r < width2)
            r0 = np.min(r[mask])
            coef[mask] = 1 - (r[mask] - r0) / dr
        coef[r > max(width, width2)] = 0
    elif profile in ('3', 'channel'):
        coef[r <= width] = density2
        dr = width2 - width
        if dr > 0:
            mask = (width < r) & (r < width2)
            r0 = np.min(r[mask])
            coef[mask] = (density2 * (1 + dr - r[mask]) + (r[mask] - r0)) / dr
    elif profile in ('4', 'parabolic-channel'):
        coef = density2 * (1 + (r / width) ** 2)
        coef[coef > 1] = 1
    elif profile in ('5', 'gaussian'):
        coef = np.exp(-r ** 2 / 2 / width ** 2)
        coef[r > 5 * width] = 0
    else:
        print(f'Unknown transverse distribution {profile}, '
              'the uniform distribution is used instead.')
    return coef


def _rshape_coef(config, t_mid, x_init, y_init):
    """profile.py:50-85."""
    profiles = {'1', 'uniform', '2', 'stepwise', '3', 'channel',
                '4', 'parabolic-channel', '5', 'gaussian'}
    rshape = config.get('plasma-rshape')
    r = np.sqrt(x_init ** 2 + y_init ** 2)
    coef = np.ones_like(x_init)
    if rshape in profiles:
        coef = _radial_coef(rshape, config.getfloat('plasma-width'),
                            config.getfloat('plasma-width-2'),
                            config.getfloat('plasma-density-2'), r)
    else:
        segs = [ln.split() for ln in rshape.splitlines() if ln.split()]
        for seg in segs:
            if t_mid < float(seg[0]):
                coef = _radial_coef(seg[1], float(seg[2]), float(seg[3]),
                                    float(seg[4]), r)
                break
            t_mid -= float(seg[0])
    return coef


def _zshape_coef(config, t_mid):
    """profile.py:87-109."""
    zshape = config.get('plasma-zshape')
    coef = 1
    if not zshape.isspace():
        segs = [ln.split() for ln in zshape.splitlines() if ln.split()]
        for seg in segs:
            if t_mid < float(seg[0]):
                if seg[2] == 'L':
                    coef = (float(seg[1]) * (float(seg[0]) - t_mid)
                            + float(seg[3]) * t_mid) / float(seg[0])
                else:
                    print(seg[2], 'segment of z shape is not available, '
                          'a density of 1 is assumed.')
                break
            t_mid -= float(seg[0])
    return coef


def profile_initial_plasma(config, current_time, x_init, y_init, q, m):
    """Density profile scaling of q and m, profile.py:111-145."""
    shape = config.getraw('plasma-shape')
    t_mid = current_time - config.getfloat('time-step') / 2
    if callable(shape):
        coef = shape(current_time, x_init, y_init)
    else:
        coef = _zshape_coef(config, t_mid) * _rshape_coef(config, t_mid, x_init, y_init)
    if np.any(np.asarray(coef) < 0):
        print('A density that is < 0 is not available, a uniform density is assumed.')
        coef = np.ones_like(x_init)
    return q * coef, m * coef


def plasma_params(config: Config):
    N = config.getint('window-width-steps')
    h = config.getfloat('transverse-step')
    bp = config.getint('bound-padding-steps')
    return dict(
        N=N, h=h, dxi=config.getfloat('xi-step'),
        boundary=h * (N / 2 - bp),
        sub_coeff=config.getfloat('field-solver-subtraction-coefficient'),
        ion_model=config.get('ion-model'),
        precision=_part_precision(config, 'field-precision'),
        deposit_precision=_part_precision(config, 'deposit-precision'),
    )


def _part_precision(config: Config, key: str) -> int:
    """'precision' sets both parts ('fp64' or 'mixed'); 'field-precision' and
    'deposit-precision' ('fp64' or 'fp32') override one part each."""
    v = config.getraw(key)
    if v is None:
        mixed = str(config.getraw('precision') or 'fp64').lower() == 'mixed'
    else:
        v = str(v).lower()
        if v not in ('fp64', 'fp32'):
            raise ValueError(f"{key} must be 'fp64' or 'fp32', not {v!r}")
        mixed = v == 'fp32'
    return _lib.LCB_PREC_MIXED if mixed else _lib.LCB_PREC_FP64


def host_initial_particles(config: Config, current_time=0.0):
    """Lattice, charge and mass of the electrons (initialization.py:107-135,
    278-330).  Returns numpy arrays (Ns, Ns)."""
    N = config.getint('window-width-steps')
    h = config.getfloat('transverse-step')
    bp = config.getint('bound-padding-steps')
    pp = config.getint('plasma-padding-steps')
    fineness = config.getfloat('plasma-fineness')
    if fineness > 1:
        fineness = int(fineness)
    if N % 2 != 1:
        raise ValueError("window-width-steps must be odd")
    if bp <= 2:
        raise Exception("'bound_padding_steps' parameter is too low.\n"
                        "Details: 'bound_padding_steps' must be bigger than 2. "
                        "By default it is 10.")
    if config.getbool('dual-plasma-approach'):
        raise NotImplementedError("dual-plasma-approach is not supported "
                                  "(the reference's own path for it is broken)")
    g = make_plasma_grid(N - pp * 2, h, fineness)
    Ns = len(g)
    y_init = np.ascontiguousarray(np.broadcast_to(g, (Ns, Ns)))
    x_init = np.ascontiguousarray(y_init.T)
    q = np.ones_like(x_init) * ELECTRON_CHARGE / fineness ** 2 * h ** 2
    m = np.ones_like(x_init) * ELECTRON_MASS / fineness ** 2 * h ** 2
    q, m = profile_initial_plasma(config, current_time, x_init, y_init, q, m)
    return x_init, y_init, np.asarray(q, dtype=np.float64), np.asarray(m, dtype=np.float64)


class PlasmaState:
    """One copy of the plasma particles of all sorts (concatenated SoA)."""

    def __init__(self, n_sorts, Ns, device):
        self.n_sorts, self.Ns = n_sorts, Ns
        self.n_per_sort = Ns * Ns
        n = n_sorts * self.n_per_sort
        self.t = {k: torch.zeros(n, dtype=torch.float64, device=device)
                  for k in PARTICLE_NAMES}
        # dx_chaotic, dy_chaotic of the first sort (the electrons): the
        # declustering filter's state, zero while it is off
        self.chaos = torch.zeros(2, self.n_per_sort, dtype=torch.float64, device=device)

    def __getattr__(self, k):
        t = self.__dict__.get("t")
        if t is not None and k in t:
            return t[k]
        raise AttributeError(k)

    def sort_arrays(self, s: int) -> Arrays:
        """Per-sort (Ns, Ns) views with the reference's attribute names."""
        a, b = s * self.n_per_sort, (s + 1) * self.n_per_sort
        views = {k: v[a:b].view(self.Ns, self.Ns) for k, v in self.t.items()}
        z = torch.zeros_like(views["x_init"])
        dx, dy = ((self.chaos[0].view(self.Ns, self.Ns), self.chaos[1].view(self.Ns, self.Ns))
                  if s == 0 else (z, z))
        return Arrays(torch, **views, dx_chaotic=dx, dy_chaotic=dy,
                      dx_chaotic_perp=z, dy_chaotic_perp=z)


def sorts_of(ion_model):
    return ("electrons", "ions") if ion_model == "mobile" else ("electrons",)
