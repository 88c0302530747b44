"""Seeded beam generator producing ``particle_dtype3d`` arrays.

Restates the reference's ``lcode.alt_beam_generator`` (beam_generator.py:28-161,
beam_shape.py, beam_segment_shape.py, rshape.py, eshape.py, xishape.py).  The
generated beam is an *input* of the xi loop, so the random stream must be
drawn in exactly the reference's order (``numpy.random.RandomState(seed)``;
per layer: xi, then r/phi/px/py, then pz) for a given ``beam_parameters``
dict to produce the same particles.
"""
from __future__ import annotations

import numpy as np

from .config import Config

particle_dtype3d = np.dtype([('xi', 'f8'), ('x', 'f8'), ('y', 'f8'),
                             ('px', 'f8'), ('py', 'f8'), ('pz', 'f8'),
                             ('q_m', 'f8'), ('q_norm', 'f8'), ('id', 'i8')])

# Longitudinal current profiles f(dxi, length), xishape.py:38-49.
XI_SHAPES = {
    'cos': lambda d, L: 0.5 * (1 - np.cos(2 * np.pi * d / L)),
    't': lambda d, L: d / L,
    'T': lambda d, L: 1 - d / L,
    'l': lambda d, L: 1,
    'half-cos': lambda d, L: 0.5 * (1 - np.cos(np.pi * d / L)),
    'b': lambda d, L: 0.5 * (1 + np.cos(np.pi * d / L)),
    'gaussian': lambda d, L: 0.5 * np.exp(-18 * (d / L) ** 2),
}
XI_SHAPES['c'] = XI_SHAPES['cos']
XI_SHAPES['h'] = XI_SHAPES['half-cos']
XI_SHAPES['g'] = XI_SHAPES['gaussian']


def _gauss3d(rng, radius, sigma_p, r_max, size, xshift, yshift):
    """Truncated radial Gaussian (rshape.py:40-48)."""
    a = 1 - np.exp(-r_max ** 2 / (2 * radius ** 2))
    r = radius * np.sqrt(-2 * np.log(1 - rng.random_sample(size) * a))
    phi = rng.uniform(0, 2 * np.pi, size)
    x = r * np.cos(phi) + xshift
    y = r * np.sin(phi) + yshift
    px = rng.normal(0, sigma_p, size)
    py = rng.normal(0, sigma_p, size)
    return x, y, px, py


R_SHAPES = {'gaussian': _gauss3d, 'g': _gauss3d}


def _energy(kind, rng, energy, espread, d, L, size):
    """Longitudinal momentum profiles (eshape.py:37-54)."""
    if kind in ('monoenergetic', 'm'):
        return np.full(size, energy)
    if kind in ('uniform', 'u'):
        return rng.uniform(energy, espread, size)
    if kind in ('linear', 'l'):
        return np.full(size, energy * d / L + espread * (1 - d / L))
    if kind in ('gaussian', 'g'):
        return rng.normal(energy, espread, size)
    if kind in tuple(str(i) for i in range(2, 10)):
        n = int(kind)
        return np.full(size, espread) + rng.randint(0, n) * (energy - espread) / (n - 1)
    raise KeyError(kind)


class BeamSegment:
    """One longitudinal segment (beam_segment_shape.py:5-63)."""

    def __init__(self, length, ampl, xishape, radius, energy, xshift, yshift,
                 rshape, angspread, angshape, espread, eshape, mass_charge_ratio):
        self.length = length
        self.ampl = ampl
        self.xishape = XI_SHAPES[xishape]
        self.radius = radius
        self.energy = energy
        self.xshift, self.yshift = xshift, yshift
        self.rshape = R_SHAPES[rshape]
        self.angspread = angspread
        self.angshape = XI_SHAPES[angshape]
        self.espread = espread
        self.eshape = eshape
        self.mass_charge_ratio = mass_charge_ratio
        self.owner_current = 0.0

    def current_at(self, d):
        if d < 0 or d > self.length:
            return 0
        return self.ampl * self.owner_current * self.xishape(d, self.length)


class BeamShape:
    """Ordered segments from xi = 0 backwards (beam_shape.py:5-43)."""

    def __init__(self, config: Config, current, particles_in_layer, rng_seed):
        if config.get('geometry').lower() == '3d':
            current *= 2 * 3.1415926535897932
        self.current = current
        self.particles_in_layer = particles_in_layer
        self.rng_seed = rng_seed
        self.segments: list[BeamSegment] = []

    def add_segment(self, seg: BeamSegment):
        self.segments.append(seg)
        seg.owner_current = self.current

    def get_segment(self, xi):
        start = 0
        for seg in self.segments:
            if 0 < start - xi < seg.length:
                return seg, start
            start -= seg.length
        return None, 0

    @property
    def total_length(self):
        return sum(s.length for s in self.segments)

    def initial_current(self, xi):
        seg, start = self.get_segment(xi)
        return 0 if seg is None else seg.current_at(start - xi)


_SHAPE_KEYS = {'current': 0.05, 'particles_in_layer': 2000, 'rng_seed': 1}
_SEGMENT_DEFAULTS = {
    'length': 5.01, 'ampl': 1., 'xishape': 'cos', 'radius': 1.,
    'energy': 1000., 'xshift': 0, 'yshift': 0, 'rshape': 'g',
    'angspread': 1e-5, 'angshape': 'l', 'espread': 0, 'eshape': 'm',
    'mass_charge_ratio': 1,
}


def generate_beam(config, beam_parameters: dict | None = None) -> np.ndarray:
    """Build the beam described by ``beam_parameters`` (beam_generator.py:28-93):
    top-level keys current / particles_in_layer / rng_seed, a 'default' dict
    overriding segment defaults, and any other dict adding a segment."""
    if isinstance(config, dict):
        config = Config(config)
    shape_params = dict(_SHAPE_KEYS)
    seg_defaults = dict(_SEGMENT_DEFAULTS)
    if beam_parameters is None:
        shape = BeamShape(config, **shape_params)
        shape.add_segment(BeamSegment(**seg_defaults))
        return generate_beam_array(config, shape)
    for k in beam_parameters:
        if k in shape_params:
            shape_params[k] = beam_parameters[k]
    shape = BeamShape(config, **shape_params)
    for k, v in beam_parameters.items():
        if isinstance(v, dict):
            if k == 'default':
                seg_defaults.update(v)
            else:
                params = dict(seg_defaults)
                params.update(v)
                shape.add_segment(BeamSegment(**params))
        elif k not in shape_params:
            raise Exception(f"The {k} key of beam_parameters dictionary"
                            "is not supported.")
    if not shape.segments:
        shape.add_segment(BeamSegment(**seg_defaults))
    return generate_beam_array(config, shape)


def generate_beam_array(config: Config, shape: BeamShape) -> np.ndarray:
    """Layer-by-layer sampling (beam_generator.py:96-161)."""
    dxi = config.getfloat('xi-step')
    three_d = config.get('geometry').lower() == '3d'
    max_radius = config.getfloat('window-width')
    if three_d:
        max_radius /= 2
    max_radius = max(0.9 * max_radius, max_radius - 1)

    rng = np.random.RandomState(shape.rng_seed)
    xi_vals = np.arange(-dxi / 2, -shape.total_length, -dxi)
    current = np.array([shape.initial_current(x) for x in xi_vals], dtype=np.float64)
    elem_charge = np.abs(2 * shape.current / shape.particles_in_layer)
    per_layer = (shape.particles_in_layer *
                 np.abs(current / shape.current)).astype(np.int_)
    total = int(per_layer.sum())
    beam = np.zeros(total, dtype=particle_dtype3d)
    beam['id'] = np.arange(1, total + 1, dtype=np.int_)
    pos = 0
    for li in range(len(current)):
        layer_xi = -dxi * li
        xi_mid = layer_xi - dxi / 2
        seg, seg_start = shape.get_segment(xi_mid)
        d = seg_start - xi_mid
        n = int(per_layer[li])
        if seg is None:
            continue
        q_m = (1 / seg.mass_charge_ratio) * (1 if current[li] > 0 else -1)
        q_norm = elem_charge * (1 if shape.current >= 0 else -1)
        sl = slice(pos, pos + n)
        beam['xi'][sl] = rng.uniform(layer_xi - dxi, layer_xi, n)
        sigma_p = seg.angspread * seg.energy * seg.angshape(d, seg.length)
        x, y, px, py = seg.rshape(rng, seg.radius, sigma_p, max_radius, n,
                                  seg.xshift, seg.yshift)
        beam['x'][sl], beam['y'][sl] = x, y
        beam['px'][sl], beam['py'][sl] = px, py
        beam['pz'][sl] = _energy(seg.eshape, rng, seg.energy, seg.espread, d,
                                 seg.length, n)
        beam['q_m'][sl] = np.full(n, q_m)
        beam['q_norm'][sl] = np.full(n, q_norm)
        pos += n
    return beam[np.argsort(-beam['xi'])]
