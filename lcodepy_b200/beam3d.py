"""Beam on the device: particle SoA, xi-layer source and drain, density
layout and substepped push (lcode/beam3d/*).

The beam is kept sorted by xi (descending) in HBM, so a layer is a
contiguous slice; layer lengths are found by binary search on a host copy of
the sorted xi taken once per time step (the reference counts them with a
device reduction and a host sync per layer, beam3d/beam_io.py:29-47).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .beam_generator import particle_dtype3d
from .config import Config

BEAM_FLOAT = ("xi", "x", "y", "px", "py", "pz", "q_m", "q_norm")
BEAM_KEYS = BEAM_FLOAT + ("id",)


class BeamParticles:
    """SoA beam (beam3d/data.py:21-178) with CUDA tensors."""

    def __init__(self, device=None, n: int = 0):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        f = lambda: torch.zeros(n, dtype=torch.float64, device=self.device)
        for k in BEAM_FLOAT:
            setattr(self, k, f())
        self.id = torch.zeros(n, dtype=torch.int64, device=self.device)
        self.dt = f()
        self.remaining_steps = torch.zeros(n, dtype=torch.int64, device=self.device)

    # -- construction / I/O (data.py:53-86) --
    def init_generated(self, beam_array: np.ndarray):
        for k in BEAM_KEYS:
            dt = torch.int64 if k == "id" else torch.float64
            setattr(self, k, torch.as_tensor(np.ascontiguousarray(beam_array[k]),
                                             dtype=dt).to(self.device))
        self.dt = torch.zeros_like(self.q_norm)
        self.remaining_steps = torch.zeros_like(self.id)
        return self

    def load(self, path):
        with np.load(path) as d:
            for k in BEAM_KEYS:
                dt = torch.int64 if k == "id" else torch.float64
                setattr(self, k, torch.as_tensor(np.ascontiguousarray(d[k]), dtype=dt).to(self.device))
        self.dt = torch.zeros_like(self.q_norm)
        self.remaining_steps = torch.zeros_like(self.id)
        return self

    def save(self, *args, **kwargs):
        np.savez_compressed(*args, **kwargs,
                            **{k: getattr(self, k).cpu().numpy() for k in BEAM_KEYS})

    @property
    def particles(self) -> np.ndarray:
        out = np.zeros(self.size, dtype=particle_dtype3d)
        for k in BEAM_KEYS:
            out[k] = getattr(self, k).cpu().numpy()
        return out

    @property
    def size(self) -> int:
        return int(self.id.numel())

    def _all(self):
        return BEAM_KEYS + ("dt", "remaining_steps")

    def take(self, sel) -> "BeamParticles":
        b = BeamParticles.__new__(BeamParticles)
        b.device = self.device
        for k in self._all():
            setattr(b, k, getattr(self, k)[sel])
        return b

    def xi_sorted(self):
        """Sort by xi, descending (data.py:88-105)."""
        order = torch.sort(-self.xi, stable=True).indices
        for k in self._all():
            setattr(self, k, getattr(self, k)[order].contiguous())

    def append(self, other: "BeamParticles") -> "BeamParticles":
        b = BeamParticles.__new__(BeamParticles)
        b.device = self.device
        for k in self._all():
            setattr(b, k, torch.cat((getattr(self, k), getattr(other, k))))
        return b

    @staticmethod
    def concat(parts, device) -> "BeamParticles":
        b = BeamParticles(device)
        if parts:
            for k in b._all():
                setattr(b, k, torch.cat([getattr(p, k) for p in parts]))
        return b


class BeamSource:
    """Hands out consecutive xi layers of a sorted beam (beam_io.py:9-47)."""

    def __init__(self, config: Config, beam_particles, device=None):
        self.dxi = config.getfloat('xi-step')
        if isinstance(beam_particles, np.ndarray):
            beam = BeamParticles(device).init_generated(beam_particles)
        else:
            beam = beam_particles
        beam.xi_sorted()
        self.beam = beam
        self.head = 0
        # descending xi on the host, once, for the layer boundaries
        self._neg_xi = (-beam.xi).cpu().numpy()

    def _n_ge(self, v):
        # number of particles with xi >= v (the array is sorted descending)
        return int(np.searchsorted(self._neg_xi, -v, side='right'))

    def layer_bounds(self, layer_idx):
        xi_min = -self.dxi * layer_idx
        xi_max = -self.dxi * (layer_idx + 1)
        lo = max(self._n_ge(xi_min), self.head)
        hi = max(self._n_ge(xi_max), self.head)
        length = hi - lo
        return self.head, self.head + length

    def get_beam_layer_to_layout(self, layer_idx) -> BeamParticles:
        a, b = self.layer_bounds(layer_idx)
        self.head = b
        return self.beam.take(slice(a, b))

    def remaining(self) -> BeamParticles:
        return self.beam.take(slice(self.head, None))


class BeamDrain:
    """Collects moved layers (beam_io.py:50-81); concatenated once on demand
    rather than on every push."""

    def __init__(self, config: Config, device=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.parts = []
        self.lost_parts = []

    def push_beam_layer(self, layer: BeamParticles):
        if layer.size > 0:
            self.parts.append(layer)

    def push_beam_lost(self, layer: BeamParticles):
        if layer.size > 0:
            self.lost_parts.append(layer)

    def beam_slice(self) -> BeamParticles:
        if len(self.parts) != 1:
            self.parts = [BeamParticles.concat(self.parts, self.device)]
        return self.parts[0]

    @property
    def beam_buffer(self):
        return self.beam_slice()

    def save(self, *args, **kwargs):
        self.beam_slice().save(*args, **kwargs)


class RigidBeamSource:
    """beam_io.py:84-94: the layout function itself is the 'layer'."""

    def __init__(self, config: Config, fn):
        self.fn = fn

    def get_beam_layer_to_layout(self, layer_idx):
        return self.fn


class RigidBeamDrain:
    def __init__(self, config: Config):
        pass

    def push_beam_layer(self, layer):
        pass

    def push_beam_lost(self, layer):
        pass

    def beam_slice(self):
        return None


class BeamCalculator:
    """Beam density layout and push (beam_calculator.py:51-143), on the device.

    Beam density planes stay undivided in HBM (the 1/h^2 of
    beam_calculator.py:91 is applied by the field solver, which receives the
    divisor), so ``rho_divisor`` must accompany any plane handed out."""

    def __init__(self, config: Config, device=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.h = config.getfloat('transverse-step')
        self.N = config.getint('window-width-steps')
        self.dxi = config.getfloat('xi-step')
        self.time_step = config.getfloat('time-step')
        self.substep_energy = config.getfloat('beam-substepping-energy')
        R = self.h * self.N / 2
        self.r_max = max(0.9 * R, R - 1)
        self.rho_divisor = self.h ** 2
        self.planes = torch.zeros(3, self.N, self.N, dtype=torch.float64, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.i = 0

    def start_time_step(self):
        self.planes.zero_()
        self.i = 0

    def rho_prev(self):
        return self.planes[(self.i - 1) % 3]

    def layout_beam_layer(self, layer: BeamParticles, layer_idx: int):
        """Deposit a layer: xi_loc weights into this step's plane, 1 - xi_loc
        into the next step's (weights.py:152-163).  Returns (full, prev)."""
        self.i = layer_idx
        full = self.planes[layer_idx % 3]
        nxt = self.planes[(layer_idx + 1) % 3]
        nxt.zero_()
        if layer.size:
            L = _lib.load()
            _lib.check(L.lcb_beam_deposit(
                layer.size, self.N, self.h, self.dxi, layer_idx,
                layer.x.data_ptr(), layer.y.data_ptr(), layer.xi.data_ptr(),
                layer.q_norm.data_ptr(), full.data_ptr(), nxt.data_ptr(),
                self.err.data_ptr(), _lib.stream_handle()), "lcb_beam_deposit")
        prev = self.planes[(layer_idx - 1) % 3] if layer_idx > 0 else self._zero()
        return full, prev

    def _zero(self):
        if not hasattr(self, "_z"):
            self._z = torch.zeros(self.N, self.N, dtype=torch.float64, device=self.device)
        return self._z

    def move_beam_layer(self, layer: BeamParticles, fell_size: int, layer_idx: int,
                        fields_k, fields_k1):
        """Substep and push the layer between the previous (k) and new (k+1)
        plasma planes; returns (lost, moved, fell) (beam_calculator.py:97-134)."""
        n = layer.size
        if n == 0:
            e = BeamParticles(self.device)
            return e, e, e
        L = _lib.load()
        fresh = n - fell_size
        st = _lib.stream_handle()
        if fresh > 0:
            _lib.check(L.lcb_beam_substepping(
                fresh, layer.q_m.data_ptr(), layer.pz.data_ptr(), self.substep_energy,
                self.time_step, layer.dt.data_ptr(), layer.remaining_steps.data_ptr(), st),
                "lcb_beam_substepping")
        flags = torch.empty(n, dtype=torch.uint8, device=self.device)
        _lib.check(L.lcb_beam_move(
            n, self.dxi, self.r_max, layer_idx - 1, self.h, self.N,
            layer.q_m.data_ptr(), layer.dt.data_ptr(), fields_k.struct, fields_k1.struct,
            layer.remaining_steps.data_ptr(), layer.id.data_ptr(), layer.x.data_ptr(),
            layer.y.data_ptr(), layer.xi.data_ptr(), layer.px.data_ptr(),
            layer.py.data_ptr(), layer.pz.data_ptr(), flags.data_ptr(),
            self.err.data_ptr(), st), "lcb_beam_move")
        lost = layer.take((flags & 1) != 0)
        moved = layer.take((flags & 2) != 0)
        fell = layer.take((flags & 4) != 0)
        return lost, moved, fell


class RigidBeamCalculator:
    """Rigid driver (beam_calculator.py:148-181): rho_b(xi) = fn(xp, xi, X, Y)
    with X, Y = meshgrid(grid, grid).  The function is evaluated on the host
    with numpy, for all xi layers of a time step at once, and the planes are
    uploaded to HBM in one copy."""

    def __init__(self, config: Config, device=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.dxi = config.getfloat('xi-step')
        N = config.getint('window-width-steps')
        h = config.getfloat('transverse-step')
        grid = (np.arange(N) - N // 2) * h
        self.x_grid, self.y_grid = np.meshgrid(grid, grid)
        self.N = N
        self.rho_divisor = 1.0
        self.table = None
        self.zero = torch.zeros(N, N, dtype=torch.float64, device=self.device)

    def start_time_step(self):
        pass

    def prepare(self, fn, first, last):
        """Evaluate fn for layers first..last (inclusive) and upload them."""
        n = last - first + 1
        host = torch.empty((n, self.N, self.N), dtype=torch.float64, pin_memory=True)
        hn = host.numpy()
        for k in range(n):
            xi = -(first + k) * self.dxi
            hn[k] = fn(np, xi, self.x_grid, self.y_grid)
        self.first = first
        self.table = host.to(self.device, non_blocking=True)
        self._host = host

    def layout_beam_layer(self, fn, layer_idx):
        full = self.table[layer_idx - self.first]
        prev = self.table[layer_idx - 1 - self.first] if layer_idx > self.first else self.zero
        return full, prev

    def move_beam_layer(self, *a, **k):
        return None, None, None
