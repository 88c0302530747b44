"""Beam on the device: particle SoA, xi-layer source and drain, density
layout and substepped push (lcode/beam3d/*).

The beam is kept sorted by xi (descending) in HBM, so a layer is a
contiguous slice; layer lengths are found by binary search on a host copy of
the sorted xi taken once per time step (the reference counts them with a
device reduction and a host sync per layer, beam3d/beam_io.py:29-47).
"""
from __future__ import annotations

import ctypes as C

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

    def all_layer_bounds(self, first=0, last=None):
        """Slices of every layer the xi loop will cut, in order, as the
        reference's successive get_beam_layer_to_layout calls would cut them
        (count in range, then cut from the head)."""
        out = {}
        head = self.head
        # deepest layer holding a particle: ceil(-min(xi) / dxi)
        n_layers = last if last is not None else int(np.ceil(
            max(float(self._neg_xi[-1]) if self._neg_xi.size else 0.0, 0.0) / self.dxi)) + 2
        saved = self.head
        for i in range(first, n_layers + 1):
            self.head = head
            a, b = self.layer_bounds(i)
            out[i] = (a, b)
            head = b
        self.head = saved
        return out

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


def _soa(b: "BeamParticles", offset: int = 0) -> "_lib.BeamSoA":
    s = _lib.BeamSoA()
    for k in BEAM_KEYS + ("dt", "remaining_steps"):
        t = getattr(b, k)
        setattr(s, k, t.data_ptr() + offset * t.element_size())
    return s


class BeamCalculator:
    """Beam density layout and push (beam_calculator.py:51-143), on the device.

    One xi step of the beam is one lcb_beam_step call: the push of layer i-1
    (between the previous and the new plasma fields) and the layout of layer
    i+1 for the next step, with every particle count kept on the device
    (drain, fell and lost buffers with device counters).  Beam density planes
    stay undivided in HBM (the 1/h^2 of beam_calculator.py:91 is applied by
    the field solver, which receives ``rho_divisor``)."""

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
        # device counters: fell A, fell B, drain, lost
        self.counts = torch.zeros(4, dtype=torch.int64, device=self.device)
        self.cap = 0
        self._plane_ptrs = [self.planes[k].data_ptr() for k in range(3)]
        self._step_args_cache = {}   # per fell buffer parity; reset with the buffers

    def _ensure(self, n_total, max_layer):
        cap = max(n_total, 1)
        stage = cap + max(max_layer, 1)
        if cap <= self.cap and stage <= self.stage_cap:
            return
        self.cap, self.stage_cap = cap, stage
        self._step_args_cache = {}
        self.drain = BeamParticles(self.device, cap)
        self.lost = BeamParticles(self.device, cap)
        self.fell = [BeamParticles(self.device, cap), BeamParticles(self.device, cap)]
        self.stage = BeamParticles(self.device, stage)
        self.flags = torch.zeros(stage, dtype=torch.uint8, device=self.device)

    def start_time_step(self, source: "BeamSource"):
        """Zero the planes and counters (the first layer is laid out by
        layout_first).  A streaming source (pipeline.StreamingSource) gives
        its layer slices as its chunks arrive; its buffers are sized for the
        whole beam."""
        self.source = source
        self._step_args_cache = {}
        n = source.beam.size
        if getattr(source, "streaming", False):
            self.bounds = None
            max_layer = n
        else:
            self.bounds = source.all_layer_bounds()
            max_layer = max((b - a for a, b in self.bounds.values()), default=0)
        self._ensure(n, max_layer)
        self.planes.zero_()
        self.counts.zero_()
        self.err.zero_()
        self.fell_cur = 0

    def layer_bounds(self, i):
        if self.bounds is None:
            return self.source.layer_bounds(i) if i >= 0 else (0, 0)
        return self.bounds.get(i, (0, 0))

    def rho(self, i):
        """(full, prev) density planes of xi step i."""
        return self.planes[i % 3], self.planes[(i - 1) % 3]

    def _args(self, layer_idx, layout, move, fields_k, fields_k1):
        a = _lib.BeamStepArgs()
        a.grid_steps, a.h, a.xi_step, a.r_max = self.N, self.h, self.dxi, self.r_max
        a.substep_energy, a.time_step = self.substep_energy, self.time_step
        a.layer_idx = layer_idx
        a.source = _soa(self.source.beam)
        a.layout_begin, a.layout_end = layout
        a.move_begin, a.move_end = move
        fi, fo = self.fell_cur, 1 - self.fell_cur
        a.fell_in = _soa(self.fell[fi])
        a.fell_in_count = self.counts[fi].data_ptr()
        a.fell_out = _soa(self.fell[fo])
        a.fell_out_count = self.counts[fo].data_ptr()
        a.fell_capacity = self.cap
        a.drain = _soa(self.drain)
        a.drain_count = self.counts[2].data_ptr()
        a.drain_capacity = self.cap
        a.lost = _soa(self.lost)
        a.lost_count = self.counts[3].data_ptr()
        a.lost_capacity = self.cap
        a.stage = _soa(self.stage)
        a.stage_flags = self.flags.data_ptr()
        a.stage_capacity = self.stage_cap
        a.ro0 = self.planes[layer_idx % 3].data_ptr()
        a.ro1 = self.planes[(layer_idx + 1) % 3].data_ptr()
        a.fields_k = C.addressof(fields_k.struct) if fields_k is not None else None
        a.fields_k1 = C.addressof(fields_k1.struct) if fields_k1 is not None else None
        a.err = self.err.data_ptr()
        return a

    def layout_first(self, i):
        """Lay out layer i alone (before the first xi step)."""
        lo = self.layer_bounds(i)
        if lo[1] > lo[0]:
            L = _lib.load()
            _lib.check(L.lcb_beam_deposit(
                lo[1] - lo[0], self.N, self.h, self.dxi, i,
                self.source.beam.x[lo[0]:].data_ptr(), self.source.beam.y[lo[0]:].data_ptr(),
                self.source.beam.xi[lo[0]:].data_ptr(), self.source.beam.q_norm[lo[0]:].data_ptr(),
                self.planes[i % 3].data_ptr(), self.planes[(i + 1) % 3].data_ptr(),
                self.err.data_ptr(), _lib.stream_handle()), "lcb_beam_deposit")

    def after_plasma_step(self, i, fields_prev, fields_new):
        """Push layer i-1 (and the particles that fell from the last push)
        between fields_prev and fields_new, then lay out layer i+1.  The
        argument struct is built once per fell-buffer parity; a step only
        sets its layer indices, ranges, planes and fields."""
        # plane (i + 2) % 3 (ro1) is cleared inside lcb_beam_step
        a = self._step_args_cache.get(self.fell_cur)
        if a is None:
            a = self._step_args_cache[self.fell_cur] = self._args(i, (0, 0), (0, 0), None, None)
        a.layer_idx = i
        a.layout_idx = i + 1
        a.layout_begin, a.layout_end = self.layer_bounds(i + 1)
        a.move_begin, a.move_end = self.layer_bounds(i - 1)
        a.ro0 = self._plane_ptrs[(i + 1) % 3]
        a.ro1 = self._plane_ptrs[(i + 2) % 3]
        a.fields_k = C.addressof(fields_prev.struct) if fields_prev is not None else None
        a.fields_k1 = C.addressof(fields_new.struct) if fields_new is not None else None
        _lib.check(_lib.load().lcb_beam_step(C.byref(a), _lib.stream_handle()),
                   "lcb_beam_step")
        self.fell_cur = 1 - self.fell_cur

    def finish(self):
        """Moved and lost particles of the time step (one host read)."""
        c = self.counts.cpu().numpy()
        out = []
        for buf, n in ((self.drain, int(c[2])), (self.lost, int(c[3]))):
            v = buf.take(slice(0, n))
            for k in v._all():  # own the data: the buffers are reused next time step
                setattr(v, k, getattr(v, k).clone())
            out.append(v)
        return out[0], out[1]


class RigidBeamCalculator:
    """Rigid driver (beam_calculator.py:148-181): rho_b(xi) = fn(xp, xi, X, Y)
    with X, Y = meshgrid(grid, grid).  The function is evaluated on the host
    with numpy, for all xi layers of a time step at once, and the planes are
    uploaded to HBM in one copy.  Each xi step copies its layer into one of
    two fixed planes (the other holds the previous layer), so the plasma
    step's captured graphs read fixed addresses: one device copy per step."""

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
        self.planes = torch.zeros(2, N, N, dtype=torch.float64, device=self.device)

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
        full = self.planes[layer_idx % 2]
        full.copy_(self.table[layer_idx - self.first])
        prev = self.planes[(layer_idx - 1) % 2] if layer_idx > self.first else self.zero
        return full, prev

    def move_beam_layer(self, *a, **k):
        return None, None, None
