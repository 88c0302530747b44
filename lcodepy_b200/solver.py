"""Device-resident plasma xi step (lcode/plasma3d/solver.py:25-78).

``Plane2d3vPlasmaSolver`` owns every device buffer of the plasma response and
advances it by one xi step through liblcb.so:

    K1 move_wo_fields -> K2 move_smart(fields_prev) -> K3 deposit
      -> compute_fields(fields_prev)          -> half A
      -> K2(half A) -> K3 -> compute_fields(half A) -> full, half B
      -> K2(half B) -> K3

Buffers rotate instead of being copied: particles (prev, full), fields
(prev, full) and currents (prev, full) swap roles after each step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .config import Config
from .data import Arrays
from .plasma3d import (CURRENT_NAMES, FIELD_NAMES, PARTICLE_NAMES, FieldOperators,
                       PlasmaState, host_initial_particles, plasma_params, sorts_of)


class FieldSet:
    """Seven N x N FP64 planes."""

    def __init__(self, N, device):
        self.buf = torch.zeros(7, N, N, dtype=torch.float64, device=device)
        self.struct = _lib.Fields7()
        for i in range(7):
            self.struct.f[i] = self.buf[i].data_ptr()

    def __getattr__(self, k):
        if k in FIELD_NAMES:
            return self.__dict__["buf"][FIELD_NAMES.index(k)]
        raise AttributeError(k)

    def arrays(self) -> Arrays:
        return Arrays(torch, **{k: self.buf[i] for i, k in enumerate(FIELD_NAMES)})


class CurrentSet:
    """ro, jx, jy, jz, each (2, N, N)."""

    def __init__(self, N, device):
        self.buf = torch.zeros(4, 2, N, N, dtype=torch.float64, device=device)
        self.struct = _lib.Currents4(*(self.buf[i].data_ptr() for i in range(4)), 2)

    def __getattr__(self, k):
        if k in CURRENT_NAMES:
            return self.__dict__["buf"][CURRENT_NAMES.index(k)]
        raise AttributeError(k)

    def arrays(self) -> Arrays:
        return Arrays(torch, **{k: self.buf[i] for i, k in enumerate(CURRENT_NAMES)})


class Plane2d3vPlasmaSolver:
    """The plasma response to one xi step, on the GPU."""

    def __init__(self, config: Config, device=None):
        # declustering noise filter of the electrons after the last move
        # (solver.py:68-72, noise_filter.py:82-239).  The reference reads the
        # damping from 'damping-declustering', which its defaults lack (a run
        # without that key fails there); here the default
        # 'declustering-damping' is the fallback.
        self.declustering = config.getbool('declustering-enabled')
        if self.declustering:
            damping = config.getraw('damping-declustering')
            self.decl = dict(
                force=config.getfloat('declustering-force'),
                damping=float(damping if damping is not None
                              else config.getfloat('declustering-damping')),
                limit=config.getfloat('declustering-limit'),
                sigma=config.getfloat('declustering-averaging'))
            self.decl_buf = None
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.config = config
        p = plasma_params(config)
        self.N, self.h, self.dxi = p["N"], p["h"], p["dxi"]
        self.boundary, self.sub_coeff = p["boundary"], p["sub_coeff"]
        self.ion_model, self.precision = p["ion_model"], p["precision"]
        self.dep_precision = p["deposit_precision"]
        self.sort_names = sorts_of(self.ion_model)
        self.n_sorts = len(self.sort_names)
        _lib.load()
        self.ops = FieldOperators(self.N, self.h, self.sub_coeff, self.device,
                                  self.precision == _lib.LCB_PREC_MIXED)
        N, dev = self.N, self.device
        self.fields = [FieldSet(N, dev) for _ in range(2)]   # prev, full (rotating)
        self.half = [FieldSet(N, dev) for _ in range(2)]     # half A, half B
        self.currents = [CurrentSet(N, dev) for _ in range(2)]
        self.ws_fields = torch.empty(
            _lib.load().lcb_compute_fields_workspace_bytes(N, self.precision),
            dtype=torch.uint8, device=dev)
        ws_dep = _lib.load().lcb_plasma_deposit_workspace_bytes(N, self.dep_precision)
        self.ws_dep = torch.empty(max(ws_dep, 256), dtype=torch.uint8, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ro_initial = torch.zeros(N, N, dtype=torch.float64, device=dev)
        self.zero_plane = torch.zeros(N, N, dtype=torch.float64, device=dev)
        self.states = None
        self.cur = 0  # index of the "prev" copy in self.states / fields / currents
        # name -> list of (start, end) CUDA events, filled while not None
        self.op_timers = None
        # CUDA graphs of one xi step, one per buffer parity; the beam density
        # planes are copied into fixed buffers so the graphs stay valid.
        pe = config.getraw('cuda-graphs')
        self.use_graphs = True if pe is None else bool(pe)
        # one fused kernel per predictor-corrector stage (K1/K2 + K3), the
        # default in both precisions; 'fused-particle-kernels': False runs
        # the three reference kernels separately
        pf = config.getraw('fused-particle-kernels')
        self.fused = True if pf is None else bool(pf)
        self.fineness = max(1, int(round(config.getfloat('plasma-fineness') or 1)))
        self.rbf = torch.zeros(N, N, dtype=torch.float64, device=dev)
        self.rbp = torch.zeros(N, N, dtype=torch.float64, device=dev)
        self.graphs = [None, None]
        self.graph_launches = [0, 0]
        self.graph_div = None
        self.plane_graphs = {}    # (parity, plane pointers, divisor) -> (graph, launches)
        self.eager_steps = 0
        # capture on the current (non-default) stream without the device-wide
        # synchronisation of torch.cuda.graph, for solvers that share the GPU
        # with others (batch members)
        self.capture_on_stream = False
        # on-axis Ez of every xi step recorded on the device as the step's
        # last kernel (inside the captured graphs): a history and its counter
        # (see record_axis); None records nothing
        self.axis = None

    def record_axis(self, capacity: int):
        """Record the new on-axis Ez at the end of every xi step into a
        device history of ``capacity`` entries (lcb_record_axis); returns
        (history, counter).  The buffers persist, so captured graphs stay
        valid; a larger capacity drops the graphs."""
        if self.axis is None or self.axis[0].numel() < capacity:
            self.axis = (torch.zeros(capacity, dtype=torch.float64, device=self.device),
                         torch.zeros(1, dtype=torch.int64, device=self.device))
            self.graphs = [None, None]
            self.plane_graphs = {}
        return self.axis

    def _timed(self, name, fn, *args):
        if self.op_timers is None:
            return fn(*args)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn(*args)
        b.record()
        self.op_timers.setdefault(name, []).append((a, b))
        return r

    # -- initial state (initialization.py:278-414) --
    def init_state(self, current_time=0.0):
        x_init, y_init, q, m = host_initial_particles(self.config, current_time)
        Ns = x_init.shape[0]
        dev = self.device
        if self.states is None or self.states[0].Ns != Ns:
            self.states = [PlasmaState(self.n_sorts, Ns, dev) for _ in range(2)]
            # graphs captured on the previous particle buffers are stale
            self.graphs = [None, None]
            self.plane_graphs = {}
        st = self.states[0]
        n = Ns * Ns
        xi_t = torch.from_numpy(x_init.ravel()).to(dev)
        yi_t = torch.from_numpy(y_init.ravel()).to(dev)
        q_t = torch.from_numpy(q.ravel()).to(dev)
        m_t = torch.from_numpy(m.ravel()).to(dev)
        for s in (self.states[0], self.states[1]):
            for k in ("x_offt", "y_offt", "px", "py", "pz"):
                s.t[k].zero_()
            s.chaos.zero_()
            for si in range(self.n_sorts):
                sl = slice(si * n, (si + 1) * n)
                s.x_init[sl] = xi_t
                s.y_init[sl] = yi_t
            s.q[:n] = q_t
            s.m[:n] = m_t
            if self.n_sorts == 2:
                s.q[n:] = -q_t
                s.m[n:] = self.config.getfloat("ion-mass") * m_t
        # background charge: minus the deposited initial electrons
        # (initialization.py:351-356)
        tmp = self.currents[1]
        self._deposit(st, tmp, with_background=False, n_sorts=1)
        self.ro_initial.copy_(-tmp.ro[0])
        for f in self.fields + self.half:
            f.buf.zero_()
        for c in self.currents:
            c.buf.zero_()
        self.err.zero_()
        self.cur = 0
        self.last_fields = self.fields[1]

    def load_state(self, state: dict):
        """Start from a stored plasma state (``plasma_state.load_plasmastate``)
        instead of the initial one: particles of every sort, the previous
        fields and currents, and the background charge if the state has it
        (initialization.py:417-460).  Call after ``init_state``; returns the
        state's xi_plasma_layer (None if it has none)."""
        st0 = self.states[0]
        n, Ns, N = st0.n_per_sort, st0.Ns, self.N
        for si, sort in enumerate(self.sort_names):
            rec = state["particles"][sort]
            if rec["x_init"].shape != (Ns, Ns):
                raise ValueError(f"plasma state '{sort}' has a {rec['x_init'].shape} lattice, "
                                 f"this configuration {Ns} x {Ns}")
            for k in PARTICLE_NAMES:
                t = torch.from_numpy(np.ascontiguousarray(rec[k]).ravel()).to(self.device)
                for s in self.states:
                    s.t[k][si * n:(si + 1) * n] = t
            if si == 0:     # the electrons' declustering state, if stored
                for c, k in enumerate(("dx_chaotic", "dy_chaotic")):
                    if k in rec:
                        t = torch.from_numpy(np.ascontiguousarray(rec[k]).ravel()).to(self.device)
                        for s in self.states:
                            s.chaos[c].copy_(t)
        for key, shape in (("fields", (N, N)), ("currents", (2, N, N))):
            for k, a in state[key].items():
                if a.shape != shape:
                    raise ValueError(f"plasma state {key} '{k}' has shape {a.shape}, expected {shape}")
        F = self.fields[self.cur]
        for i, k in enumerate(FIELD_NAMES):
            F.buf[i].copy_(torch.from_numpy(state["fields"][k]))
        Cs = self.currents[self.cur]
        for i, k in enumerate(CURRENT_NAMES):
            Cs.buf[i].copy_(torch.from_numpy(state["currents"][k]))
        if state.get("rho_initial") is not None:
            self.ro_initial.copy_(torch.from_numpy(state["rho_initial"]))
        return state.get("xi_plasma_layer")

    # -- kernels --
    def _deposit(self, st: PlasmaState, out: CurrentSet, with_background=True, n_sorts=None):
        L = _lib.load()
        n_sorts = n_sorts or self.n_sorts
        bg = self.ro_initial if (with_background and self.ion_model == "background") else None
        _lib.check(L.lcb_plasma_deposit(
            st.n_per_sort, n_sorts, self.N, self.h, st.Ns, self.dep_precision,
            st.x_init.data_ptr(), st.y_init.data_ptr(), st.x_offt.data_ptr(),
            st.y_offt.data_ptr(), st.px.data_ptr(), st.py.data_ptr(), st.pz.data_ptr(),
            st.q.data_ptr(), st.m.data_ptr(), _lib.ptr(bg),
            out.ro.data_ptr(), out.jx.data_ptr(), out.jy.data_ptr(), out.jz.data_ptr(),
            self.ws_dep.data_ptr(), self.ws_dep.numel(), self.err.data_ptr(),
            _lib.stream_handle()), "lcb_plasma_deposit")

    def _move_wo_fields(self, prev: PlasmaState, full: PlasmaState):
        L = _lib.load()
        _lib.check(L.lcb_plasma_move_wo_fields(
            prev.x_offt.numel(), self.dxi, prev.m.data_ptr(),
            prev.x_offt.data_ptr(), prev.y_offt.data_ptr(), prev.px.data_ptr(),
            prev.py.data_ptr(), prev.pz.data_ptr(), prev.q.data_ptr(),
            full.x_offt.data_ptr(), full.y_offt.data_ptr(), full.px.data_ptr(),
            full.py.data_ptr(), full.pz.data_ptr(), full.q.data_ptr(),
            _lib.stream_handle()), "lcb_plasma_move_wo_fields")

    def _move_smart(self, F: FieldSet, prev: PlasmaState, full: PlasmaState):
        L = _lib.load()
        fb = F.buf
        _lib.check(L.lcb_plasma_move_smart(
            prev.x_offt.numel(), self.dxi, self.boundary, self.h, self.N,
            *(fb[i].data_ptr() for i in range(6)),
            prev.x_init.data_ptr(), prev.y_init.data_ptr(),
            prev.x_offt.data_ptr(), prev.y_offt.data_ptr(), prev.px.data_ptr(),
            prev.py.data_ptr(), prev.pz.data_ptr(), full.m.data_ptr(),
            full.q.data_ptr(), full.x_offt.data_ptr(), full.y_offt.data_ptr(),
            full.px.data_ptr(), full.py.data_ptr(), full.pz.data_ptr(),
            self.err.data_ptr(), _lib.stream_handle()), "lcb_plasma_move_smart")

    def _move_deposit(self, F: FieldSet, prev: PlasmaState, full: PlasmaState,
                      out: CurrentSet, first: bool):
        a = _lib.MoveDepositArgs()
        a.n_per_sort, a.n_sorts, a.particles_side = prev.n_per_sort, self.n_sorts, prev.Ns
        a.grid_steps, a.precision, a.first = self.N, self.dep_precision, int(first)
        a.lattice_fineness = self.fineness
        a.xi_step, a.boundary, a.h = self.dxi, self.boundary, self.h
        for i in range(6):
            a.fields[i] = F.buf[i].data_ptr()
        a.prev = _lib.PlasmaParticles(*(prev.t[k].data_ptr() for k in PARTICLE_NAMES))
        a.full = _lib.PlasmaParticles(*(full.t[k].data_ptr() for k in PARTICLE_NAMES))
        a.ro_initial = self.ro_initial.data_ptr() if self.ion_model == "background" else None
        a.ro, a.jx, a.jy, a.jz = (out.buf[i].data_ptr() for i in range(4))
        a.workspace, a.workspace_bytes = self.ws_dep.data_ptr(), self.ws_dep.numel()
        a.err = self.err.data_ptr()
        _lib.check(_lib.load().lcb_plasma_move_deposit(C.byref(a), _lib.stream_handle()),
                   "lcb_plasma_move_deposit")

    def _compute_fields(self, F: FieldSet, Fprev: FieldSet, cprev: CurrentSet,
                        cfull: CurrentSet, rb_full, rb_prev, rb_div,
                        out_full: FieldSet | None, out_half: FieldSet):
        a = _lib.ComputeFieldsArgs()
        a.grid_steps, a.h, a.xi_step = self.N, self.h, self.dxi
        a.subtraction_coeff, a.precision = self.sub_coeff, self.precision
        a.operators = self.ops.ptr
        a.fields, a.fields_prev = F.struct, Fprev.struct
        a.currents_prev, a.currents_full = cprev.struct, cfull.struct
        a.rho_beam_full, a.rho_beam_prev = rb_full.data_ptr(), rb_prev.data_ptr()
        a.rho_beam_divisor = rb_div
        if out_full is not None:
            a.out_full = out_full.struct
        a.out_half = out_half.struct
        a.workspace, a.workspace_bytes = self.ws_fields.data_ptr(), self.ws_fields.numel()
        _lib.check(_lib.load().lcb_compute_fields(C.byref(a), _lib.stream_handle()),
                   "lcb_compute_fields")

    def _declustering(self, full: PlasmaState, prev: PlasmaState):
        """The noise filter on the moved electrons (noise_filter.py:82-239):
        inhomogeneity kernel, Gaussian average of both planes by a Fourier
        multiply (cuFFT; scipy's fourier_gaussian factor exp(-2 pi^2 sigma^2
        f^2) per axis, f the FFT frequencies), then the kick kernel."""
        L = _lib.load()
        n = prev.Ns
        st = _lib.stream_handle()
        if self.decl_buf is None:
            self.decl_buf = torch.zeros(4, n, n, dtype=torch.float64, device=self.device)
            f = torch.fft.fftfreq(n, dtype=torch.float64, device=self.device)
            g = torch.exp(-2 * np.pi ** 2 * self.decl["sigma"] ** 2 * f * f)
            self.decl_gauss = g[:, None] * g[None, :]
        b = self.decl_buf
        _lib.check(L.lcb_declustering_inhomogeneity(
            n, full.x_offt.data_ptr(), full.y_offt.data_ptr(), b[0].data_ptr(),
            b[1].data_ptr(), st), "lcb_declustering_inhomogeneity")
        b[2:4].copy_(torch.fft.ifft2(torch.fft.fft2(b[0:2]) * self.decl_gauss).real)
        a = _lib.DeclusteringArgs()
        a.n, a.xi_step = n, self.dxi
        a.force, a.damping, a.limit = self.decl["force"], self.decl["damping"], self.decl["limit"]
        a.dx_inhom, a.dy_inhom = b[0].data_ptr(), b[1].data_ptr()
        a.dx_average, a.dy_average = b[2].data_ptr(), b[3].data_ptr()
        a.dx_chaotic_prev, a.dy_chaotic_prev = prev.chaos[0].data_ptr(), prev.chaos[1].data_ptr()
        a.px, a.py = full.px.data_ptr(), full.py.data_ptr()
        a.dx_chaotic, a.dy_chaotic = full.chaos[0].data_ptr(), full.chaos[1].data_ptr()
        _lib.check(L.lcb_declustering_apply(C.byref(a), st), "lcb_declustering_apply")

    # -- the xi step --
    @property
    def prev_fields(self) -> FieldSet:
        return self.fields[self.cur]

    @property
    def prev_currents(self) -> CurrentSet:
        return self.currents[self.cur]

    @property
    def prev_particles(self) -> PlasmaState:
        return self.states[self.cur]

    def step_dxi(self, rb_full: torch.Tensor, rb_prev: torch.Tensor, rb_div: float = 1.0,
                 stable_planes: bool = False):
        """Advance the plasma by one xi step; afterwards the new state is the
        "prev" state (fields / currents / particles) and the step's input
        fields remain readable as ``last_fields`` until the next step.

        After two eager steps the step runs as a captured CUDA graph (one per
        parity of the rotating buffers), unless per-op timing is requested.
        The beam density planes are copied into fixed buffers that the graphs
        read; with ``stable_planes`` (the caller rotates a few persistent
        planes, as the non-rigid beam does) one graph per parity and plane
        pair reads them in place instead."""
        if not self.use_graphs or self.op_timers is not None:
            self._step_ops(rb_full, rb_prev, rb_div)
            self.eager_steps += 1
            return
        p = self.cur
        if stable_planes:
            key = (p, rb_full.data_ptr(), rb_prev.data_ptr(), rb_div)
            if key not in self.plane_graphs:
                if self.eager_steps < 2:
                    self._step_ops(rb_full, rb_prev, rb_div)
                    self.eager_steps += 1
                    return
                self.plane_graphs[key] = self._capture(rb_full, rb_prev, rb_div)
            g, nl = self.plane_graphs[key]
        else:
            self.rbf.copy_(rb_full)
            self.rbp.copy_(rb_prev)
            if self.graph_div != rb_div:
                self.graphs = [None, None]
                self.graph_div = rb_div
            if self.graphs[p] is None:
                if self.eager_steps < 2:
                    self._step_ops(self.rbf, self.rbp, rb_div)
                    self.eager_steps += 1
                    return
                self.graphs[p], self.graph_launches[p] = self._capture(self.rbf, self.rbp, rb_div)
            g, nl = self.graphs[p], self.graph_launches[p]
        g.replay()
        _lib.add_replayed(nl)
        self.cur = 1 - p
        self.last_fields = self.fields[p]

    def _capture(self, rb_full, rb_prev, rb_div):
        """Capture one xi step (for the current buffer parity) reading the
        given beam density planes; returns (graph, launches in it)."""
        g = torch.cuda.CUDAGraph()
        n0 = _lib.load().lcb_launch_count()
        if self.capture_on_stream:
            g.capture_begin(capture_error_mode="thread_local")
            try:
                self._step_ops(rb_full, rb_prev, rb_div, advance=False)
            finally:
                g.capture_end()
        else:
            with torch.cuda.graph(g):
                self._step_ops(rb_full, rb_prev, rb_div, advance=False)
        return g, _lib.load().lcb_launch_count() - n0

    def _step_ops(self, rb_full, rb_prev, rb_div, advance=True):
        p, f = self.cur, 1 - self.cur
        prev, full = self.states[p], self.states[f]
        Fp, Ff = self.fields[p], self.fields[f]
        cp, cf = self.currents[p], self.currents[f]
        hA, hB = self.half
        T = self._timed
        if self.fused:
            T("move_deposit", self._move_deposit, Fp, prev, full, cf, True)
        else:
            T("move_wo_fields", self._move_wo_fields, prev, full)
            T("move_smart", self._move_smart, Fp, prev, full)
            T("deposit", self._deposit, full, cf)
        T("compute_fields", self._compute_fields, Fp, Fp, cp, cf, rb_full, rb_prev,
          rb_div, None, hA)
        if self.fused:
            T("move_deposit", self._move_deposit, hA, prev, full, cf, False)
        else:
            T("move_smart", self._move_smart, hA, prev, full)
            T("deposit", self._deposit, full, cf)
        T("compute_fields", self._compute_fields, hA, Fp, cp, cf, rb_full, rb_prev,
          rb_div, Ff, hB)
        if self.declustering:
            # the filter acts between the last move and its deposit
            T("move_smart", self._move_smart, hB, prev, full)
            T("declustering", self._declustering, full, prev)
            T("deposit", self._deposit, full, cf)
        elif self.fused:
            T("move_deposit", self._move_deposit, hB, prev, full, cf, False)
        else:
            T("move_smart", self._move_smart, hB, prev, full)
            T("deposit", self._deposit, full, cf)
        if self.axis is not None:
            hist, counter = self.axis
            _lib.check(_lib.load().lcb_record_axis(
                Ff.buf[FIELD_NAMES.index("Ez")].data_ptr(), self.N, counter.data_ptr(),
                hist.data_ptr(), hist.numel(), _lib.stream_handle()), "lcb_record_axis")
        if advance:
            self.cur = f
            self.last_fields = Fp

    # -- views with the reference's names --
    def particles_dict(self) -> dict:
        st = self.prev_particles
        return {name: st.sort_arrays(s) for s, name in enumerate(self.sort_names)}

    def check_errors(self):
        e = int(self.err.item())
        if e:
            self.err.zero_()
            why = []
            if e & _lib.DEVERR_PLASMA_STENCIL:
                why.append("a plasma particle stencil left the grid (NaN or runaway particle)")
            if e & _lib.DEVERR_FIXED_RANGE:
                why.append("a deposit contribution approached the fixed-point range of the "
                           "mixed-precision deposit (use 'deposit-precision': 'fp64')")
            raise RuntimeError(f"device error word 0x{e:x}: " + "; ".join(why or ["unknown"]))
