"""Many simulations on one GPU: batched parameter scans and a served request
stream.

Each ``Member`` is one quasistatic 3D simulation with a rigid Gaussian driver.
Its whole xi step -- driver evaluated on the device from a step counter,
predictor-corrector plasma step, on-axis Ez record -- is captured once in two
CUDA graphs (one per parity of the rotating buffers) and replayed on the
member's own stream, so members of any grid size advance concurrently and a
host loop only issues one graph launch per member and xi step.

A ``BeamMember`` has a non-rigid driver (macroparticles of a bi-Gaussian
beam): its plasma step is the same captured graph, and the beam layer step
(push, ordered compaction, layout of the next layer, with device counters)
is launched beside it on the member's stream, without host round trips.

``BatchRunner`` advances a fixed set of members together (a parameter scan).
``Server`` admits requests that arrive over time into free slots while others
run (continuous batching), bounded by an HBM budget, and reports each
request's completion latency.

Slots can be checkpointed between xi steps and resumed (``Member.checkpoint``,
``restore_member``, ``Server.checkpoint`` / ``Server.restore``): a member's
plasma state goes to a plasma state file in the format the reference's
``Simulation`` loads with ``external_plasmastate`` (plasma_state.py), its
metadata (config, driver, steps done, on-axis Ez so far, and for a beam
driver the beam step's device buffers) to a slot file beside it.
"""
from __future__ import annotations

import collections
import dataclasses
import json
import math
import os
import time

import numpy as np
import torch

from . import _lib
from .config import Config
from .solver import Plane2d3vPlasmaSolver

XI_LEN = math.sqrt(2 * math.pi)


@dataclasses.dataclass
class GaussianDriver:
    """rho_b = amplitude exp(-r^2 / (2 sigma_r^2)) (1 + cos(sqrt(pi/2) xi)) / 2
    on -xi_len <= xi <= 0.  Callable with the reference's rigid-beam
    signature fn(xp, xi, x_grid, y_grid) as well."""
    amplitude: float = 0.1
    sigma_r: float = 1.0
    xi_len: float = XI_LEN

    def __call__(self, xp, xi, x, y):
        if -self.xi_len <= xi <= 0:
            return (self.amplitude * xp.exp(-(x ** 2 + y ** 2) / (2 * self.sigma_r ** 2))
                    * (1 + np.cos(np.sqrt(np.pi / 2) * xi)) / 2)
        return xp.zeros_like(x)


@dataclasses.dataclass
class BeamDriver:
    """A non-rigid electron driver: n macroparticles, bi-Gaussian (sigma_r,
    sigma_z) around xi0 (cut to 2 xi0 < xi < 0 and r < r_max), peak density
    `amplitude` (in n0; the beam charge is negative), gamma with a relative
    spread, normalised emittance; generated on the device from `seed`."""
    n: int = 100_000
    amplitude: float = 0.1
    sigma_r: float = 1.0
    sigma_z: float = 1.0
    xi0: float = -3.0
    gamma: float = 1000.0
    espread: float = 0.01
    emittance: float = 1e-2
    seed: int = 0
    r_max: float = 4.0        # radial cut (keep it inside the window)

    def device_beam(self, dxi: float, device=None):
        """The beam generated on the device (seeded Philox stream of
        torch.Generator), sorted by xi descending, as BeamParticles: the
        distribution of bigaussian_beam in milliseconds instead of the host's
        tenths of a second, so that admitting a request does not stall the
        server loop."""
        from .beam3d import BeamParticles
        dev = device or torch.device("cuda", torch.cuda.current_device())
        g = torch.Generator(device=dev)
        g.manual_seed(int(self.seed))
        f64 = dict(dtype=torch.float64, device=dev, generator=g)
        xi = torch.randn(2 * self.n, **f64) * self.sigma_z + self.xi0
        xi = xi[(xi < 0) & (xi > 2 * self.xi0)][:self.n]
        m = xi.numel()
        cut = 1 - math.exp(-self.r_max ** 2 / (2 * self.sigma_r ** 2))
        r = self.sigma_r * torch.sqrt(-2 * torch.log1p(-torch.rand(m, **f64) * cut))
        phi = torch.rand(m, **f64) * (2 * math.pi)
        sp = self.emittance / self.sigma_r
        b = BeamParticles(dev)
        b.xi = xi
        b.x, b.y = r * torch.cos(phi), r * torch.sin(phi)
        b.px = torch.randn(m, **f64) * sp
        b.py = torch.randn(m, **f64) * sp
        b.pz = torch.randn(m, **f64) * (self.gamma * self.espread) + self.gamma
        b.q_m = torch.full((m,), -1.0, dtype=torch.float64, device=dev)
        q_total = (-self.amplitude * (math.sqrt(2 * math.pi) * self.sigma_z)
                   * (2 * math.pi * self.sigma_r ** 2) / dxi)
        b.q_norm = torch.full((m,), q_total / max(m, 1), dtype=torch.float64, device=dev)
        b.id = torch.arange(1, m + 1, dtype=torch.int64, device=dev)
        b.dt = torch.zeros_like(b.q_norm)
        b.remaining_steps = torch.zeros_like(b.id)
        b.xi_sorted()
        return b

    def particles(self, dxi: float) -> np.ndarray:
        """The same beam as a host particle_dtype3d array (for beam files)."""
        from .beam_generator import particle_dtype3d
        b = self.device_beam(dxi)
        out = np.zeros(b.xi.numel(), dtype=particle_dtype3d)
        for k in ('xi', 'x', 'y', 'px', 'py', 'pz', 'q_m', 'q_norm', 'id'):
            out[k] = getattr(b, k).cpu().numpy()
        return out


def bigaussian_beam(n=1_000_000, seed=2024, sigma_r=0.5, sigma_z=1.0, xi0=-3.0,
                    gamma=1000.0, espread=0.01, emittance=1e-2, peak=-0.5, dxi=0.02,
                    r_max=4.0) -> np.ndarray:
    """Seeded bi-Gaussian beam as a particle_dtype3d array, sorted by xi
    (descending), cut to xi in (2 xi0, 0) and r < r_max.  q_norm makes the
    deposited on-axis peak density equal `peak` (layer charge per cell area):
    rho = Q dxi / (sqrt(2 pi) sigma_z) / (2 pi sigma_r^2)."""
    from .beam_generator import particle_dtype3d
    rng = np.random.default_rng(seed)
    xi = rng.normal(xi0, sigma_z, 2 * n)
    xi = xi[(xi < 0) & (xi > 2 * xi0)][:n]
    m = xi.size
    r = sigma_r * np.sqrt(-2 * np.log(1 - rng.random(m) * (1 - np.exp(-r_max ** 2 / (2 * sigma_r ** 2)))))
    phi = rng.uniform(0, 2 * np.pi, m)
    b = np.zeros(m, dtype=particle_dtype3d)
    b['xi'] = xi
    b['x'], b['y'] = r * np.cos(phi), r * np.sin(phi)
    sp = emittance / sigma_r
    b['px'], b['py'] = rng.normal(0, sp, m), rng.normal(0, sp, m)
    b['pz'] = rng.normal(gamma, gamma * espread, m)
    b['q_m'] = -1.0
    q_total = peak * (np.sqrt(2 * np.pi) * sigma_z) * (2 * np.pi * sigma_r ** 2) / dxi
    b['q_norm'] = q_total / m
    b['id'] = np.arange(1, m + 1)
    return b[np.argsort(-b['xi'], kind='stable')]


# device bytes per beam macroparticle: the sorted source, the drain, the two
# fell-through buffers and the lost buffer (11 eight-byte fields each)
BEAM_BYTES_PER_PARTICLE = 5 * 11 * 8


def footprint_bytes(config: dict, driver=None) -> int:
    """Device memory one member needs (particles, fields, currents, solver
    workspaces), for admission decisions."""
    cfg = Config(config)
    cfg._adjust_config_values_3d()
    N = cfg.getint('window-width-steps')
    f = max(1, int(round(cfg.getfloat('plasma-fineness') or 1)))
    Ns = (N - 2 * cfg.getint('plasma-padding-steps')) * f
    sorts = 2 if cfg.get('ion-model') == 'mobile' else 1
    mixed = str(cfg.getraw('precision') or 'fp64').lower() == 'mixed'
    L = _lib.load()
    prec = _lib.LCB_PREC_MIXED if mixed else _lib.LCB_PREC_FP64
    particles = 2 * 9 * 8 * sorts * Ns * Ns
    planes = (4 * 7 + 2 * 4 * 2 + 4) * 8 * N * N
    beam = BEAM_BYTES_PER_PARTICLE * driver.n if isinstance(driver, BeamDriver) else 0
    return int(particles + planes + beam + L.lcb_compute_fields_workspace_bytes(N, prec)
               + L.lcb_field_operators_bytes(N, prec)
               + L.lcb_plasma_deposit_workspace_bytes(N, prec) + (8 << 20))


class Member:
    """One simulation whose xi step is a pair of captured CUDA graphs."""

    def __init__(self, config: dict, driver: GaussianDriver, device=None, name=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.config_dict = dict(config)
        cfg = Config({**config, 'cuda-graphs': False})
        cfg._adjust_config_values_3d()
        self.config = cfg
        self.name = name
        self.driver = driver
        self.N = cfg.getint('window-width-steps')
        self.h = cfg.getfloat('transverse-step')
        self.dxi = cfg.getfloat('xi-step')
        self.n_steps = round(cfg.getfloat('window-length') / self.dxi) + 1
        self.cells = self.N * self.N
        self.stream = torch.cuda.Stream(self.device)
        with torch.cuda.stream(self.stream):
            self.solver = Plane2d3vPlasmaSolver(cfg, self.device)
            self.solver.init_state(cfg.getfloat('time-step'))
            self.counter = torch.zeros(1, dtype=torch.int64, device=self.device)
            self.ez = torch.zeros(self.n_steps, dtype=torch.float64, device=self.device)
        self.graphs = [None, None]
        self.eager = 0
        self.done = 0
        self.marks = collections.deque()
        self.end_event = None
        self.t_admit = self.t_done = None

    @property
    def finished(self) -> bool:
        return self.done >= self.n_steps

    def _ops(self):
        L = _lib.load()
        ps = self.solver
        st = _lib.stream_handle()
        d = self.driver
        _lib.check(L.lcb_rigid_gaussian(self.N, self.h, self.dxi, d.amplitude, d.sigma_r,
                                        d.xi_len, 0, self.counter.data_ptr(),
                                        ps.rbf.data_ptr(), ps.rbp.data_ptr(), st),
                   "lcb_rigid_gaussian")
        ps._step_ops(ps.rbf, ps.rbp, 1.0, advance=False)
        new = ps.fields[1 - ps.cur]
        _lib.check(L.lcb_record_axis(new.Ez.data_ptr(), self.N, self.counter.data_ptr(),
                                     self.ez.data_ptr(), self.n_steps, st), "lcb_record_axis")

    MARK_EVERY = 16
    MAX_AHEAD = 4

    def step(self):
        """Issue one xi step on the member's stream (asynchronous).  The host
        stays at most MARK_EVERY * MAX_AHEAD steps ahead of the device."""
        ps = self.solver
        p = ps.cur
        if len(self.marks) >= self.MAX_AHEAD:
            self.marks.popleft().synchronize()
        with torch.cuda.stream(self.stream):
            if self.eager < 2:
                self._ops()
                self.eager += 1
            else:
                if self.graphs[p] is None:
                    # capture on the member's own stream without the
                    # device-wide synchronisation torch.cuda.graph performs,
                    # so other members keep running meanwhile
                    g = torch.cuda.CUDAGraph()
                    n0 = _lib.load().lcb_launch_count()
                    g.capture_begin(capture_error_mode="thread_local")
                    try:
                        self._ops()
                    finally:
                        g.capture_end()
                    self.graphs[p] = (g, _lib.load().lcb_launch_count() - n0)
                g, nl = self.graphs[p]
                g.replay()
                _lib.add_replayed(nl)
            self.done += 1
            if self.done % self.MARK_EVERY == 0 or self.done >= self.n_steps:
                ev = torch.cuda.Event()
                ev.record(self.stream)
                self.marks.append(ev)
                if self.done >= self.n_steps:
                    self.end_event = ev
        ps.cur = 1 - p
        ps.last_fields = ps.fields[p]

    def complete(self) -> bool:
        """All steps issued and executed."""
        return self.end_event is not None and self.end_event.query()

    def check(self):
        """Raise if a kernel of this member set a bit of a device error word."""
        self.stream.synchronize()
        self.solver.check_errors()

    def result(self):
        """On-axis Ez per xi step and the final fields (host arrays); raises if
        a kernel set a bit of the device error word."""
        self.check()
        return {"ez": self.ez.cpu().numpy(),
                "fields": self.solver.prev_fields.buf.cpu().numpy()}

    def checkpoint(self, directory) -> str:
        """Write this member's state between xi steps: ``<name>.plasma.npz``
        (a plasma state file: the last computed layer's particles, fields,
        currents and background charge, with its xi) and ``<name>.slot.npz``
        (config, driver, steps done, on-axis Ez so far, driver-specific
        state).  Waits for the member's stream; raises if a device error word
        is set.  Returns the common path prefix for ``restore_member``."""
        from .plasma_state import save_plasmastate
        self.check()
        os.makedirs(directory, exist_ok=True)
        base = os.path.join(directory, str(self.name if self.name is not None else "member"))
        ps = self.solver
        # each file is written under a temporary name and renamed, so that an
        # interrupted checkpoint leaves the previous files, not truncated ones
        save_plasmastate(base + ".plasma.tmp.npz", ps.particles_dict(), ps.prev_fields.arrays(),
                         ps.prev_currents.arrays(), ro_initial=ps.ro_initial,
                         xi_plasma_layer=-self.dxi * (self.done - 1))
        meta = {"format": np.array(SLOT_FORMAT), "name": np.array(str(self.name)),
                "config": np.array(json.dumps(self.config_dict)),
                "driver": np.array(driver_record(self.driver)),
                "done": np.array(self.done),
                "ez": self.ez[:self.done].cpu().numpy(),
                "arrival": np.array(float(getattr(self, "t_arrival", 0.0) or 0.0))}
        meta.update(self._slot_state())
        np.savez(base + ".slot.tmp.npz", **meta)
        os.replace(base + ".plasma.tmp.npz", base + ".plasma.npz")
        os.replace(base + ".slot.tmp.npz", base + ".slot.npz")
        return base

    def _slot_state(self) -> dict:
        return {}

    def _restore_slot_state(self, meta: dict):
        pass

    def release(self):
        self.graphs = [None, None]
        self.solver = None
        self.marks.clear()


class BeamMember(Member):
    """One simulation with a non-rigid driver.  Its plasma step is the
    solver's captured graph (one per buffer parity); the beam layer step
    (push of layer i - 1 between the previous and the new fields, layout of
    layer i + 1, all on the device) and the on-axis Ez record are launched
    around it on the member's stream."""

    def __init__(self, config: dict, driver: BeamDriver, device=None, name=None):
        from .beam3d import BeamCalculator, BeamSource
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.config_dict = dict(config)
        cfg = Config(config)
        cfg._adjust_config_values_3d()
        self.config = cfg
        self.name = name
        self.driver = driver
        self.N = cfg.getint('window-width-steps')
        self.dxi = cfg.getfloat('xi-step')
        self.n_steps = round(cfg.getfloat('window-length') / self.dxi) + 1
        self.cells = self.N * self.N
        self.stream = torch.cuda.Stream(self.device)
        with torch.cuda.stream(self.stream):
            self.solver = Plane2d3vPlasmaSolver(cfg, self.device)
            self.solver.init_state(cfg.getfloat('time-step'))
            self.solver.capture_on_stream = True
            self.bc = BeamCalculator(cfg, self.device)
            self.source = BeamSource(cfg, driver.device_beam(self.dxi, self.device), self.device)
            self.bc.start_time_step(self.source)
            self.bc.layout_first(0)
            self.counter = torch.zeros(1, dtype=torch.int64, device=self.device)
            self.ez = torch.zeros(self.n_steps, dtype=torch.float64, device=self.device)
        self.done = 0
        self.marks = collections.deque()
        self.end_event = None
        self.t_admit = None

    def step(self):
        if len(self.marks) >= self.MAX_AHEAD:
            self.marks.popleft().synchronize()
        ps, bc, i = self.solver, self.bc, self.done
        L = _lib.load()
        with torch.cuda.stream(self.stream):
            rb_full, rb_prev = bc.rho(i)
            ps.step_dxi(rb_full, rb_prev, bc.rho_divisor, stable_planes=True)
            bc.after_plasma_step(i, ps.last_fields, ps.prev_fields)
            _lib.check(L.lcb_record_axis(ps.prev_fields.Ez.data_ptr(), self.N,
                                         self.counter.data_ptr(), self.ez.data_ptr(),
                                         self.n_steps, _lib.stream_handle()), "lcb_record_axis")
            self.done += 1
            if self.done % self.MARK_EVERY == 0 or self.done >= self.n_steps:
                ev = torch.cuda.Event()
                ev.record(self.stream)
                self.marks.append(ev)
                if self.done >= self.n_steps:
                    self.end_event = ev

    def check(self):
        super().check()
        e = int(self.bc.err.item())
        if e:
            raise RuntimeError(f"beam device error word 0x{e:x} in member {self.name}")

    def _beam_buffers(self):
        bc = self.bc
        return (("drain", bc.drain, 2), ("lost", bc.lost, 3), ("fell0", bc.fell[0], 0),
                ("fell1", bc.fell[1], 1))

    def _slot_state(self) -> dict:
        """The beam step's state between xi steps: the three density planes
        (layouts in progress), the device counters, the fell-buffer parity
        and the filled part of the drain, lost and fell buffers.  The source
        beam is regenerated from the driver's seed."""
        bc = self.bc
        counts = bc.counts.cpu().numpy()
        out = {"beam_planes": bc.planes.cpu().numpy(), "beam_counts": counts,
               "beam_fell_cur": np.array(bc.fell_cur)}
        for tag, buf, c in self._beam_buffers():
            for k in buf._all():
                out[f"beam_{tag}_{k}"] = getattr(buf, k)[:int(counts[c])].cpu().numpy()
        return out

    def _restore_slot_state(self, meta: dict):
        bc = self.bc
        bc.planes.copy_(torch.from_numpy(meta["beam_planes"]))
        bc.counts.copy_(torch.from_numpy(meta["beam_counts"]))
        bc.fell_cur = int(meta["beam_fell_cur"])
        for tag, buf, _ in self._beam_buffers():
            for k in buf._all():
                a = torch.from_numpy(meta[f"beam_{tag}_{k}"])
                getattr(buf, k)[:a.numel()].copy_(a)

    def release(self):
        self.solver = None
        self.bc = None
        self.source = None
        self.marks.clear()


def make_member(config: dict, driver, device=None, name=None) -> Member:
    """A Member for a rigid Gaussian driver, a BeamMember for a beam."""
    if isinstance(driver, BeamDriver):
        return BeamMember(config, driver, device, name)
    return Member(config, driver, device, name)


SLOT_FORMAT = 1


def driver_record(driver) -> str:
    """A driver as JSON (kind and parameters)."""
    kind = "beam" if isinstance(driver, BeamDriver) else "rigid"
    return json.dumps({"kind": kind, **dataclasses.asdict(driver)})


def driver_from_record(record: str):
    d = json.loads(record)
    kind = d.pop("kind")
    if kind == "beam":
        return BeamDriver(**d)
    if kind == "rigid":
        return GaussianDriver(**d)
    raise ValueError(f"unknown driver kind {kind!r}")


def restore_member(base: str, device=None) -> Member:
    """Rebuild a member from ``Member.checkpoint``'s files (``base`` is the
    path prefix it returned) and put it where it stopped: the next step is
    the one after the stored layer."""
    from .plasma_state import load_plasmastate
    with np.load(base + ".slot.npz") as z:
        meta = {k: z[k] for k in z.files}
    if int(meta["format"]) != SLOT_FORMAT:
        raise ValueError(f"{base}.slot.npz: slot format {int(meta['format'])}, "
                         f"expected {SLOT_FORMAT}")
    config = json.loads(str(meta["config"]))
    driver = driver_from_record(str(meta["driver"]))
    m = make_member(config, driver, device, name=str(meta["name"]))
    state = load_plasmastate(base + ".plasma.npz", m.solver.sort_names)
    done = int(meta["done"])
    xi = state["xi_plasma_layer"]
    if xi is None or abs(xi + m.dxi * (done - 1)) > 1e-9 * max(1.0, abs(xi)):
        raise ValueError(f"{base}: the plasma state (xi {xi}) is not the layer of the "
                         f"slot file ({done} steps done)")
    with torch.cuda.stream(m.stream):
        m.solver.load_state(state)
        m.counter.fill_(done)
        if done:
            m.ez[:done].copy_(torch.from_numpy(meta["ez"]))
        m._restore_slot_state(meta)
    m.stream.synchronize()
    m.done = done
    m.t_arrival = float(meta["arrival"])
    return m


def solo_ez(config: dict, driver, **overrides) -> np.ndarray:
    """On-axis Ez of the same simulation run alone through the drop-in
    Simulation API (one time step), with config keys overridden."""
    import os
    import tempfile
    from .simulation import Simulation
    c = {**config, **overrides}
    if isinstance(driver, BeamDriver):
        c['rigid-beam'] = False
        c.setdefault('time-limit', 1.0)
        c['time-step'] = c.get('time-step', 1.0)
        sim = Simulation(config=c, runas_filename='')
        arr = driver.particles(float(c['xi-step']))
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, 'beam.npz')
            np.savez(path, **{k: arr[k] for k in arr.dtype.names})
            sim.load_beamfile(path)
        sim.step(1)
    else:
        sim = Simulation(config=c, beam_parameters=driver, runas_filename='')
        sim.step()
    return sim.push_solver.ez_axis.cpu().numpy()


class BatchRunner:
    """Advance a fixed set of members together, one xi step at a time.

    With ``single_graph`` (rigid-driver members of one length, advancing in
    lockstep) every batched xi step after the members' two eager steps is ONE
    graph launch: the members' steps are captured together, each on its own
    stream forked from and joined back into the capturing stream, once per
    buffer parity; otherwise each member replays its own graph on its
    stream."""

    MARK_EVERY = 16
    MAX_AHEAD = 4

    def __init__(self, members, single_graph=False):
        self.members = list(members)
        self.single_graph = single_graph and len(self.members) > 0 and all(
            type(m) is Member for m in self.members) and len(
            {m.n_steps for m in self.members}) == 1
        self.graphs = [None, None]
        self.stream = torch.cuda.Stream(self.members[0].device) if self.single_graph else None
        self.marks = collections.deque()
        self.launches = 0

    def _capture(self):
        """One graph holding every member's xi step for the current parity."""
        g = torch.cuda.CUDAGraph()
        n0 = _lib.load().lcb_launch_count()
        with torch.cuda.stream(self.stream):
            g.capture_begin(capture_error_mode="thread_local")
            try:
                fork = torch.cuda.Event()
                fork.record(self.stream)
                for m in self.members:
                    m.stream.wait_event(fork)
                    with torch.cuda.stream(m.stream):
                        m._ops()
                    join = torch.cuda.Event()
                    join.record(m.stream)
                    self.stream.wait_event(join)
            finally:
                g.capture_end()
        return g, _lib.load().lcb_launch_count() - n0

    def step(self):
        if not self.single_graph or any(m.eager < 2 for m in self.members):
            for m in self.members:
                if not m.finished:
                    m.step()
            return
        if self.members[0].finished:
            return
        p = self.members[0].solver.cur
        if len(self.marks) >= self.MAX_AHEAD:
            self.marks.popleft().synchronize()
        if self.graphs[p] is None:
            # the members' streams have work queued from their eager steps
            for m in self.members:
                self.stream.wait_stream(m.stream)
            self.graphs[p] = self._capture()
        g, nl = self.graphs[p]
        # members' earlier work (eager steps) precedes the batch graph
        for m in self.members:
            self.stream.wait_stream(m.stream)
        with torch.cuda.stream(self.stream):
            g.replay()
        _lib.add_replayed(nl)
        for m in self.members:
            ps = m.solver
            m.done += 1
            ps.cur = 1 - p
            ps.last_fields = ps.fields[p]
            if m.done >= m.n_steps:
                ev = torch.cuda.Event()
                ev.record(self.stream)
                m.end_event = ev
        if self.members[0].done % self.MARK_EVERY == 0:
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self.marks.append(ev)

    def join(self):
        """Make the members' streams wait for the batch graphs (before reading
        results on a member's stream)."""
        if self.single_graph:
            for m in self.members:
                m.stream.wait_stream(self.stream)

    def run(self, steps=None):
        n = steps if steps is not None else max(m.n_steps for m in self.members)
        for _ in range(n):
            self.step()
        self.join()
        torch.cuda.synchronize()

    @property
    def cell_steps_per_step(self):
        return sum(m.cells for m in self.members if not m.finished)


def request_stream(n=500, rate=20.0, seed=4321, dxi=0.05, h=0.05, sizes=(129, 257, 513),
                   min_steps=200, max_steps=2000, precision="mixed", beam_fraction=0.5,
                   beam_particles=(100_000, 1_000_000)):
    """The served stream: n requests with Poisson arrivals of the given mean
    rate (exponential gaps), grid drawn from sizes, xi length uniform in
    [min_steps, max_steps] steps of dxi, and a driver with amplitude ~
    U[0.01, 0.5] and sigma_r ~ U[0.5, 2]: with probability beam_fraction a
    non-rigid bi-Gaussian beam of U[beam_particles] macroparticles, else a
    rigid Gaussian; all drawn from numpy.random.default_rng(seed).  Returns
    (arrival, id, config, driver)."""
    widths = {129: 3.25, 257: 6.45, 513: 12.85}
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(n):
        t += float(rng.exponential(1.0 / rate))
        N = int(sizes[rng.integers(len(sizes))])
        steps = int(rng.integers(min_steps, max_steps + 1))
        amp, sig = float(rng.uniform(0.01, 0.5)), float(rng.uniform(0.5, 2.0))
        width = widths.get(N, N * h / 2)
        if rng.random() < beam_fraction:
            # radial cut at 4 sigma_r, or at 80% of the window's half width
            drv = BeamDriver(n=int(rng.integers(beam_particles[0], beam_particles[1] + 1)),
                             amplitude=amp, sigma_r=sig, seed=seed * 1000 + r,
                             r_max=min(4 * sig, 0.4 * width))
        else:
            drv = GaussianDriver(amplitude=amp, sigma_r=sig)
        cfg = {'geometry': '3d', 'window-width': width, 'transverse-step': h,
               'window-length': (steps - 1) * dxi, 'xi-step': dxi,
               'ion-model': 'background', 'plasma-particles-per-cell': 4,
               'rigid-beam': not isinstance(drv, BeamDriver), 'print-every': 0,
               'precision': precision, 'time-step': 1.0}
        out.append((t, f"req{r:04d}", cfg, drv))
    return out


def scan_members(n=64, seed=1234, n_steps=1000, precision="mixed", dxi=0.05, h=0.05,
                 sizes=(129, 257, 513), device=None):
    """The batched parameter scan: member m has grid sizes[m % 3] at step h,
    2 x 2 particles per cell, background ions, xi step dxi for n_steps steps,
    and a rigid Gaussian driver with amplitude ~ U[0.01, 0.5] and sigma_r ~
    U[0.5, 2] drawn from numpy.random.default_rng(seed + m)."""
    widths = {129: 3.25, 257: 6.45, 513: 12.85}
    out = []
    for m in range(n):
        rng = np.random.default_rng(seed + m)
        N = sizes[m % len(sizes)]
        drv = GaussianDriver(amplitude=float(rng.uniform(0.01, 0.5)),
                             sigma_r=float(rng.uniform(0.5, 2.0)))
        cfg = {'geometry': '3d', 'window-width': widths.get(N, N * h / 2), 'transverse-step': h,
               'window-length': (n_steps - 1) * dxi, 'xi-step': dxi,
               'ion-model': 'background', 'plasma-particles-per-cell': 4,
               'rigid-beam': True, 'print-every': 0, 'precision': precision,
               'time-step': 1.0}
        out.append((cfg, drv))
    return out


class Server:
    """Continuous batching of simulation requests on one GPU.

    Requests arrive over time; ``poll`` admits waiting requests (in arrival
    order) into free slots when their HBM footprint fits the budget, every
    ``tick`` advances each running request by one xi step (one graph launch on
    its own stream), and ``retire`` collects requests whose last step has
    executed, releasing their memory so that waiting ones are admitted while
    others are still running.  Latency is measured from a request's arrival
    to the moment its completion is observed.

    A request that cannot be set up (an invalid config, no device memory),
    whose launches fail, or whose kernels set a bit of a device error word is
    finished with ``done[id]["error"]`` (the exception text) and its memory is
    released; the other requests carry on."""

    def __init__(self, hbm_budget_bytes: int, max_slots: int = 64, device=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = hbm_budget_bytes
        self.max_slots = max_slots
        self.waiting = collections.deque()   # (arrival, request_id, config, driver)
        self.running = []                    # (request_id, Member, footprint)
        self.draining = []                   # all steps issued, not yet complete
        self.done = {}
        self.used = 0
        self.t0 = time.perf_counter()

    def now(self):
        return time.perf_counter() - self.t0

    def submit(self, request_id, config, driver, arrival=None):
        item = (self.now() if arrival is None else arrival, request_id, config, driver)
        if self.waiting and item[0] < self.waiting[-1][0]:
            w = sorted([*self.waiting, item], key=lambda r: r[0])
            self.waiting = collections.deque(w)
        else:
            self.waiting.append(item)

    def _fail(self, rid, arrival, admitted, err: Exception):
        t = self.now()
        self.done[rid] = {"error": f"{type(err).__name__}: {err}", "ez": None,
                          "latency": t - arrival, "arrival": arrival, "admitted": admitted,
                          "finished": t}

    def _drop(self, m, err: Exception):
        self._fail(m.name, m.t_arrival, m.t_admit, err)
        # work queued earlier on the member's stream may still read or write
        # its buffers: wait for it before they go back to the allocator (a
        # stream in an error state raises again; its work is over then)
        try:
            m.stream.synchronize()
        except Exception:
            pass
        try:
            m.release()
        finally:
            self.used -= m.footprint

    def poll(self):
        """Admit arrived requests, first come first served, while a slot is
        free and the footprint fits; a request that does not fit waits (and so
        do the ones behind it, so large requests are not starved)."""
        t = self.now()
        while self.waiting:
            arr, rid, cfg, drv = self.waiting[0]
            if arr > t or len(self.running) + len(self.draining) >= self.max_slots:
                break
            try:
                fp = footprint_bytes(cfg, drv)
            except Exception as e:      # an invalid config
                self.waiting.popleft()
                self._fail(rid, arr, None, e)
                continue
            if self.used + fp > self.budget and (self.running or self.draining):
                break
            self.waiting.popleft()
            try:
                m = make_member(cfg, drv, self.device, name=rid)
            except Exception as e:      # set-up failed (config, device memory)
                self._fail(rid, arr, t, e)
                continue
            m.t_arrival = arr
            m.t_admit = t
            m.footprint = fp
            self.running.append(m)
            self.used += fp

    def tick(self):
        """One xi step for every running request."""
        keep = []
        for m in self.running:
            try:
                m.step()
            except Exception as e:      # a launch failed
                self._drop(m, e)
                continue
            (self.draining if m.finished else keep).append(m)
        self.running = keep

    def retire(self):
        keep = []
        for m in self.draining:
            if m.complete():
                t = self.now()
                try:
                    m.check()
                except Exception as e:  # a device error word was set
                    self._drop(m, e)
                    continue
                self.done[m.name] = {"ez": m.ez.cpu().numpy(), "latency": t - m.t_arrival,
                                     "arrival": m.t_arrival, "admitted": m.t_admit,
                                     "finished": t, "cells": m.cells, "steps": m.n_steps}
                m.release()
                self.used -= m.footprint
            else:
                keep.append(m)
        self.draining = keep

    def idle(self):
        return not self.running and not self.draining and not self.waiting

    def checkpoint(self, directory):
        """Write the server's requests to ``directory``: requests whose steps
        are all issued are finished first (their results stay in ``done``),
        every running request's slot is written (``Member.checkpoint``) and
        the waiting queue goes to ``server.json`` with the arrival times
        relative to now.  The server itself is left as it was."""
        for m in list(self.draining):
            m.end_event.synchronize()
        self.retire()
        os.makedirs(directory, exist_ok=True)
        t = self.now()
        running = []
        for m in self.running:
            base = m.checkpoint(directory)
            running.append({"base": os.path.basename(base), "arrival": m.t_arrival - t})
        waiting = [{"id": rid, "config": cfg, "driver": driver_record(drv),
                    "arrival": arr - t} for arr, rid, cfg, drv in self.waiting]
        path = os.path.join(directory, "server.json")
        with open(path + ".tmp", "w") as f:
            json.dump({"format": SLOT_FORMAT, "running": running, "waiting": waiting}, f)
        os.replace(path + ".tmp", path)

    @classmethod
    def restore(cls, directory, hbm_budget_bytes: int, max_slots: int = 64, device=None):
        """A server holding ``checkpoint``'s requests: the running ones
        admitted at once (in their stored state), the waiting ones queued
        with their arrival times relative to the restore."""
        srv = cls(hbm_budget_bytes, max_slots, device)
        with open(os.path.join(directory, "server.json")) as f:
            meta = json.load(f)
        if meta.get("format") != SLOT_FORMAT:
            raise ValueError(f"{directory}/server.json: format {meta.get('format')}, "
                             f"expected {SLOT_FORMAT}")
        for r in meta["running"]:
            m = restore_member(os.path.join(directory, r["base"]), srv.device)
            m.t_arrival = r["arrival"]
            m.t_admit = 0.0
            m.footprint = footprint_bytes(m.config_dict, m.driver)
            srv.running.append(m)
            srv.used += m.footprint
        for w in meta["waiting"]:
            srv.submit(w["id"], w["config"], driver_from_record(w["driver"]),
                       arrival=max(0.0, w["arrival"]))
        return srv

    def run(self):
        """Serve until every submitted request is done."""
        while not self.idle():
            self.poll()
            if self.running:
                self.tick()
            elif self.draining:
                self.draining[0].end_event.synchronize()
            elif self.waiting:
                time.sleep(max(0.0, min(self.waiting[0][0] - self.now(), 0.01)))
            self.retire()
