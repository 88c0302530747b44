#!/usr/bin/env python
"""Benchmark: xi-steps x cells per second of the quasistatic 3D xi loop.

Workload (the production FP64 drop-in configuration): 513 x 513 grid
(window-width 5.13, transverse-step 0.02), 2 x 2 plasma macroparticles per
cell (929,296 electrons, background ions), xi-step 0.02, window-length 60
(3001 xi iterations), and a non-rigid seeded bi-Gaussian electron driver of
1,000,000 macroparticles (sigma_r 0.5, sigma_z 1, peak n_b/n0 = 0.5,
gamma = 1000 +- 1 %, normalised emittance 1e-2), pushed every xi layer.

One bench step = one xi step (plasma predictor-corrector + beam layout and
push) of that workload; the xi loop of one time step runs once, the first
--warmup xi steps untimed and the next --steps timed with CUDA events.  All
inputs live in HBM and exceed L2 (plasma state 134 MB, beam 88 MB), so no
extra L2 flush is done.  With --gpus N (torchrun) every rank runs its own
replica (the xi loop does not shard): weak scaling.

The default line also carries the many-simulation forms (at one GPU):
"batched" -- the 64-member scan in mixed precision against the same members
run one by one through the plain FP64 drop-in path -- and "served" -- the
request stream in mixed precision against the same requests run one by one,
first come first served, through the plain FP64 path (each timed for real).

--impl reference times the CPU restatement of the reference algorithm
(oracle/: the reference's Python package cannot travel with this tree) on
the host cores, on a bounded sample of the same xi loop.
"""
from __future__ import annotations

import argparse
import contextlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

# many member streams run concurrently in the batch and serve workloads
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "lcode3d-production-fp64: N=513 h=0.02 ppc=4 dxi=0.02 L=60 beam=1e6 bi-gaussian"
METRIC = "xi-steps*cells/s"


def workload_config(precision="fp64", window_length=60.0):
    return {'geometry': '3d', 'processing-unit-type': 'gpu',
            'window-width': 5.13, 'transverse-step': 0.02,
            'window-length': window_length, 'xi-step': 0.02,
            'time-limit': 1.0, 'time-step': 1.0,
            'ion-model': 'background', 'plasma-particles-per-cell': 4,
            'rigid-beam': False, 'print-every': 0, 'precision': precision}


def make_beam(n=1_000_000, seed=2024, sigma_r=0.5, sigma_z=1.0, xi0=-3.0,
              gamma=1000.0, espread=0.01, emittance=1e-2, peak=-0.5, dxi=0.02,
              r_max=4.0):
    """The workload's seeded bi-Gaussian driver (a particle_dtype3d array)."""
    from lcodepy_b200.batch import bigaussian_beam
    return bigaussian_beam(n, seed, sigma_r, sigma_z, xi0, gamma, espread, emittance, peak,
                           dxi, r_max)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [ln.split(",") for ln in open(self.f.name).read().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64,
                     device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_gpu(args, ws, rank, local):
    import torch
    from lcodepy_b200 import Simulation, _lib
    from lcodepy_b200.beam3d import BeamParticles, BeamSource, BeamDrain

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfg = workload_config(args.precision, args.window_length)
    beam_host = make_beam()
    sim = Simulation(config=cfg, beam_parameters={}, runas_filename='')
    ps = sim.push_solver
    conf = sim.effective_config
    N = conf.getint('window-width-steps')
    n_iter = ps.xi_steps + 1
    W, K = args.warmup, args.steps
    if W + K > n_iter:
        raise SystemExit(f"--warmup + --steps must be <= {n_iter} xi steps")

    # ---- device-resident timed run: one xi loop, events at W and W+K ----
    source = BeamSource(conf, BeamParticles(dev).init_generated(beam_host), dev)
    drain = BeamDrain(conf, dev)
    ps.plasma_solver.init_state(1.0)
    torch.cuda.synchronize()
    ev = {}
    op_times = {}
    op_marks = []     # (xi step, per-op launch counts before it): --op-timeline

    def hook(k):
        if k == W:
            barrier(ws)
            torch.cuda.synchronize()
            ev["clock"] = ClockSampler(local) if rank == 0 else None
            ev["l0"] = _lib.launch_count()
            ev["t0"] = torch.cuda.Event(enable_timing=True)
            ev["t0"].record()
        if W <= k < W + K:
            # every 16th timed step runs eagerly with per-op CUDA events (the
            # kernels are the same; the others replay the captured graphs)
            every = args.op_every
            ps.plasma_solver.op_timers = op_times if (k - W) % every == 0 else None
            if (k - W) % every == 0:
                op_marks.append((k, {n: len(v) for n, v in op_times.items()}))
        if k == W + K:
            ev["t1"] = torch.cuda.Event(enable_timing=True)
            ev["t1"].record()
            ps.plasma_solver.op_timers = None
            torch.cuda.synchronize()
            ev["l1"] = _lib.launch_count()
            ev["clocks"] = ev["clock"].stop() if ev.get("clock") else None

    ps.step_dt(conf.getfloat('xi-step'), source, drain, 1.0, [], step_hook=hook)
    if "t1" not in ev:
        hook(W + K)
    torch.cuda.synchronize()
    ms_total = ev["t0"].elapsed_time(ev["t1"])
    ms_total = max_over_ranks(ms_total, ws)
    barrier(ws)
    ms_per_step = ms_total / K
    cells = N * N
    value = ws * K * cells / (ms_total / 1e3)

    # ---- per-op device time over the timed region (CUDA events) ----
    ops = {}
    for name, evs in op_times.items():
        tot = sum(a.elapsed_time(b) for a, b in evs)
        ops[name] = {"launches": len(evs), "ms_total": tot, "ms_avg": tot / max(len(evs), 1)}
    if args.op_timeline and rank == 0:
        # per eagerly timed xi step: each op's launches, in microseconds
        line = {}
        ends = op_marks[1:] + [(None, {n: len(v) for n, v in op_times.items()})]
        for (k, a), (_, b) in zip(op_marks, ends):
            line[k] = {n: [round(e0.elapsed_time(e1) * 1e3, 1)
                           for e0, e1 in op_times[n][a.get(n, 0):b.get(n, 0)]]
                       for n in op_times}
        with open(args.op_timeline, "w") as f:
            json.dump(line, f)

    # ---- end to end through the public API, host buffers in and out ----
    e2e = None if args.no_e2e else run_e2e(cfg, beam_host, dev)

    Ns = ps.plasma_solver.states[0].Ns
    n_particles = Ns * Ns * (2 if conf.get('ion-model') == 'mobile' else 1)
    del source, drain, sim, ps
    return dict(value=value, ms_per_step=ms_per_step, N=N, ops=ops, n_particles=n_particles,
                launches=int(ev["l1"] - ev["l0"]), clocks=ev.get("clocks"),
                e2e=e2e, n_iter=n_iter)


def rigid_driver(xp, xi, x, y):
    """rho_b = 0.1 exp(-r^2/2) (1 + cos(sqrt(pi/2) xi))/2 on -sqrt(2 pi) <= xi <= 0."""
    if -np.sqrt(2 * np.pi) <= xi <= 0:
        return 0.1 * xp.exp(-(x ** 2 + y ** 2) / 2) * (1 + np.cos(np.sqrt(np.pi / 2) * xi)) / 2
    return xp.zeros_like(x)


def run_rigid129(args, ws, rank, local):
    """The CPU-runnable plain configuration: 129 x 129 (window-width 6.5, step
    0.1), 2 x 2 per cell, background ions, xi-step 0.1, 201 xi iterations,
    rigid Gaussian driver; --precision picks FP64 or the mixed form."""
    import torch
    from lcodepy_b200 import Simulation
    from lcodepy_b200.beam3d import RigidBeamSource
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfg = {'geometry': '3d', 'processing-unit-type': 'gpu', 'window-width': 6.5,
           'transverse-step': 0.1, 'window-length': 20.0, 'xi-step': 0.1,
           'ion-model': 'background', 'plasma-particles-per-cell': 4, 'rigid-beam': True,
           'print-every': 0, 'precision': args.precision}
    times = []
    for rep in range(args.warmup + args.steps):
        sim = Simulation(config={**cfg, 'time-step-pipeline': False},
                         beam_parameters=rigid_driver, runas_filename='')
        ps = sim.push_solver
        ev = {}

        def hook(k, ps=ps, ev=ev):
            if k == 0:
                torch.cuda.synchronize()
                ev["t0"] = torch.cuda.Event(enable_timing=True)
                ev["t0"].record()
            if k == ps.xi_steps + 1:
                ev["t1"] = torch.cuda.Event(enable_timing=True)
                ev["t1"].record()
        ps.plasma_solver.init_state(1.0)
        ps.step_dt(0.1, RigidBeamSource(None, rigid_driver), None, 1.0, [], step_hook=hook)
        torch.cuda.synchronize()
        if rep >= args.warmup:
            times.append(ev["t0"].elapsed_time(ev["t1"]))
    N = sim.effective_config.getint('window-width-steps')
    n_iter = ps.xi_steps + 1
    ms = float(np.median(times))
    return {"value": ws * n_iter * N * N / (ms / 1e3), "ms_per_step": ms / n_iter, "N": N,
            "n_iter": n_iter}


def run_batch(args, ws, rank, local):
    """The batched parameter scan: 64 simulations (grids 129, 257, 513 at step
    0.05, 2 x 2 per cell, rigid Gaussian drivers with seeded amplitudes and
    widths), advanced together in mixed precision: a bench step is one graph
    launch that advances every member by one xi step (the members' steps are
    captured together, each on its own stream).  The same members
    are then run one after another through the plain FP64 drop-in path
    (Simulation with its default settings) for the plain-path comparison and
    the on-axis Ez error."""
    import torch
    from lcodepy_b200 import Simulation
    from lcodepy_b200.batch import BatchRunner, make_member, scan_members
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W, K = args.warmup, args.steps
    specs = scan_members(n=args.members, n_steps=max(W, 4) + K, precision=args.precision)
    members = [make_member(c, d, dev) for c, d in specs]
    runner = BatchRunner(members, single_graph=True)
    # two eager steps, then one capture per buffer parity: all before timing
    for _ in range(max(W, 4)):
        runner.step()
    torch.cuda.synchronize()
    barrier(ws)
    clock = ClockSampler(local) if rank == 0 else None
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    # all member streams join the current stream around the timed region
    from lcodepy_b200 import _lib
    n0 = _lib.launch_count()
    cur = torch.cuda.current_stream()
    t0.record(cur)
    for m in members:
        m.stream.wait_stream(cur)
    if runner.stream is not None:
        runner.stream.wait_stream(cur)
    for _ in range(K):
        runner.step()
    for m in members:
        cur.wait_stream(m.stream)
    if runner.stream is not None:
        cur.wait_stream(runner.stream)
    t1.record(cur)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - n0
    clocks = clock.stop() if clock else None
    ms = max_over_ranks(t0.elapsed_time(t1), ws)
    cells = sum(m.cells for m in members)
    value = ws * cells * K / (ms / 1e3)
    runner.join()
    ez_batch = [m.result()["ez"] for m in members]
    for m in members:
        m.release()
    del members, runner
    torch.cuda.empty_cache()

    # plain FP64: each member alone through the drop-in path with its default
    # settings (captured graphs, fused particle stage): the fastest FP64 form
    plain_ms, errs = 0.0, []
    for (cfg, drv), ezb in zip(specs, ez_batch):
        c = {**cfg, 'precision': 'fp64'}
        sim = Simulation(config=c, beam_parameters=drv, runas_filename='')
        ps = sim.push_solver
        ev = {}

        def hook(k, ev=ev):
            if k == W:
                ev["a"] = torch.cuda.Event(enable_timing=True)
                ev["a"].record()
            if k == W + K:
                ev["b"] = torch.cuda.Event(enable_timing=True)
                ev["b"].record()
        ps.plasma_solver.init_state(1.0)
        from lcodepy_b200.beam3d import RigidBeamSource
        ps.step_dt(cfg['xi-step'], RigidBeamSource(None, drv), None, 1.0, [], step_hook=hook)
        torch.cuda.synchronize()
        plain_ms += ev["a"].elapsed_time(ev["b"])
        ez64 = ps.ez_axis.cpu().numpy()
        errs.append(float(np.linalg.norm(ezb - ez64) / max(np.linalg.norm(ez64), 1e-300)))
        del sim, ps
    plain = cells * K / (plain_ms / 1e3)
    return {"value": value, "ms_per_step": ms / K, "plain": plain, "ratio": value / plain,
            "ez_err_max": max(errs), "ez_err_median": float(np.median(errs)),
            "clocks": clocks, "cells": cells, "members": len(specs), "launches": launches}


def run_plain_requests(reqs, dev, extra=None):
    """Run each (arrival, id, config, driver) request alone through the
    drop-in Simulation API in FP64 (config keys in `extra` added); returns
    {id: {seconds, ez}}, or {id: {seconds, error}} for a request whose run
    raised (a device error word: a runaway plasma particle).  A beam
    driver's particle file is written before its clock starts (the served
    path generates beams on the device in milliseconds)."""
    import torch
    from lcodepy_b200 import Simulation
    from lcodepy_b200.batch import BeamDriver
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for arr, rid, cfg, drv in reqs:
            c = {**cfg, 'precision': 'fp64', 'time-step-pipeline': False, **(extra or {})}
            path = None
            if isinstance(drv, BeamDriver):
                c['rigid-beam'] = False
                c.setdefault('time-limit', 1.0)
                beam = drv.particles(float(c['xi-step']))
                path = os.path.join(td, "beam.npz")
                np.savez(path, **{k: beam[k] for k in beam.dtype.names})
                del beam
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sim = None
            try:
                with contextlib.redirect_stdout(sys.stderr):   # Simulation's progress notes
                    if path is None:
                        sim = Simulation(config=c, beam_parameters=drv, runas_filename='')
                        sim.step()
                    else:
                        sim = Simulation(config=c, runas_filename='')
                        sim.load_beamfile(path)
                        sim.step(1)
                ez = sim.push_solver.ez_axis.cpu().numpy()
                torch.cuda.synchronize()
                out[rid] = {"seconds": time.perf_counter() - t0, "ez": ez}
            except RuntimeError as e:
                torch.cuda.synchronize()
                out[rid] = {"seconds": time.perf_counter() - t0, "error": str(e)}
            del sim
    return out


def run_serve(args, ws, rank, local):
    """The served stream: requests with Poisson arrivals (20 per second,
    seeded), grids 129/257/513 at h = 0.05, xi lengths uniform in 200..2000
    steps of 0.05, half of the drivers rigid Gaussians and half non-rigid
    bi-Gaussian beams of 100k..1M macroparticles; admitted by HBM footprint into at
    most --slots concurrent members, each advanced by captured graphs on its
    own stream.  The plain comparison runs the same requests one by one, first
    come first served, through the plain FP64 drop-in path (Simulation with
    its default settings), each timed for real; its queue follows from the
    arrivals and the measured durations."""
    import torch
    from lcodepy_b200 import _lib
    from lcodepy_b200.batch import BeamDriver, Server, request_stream
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    reqs = request_stream(n=args.requests, precision=args.precision)
    # warm the library, the allocator and the graph path on a short request
    warm = Server(hbm_budget_bytes=args.hbm_budget_gb << 30, max_slots=args.slots, device=dev)
    for N in (129, 257, 513):
        for bf in (0.0, 1.0):
            _, _, c, d = request_stream(n=1, sizes=(N,), min_steps=8, max_steps=8,
                                        precision=args.precision, beam_fraction=bf,
                                        beam_particles=(50_000, 50_000))[0]
            warm.submit(f"warm{N}{bf}", c, d, arrival=0.0)
    warm.run()
    torch.cuda.synchronize()
    barrier(ws)
    srv = Server(hbm_budget_bytes=args.hbm_budget_gb << 30, max_slots=args.slots, device=dev)
    for arr, rid, cfg, drv in reqs:
        srv.submit(rid, cfg, drv, arrival=arr)
    clock = ClockSampler(local) if rank == 0 else None
    n0 = _lib.launch_count()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    srv.t0 = time.perf_counter()
    t0.record()
    srv.run()
    torch.cuda.synchronize()
    t1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - srv.t0
    clocks = clock.stop() if clock else None
    launches = _lib.launch_count() - n0
    ms = max_over_ranks(t0.elapsed_time(t1), ws)
    done = {r: d for r, d in srv.done.items() if "error" not in d}
    failed = len(srv.done) - len(done)
    failed_ids = {r: d["error"][:160] for r, d in sorted(srv.done.items()) if "error" in d}
    cell_steps = sum(d["cells"] * d["steps"] for d in done.values())
    lat = np.array([done[r]["latency"] for _, r, _, _ in reqs if r in done])
    value = ws * cell_steps / (ms / 1e3)
    # plain path, request by request, first come first served: every request
    # runs alone through the drop-in Simulation API in FP64 (its defaults:
    # graphs and the fused particle stage), timed by wall clock from
    # construction to the synchronised end of its xi loop.  One request runs
    # at a time, so the queue is exact from the measured durations: request i
    # starts at max(arrival_i, end of request i-1).
    plain = ({} if args.no_plain else
             run_plain_requests([r for r in reqs if r[1] in done], dev))
    finish, plain_lat = 0.0, []
    for arr, rid, _, _ in reqs:
        if rid not in plain:
            continue
        finish = max(finish, arr) + plain[rid]["seconds"]
        plain_lat.append(finish - arr)
    plain_lat = np.array(plain_lat)
    plain_value = cell_steps / finish if finish > 0 else None
    pct = lambda a, q: float(np.percentile(a, q)) if a.size else None
    # accuracy: every served result against the same request alone in FP64
    def rel_l2(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    plain_failed = sorted(rid for rid, v in plain.items() if "error" in v)
    err_of = {rid: rel_l2(done[rid]["ez"], v["ez"]) for rid, v in plain.items() if "ez" in v}
    errs = list(err_of.values())
    worst = sorted(err_of.items(), key=lambda kv: -kv[1])[:3]
    # requests over 1e-5 run once more in FP64 with the reference's three
    # separate particle kernels (FP64 atomics in another order): how far two
    # FP64 runs that differ only in rounding drift apart on that request
    over = [r for r in reqs if r[1] in err_of and err_of[r[1]] > 1e-5]
    alt = run_plain_requests(over, dev, extra={'fused-particle-kernels': False})
    fp64_spread = {rid: {"mixed_vs_fp64": err_of[rid],
                         "fp64_vs_fp64_separate_kernels": (
                             rel_l2(alt[rid]["ez"], plain[rid]["ez"]) if "ez" in alt[rid]
                             else alt[rid]["error"])}
                   for rid in alt}
    return {"value": value, "ms": ms, "wall_s": wall, "cell_steps": cell_steps,
            "p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "plain_value": plain_value, "plain_p50": pct(plain_lat, 50),
            "plain_p99": pct(plain_lat, 99),
            "plain_busy_s": sum(v["seconds"] for v in plain.values()), "failed": failed,
            "beam_requests": sum(isinstance(r[3], BeamDriver) for r in reqs),
            "errs": errs, "worst": worst, "fp64_spread": fp64_spread,
            "plain_failed": plain_failed, "failed_ids": failed_ids,
            "clocks": clocks, "launches": launches,
            "span_arrivals_s": reqs[-1][0]}


def run_e2e(cfg, beam_host, dev):
    """Simulation.step() from a host beam file to host results: the H2D copy of
    the beam and of the initial plasma and the D2H read of fields, on-axis Ez
    and the moved beam are inside the timed region."""
    import torch
    from lcodepy_b200 import Simulation
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "beam.npz")
        np.savez(path, **{k: beam_host[k] for k in beam_host.dtype.names})
        # every rank is an independent replica, not a time-step pipeline stage
        sim = Simulation(config={**cfg, 'time-step-pipeline': False}, beam_parameters={},
                         runas_filename='')
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.load_beamfile(path)
        sim.step(1)
        particles, fields, currents = sim.push_solver._plasmastate
        host_fields = fields.to_numpy()
        ez = sim.push_solver.ez_axis.cpu().numpy()
        moved = sim.beam_drain.beam_slice().particles
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    conf = sim.effective_config
    N = conf.getint('window-width-steps')
    n_iter = sim.push_solver.xi_steps + 1
    Ns = sim.push_solver.plasma_solver.states[0].Ns
    h2d = beam_host.nbytes + 4 * Ns * Ns * 8
    d2h = 7 * N * N * 8 + ez.nbytes + moved.nbytes
    return {"value": n_iter * N * N / dt, "unit": METRIC, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "seconds": dt, "xi_steps": n_iter}


# ---------------------------------------------------------------------------
# CPU arm (oracle restatement of the reference algorithm)
# ---------------------------------------------------------------------------

def run_headline(args, ws, rank, local):
    """The many-simulation forms carried by the default line: the batched
    scan (64 members, mixed precision, 30 timed batched xi steps) and the
    served stream (`--requests` requests, mixed precision), each against the
    plain FP64 drop-in path run member by member / request by request."""
    import torch
    out = {}
    torch.cuda.empty_cache()
    bargs = argparse.Namespace(**{**vars(args), "steps": 30, "warmup": 3, "precision": "mixed"})
    try:
        b = run_batch(bargs, ws, rank, local)
        out["batched"] = {
            "workload": f"batched scan: {b['members']} members, grids 129/257/513 at h=0.05, "
                        "dxi=0.05, ppc=4, seeded rigid Gaussian drivers; 30 timed batched xi "
                        "steps after 3",
            "precision": "mixed", "value": b["value"], "unit": METRIC,
            "ms_per_batched_step": b["ms_per_step"], "plain_fp64_value": b["plain"],
            "batched_vs_plain": b["ratio"],
            "ez_rel_l2_vs_fp64": {"max": b["ez_err_max"], "median": b["ez_err_median"]},
            "gpu_launches": b["launches"], "clocks": b["clocks"]}
    except Exception as e:  # reported, not fatal to the production line
        out["batched"] = {"error": f"{type(e).__name__}: {e}"}
    torch.cuda.empty_cache()
    sargs = argparse.Namespace(**{**vars(args), "precision": "mixed"})
    try:
        v = run_serve(sargs, ws, rank, local)
        out["served"] = {
            "workload": f"served stream: {args.requests} requests (Poisson 20/s, seeded), grids "
                        "129/257/513 at h=0.05, 200-2000 xi steps of 0.05, half rigid "
                        "Gaussian, half bi-Gaussian beams of 100k-1M macroparticles",
            "precision": "mixed", "slots": args.slots, "hbm_budget_gb": args.hbm_budget_gb,
            "value": v["value"], "unit": METRIC,
            "latency_s": {"p50": v["p50"], "p99": v["p99"]},
            "plain_fp64": {"value": v["plain_value"], "p50": v["plain_p50"],
                           "p99": v["plain_p99"], "busy_s": v["plain_busy_s"],
                           "how": "each request alone through Simulation, timed; FCFS queue "
                                  "from the arrivals and the measured durations"},
            "served_vs_plain": v["value"] / v["plain_value"] if v["plain_value"] else None,
            "ez_rel_l2_vs_fp64": {"max": max(v["errs"]) if v["errs"] else None,
                                  "median": float(np.median(v["errs"])) if v["errs"] else None,
                                  "over_1e-5": int(sum(e > 1e-5 for e in v["errs"])),
                                  "worst": v["worst"],
                                  "over_1e-5_fp64_spread": v["fp64_spread"]},
            "failed_requests": v["failed"], "failed_ids": v["failed_ids"],
            "plain_fp64_failed_requests": v["plain_failed"], "gpu_launches": v["launches"],
            "clocks": v["clocks"]}
    except Exception as e:
        out["served"] = {"error": f"{type(e).__name__}: {e}"}
    return out


class _Budget(Exception):
    pass


def run_cpu_sample(warmup, steps, beam_host, budget_s=90.0):
    """The oracle on the host cores over the workload's xi loop: `warmup` xi
    steps untimed, then up to `steps` timed xi steps, stopping early once
    `budget_s` seconds of timed work are done.  Returns (xi-steps*cells/s,
    seconds, timed steps, threads)."""
    from oracle import oracle as O
    p = O.make_params(5.13, 0.02, 0.02)
    sorts, consts = O.init_plasma(p)
    F, cur = O.Fields.zeros(p.N), O.Currents.zeros(p.N)
    beam = O.Beam.from_array(beam_host).sorted()
    stamps = []

    def record(i, *_):
        stamps.append(time.perf_counter())
        timed = len(stamps) - 1 - warmup
        if timed >= steps or (timed > 0 and stamps[-1] - stamps[warmup] > budget_s):
            raise _Budget
    try:
        O.step_dt(p, sorts, F, cur, consts, warmup + steps, beam=beam, time_step=1.0,
                  record=record)
    except _Budget:
        pass
    n = len(stamps) - 1 - warmup
    dt = stamps[-1] - stamps[warmup]
    return n * p.N * p.N / dt, dt, n, O.num_threads()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2997)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--members", type=int, default=64, help="batch: scan members")
    ap.add_argument("--requests", type=int, default=64, help="serve: requests in the stream")
    ap.add_argument("--slots", type=int, default=32, help="serve: concurrent members")
    ap.add_argument("--no-plain", action="store_true",
                    help="serve: skip the request-by-request plain FP64 comparison")
    ap.add_argument("--hbm-budget-gb", type=int, default=64, help="serve: HBM admission budget")
    ap.add_argument("--workload", default="production",
                    choices=["production", "rigid129", "batch", "serve"],
                    help="production: the N=513 FP64 drop-in run (default); rigid129: "
                         "the 129 x 129 rigid-driver configuration")
    ap.add_argument("--cpu-sample", type=int, default=8,
                    help="timed xi steps of the CPU baseline sample")
    ap.add_argument("--cpu-budget", type=float, default=90.0,
                    help="reference arm: seconds of timed CPU work at most")
    ap.add_argument("--no-headline", action="store_true",
                    help="production line only: skip the batched scan and the served "
                         "stream that the default line carries")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end Simulation run (profiling runs)")
    ap.add_argument("--op-every", type=int, default=16,
                    help="per-op CUDA events on every K-th timed xi step (run eagerly)")
    ap.add_argument("--op-timeline", default=None,
                    help="write each eagerly timed xi step's per-op launch times (us) "
                         "to this JSON file")
    ap.add_argument("--window-length", type=float, default=60.0,
                    help="xi window length; smaller values give the small "
                         "profiling case of the same grid and beam")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.op_every < 1:
        raise SystemExit("--op-every must be >= 1")
    ws, rank, local = dist_init()

    if args.impl == "reference":
        if rank == 0:
            W = min(args.warmup, 3)
            v, dt, n, thr = run_cpu_sample(W, args.steps, make_beam(), args.cpu_budget)
            line = {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
                    "steps": n, "warmup": W, "ms_per_step": dt * 1e3 / n,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic (seeded bi-Gaussian beam, uniform plasma)",
                    "impl": "reference",
                    "config": {"workload": WORKLOAD, "parallelism": "replicas",
                               "l2": "inputs larger than L2"},
                    "cpu_baseline": {"value": v, "unit": METRIC, "cores": thr, "kind": "port",
                                     "sample": f"xi steps {W + 1}..{W + n} of the workload "
                                               f"({dt:.1f} s; the oracle's C particle loops "
                                               f"with OpenMP + scipy DST/DCT; at most "
                                               f"{args.cpu_budget:g} s of timed work)"},
                    "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    if args.workload == "batch":
        r = run_batch(args, ws, rank, local)
        if rank == 0:
            print(json.dumps({
                "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "mixed" if args.precision == "mixed" else "f64",
                "data": "synthetic (seeded rigid Gaussian drivers)",
                "config": {"workload": f"batched scan: {r['members']} members, grids "
                                       "129/257/513 at h=0.05, dxi=0.05, ppc=4",
                           "precision": args.precision,
                           "steps_are": "batched xi steps (every member advances one)"},
                "plain_fp64_value": r["plain"], "batched_vs_plain": r["ratio"],
                "ez_rel_l2_vs_fp64": {"max": r["ez_err_max"], "median": r["ez_err_median"]},
                "gpu_launches": r["launches"], "clocks": r["clocks"]}), flush=True)
        return
    if args.workload == "serve":
        r = run_serve(args, ws, rank, local)
        if rank == 0:
            print(json.dumps({
                "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": ws,
                "steps": args.requests, "warmup": args.warmup,
                "ms_per_step": r["ms"] / args.requests,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "mixed" if args.precision == "mixed" else "f64",
                "data": "synthetic (seeded Poisson request stream; rigid Gaussian and "
                        "seeded bi-Gaussian beam drivers)",
                "config": {"workload": f"served stream: {args.requests} requests, Poisson "
                                       "20/s, grids 129/257/513 at h=0.05, 200-2000 xi "
                                       "steps of 0.05, ppc=4, drivers half rigid, half "
                                       "beams of 100k-1M macroparticles",
                           "beam_requests": r["beam_requests"],
                           "precision": args.precision, "slots": args.slots,
                           "hbm_budget_gb": args.hbm_budget_gb,
                           "steps_are": "requests; ms_per_step = makespan / requests",
                           "l2": "aggregate member state larger than L2"},
                "latency_s": {"p50": r["p50"], "p99": r["p99"]},
                "failed_requests": r["failed"], "failed_ids": r["failed_ids"],
                "plain_fp64_failed_requests": r["plain_failed"],
                "makespan_s": r["ms"] / 1e3, "cell_steps": r["cell_steps"],
                "plain_fp64": {"value": r["plain_value"], "p50": r["plain_p50"],
                               "p99": r["plain_p99"], "busy_s": r["plain_busy_s"]},
                "served_vs_plain": r["value"] / r["plain_value"] if r["plain_value"] else None,
                "ez_rel_l2_vs_fp64": {"max": max(r["errs"]) if r["errs"] else None,
                                      "median": float(np.median(r["errs"])) if r["errs"] else None,
                                      "over_1e-5": int(sum(e > 1e-5 for e in r["errs"])),
                                      "worst": r["worst"],
                                      "over_1e-5_fp64_spread": r["fp64_spread"]},
                "gpu_launches": r["launches"], "clocks": r["clocks"]}), flush=True)
        return
    if args.workload == "rigid129":
        r = run_rigid129(args, ws, rank, local)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": r["value"], "unit": METRIC,
                              "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None,
                              "dtype": "f64" if args.precision == "fp64" else "mixed",
                              "data": "synthetic", "config": {
                                  "workload": f"rigid Gaussian driver, N={r['N']}, h=0.1, "
                                              f"dxi=0.1, {r['n_iter']} xi steps, ppc=4",
                                  "precision": args.precision,
                                  "steps_are": "whole xi loops (201 xi steps each)"}}),
                  flush=True)
        return
    r = run_gpu(args, ws, rank, local)
    headline = {}
    if not args.no_headline and ws == 1:
        headline = run_headline(args, ws, rank, local)
    if rank == 0:
        N = r["N"]
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        r["precision"] = args.precision
        roof = roofline(r, N, peaks)
        cpu = None
        if not args.no_cpu_baseline:
            v, dt, n, thr = run_cpu_sample(1, args.cpu_sample, make_beam(), 30.0)
            cpu = {"value": v, "unit": METRIC, "cores": thr, "kind": "port",
                   "sample": f"xi steps 2..{n + 1} of the workload on the host ({dt:.1f} s; "
                             "the oracle's C particle loops with OpenMP + scipy DST/DCT)"}
        line = {"metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64-particles/f32-fields",
                "data": "synthetic (seeded bi-Gaussian beam, uniform plasma)",
                "config": {"workload": WORKLOAD if args.window_length == 60.0 else
                           WORKLOAD.replace("L=60", f"L={args.window_length:g}"),
                           "grid": N, "xi_iterations": r["n_iter"],
                           "precision": args.precision, "parallelism": "replicas",
                           "l2": "inputs larger than L2 (no flush)"},
                "e2e": (None if r["e2e"] is None else
                        {k: r["e2e"][k] for k in ("value", "unit", "h2d_bytes_per_step",
                                                  "d2h_bytes_per_step")}),
                "gpu_launches": r["launches"], "clocks": r["clocks"],
                "roofline": roof, "cpu_baseline": cpu,
                "ops": {k: {"launches": v["launches"], "ms_avg": round(v["ms_avg"], 5),
                            "ms_total": round(v["ms_total"], 2)} for k, v in r["ops"].items()}}
        line.update(headline)
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# DRAM bytes (read + written) per call of each op, summed over all of the
# op's kernels, from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum, cold caches) of the small case of the same workload
# (N=513, window 0.2: 11 xi steps; profiles/launches_production_n513.md):
# compute_fields = RHS + four folds + four waves + finish; move_deposit = the
# fused stage averaged over the xi step's three stages (+ the fixed-point
# finish in mixed precision).
NCU_TRAFFIC = {("compute_fields", "fp64"): 197.9e6, ("compute_fields", "mixed"): 128.2e6,
               ("move_deposit", "fp64"): 110.8e6, ("move_deposit", "mixed"): 125.7e6}

# algorithmic bytes per plasma particle and xi step: K1 64 B (read m, px, py,
# pz, x_offt, y_offt; write x_offt, y_offt) + 3 x K2 128 B (read 11 x 8 B,
# write 5 x 8 B) + 3 x K3 72 B (read 9 x 8 B) = 664 B, over the xi step's
# three fused stages (K1 runs in the first): 664 / 3 B per stage on average
STAGE_BYTES = 664.0 / 3


def op_roofline(name, o, N, Np, precision, peaks):
    """Roofline of one op from its per-call CUDA-event time `o["ms_avg"]`:
    compute_fields against the measured bf16 burst peak with the useful
    dense-transform flops 56 N^3 per call (two calls per xi step make the
    112 N^3 per xi step of the transforms as dense contractions), the fused
    particle stage against the measured HBM copy bandwidth with 664 / 3 B
    per particle (the xi step's 664 B over its three stages)."""
    sec = o["ms_avg"] / 1e3
    if name == "compute_fields":
        # without the measured peaks: 1.59 PFLOP/s, an earlier burst
        # measurement of cuBLAS bf16 on B200
        peak = peaks.get("bf16_tflops", 1590.0)
        flops = 56.0 * N ** 3
        achieved = flops / sec / 1e12
        return {"bound": "tensor", "kernel": name, "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak,
                "work_per_launch": f"{flops:.4g} flop (56 N^3, N={N})",
                "traffic": NCU_TRAFFIC.get((name, precision)),
                "peak_source": ("measured bf16 burst" if "bf16_tflops" in peaks
                                else "fallback 1590 TFLOP/s")}
    peak = peaks.get("hbm_gbs", 6650.0)
    nbytes = STAGE_BYTES * Np
    achieved = nbytes / sec / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak,
            "work_per_launch": f"{nbytes:.4g} B (664/3 B x {Np} particles)",
            "traffic": NCU_TRAFFIC.get((name, precision)),
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}


def roofline(r, N, peaks):
    """The dominant op's roofline (largest device time in the timed region),
    with every measured op's roofline under "ops"."""
    ops = {k: v for k, v in r["ops"].items() if k in ("compute_fields", "move_deposit")}
    if not ops:
        return None
    Np = r["n_particles"]
    each = {k: op_roofline(k, v, N, Np, r["precision"], peaks) for k, v in ops.items()}
    name = max(ops, key=lambda k: ops[k]["ms_total"])
    return {**each[name], "ops": each}


if __name__ == "__main__":
    main()
