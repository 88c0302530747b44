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

--impl reference times the CPU restatement of the reference algorithm
(oracle/, the reference's own numba path cannot be shipped here) on the
host cores, on a bounded prefix of the same xi loop.
"""
from __future__ import annotations

import argparse
import json
import math
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
            ps.plasma_solver.op_timers = op_times if (k - W) % 16 == 0 else None
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

    # ---- end to end through the public API, host buffers in and out ----
    e2e = None if args.no_e2e else run_e2e(cfg, beam_host, dev)

    return dict(value=value, ms_per_step=ms_per_step, N=N, ops=ops,
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
        sim = Simulation(config=cfg, beam_parameters=rigid_driver, runas_filename='')
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
    widths), advanced together in mixed precision, one xi step per member per
    bench step on concurrent streams with captured graphs.  The same members
    are then run one after another through the plain FP64 drop-in path
    (Simulation with its default settings) for the plain-path comparison and
    the on-axis Ez error."""
    import torch
    from lcodepy_b200 import Simulation
    from lcodepy_b200.batch import BatchRunner, make_member, scan_members
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W, K = args.warmup, args.steps
    specs = scan_members(n=args.members, n_steps=W + K, precision=args.precision)
    members = [make_member(c, d, dev) for c, d in specs]
    runner = BatchRunner(members)
    for _ in range(W):
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
    for _ in range(K):
        runner.step()
    for m in members:
        cur.wait_stream(m.stream)
    t1.record(cur)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - n0
    clocks = clock.stop() if clock else None
    ms = max_over_ranks(t0.elapsed_time(t1), ws)
    cells = sum(m.cells for m in members)
    value = ws * cells * K / (ms / 1e3)
    ez_batch = [m.result()["ez"] for m in members]
    for m in members:
        m.release()
    del members, runner
    torch.cuda.empty_cache()

    # plain FP64: each member alone, eager, no graphs, separate kernels
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


def plain_ms_per_step(N, precision="fp64", n_steps=120, skip=20, beam=None):
    """Device ms per xi step of the plain drop-in path (PusherAndSolver3D
    with default settings) on an N x N grid at h = dxi = 0.05, with a rigid
    Gaussian driver or the given BeamDriver."""
    import torch
    from lcodepy_b200.batch import GaussianDriver, request_stream
    from lcodepy_b200.beam3d import BeamDrain, BeamSource, RigidBeamSource
    from lcodepy_b200.config import Config
    from lcodepy_b200.push_solver import PusherAndSolver3D
    cfg = dict(request_stream(n=1, sizes=(N,), min_steps=n_steps, max_steps=n_steps,
                              beam_fraction=0.0)[0][2])
    cfg['precision'] = precision
    cfg['rigid-beam'] = beam is None
    conf = Config(cfg)
    conf._adjust_config_values_3d()
    dev = torch.device("cuda", torch.cuda.current_device())
    ps = PusherAndSolver3D(conf, dev)
    ev = {}

    def hook(k):
        if k in (skip, n_steps):
            ev[k] = torch.cuda.Event(enable_timing=True)
            ev[k].record()
    ps.plasma_solver.init_state(1.0)
    if beam is None:
        src, drain = RigidBeamSource(None, GaussianDriver()), None
    else:
        import dataclasses
        beam = dataclasses.replace(beam, r_max=min(beam.r_max, 0.4 * cfg['window-width']))
        src = BeamSource(conf, beam.device_beam(cfg['xi-step'], dev), dev)
        drain = BeamDrain(conf, dev)
    ps.step_dt(cfg['xi-step'], src, drain, 1.0, [], step_hook=hook)
    torch.cuda.synchronize()
    return ev[skip].elapsed_time(ev[n_steps]) / (n_steps - skip)


def run_serve(args, ws, rank, local):
    """The served stream: requests with Poisson arrivals (20 per second,
    seeded), grids 129/257/513 at h = 0.05, xi lengths uniform in 200..2000
    steps of 0.05, half of the drivers rigid Gaussians and half non-rigid
    bi-Gaussian beams of 100k..1M macroparticles; admitted by HBM footprint into at
    most --slots concurrent members, each advanced by captured graphs on its
    own stream.  The plain comparison runs the same requests one by one, first
    come first served, through the plain FP64 drop-in path; its per-step cost
    per grid size is measured here and its schedule computed from the
    arrivals."""
    import torch
    from lcodepy_b200 import _lib
    from lcodepy_b200.batch import Server, request_stream
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
    cell_steps = sum(d["cells"] * d["steps"] for d in done.values())
    lat = np.array([done[r]["latency"] for _, r, _, _ in reqs if r in done])
    value = ws * cell_steps / (ms / 1e3)
    # plain path, request by request, first come first served: per-step cost
    # per grid size, measured with a rigid driver and with a beam of the mean
    # size (550k macroparticles)
    from lcodepy_b200.batch import BeamDriver
    per = {N: plain_ms_per_step(N) for N in (129, 257, 513)}
    per_beam = ({N: plain_ms_per_step(N, beam=BeamDriver(n=550_000, amplitude=0.1))
                 for N in (129, 257, 513)}
                if any(isinstance(r[3], BeamDriver) for r in reqs) else per)
    finish, plain_lat, busy = 0.0, [], 0.0
    for arr, rid, cfg, drv in reqs:
        if rid not in done:
            continue
        d = done[rid]
        N = int(round(math.sqrt(d["cells"])))
        dur = d["steps"] * (per_beam if isinstance(drv, BeamDriver) else per)[N] / 1e3
        finish = max(finish, arr) + dur
        busy += dur
        plain_lat.append(finish - arr)
    plain_lat = np.array(plain_lat)
    plain_value = cell_steps / finish
    # accuracy: a few requests rerun alone through the plain FP64 path
    errs = []
    if args.check_requests:
        from lcodepy_b200.batch import solo_ez
        for arr, rid, cfg, drv in sorted((r for r in reqs if r[1] in done),
                                         key=lambda r: r[2]['window-length'])[:args.check_requests]:
            ez64 = solo_ez(cfg, drv, precision='fp64')
            errs.append(float(np.linalg.norm(done[rid]["ez"] - ez64) / np.linalg.norm(ez64)))
    return {"value": value, "ms": ms, "wall_s": wall, "cell_steps": cell_steps,
            "p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "plain_value": plain_value, "plain_p50": float(np.percentile(plain_lat, 50)),
            "plain_p99": float(np.percentile(plain_lat, 99)), "plain_ms_per_step": per,
            "plain_ms_per_step_beam": per_beam, "failed": failed,
            "beam_requests": sum(isinstance(r[3], BeamDriver) for r in reqs),
            "errs": errs, "clocks": clocks, "launches": launches,
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
        sim = Simulation(config=cfg, beam_parameters={}, runas_filename='')
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

def run_cpu_sample(xi_steps_sample, beam_host):
    """The oracle on the host cores for the first `xi_steps_sample` xi steps of
    the workload; returns (xi-steps*cells/s, seconds, threads)."""
    from oracle import oracle as O
    p = O.make_params(5.13, 0.02, 0.02)
    sorts, consts = O.init_plasma(p)
    F, cur = O.Fields.zeros(p.N), O.Currents.zeros(p.N)
    beam = O.Beam.from_array(beam_host).sorted()
    t0 = time.perf_counter()
    O.step_dt(p, sorts, F, cur, consts, xi_steps_sample - 1, beam=beam, time_step=1.0)
    dt = time.perf_counter() - t0
    return xi_steps_sample * p.N * p.N / dt, dt, O.num_threads()


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
    ap.add_argument("--hbm-budget-gb", type=int, default=64, help="serve: HBM admission budget")
    ap.add_argument("--check-requests", type=int, default=3,
                    help="serve: requests rerun alone in FP64 for the Ez error")
    ap.add_argument("--workload", default="production",
                    choices=["production", "rigid129", "batch", "serve"],
                    help="production: the N=513 FP64 drop-in run (default); rigid129: "
                         "the 129 x 129 rigid-driver configuration")
    ap.add_argument("--cpu-sample", type=int, default=8,
                    help="xi steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end Simulation run (profiling runs)")
    ap.add_argument("--window-length", type=float, default=60.0,
                    help="xi window length; smaller values give the small "
                         "profiling case of the same grid and beam")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    ws, rank, local = dist_init()

    if args.impl == "reference":
        if rank == 0:
            beam = make_beam()
            n = max(2, min(args.steps, args.cpu_sample))
            v, dt, thr = run_cpu_sample(n, beam)
            line = {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
                    "steps": n, "warmup": 0, "ms_per_step": dt * 1e3 / n,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic", "impl": "reference",
                    "config": {"workload": WORKLOAD, "parallelism": "replicas",
                               "l2": "inputs larger than L2"},
                    "cpu_baseline": {"value": v, "unit": METRIC, "cores": thr, "kind": "port",
                                     "sample": f"first {n} xi steps of the workload "
                                               "(oracle/: C particle loops + scipy DST/DCT)"},
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
                "failed_requests": r["failed"],
                "makespan_s": r["ms"] / 1e3, "cell_steps": r["cell_steps"],
                "plain_fp64": {"value": r["plain_value"], "p50": r["plain_p50"],
                               "p99": r["plain_p99"],
                               "ms_per_step": r["plain_ms_per_step"],
                               "ms_per_step_beam": r["plain_ms_per_step_beam"]},
                "served_vs_plain": r["value"] / r["plain_value"],
                "ez_rel_l2_vs_fp64": r["errs"],
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
    if rank == 0:
        N = r["N"]
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        r["precision"] = args.precision
        roof = roofline(r, N, hbm_peak, peak_src, peaks)
        cpu = None
        if not args.no_cpu_baseline:
            v, dt, thr = run_cpu_sample(args.cpu_sample, make_beam())
            cpu = {"value": v, "unit": METRIC, "cores": thr, "kind": "port",
                   "sample": f"first {args.cpu_sample} xi steps of the workload on the host "
                             f"({dt:.1f} s; oracle/: C particle loops, scipy DST/DCT)"}
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
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# DRAM bytes (read + written) per call of the dominant op, from one ncu
# capture of the small case of the same workload (N=513, 11 xi steps):
# compute_fields counts its four tensor-core waves, move_deposit the fused
# kernel of a non-first stage.
NCU_TRAFFIC = {("compute_fields", "fp64"): 85.1e6, ("compute_fields", "mixed"): 43.8e6,
               ("move_deposit", "fp64"): 118.2e6, ("move_deposit", "mixed"): 115.5e6}


def transform_flops(N):
    """Flops of the dense transforms of one compute_fields call: four waves
    of even/odd folded products (2 M K N each) over the seven problems, Phi
    counted in one call of two (the predictor does not need it)."""
    n = N - 2
    rows = [n, n, N, N, n, n, N]
    cols = [N, N, n, n, n, n, N]
    tot = 0.0
    for p in range(7):
        R, C = rows[p], cols[p]
        right = 2 * R * (((C + 1) // 2) ** 2 + ((C - 1) // 2) ** 2)
        left = 2 * C * (((R + 1) // 2) ** 2 + ((R - 1) // 2) ** 2)
        tot += (0.5 if p == 5 else 1.0) * 2 * (right + left)
    return tot


def roofline(r, N, hbm_peak, peak_src, peaks):
    """Roofline of the dominant operation over the timed region."""
    ops = r["ops"]
    if not ops:
        return None
    name = max(ops, key=lambda k: ops[k]["ms_total"])
    o = ops[name]
    Np = 964 * 964
    if name == "compute_fields":
        # executed int8 operations: one slice-pair product per pair i + j < NS
        prec = r.get("precision", "fp64")
        ns = 8 if prec == "fp64" else 4
        ops_int8 = ns * (ns + 1) // 2 * transform_flops(N)
        achieved = ops_int8 / (o["ms_avg"] / 1e3) / 1e12
        return {"bound": "tensor", "kernel": name + f" (int8 tcgen05 waves, {ns} slices)",
                "achieved": achieved, "peak": 4500.0, "unit": "TOP/s", "frac": achieved / 4500.0,
                "traffic": NCU_TRAFFIC.get((name, prec)),
                "peak_source": "nominal B200 dense int8 (no measured int8 peak on this pool)"}
    per = {"deposit": 72, "move_smart": 128, "move_wo_fields": 64,
           "move_deposit": 128 + 72}.get(name, 0)
    achieved = per * Np / (o["ms_avg"] / 1e3) / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm_peak,
            "unit": "GB/s", "frac": achieved / hbm_peak,
            "traffic": NCU_TRAFFIC.get((name, r.get("precision", "fp64"))),
            "peak_source": peak_src}


if __name__ == "__main__":
    main()
