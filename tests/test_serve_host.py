"""Admission and retirement logic of the request server, with the GPU member
replaced by a host fake (no device needed)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lcodepy_b200 import batch  # noqa: E402


class FakeMember:
    def __init__(self, cfg, drv, device=None, name=None):
        if cfg.get("setup") == "fail":
            raise MemoryError("no device memory")
        self.fail_at = cfg.get("fail_at")
        self.name = name
        self.n_steps = cfg["steps"]
        self.cells = cfg["cells"]
        self.done = 0
        self.ez = torch.zeros(self.n_steps)

    @property
    def finished(self):
        return self.done >= self.n_steps

    def step(self):
        if self.fail_at is not None and self.done == self.fail_at:
            raise RuntimeError("launch failed")
        self.ez[self.done] = self.done
        self.done += 1

    def complete(self):
        return self.finished

    def check(self):
        if self.cells == "device-error" and self.finished:
            raise RuntimeError("device error word 0x1")

    def release(self):
        self.released = True


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(batch, "Member", FakeMember)
    monkeypatch.setattr(batch, "footprint_bytes", lambda cfg, drv=None: cfg["bytes"])


def req(steps, nbytes, cells=1):
    return {"steps": steps, "bytes": nbytes, "cells": cells}


def test_budget_and_slots_bound_admission(fake):
    srv = batch.Server(hbm_budget_bytes=10, max_slots=2, device="cpu")
    srv.submit("a", req(3, 6), None, arrival=0.0)
    srv.submit("b", req(2, 4), None, arrival=0.0)
    srv.submit("c", req(2, 1), None, arrival=0.0)
    srv.poll()
    assert [m.name for m in srv.running] == ["a", "b"]      # slots full
    srv.tick(); srv.tick(); srv.retire()
    assert "b" in srv.done and srv.used == 6
    srv.poll()
    assert [m.name for m in srv.running] == ["a", "c"]      # admitted while a runs
    srv.run()
    assert set(srv.done) == {"a", "b", "c"} and srv.used == 0


def test_first_come_first_served_under_memory_pressure(fake):
    srv = batch.Server(hbm_budget_bytes=10, max_slots=8, device="cpu")
    srv.submit("big0", req(5, 8), None, arrival=0.0)
    srv.submit("big1", req(2, 8), None, arrival=0.0)
    srv.submit("small", req(2, 1), None, arrival=0.0)
    srv.poll()
    # small fits next to big0 but must not overtake big1
    assert [m.name for m in srv.running] == ["big0"]
    srv.run()
    d = srv.done
    assert d["big1"]["admitted"] <= d["small"]["admitted"]


def test_oversized_request_runs_alone(fake):
    srv = batch.Server(hbm_budget_bytes=4, max_slots=8, device="cpu")
    srv.submit("huge", req(2, 100), None, arrival=0.0)
    srv.run()
    assert list(srv.done) == ["huge"]


def test_results_and_arrivals(fake):
    srv = batch.Server(hbm_budget_bytes=100, max_slots=4, device="cpu")
    srv.submit("late", req(3, 1), None, arrival=0.05)
    srv.submit("now", req(4, 1), None, arrival=0.0)
    srv.run()
    assert srv.done["late"]["admitted"] >= 0.05
    assert list(srv.done["now"]["ez"]) == [0, 1, 2, 3]


def test_request_stream_is_seeded():
    a = batch.request_stream(n=20)
    b = batch.request_stream(n=20)
    assert [(r[0], r[2]['window-length'], r[3]) for r in a] == \
           [(r[0], r[2]['window-length'], r[3]) for r in b]
    arr = [r[0] for r in a]
    assert arr == sorted(arr) and arr[0] > 0


def test_beam_driver_routes_to_beam_member_and_costs_more(monkeypatch):
    made = []
    monkeypatch.setattr(batch, "BeamMember", lambda *a: made.append(("beam", a[1])) or a)
    monkeypatch.setattr(batch, "Member", lambda *a: made.append(("rigid", a[1])) or a)
    drv = batch.BeamDriver(n=1000, amplitude=0.1, sigma_r=0.5)
    batch.make_member({}, drv)
    batch.make_member({}, batch.GaussianDriver(0.1, 1.0))
    assert [k for k, _ in made] == ["beam", "rigid"]
    cfg = {"geometry": "3d", "window-width-step-size": 0.05, "window-width": 6.4,
           "xi-step": 0.05, "window-length": 1.0}
    rigid = batch.footprint_bytes(cfg)
    assert batch.footprint_bytes(cfg, drv) == rigid + 1000 * batch.BEAM_BYTES_PER_PARTICLE


def test_request_stream_mixes_rigid_and_beam_drivers():
    reqs = list(batch.request_stream(200, rate=20.0, seed=5))
    kinds = {type(r[3]).__name__ for r in reqs}
    assert kinds == {"BeamDriver", "GaussianDriver"}
    for _, _, cfg, drv in reqs:
        if isinstance(drv, batch.BeamDriver):
            assert 100_000 <= drv.n <= 1_000_000
            half = cfg["window-width"] / 2
            assert drv.r_max < half


def test_device_beam_distribution_on_cpu():
    """The served drivers' beam generator (run here on CPU tensors): the
    cuts, the charge normalisation and the moments of the bi-Gaussian."""
    import math
    drv = batch.BeamDriver(n=200_000, amplitude=0.3, sigma_r=0.8, sigma_z=1.0, xi0=-3.0,
                           gamma=1000.0, espread=0.01, emittance=1e-2, seed=11, r_max=2.4)
    b = drv.device_beam(0.05, torch.device("cpu"))
    xi, x, y = b.xi.numpy(), b.x.numpy(), b.y.numpy()
    n = xi.size
    assert 0.95 * drv.n < n <= drv.n
    assert (xi < 0).all() and (xi > 2 * drv.xi0).all()
    assert (np.diff(xi) <= 0).all()                           # sorted, xi descending
    r = np.hypot(x, y)
    assert r.max() < drv.r_max
    assert abs(np.std(b.pz.numpy()) / 1000.0 - 0.01) < 1e-3
    assert abs(np.std(b.px.numpy()) - drv.emittance / drv.sigma_r) < 2e-4
    q_total = (-drv.amplitude * math.sqrt(2 * math.pi) * drv.sigma_z
               * 2 * math.pi * drv.sigma_r ** 2 / 0.05)
    assert np.isclose(b.q_norm.numpy().sum(), q_total)
    assert (b.q_m.numpy() == -1).all() and (np.sort(b.id.numpy()) == np.arange(1, n + 1)).all()
    # seeded: the same driver gives the same beam
    b2 = drv.device_beam(0.05, torch.device("cpu"))
    assert np.array_equal(b2.x.numpy(), x)


def test_failing_requests_are_isolated(fake):
    srv = batch.Server(hbm_budget_bytes=100, max_slots=8, device="cpu")
    srv.submit("ok", req(4, 10), None, arrival=0.0)
    srv.submit("setup", {**req(4, 10), "setup": "fail"}, None, arrival=0.0)
    srv.submit("launch", {**req(6, 10), "fail_at": 2}, None, arrival=0.0)
    srv.submit("deverr", req(3, 10, cells="device-error"), None, arrival=0.0)
    srv.submit("ok2", req(5, 10), None, arrival=0.0)
    srv.run()
    assert set(srv.done) == {"ok", "setup", "launch", "deverr", "ok2"}
    assert "MemoryError" in srv.done["setup"]["error"]
    assert "launch failed" in srv.done["launch"]["error"]
    assert "device error" in srv.done["deverr"]["error"]
    for rid in ("ok", "ok2"):
        assert "error" not in srv.done[rid] and srv.done[rid]["ez"] is not None
    assert srv.used == 0


def test_driver_records_round_trip():
    """Slot files store drivers as JSON; both kinds come back equal."""
    for d in (batch.GaussianDriver(0.3, 0.8),
              batch.BeamDriver(n=1234, amplitude=0.2, sigma_r=0.5, seed=9, r_max=1.0)):
        assert batch.driver_from_record(batch.driver_record(d)) == d
    with pytest.raises(ValueError):
        batch.driver_from_record('{"kind": "other"}')
