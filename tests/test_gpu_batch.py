"""Batched and served simulations: every member's result equals the same
simulation run alone through the drop-in Simulation API."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs CUDA", allow_module_level=True)

from lcodepy_b200 import Simulation  # noqa: E402
from lcodepy_b200.batch import (BatchRunner, BeamDriver, BeamMember, GaussianDriver,  # noqa: E402
                                Member, Server, solo_ez)


def cfg(ww, n_steps, precision="fp64", dxi=0.05):
    return {'geometry': '3d', 'window-width': ww, 'transverse-step': 0.05,
            'window-length': (n_steps - 1) * dxi, 'xi-step': dxi,
            'ion-model': 'background', 'plasma-particles-per-cell': 4,
            'rigid-beam': True, 'print-every': 0, 'precision': precision, 'time-step': 1.0}


def solo(config, driver):
    sim = Simulation(config=config, beam_parameters=driver, runas_filename='')
    sim.step()
    return sim.push_solver.ez_axis.cpu().numpy()


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_single_graph_batch_equals_solo_runs():
    """Every member's xi step captured into one graph per buffer parity (one
    graph launch per batched xi step): each member equals its solo run."""
    specs = [(cfg(1.6, 30), GaussianDriver(0.3, 0.8)),
             (cfg(3.25, 30, precision="mixed"), GaussianDriver(0.05, 1.5)),
             (cfg(1.6, 30), GaussianDriver(0.5, 0.6))]
    members = [Member(c, d) for c, d in specs]
    runner = BatchRunner(members, single_graph=True)
    assert runner.single_graph
    runner.run()
    assert all(g is not None for g in runner.graphs)
    assert all(m.graphs == [None, None] for m in members)   # no per-member graphs
    for (c, d), m in zip(specs, members):
        got = m.result()["ez"]
        assert m.done == 30 and got.shape == (30,)
        assert rel(got, solo(c, d)) < 1e-9


def test_batched_members_equal_solo_runs():
    specs = [(cfg(1.6, 30), GaussianDriver(0.3, 0.8)),
             (cfg(3.25, 25), GaussianDriver(0.05, 1.5)),
             (cfg(1.6, 40), GaussianDriver(0.5, 0.6))]
    members = [Member(c, d) for c, d in specs]
    BatchRunner(members).run()
    for (c, d), m in zip(specs, members):
        got = m.result()["ez"]
        ref = solo(c, d)
        assert got.shape == ref.shape
        assert rel(got, ref) < 1e-9


def _beam(seed, amplitude=0.2):
    # a short narrow electron driver that stays inside the 1.6-wide window
    return BeamDriver(n=20_000, amplitude=amplitude, sigma_r=0.15, sigma_z=0.3, xi0=-0.5,
                      seed=seed, r_max=0.5)


def test_beam_member_equals_solo_run():
    """A non-rigid driver in the batch engine (device beam layer step between
    captured plasma steps) gives the drop-in Simulation's on-axis Ez."""
    c, d = cfg(1.6, 30), _beam(3)
    m = BeamMember(c, d)
    BatchRunner([m]).run()
    ref = solo_ez(c, d)
    assert rel(m.result()["ez"], ref) < 1e-9
    assert np.abs(ref).max() > 0


def test_server_results_same_alone_and_in_the_mix():
    """Requests of different sizes and lengths admitted while others run, under
    a memory budget that forces some to wait: each result equals its solo run."""
    specs = {"a": (cfg(1.6, 40), GaussianDriver(0.2, 1.0)),
             "b": (cfg(3.25, 20), GaussianDriver(0.4, 0.7)),
             "c": (cfg(1.6, 15), GaussianDriver(0.1, 1.2)),
             "d": (cfg(3.25, 35), GaussianDriver(0.3, 1.8)),
             "e": (cfg(1.6, 25), _beam(7, 0.3))}
    from lcodepy_b200.batch import footprint_bytes
    budget = footprint_bytes(specs["b"][0]) + footprint_bytes(specs["a"][0]) + (1 << 20)
    srv = Server(hbm_budget_bytes=budget, max_slots=2)
    for i, (rid, (c, d)) in enumerate(specs.items()):
        srv.submit(rid, c, d, arrival=0.0)
    srv.run()
    assert set(srv.done) == set(specs)
    # two slots: some request was admitted only after another one finished
    d = srv.done
    assert any(d[x]["admitted"] >= d[y]["finished"] for x in d for y in d if x != y)
    for rid, (c, d) in specs.items():
        assert rel(srv.done[rid]["ez"], solo_ez(c, d)) < 1e-9, rid


def _steps(m, n):
    for _ in range(n):
        m.step()
    m.stream.synchronize()


@pytest.mark.parametrize("kind,precision", [("rigid", "fp64"), ("rigid", "mixed"),
                                            ("beam", "fp64")])
def test_member_checkpoint_and_resume(tmp_path, kind, precision):
    """A member written between xi steps (plasma state file + slot file) and
    rebuilt by restore_member continues to the result of an uninterrupted
    run; writing the checkpoint leaves the running member unchanged."""
    from lcodepy_b200.batch import make_member, restore_member
    n, k = 40, 17
    c = cfg(1.6, n, precision=precision)
    d = GaussianDriver(0.3, 0.8) if kind == "rigid" else _beam(5, 0.3)
    ref = make_member(c, d, name="ref")
    _steps(ref, n)
    want = ref.result()
    m = make_member(c, d, name="slot")
    _steps(m, k)
    base = m.checkpoint(str(tmp_path))
    _steps(m, n - k)
    r = restore_member(base)
    assert r.done == k and r.name == "slot" and r.config_dict == c
    _steps(r, n - k)
    tol = 1e-12
    for got in (m.result(), r.result()):
        assert rel(got["ez"], want["ez"]) < tol
        assert rel(got["fields"], want["fields"]) < tol
    assert np.abs(want["ez"]).max() > 0


def test_server_checkpoint_and_restore(tmp_path):
    """A server checkpointed with requests running and waiting, rebuilt by
    Server.restore: every request finishes with its solo result."""
    specs = {"r0": (cfg(1.6, 30), GaussianDriver(0.3, 0.8)),
             "r1": (cfg(1.6, 40), _beam(4, 0.3)),
             "r2": (cfg(3.25, 25), GaussianDriver(0.1, 1.2))}
    srv = Server(hbm_budget_bytes=8 << 30, max_slots=2)
    for rid, (c, d) in specs.items():
        srv.submit(rid, c, d, arrival=0.0)
    srv.poll()
    for _ in range(10):
        srv.tick()
    assert [m.name for m in srv.running] == ["r0", "r1"] and len(srv.waiting) == 1
    srv.checkpoint(str(tmp_path))
    srv2 = Server.restore(str(tmp_path), hbm_budget_bytes=8 << 30, max_slots=2)
    assert [m.done for m in srv2.running] == [10, 10]
    srv2.run()
    assert set(srv2.done) == set(specs)
    for rid, (c, d) in specs.items():
        assert "error" not in srv2.done[rid], rid
        assert rel(srv2.done[rid]["ez"], solo_ez(c, d)) < 1e-9, rid
