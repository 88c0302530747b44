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
