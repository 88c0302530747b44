"""Whole xi loops through the drop-in ``Simulation`` on the GPU, against runs
of the reference (tests/golden/run_*.npz, made by make_golden.py) and the
CPU oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs CUDA", allow_module_level=True)

from lcodepy_b200 import Simulation  # noqa: E402
from oracle import oracle as O  # noqa: E402


def rigid_driver(xp, xi, x, y):
    if -np.sqrt(2 * np.pi) <= xi <= 0:
        return 0.1 * xp.exp(-(x ** 2 + y ** 2) / 2) * (1 + np.cos(np.sqrt(np.pi / 2) * xi)) / 2
    return xp.zeros_like(x)


def cfg(**kw):
    c = {'geometry': '3d', 'processing-unit-type': 'gpu',
         'window-width': 1.6, 'transverse-step': 0.05,
         'window-length': 2.0, 'xi-step': 0.05,
         'time-limit': 1, 'time-step': 1,
         'ion-model': 'background', 'plasma-particles-per-cell': 4,
         'print-every': 0}
    c.update(kw)
    return c


def run(config, beam, n_steps=None):
    sim = Simulation(config=config, beam_parameters=beam, diagnostics=[], runas_filename='')
    sim.step(n_steps)
    ps = sim.push_solver
    particles, fields, currents = ps._plasmastate
    return sim, particles, fields, currents, ps.ez_axis.cpu().numpy()


def rel_err(got, ref):
    return np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)


def check(ref, particles, fields, currents, sorts, rel):
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
        e = rel_err(getattr(fields, k).cpu().numpy(), ref["f_" + k])
        assert e < rel, f"{k}: {e:.2e}"
    for k in ("ro", "jx", "jy", "jz"):
        e = rel_err(getattr(currents, k).cpu().numpy(), ref["c_" + k])
        assert e < rel, f"{k}: {e:.2e}"
    for s in sorts:
        for k in ("x_offt", "y_offt", "px", "py", "pz", "q"):
            e = rel_err(getattr(particles[s], k).cpu().numpy(), ref[f"p_{s}_{k}"])
            assert e < rel, f"{s}.{k}: {e:.2e}"


@pytest.mark.parametrize("fixture,extra,sorts", [
    ("run_rigid_bg.npz", {}, ["electrons"]),
    ("run_rigid_mobile.npz", {'ion-model': 'mobile', 'window-length': 1.0, 'xi-step': 0.1},
     ["electrons", "ions"]),
    ("run_profile_channel.npz", {'window-length': 1.0, 'plasma-particles-per-cell': 9,
                                 'plasma-rshape': 'channel', 'plasma-width': 0.6,
                                 'plasma-width-2': 0.9, 'plasma-density-2': 0.5}, ["electrons"]),
    ("run_profile_gauss.npz", {'window-length': 1.0, 'plasma-particles-per-cell': 1,
                               'ion-model': 'mobile', 'plasma-rshape': 'gaussian',
                               'plasma-width': 0.5}, ["electrons", "ions"]),
])
def test_rigid_vs_reference(golden, fixture, extra, sorts):
    ref = golden(fixture)
    _, particles, fields, currents, ez = run(cfg(**{'rigid-beam': True, **extra}), rigid_driver)
    assert rel_err(ez, ref["ez_axis"]) < 1e-9
    check(ref, particles, fields, currents, sorts, 1e-8)


def test_declustering_vs_reference(golden):
    """The declustering noise filter on (noise_filter.py:82-239; the
    reference reads 'damping-declustering') over 21 xi steps of the rigid
    configuration, against the reference's run.  With the filter on, this
    configuration amplifies rounding differences about tenfold every 1.5 xi
    steps (measured), so after 21 steps the electrons' momenta, where the
    filter's kicks act, agree to 1e-6 of their largest value; on-axis Ez,
    fields and currents to 1e-9 / 1e-8."""
    ref = golden("run_declustering.npz")
    extra = {'window-length': 1.0, 'declustering-enabled': True,
             'declustering-averaging': 3, 'declustering-force': 0.3,
             'damping-declustering': 0.1, 'declustering-limit': 2e-3}
    _, particles, fields, currents, ez = run(cfg(**{'rigid-beam': True, **extra}), rigid_driver)
    assert rel_err(ez, ref["ez_axis"]) < 1e-9
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
        assert rel_err(getattr(fields, k).cpu().numpy(), ref["f_" + k]) < 1e-8, k
    for k in ("ro", "jx", "jy", "jz"):
        assert rel_err(getattr(currents, k).cpu().numpy(), ref["c_" + k]) < 1e-8, k
    for k in ("x_offt", "y_offt", "px", "py", "pz", "q"):
        e = rel_err(getattr(particles["electrons"], k).cpu().numpy(), ref["p_electrons_" + k])
        assert e < 1e-6, (k, e)


def test_generated_beam_vs_reference(golden):
    ref = golden("run_beam.npz")
    _, particles, fields, currents, ez = run(
        cfg(**{'window-length': 1.5}),
        {'current': 0.05, 'particles_in_layer': 400, 'default': {'length': 2.0}})
    assert rel_err(ez, ref["ez_axis"]) < 1e-9
    check(ref, particles, fields, currents, ["electrons"], 1e-8)


def test_reference_golden_configuration(golden):
    """The reference's own 3D golden case (N=321, 201 xi steps, generated beam),
    checked exactly as the reference's test checks it (rtol 5e-8)."""
    ref = golden("run_test1.npz")
    c = {'geometry': '3d', 'processing-unit-type': 'gpu', 'window-width': 8,
         'transverse-step': 0.05, 'window-length': 10, 'xi-step': 0.05,
         'time-limit': 1, 'time-step': 1, 'ion-model': 'background',
         'plasma-particles-per-cell': 4, 'field-solver-subtraction-coefficient': 1.0,
         'print-every': 0}
    _, particles, fields, currents, ez = run(
        c, {'current': 0.05, 'particles_in_layer': 5000, 'default': {'length': 5.013256548}})
    el = particles["electrons"]
    for a in ("x_offt", "y_offt", "px", "py", "pz"):
        np.testing.assert_allclose(getattr(el, a).cpu().numpy()[::10, ::10],
                                   ref["p_electrons_" + a], rtol=5e-8,
                                   atol=1e-8 * np.abs(ref["p_electrons_" + a]).max())
    for a in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        np.testing.assert_allclose(getattr(fields, a).cpu().numpy()[::10, ::10],
                                   ref["f_" + a], rtol=5e-8, atol=1e-8 * np.abs(ref["f_" + a]).max())
    for a in ("ro", "jx", "jy", "jz"):
        np.testing.assert_allclose(getattr(currents, a).cpu().numpy()[:, ::10, ::10].sum(axis=0),
                                   ref["c_" + a], rtol=5e-8, atol=1e-8 * np.abs(ref["c_" + a]).max())
    assert rel_err(ez, ref["ez_axis"]) < 5e-8


def test_two_time_steps_beam_push_vs_oracle():
    """Second time step depends on the beam push (GPU Higuera-Cary algorithm),
    checked against the oracle's restatement of it."""
    from lcodepy_b200.beam_generator import generate_beam
    from lcodepy_b200.config import Config
    config = cfg(**{'window-length': 1.5, 'time-limit': 2, 'time-step': 5.0})
    beam_params = {'current': -0.5, 'particles_in_layer': 300,
                   'default': {'length': 1.2, 'energy': 5.0, 'angspread': 1e-2}}
    sim, particles, fields, currents, ez = run(config, beam_params, n_steps=2)
    c = Config(config)
    c._adjust_config_values_3d()
    beam = O.Beam.from_array(generate_beam(c, beam_params)).sorted()
    p = O.make_params(1.6, 0.05, 0.05)
    xi_steps = round(1.5 / 0.05)
    for t in range(2):
        sorts, consts = O.init_plasma(p)
        F, cur = O.Fields.zeros(p.N), O.Currents.zeros(p.N)
        ez_o = []
        rec = lambda i, s, f, cc, rb: ez_o.append(f.Ez[p.N // 2, p.N // 2])
        sorts, F, cur, drain = O.step_dt(p, sorts, F, cur, consts, xi_steps, beam=beam,
                                         time_step=5.0, record=rec)
        beam = drain.sorted()
    assert rel_err(ez, np.array(ez_o)) < 1e-8
    assert rel_err(fields.Ez.cpu().numpy(), F.Ez) < 1e-8
    got = sim.beam_drain.beam_slice()
    order = np.argsort(got.id.cpu().numpy())
    ref_order = np.argsort(drain.id)
    np.testing.assert_array_equal(got.id.cpu().numpy()[order], drain.id[ref_order])
    for k in ("x", "y", "xi", "px", "py", "pz"):
        assert rel_err(getattr(got, k).cpu().numpy()[order], getattr(drain, k)[ref_order]) < 1e-9, k


def test_mixed_precision_on_axis_ez():
    """FP32 deposition and FP32 transforms, FP64 particles: on-axis Ez within
    relative L2 1e-5 of the FP64 run (rigid driver, 129 x 129, 201 xi steps)."""
    base = cfg(**{'rigid-beam': True, 'window-width': 6.5, 'transverse-step': 0.1,
                  'xi-step': 0.1, 'window-length': 20})
    _, _, f64, _, ez64 = run(base, rigid_driver)
    _, _, fmx, _, ezmx = run({**base, 'precision': 'mixed'}, rigid_driver)
    l2 = np.linalg.norm(ezmx - ez64) / np.linalg.norm(ez64)
    print("mixed vs fp64 on-axis Ez rel L2:", l2)
    assert l2 < 1e-5


@pytest.mark.parametrize("rigid", [True, False])
def test_cuda_graphs_match_eager(rigid):
    """The captured-graph xi step gives the eager step's results."""
    extra = {'rigid-beam': True} if rigid else {'window-length': 1.5}
    beam = rigid_driver if rigid else {'current': 0.05, 'particles_in_layer': 400,
                                       'default': {'length': 2.0}}
    _, p0, f0, c0, ez0 = run(cfg(**extra, **{'cuda-graphs': False}), beam)
    sim, p1, f1, c1, ez1 = run(cfg(**extra, **{'cuda-graphs': True}), beam)
    ps = sim.push_solver.plasma_solver
    if rigid:   # the driver's layers alternate between two fixed planes
        assert ps.graphs[0] is None and len(ps.plane_graphs) == 2
    else:       # the beam's three rotating planes are read in place
        assert ps.graphs[0] is None and len(ps.plane_graphs) == 6
    assert rel_err(ez1, ez0) < 1e-12
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
        assert rel_err(getattr(f1, k).cpu().numpy(), getattr(f0, k).cpu().numpy()) < 1e-12, k


@pytest.mark.parametrize("extra", [{'rigid-beam': True},
                                   {'rigid-beam': True, 'ion-model': 'mobile'},
                                   {'rigid-beam': True, 'plasma-particles-per-cell': 1},
                                   {'rigid-beam': True, 'precision': 'mixed'}])
def test_fused_stage_matches_separate_kernels(extra):
    """The fused move+deposit stage equals K1 + K2 + K3 launched separately."""
    _, p0, f0, c0, ez0 = run(cfg(**extra, **{'fused-particle-kernels': False}), rigid_driver)
    _, p1, f1, c1, ez1 = run(cfg(**extra, **{'fused-particle-kernels': True}), rigid_driver)
    tol = 1e-5 if extra.get('precision') == 'mixed' else 1e-12
    assert rel_err(ez1, ez0) < tol
    for k in ("Ex", "Ez", "Bz"):
        assert rel_err(getattr(f1, k).cpu().numpy(), getattr(f0, k).cpu().numpy()) < tol, k
    for s in p0:
        for k in ("x_offt", "px", "q"):
            assert rel_err(getattr(p1[s], k).cpu().numpy(), getattr(p0[s], k).cpu().numpy()) < tol


def test_device_diagnostics_record_the_run(tmp_path, monkeypatch):
    """FXiDiag / SliceDiag / ParticlesDiag attached to the drop-in Simulation:
    the on-axis Ez they write equals the solver's own record, the slices are
    the final fields, and the snapshots hold the final particles."""
    from lcodepy_b200.diagnostics import (FXiDiag, FXiType, ParticlesDiag, SliceDiag,
                                          SliceType, SliceValue)
    monkeypatch.chdir(tmp_path)
    fxi = FXiDiag(output_period=1, f_xi=FXiType.Ez | FXiType.ne | FXiType.Sf)
    sl = SliceDiag(SliceType.XI_X, slice_value=SliceValue.Ez, output_period=1)
    pd = ParticlesDiag(save_plasma=True, output_period=1, saving_xi_period=1.0)
    sim = Simulation(config=cfg(**{'rigid-beam': True}), beam_parameters=rigid_driver,
                     diagnostics=[fxi, sl, pd], runas_filename='')
    sim.step(1)
    ps = sim.push_solver
    ez = ps.ez_axis.cpu().numpy()
    diag = tmp_path / 'diagnostics'

    def one(pattern):
        files = sorted(diag.glob(pattern))
        assert len(files) == 1, files
        return files[0]

    with np.load(one('f_xi_*.npz')) as z:
        assert np.array_equal(z['Ez'], ez)
        assert z['xi'].shape == ez.shape and z['ne'].shape == ez.shape and z['Sf'].shape == ez.shape
    _, fields, _ = ps._plasmastate
    N = fields.Ez.shape[0]
    with np.load(one('slice_*.npz')) as z:
        n = z['x'].size   # the reference's default x range: the first N - 1 rows
        assert z['Ez'].shape == (ez.size, n) and n == N - 1
        assert np.array_equal(z['Ez'][-1], fields.Ez[:n, N // 2].cpu().numpy())
    particles, _, _ = ps._plasmastate
    with np.load(one('plasma_electrons_*.npz')) as z:
        assert np.array_equal(z['px'], particles['electrons'].px.cpu().numpy())
    assert len(list((diag / 'snapshots').glob('plasma_electrons_*.npz'))) >= 1


def test_resume_from_a_stored_plasma_state(tmp_path):
    """A state stored by a diagnostic at layer k and loaded through
    external_plasmastate continues the xi loop as the uninterrupted run.  As
    in the reference, a resumed time step starts with a zero beam density for
    the stored layer, so the layer is taken behind the driver (xi < -2.51)."""
    from lcodepy_b200.plasma_state import save_plasmastate
    path = tmp_path / "plasmastate.npz"
    k_store = 56

    class Store:
        def pull_config(self, config):
            self.k = 0

        def after_step_dxi(self, t, xi, particles, fields, currents, rho_beam):
            if self.k == k_store:
                save_plasmastate(path, particles, fields, currents, xi_plasma_layer=xi)
            self.k += 1

        def dump(self, *a, **k):
            pass

    c = cfg(**{'rigid-beam': True, 'window-length': 4.0})
    sim = Simulation(config=c, beam_parameters=rigid_driver, diagnostics=[Store()], runas_filename='')
    sim.step(1)
    ez_all = sim.push_solver.ez_axis.cpu().numpy()
    sim2 = Simulation(config=c, beam_parameters=rigid_driver, runas_filename='')
    sim2.external_plasmastate = True
    sim2.path_to_plasmastate = str(path)
    sim2.step(1)
    ez_resumed = sim2.push_solver.ez_axis.cpu().numpy()
    assert ez_resumed.shape == ez_all[k_store + 1:].shape
    assert rel_err(ez_resumed, ez_all[k_store + 1:]) < 1e-10


def _production_beam(shift=2.9):
    """The production workload's seeded 1M-particle bi-Gaussian driver
    (sigma_r 0.5, sigma_z 1, peak n_b/n0 0.5, gamma 1000 +- 1 %, emittance
    1e-2), moved forward by `shift` in xi so that a short window starts inside
    the beam; particles that end up ahead of xi = 0 are dropped."""
    from lcodepy_b200.batch import bigaussian_beam
    b = bigaussian_beam(1_000_000, 2024, 0.5, 1.0, -3.0, 1000.0, 0.01, 1e-2, -0.5, 0.02, 4.0)
    b['xi'] += shift
    return b[b['xi'] < 0]


@pytest.mark.parametrize("precision,rel", [("fp64", 1e-8), ("mixed", 1e-5)])
def test_production_configuration_vs_oracle(tmp_path, precision, rel):
    """The benchmarked production grid (N=513, h 0.02, dxi 0.02, 929,296
    electrons, background ions) with the production beam, pushed every
    layer: 16 xi steps inside the beam, every layer with beam particles.
    FP64: on-axis Ez, the final fields and the drained beam against the
    oracle within 1e-8 relative.  Mixed precision: on-axis Ez relative L2 and
    the final Ez within 1e-5 of the FP64 oracle."""
    beam = _production_beam()
    path = tmp_path / "beam.npz"
    np.savez(path, **{k: beam[k] for k in beam.dtype.names})
    config = {'geometry': '3d', 'processing-unit-type': 'gpu', 'window-width': 5.13,
              'transverse-step': 0.02, 'window-length': 0.3, 'xi-step': 0.02,
              'time-limit': 1.0, 'time-step': 1.0, 'ion-model': 'background',
              'plasma-particles-per-cell': 4, 'print-every': 0, 'precision': precision}
    sim = Simulation(config=config, beam_parameters={}, diagnostics=[], runas_filename='')
    sim.load_beamfile(str(path))
    sim.step(1)
    ps = sim.push_solver
    particles, fields, currents = ps._plasmastate
    ez = ps.ez_axis.cpu().numpy()
    N = fields.Ez.shape[0]
    assert N == 513 and ez.size == 16

    p = O.make_params(5.13, 0.02, 0.02)
    sorts, consts = O.init_plasma(p)
    F, cur = O.Fields.zeros(p.N), O.Currents.zeros(p.N)
    ez_o, layers = [], []
    ob = O.Beam.from_array(beam).sorted()
    sorts, F, cur, drain = O.step_dt(
        p, sorts, F, cur, consts, 15, beam=ob, time_step=1.0,
        record=lambda i, s, f, c, rb: (ez_o.append(f.Ez[p.N // 2, p.N // 2]),
                                       layers.append(np.abs(rb).max())))
    ez_o = np.array(ez_o)
    assert min(layers[1:]) > 0   # the beam is present in every layer
    if precision == "fp64":
        assert rel_err(ez, ez_o) < rel
        for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
            assert rel_err(getattr(fields, k).cpu().numpy(), getattr(F, k)) < rel, k
        e = particles["electrons"]
        for k in ("x_offt", "y_offt", "px", "py", "pz"):
            assert rel_err(getattr(e, k).cpu().numpy(), getattr(sorts[0], k)) < rel, k
        got = sim.beam_drain.beam_slice()
        gid = got.id.cpu().numpy()
        assert gid.size == drain.id.size and gid.size > 0
        order, ref_order = np.argsort(gid), np.argsort(drain.id)
        np.testing.assert_array_equal(gid[order], drain.id[ref_order])
        for k in ("x", "y", "xi", "px", "py", "pz"):
            assert rel_err(getattr(got, k).cpu().numpy()[order],
                           getattr(drain, k)[ref_order]) < rel, k
    else:
        l2 = np.linalg.norm(ez - ez_o) / np.linalg.norm(ez_o)
        print(f"N=513 production beam, mixed vs FP64 oracle: on-axis Ez rel L2 {l2:.2e}")
        assert l2 < rel
        assert np.linalg.norm(fields.Ez.cpu().numpy() - F.Ez) / np.linalg.norm(F.Ez) < rel


class _SliceRecorder:
    """A diagnostic with the reference's after_step_dxi signature that keeps
    on-axis Ez every xi step and the rho (sorts summed) and Ez slices every
    `every` xi steps."""

    def __init__(self, every=20):
        self.every = every

    def pull_config(self, config):
        self.k, self.rho, self.ez = 0, [], []

    def after_step_dxi(self, t, xi, particles, fields, currents, rho_beam):
        if self.k % self.every == 0:
            self.rho.append(currents.ro.get().sum(axis=0))
            self.ez.append(fields.Ez.get())
        self.k += 1

    def dump(self, *a, **k):
        pass


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_mixed_precision_slices_and_axis():
    """The precision form of the 129 x 129 rigid configuration (201 xi steps):
    on-axis Ez over the run, and the rho (sorts summed) and Ez slices taken
    every 20 xi steps, over the run, within relative L2 1e-5 of the FP64 run.
    The per-slice errors are printed too; the first rho slice, at xi = 0, is
    the small first response of a neutral plasma (electrons and ions cancel),
    so its own relative error is larger than the run's."""
    base = cfg(**{'rigid-beam': True, 'window-width': 6.5, 'transverse-step': 0.1,
                  'xi-step': 0.1, 'window-length': 20})
    out = {}
    for prec in ("fp64", "mixed"):
        rec = _SliceRecorder(20)
        sim = Simulation(config={**base, 'precision': prec}, beam_parameters=rigid_driver,
                         diagnostics=[rec], runas_filename='')
        sim.step()
        out[prec] = (sim.push_solver.ez_axis.cpu().numpy(), rec)
    ez64, r64 = out["fp64"]
    ezmx, rmx = out["mixed"]
    assert len(r64.rho) == 11
    e_axis = _rel_l2(ezmx, ez64)
    e_rho = _rel_l2(np.stack(rmx.rho), np.stack(r64.rho))
    e_ez = _rel_l2(np.stack(rmx.ez), np.stack(r64.ez))
    per_rho = [_rel_l2(a, b) for a, b in zip(rmx.rho, r64.rho)]
    per_ez = [_rel_l2(a, b) for a, b in zip(rmx.ez[1:], r64.ez[1:])]
    print(f"mixed vs FP64, 129^2 201 steps: on-axis Ez {e_axis:.2e}; rho slices {e_rho:.2e} "
          f"(per slice {' '.join(f'{e:.1e}' for e in per_rho)}); Ez slices {e_ez:.2e} "
          f"(per slice max {max(per_ez):.1e})")
    assert e_axis < 1e-5
    assert e_rho < 1e-5
    assert e_ez < 1e-5


def test_mixed_precision_beam_energy():
    """The precision form with a non-rigid beam (129 x 129, two time steps of
    5, a generated gamma ~ 10 beam): the drained beam's mean energy, and its
    change over the run, within 1e-5 relative of the FP64 run; on-axis Ez of
    the second time step within relative L2 1e-5."""
    base = cfg(**{'window-width': 6.5, 'transverse-step': 0.1, 'xi-step': 0.1,
                  'window-length': 8, 'time-limit': 2, 'time-step': 5.0})
    beam = {'current': -0.5, 'particles_in_layer': 500,
            'default': {'length': 4.0, 'energy': 10.0, 'angspread': 1e-2}}
    res = {}
    for prec in ("fp64", "mixed"):
        sim, _, _, _, ez = run({**base, 'precision': prec}, beam, n_steps=2)
        b = sim.beam_drain.beam_slice()
        p2 = b.px.cpu().numpy() ** 2 + b.py.cpu().numpy() ** 2 + b.pz.cpu().numpy() ** 2
        energy = np.sqrt(1 / b.q_m.cpu().numpy() ** 2 + p2)
        res[prec] = (ez, energy, b.id.cpu().numpy())
    ez64, en64, id64 = res["fp64"]
    ezmx, enmx, idmx = res["mixed"]
    np.testing.assert_array_equal(np.sort(id64), np.sort(idmx))
    from lcodepy_b200.beam_generator import generate_beam
    from lcodepy_b200.config import Config
    c = Config(base)
    c._adjust_config_values_3d()
    g = generate_beam(c, beam)
    e0 = np.sqrt(1 / g['q_m'] ** 2 + g['px'] ** 2 + g['py'] ** 2 + g['pz'] ** 2).mean()
    m64, mmx = en64.mean(), enmx.mean()
    e_mean = abs(mmx - m64) / m64
    e_change = abs(mmx - m64) / abs(m64 - e0)
    e_axis = _rel_l2(ezmx, ez64)
    print(f"mixed vs FP64 beam: mean energy {e_mean:.2e}, energy change {e_change:.2e} "
          f"(FP64 change {m64 - e0:.3e} of {e0:.3f}), on-axis Ez {e_axis:.2e}")
    assert e_mean < 1e-5 and e_change < 1e-5 and e_axis < 1e-5


def test_resume_matches_reference_resume(golden):
    """A plasma state file written by plasma_state.save_plasmastate from the
    reference's own run (after xi layer 56), resumed through the drop-in
    Simulation with external_plasmastate, against the reference's Simulation
    resuming from the same file (tests/golden/make_resume_golden.py)."""
    import os
    ref = golden("run_resume.npz")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "resume_state.npz")
    sim = Simulation(config=cfg(**{'rigid-beam': True, 'window-length': 4.0}),
                     beam_parameters=rigid_driver, runas_filename='')
    sim.external_plasmastate = True
    sim.path_to_plasmastate = path
    sim.step(1)
    ps = sim.push_solver
    particles, fields, currents = ps._plasmastate
    ez = ps.ez_axis.cpu().numpy()
    assert ez.shape == ref["ez_axis"].shape
    assert rel_err(ez, ref["ez_axis"]) < 1e-8
    check(ref, particles, fields, currents, ["electrons"], 1e-8)
