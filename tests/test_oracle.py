"""The CPU oracle against the reference: per-kernel known answers and whole
xi-loop runs produced by the reference itself (tests/golden/make_golden.py),
and the reference's own golden states (tests/integration/data/*.npz)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import REFERENCE_DATA

RTOL = 5e-8  # the reference's own golden tolerance (test_3D_part.py:7)


def test_kernel_known_answers(golden):
    d = golden("kat_kernels.npz")
    N, h, dxi, bnd = int(d["N"]), float(d["h"]), float(d["dxi"]), float(d["boundary"])
    p = O.Params(N=N, h=h, dxi=dxi, sub_coeff=1 + dxi, boundary=bnd)
    prev = O.Sort(d["x_init"], d["y_init"], d["xo_prev"], d["yo_prev"],
                  d["px_prev"], d["py_prev"], d["pz_prev"], d["q"].copy(), d["m"])
    full = O.move_wo_fields(p, prev)
    np.testing.assert_array_equal(full.x_offt, d["k1_xo"])
    np.testing.assert_array_equal(full.y_offt, d["k1_yo"])
    F = O.Fields(*(d["F_" + k] for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")),
                 np.zeros((N, N)))
    O.move_smart(p, F, prev, full)
    for a, b in (("x_offt", "k2_xo"), ("y_offt", "k2_yo"), ("px", "k2_px"),
                 ("py", "k2_py"), ("pz", "k2_pz"), ("q", "k2_q")):
        # reflected particles lose a few digits to x_offt = x - x_init
        np.testing.assert_allclose(getattr(full, a), d[b], rtol=1e-13,
                                   atol=1e-12 * np.abs(d[b]).max())
    cur = O.Currents.zeros(N)
    O.deposit_sort(p, full, cur, 0)
    for k in ("ro", "jx", "jy", "jz"):
        np.testing.assert_allclose(getattr(cur, k)[0], d["k3_" + k], rtol=1e-13,
                                   atol=1e-13 * np.abs(d["k3_" + k]).max())
    b = O.Beam(xi=d["b_xi"].copy(), x=d["b_x"].copy(), y=d["b_y"].copy(),
               q_norm=d["b_q"].copy(), id=np.arange(d["b_x"].size))
    r0, r1 = np.zeros((N, N)), np.zeros((N, N))
    O.deposit_beam(p, int(d["b_layer"]), b, r0, r1)
    np.testing.assert_allclose(r0, d["k4_ro0"], rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(r1, d["k4_ro1"], rtol=1e-13, atol=1e-16)
    n = d["k6_qm"].size
    dt, rs = np.empty(n), np.empty(n, np.int64)
    import ctypes
    O.lib().orc_beam_substepping(ctypes.c_int64(n), O._p(d["k6_qm"].copy()),
                                 O._p(d["k6_pz"].copy()), ctypes.c_double(2.0),
                                 ctypes.c_double(1.0), O._p(dt), O._p(rs))
    np.testing.assert_array_equal(dt, d["k6_dt"])
    np.testing.assert_array_equal(rs, (1.0 / d["k6_dt"]).astype(np.int64))


def test_field_solver_known_answer(golden):
    d = golden("kat_fields.npz")
    N, h, dxi, sub = int(d["N"]), float(d["h"]), float(d["dxi"]), float(d["sub"])
    p = O.Params(N=N, h=h, dxi=dxi, sub_coeff=sub, boundary=0)
    consts = O.Consts(None, O.dirichlet_matrix(N, h), O.mixed_matrix(N, h, sub),
                      O.neumann_matrix(N, h))
    F = O.Fields(*(d["in_" + k] for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")))
    Fp = O.Fields(*(d["prev_" + k] for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")))
    cp = O.Currents(*(d["cp_" + k] for k in ("ro", "jx", "jy", "jz")))
    cf = O.Currents(*(d["cf_" + k] for k in ("ro", "jx", "jy", "jz")))
    full, half = O.compute_fields(p, F, Fp, consts, d["rb_full"], d["rb_prev"], cp, cf)
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
        for tag, got in (("full_", full), ("half_", half)):
            ref = d[tag + k]
            np.testing.assert_allclose(getattr(got, k), ref, rtol=0,
                                       atol=1e-12 * np.abs(ref).max())


def rigid_driver(xp, xi, x, y):
    if -np.sqrt(2 * np.pi) <= xi <= 0:
        return 0.1 * xp.exp(-(x ** 2 + y ** 2) / 2) * (1 + np.cos(np.sqrt(np.pi / 2) * xi)) / 2
    return xp.zeros_like(x)


def _run_oracle(window_width, h, dxi, window_length, ion_model, rigid=None,
                beam=None, ppc=4):
    p = O.make_params(window_width, h, dxi, ion_model=ion_model)
    sorts, consts = O.init_plasma(p, ppc=ppc)
    N = p.N
    F, cur = O.Fields.zeros(N), O.Currents.zeros(N)
    ez = []
    rec = lambda i, s, f, c, rb: ez.append(f.Ez[N // 2, N // 2])
    xi_steps = round(window_length / dxi)
    sorts, F, cur, drain = O.step_dt(p, sorts, F, cur, consts, xi_steps,
                                     beam=beam, rigid=rigid, record=rec)
    return p, sorts, F, cur, np.array(ez), drain


def _check_state(ref, sorts, F, cur, names, rtol):
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
        r = ref["f_" + k]
        np.testing.assert_allclose(getattr(F, k), r, rtol=rtol, atol=1e-9 * np.abs(r).max())
    for k in ("ro", "jx", "jy", "jz"):
        r = ref["c_" + k]
        np.testing.assert_allclose(getattr(cur, k), r, rtol=rtol, atol=1e-9 * np.abs(r).max())
    for s, name in zip(sorts, names):
        for k in ("x_offt", "y_offt", "px", "py", "pz", "q"):
            r = ref[f"p_{name}_{k}"]
            np.testing.assert_allclose(getattr(s, k), r, rtol=rtol,
                                       atol=1e-9 * max(np.abs(r).max(), 1e-300))


@pytest.mark.parametrize("fixture,ion,dxi,length,names", [
    ("run_rigid_bg.npz", "background", 0.05, 2.0, ["electrons"]),
    ("run_rigid_mobile.npz", "mobile", 0.1, 1.0, ["electrons", "ions"]),
])
def test_whole_run_rigid(golden, fixture, ion, dxi, length, names):
    ref = golden(fixture)
    p, sorts, F, cur, ez, _ = _run_oracle(1.6, 0.05, dxi, length, ion, rigid=rigid_driver)
    np.testing.assert_allclose(ez, ref["ez_axis"], rtol=1e-9,
                               atol=1e-12 * np.abs(ref["ez_axis"]).max())
    _check_state(ref, sorts, F, cur, names, rtol=1e-8)


def test_whole_run_generated_beam(golden):
    from lcodepy_b200.beam_generator import generate_beam
    from lcodepy_b200.config import Config
    ref = golden("run_beam.npz")
    cfg = Config({'geometry': '3d', 'window-width': 1.6, 'transverse-step': 0.05,
                  'xi-step': 0.05})
    cfg._adjust_config_values_3d()
    arr = generate_beam(cfg, {'current': 0.05, 'particles_in_layer': 400,
                              'default': {'length': 2.0}})
    beam = O.Beam.from_array(arr).sorted()
    p, sorts, F, cur, ez, _ = _run_oracle(1.6, 0.05, 0.05, 1.5, "background", beam=beam)
    np.testing.assert_allclose(ez, ref["ez_axis"], rtol=1e-9,
                               atol=1e-12 * np.abs(ref["ez_axis"]).max())
    _check_state(ref, sorts, F, cur, ["electrons"], rtol=1e-8)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_DATA),
                    reason="reference golden data not present")
def test_reference_golden_test1():
    """The reference's own golden state (tests/integration/test_3D_part.py:32-56):
    N=321, 201 xi steps, generated beam of current 0.05, one time step."""
    from lcodepy_b200.beam_generator import generate_beam
    from lcodepy_b200.config import Config
    cfg = Config({'geometry': '3d', 'window-width': 8, 'transverse-step': 0.05,
                  'xi-step': 0.05, 'window-length': 10, 'plasma-particles-per-cell': 4,
                  'ion-model': 'background', 'field-solver-subtraction-coefficient': 1.0})
    cfg._adjust_config_values_3d()
    arr = generate_beam(cfg, {'current': 0.05, 'particles_in_layer': 5000,
                              'default': {'length': 5.013256548}})
    beam = O.Beam.from_array(arr).sorted()
    p = O.make_params(8, 0.05, 0.05, sub_coeff=1.0)
    assert p.N == 321 and p.sub_coeff == 1.0
    sorts, consts = O.init_plasma(p, ppc=4)
    F, cur = O.Fields.zeros(p.N), O.Currents.zeros(p.N)
    sorts, F, cur, _ = O.step_dt(p, sorts, F, cur, consts, 200, beam=beam)
    ref = np.load(os.path.join(REFERENCE_DATA, "3D_test1.npz"))
    for a in ("x_offt", "y_offt", "px", "py", "pz"):
        assert np.allclose(getattr(sorts[0], a)[::10, ::10], ref[a], rtol=RTOL, atol=1e-125), a
    for a in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        assert np.allclose(getattr(F, a)[::10, ::10], ref[a], rtol=RTOL, atol=1e-125), a
    for a in ("ro", "jx", "jy", "jz"):
        assert np.allclose(getattr(cur, a)[:, ::10, ::10].sum(axis=0), ref[a],
                           rtol=RTOL, atol=1e-125), a
