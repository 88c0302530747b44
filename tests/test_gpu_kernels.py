"""Per-kernel parity of liblcb.so (called through its C ABI) against the CPU
oracle and the reference's own known answers (tests/golden/kat_*.npz).

Tolerances: the kernels compute in FP64 like the reference; the GPU sums in
a different order (atomics, fused multiply-adds, dense transforms instead of
FFTs), so results agree to a few ulps of the largest element."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs CUDA", allow_module_level=True)

from lcodepy_b200 import _lib  # noqa: E402
from lcodepy_b200.plasma3d import FieldOperators  # noqa: E402
from oracle import oracle as O  # noqa: E402

DEV = torch.device("cuda")


def T(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def N_(t):
    return t.detach().cpu().numpy()


def close(got, ref, rel=1e-12, what=""):
    scale = max(np.abs(ref).max(), 1e-300)
    err = np.abs(got - ref).max() / scale
    assert err <= rel, f"{what}: max |diff| / max |ref| = {err:.3e} > {rel:.1e}"


@pytest.fixture(scope="module")
def kat(golden):
    return golden("kat_kernels.npz")


def _plasma_from_kat(d):
    n = d["x_init"].size
    st = {k: T(d[v].ravel()) for k, v in (
        ("x_init", "x_init"), ("y_init", "y_init"), ("x_offt", "xo_prev"),
        ("y_offt", "yo_prev"), ("px", "px_prev"), ("py", "py_prev"),
        ("pz", "pz_prev"), ("q", "q"), ("m", "m"))}
    return n, st


def test_move_wo_fields_and_smart(kat):
    d = kat
    L = _lib.load()
    N, h, dxi, bnd = int(d["N"]), float(d["h"]), float(d["dxi"]), float(d["boundary"])
    n, p = _plasma_from_kat(d)
    full = {k: torch.empty_like(p["x_offt"]) for k in ("x_offt", "y_offt", "px", "py", "pz", "q")}
    st = _lib.stream_handle()
    _lib.check(L.lcb_plasma_move_wo_fields(
        n, dxi, p["m"].data_ptr(), p["x_offt"].data_ptr(), p["y_offt"].data_ptr(),
        p["px"].data_ptr(), p["py"].data_ptr(), p["pz"].data_ptr(), p["q"].data_ptr(),
        full["x_offt"].data_ptr(), full["y_offt"].data_ptr(), full["px"].data_ptr(),
        full["py"].data_ptr(), full["pz"].data_ptr(), full["q"].data_ptr(), st), "k1")
    close(N_(full["x_offt"]).reshape(d["k1_xo"].shape), d["k1_xo"], 1e-15, "K1 x_offt")
    close(N_(full["y_offt"]).reshape(d["k1_yo"].shape), d["k1_yo"], 1e-15, "K1 y_offt")
    F = [T(d["F_" + k]) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")]
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    _lib.check(L.lcb_plasma_move_smart(
        n, dxi, bnd, h, N, *(f.data_ptr() for f in F),
        p["x_init"].data_ptr(), p["y_init"].data_ptr(), p["x_offt"].data_ptr(),
        p["y_offt"].data_ptr(), p["px"].data_ptr(), p["py"].data_ptr(), p["pz"].data_ptr(),
        p["m"].data_ptr(), full["q"].data_ptr(), full["x_offt"].data_ptr(),
        full["y_offt"].data_ptr(), full["px"].data_ptr(), full["py"].data_ptr(),
        full["pz"].data_ptr(), err.data_ptr(), st), "k2")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for k, ref in (("x_offt", "k2_xo"), ("y_offt", "k2_yo"), ("px", "k2_px"),
                   ("py", "k2_py"), ("pz", "k2_pz"), ("q", "k2_q")):
        close(N_(full[k]).reshape(d[ref].shape), d[ref], 1e-12, "K2 " + k)


@pytest.mark.parametrize("precision,rel", [(_lib.LCB_PREC_FP64, 1e-12),
                                           (_lib.LCB_PREC_MIXED, 1e-8)])
def test_deposit(kat, precision, rel):
    d = kat
    L = _lib.load()
    N, h = int(d["N"]), float(d["h"])
    Ns = d["x_init"].shape[0]
    n = Ns * Ns
    x_init, y_init = T(d["x_init"].ravel()), T(d["y_init"].ravel())
    xo, yo = T(d["k2_xo"].ravel()), T(d["k2_yo"].ravel())
    px, py, pz = T(d["k2_px"].ravel()), T(d["k2_py"].ravel()), T(d["k2_pz"].ravel())
    q, m = T(d["k2_q"].ravel()), T(d["m"].ravel())
    out = [torch.full((2, N, N), 7.0, dtype=torch.float64, device=DEV) for _ in range(4)]
    ro_init = T(np.arange(N * N, dtype=np.float64).reshape(N, N))
    ws = torch.empty(max(L.lcb_plasma_deposit_workspace_bytes(N, precision), 256),
                     dtype=torch.uint8, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    _lib.check(L.lcb_plasma_deposit(
        n, 1, N, h, Ns, precision, x_init.data_ptr(), y_init.data_ptr(), xo.data_ptr(),
        yo.data_ptr(), px.data_ptr(), py.data_ptr(), pz.data_ptr(), q.data_ptr(),
        m.data_ptr(), ro_init.data_ptr(), *(o.data_ptr() for o in out),
        ws.data_ptr(), ws.numel(), err.data_ptr(), _lib.stream_handle()), "k3")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for o, k in zip(out, ("ro", "jx", "jy", "jz")):
        close(N_(o[0]), d["k3_" + k], rel, "K3 " + k)
    np.testing.assert_array_equal(N_(out[0][1]), N_(ro_init))
    for o in out[1:]:
        assert float(o[1].abs().max()) == 0.0


def test_mixed_deposit_is_order_independent(kat):
    """The fixed-point sums of the mixed-precision deposit are exact, so three
    calls on the same particles agree bit for bit (the atomics' order varies
    between calls), and the sums stay within 2^-32 per contribution of the
    FP64 deposit."""
    d = kat
    L = _lib.load()
    N, h = int(d["N"]), float(d["h"])
    Ns = d["x_init"].shape[0]
    n = Ns * Ns
    names = ("x_init", "y_init", "k2_xo", "k2_yo", "k2_px", "k2_py", "k2_pz", "k2_q", "m")
    inp = [T(d[k].ravel()) for k in names]
    prec = _lib.LCB_PREC_MIXED
    ws = torch.empty(L.lcb_plasma_deposit_workspace_bytes(N, prec), dtype=torch.uint8,
                     device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    runs = []
    for _ in range(3):
        out = [torch.zeros((2, N, N), dtype=torch.float64, device=DEV) for _ in range(4)]
        _lib.check(L.lcb_plasma_deposit(
            n, 1, N, h, Ns, prec, *(t.data_ptr() for t in inp), None,
            *(o.data_ptr() for o in out), ws.data_ptr(), ws.numel(), err.data_ptr(),
            _lib.stream_handle()), "k3")
        runs.append([N_(o) for o in out])
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for r in runs[1:]:
        for a, b in zip(r, runs[0]):
            np.testing.assert_array_equal(a, b)
    for o, k in zip(runs[0], ("ro", "jx", "jy", "jz")):
        assert np.abs(o[0] - d["k3_" + k]).max() < 1e-8


def test_deposit_runaway_particles_take_global_path(kat):
    """Particles far from their tile's window still deposit (global atomics)."""
    d = kat
    L = _lib.load()
    N, h = int(d["N"]), float(d["h"])
    Ns = d["x_init"].shape[0]
    p = O.Params(N=N, h=h, dxi=float(d["dxi"]), sub_coeff=1, boundary=float(d["boundary"]))
    rng = np.random.default_rng(3)
    xo = rng.uniform(-0.8, 0.8, (Ns, Ns))  # up to 16 cells away from the lattice
    yo = rng.uniform(-0.8, 0.8, (Ns, Ns))
    xo = np.clip(d["x_init"] + xo, -1.0, 1.0) - d["x_init"]
    yo = np.clip(d["y_init"] + yo, -1.0, 1.0) - d["y_init"]
    s = O.Sort(d["x_init"], d["y_init"], xo, yo, d["k2_px"], d["k2_py"], d["k2_pz"],
               d["k2_q"].copy(), d["m"])
    cur = O.Currents.zeros(N)
    O.deposit_sort(p, s, cur, 0)
    out = [torch.zeros((2, N, N), dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = torch.empty(256, dtype=torch.uint8, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    inputs = [T(a.ravel()) for a in (d["x_init"], d["y_init"], xo, yo, d["k2_px"],
                                     d["k2_py"], d["k2_pz"], d["k2_q"], d["m"])]
    _lib.check(L.lcb_plasma_deposit(
        Ns * Ns, 1, N, h, Ns, _lib.LCB_PREC_FP64, *(t.data_ptr() for t in inputs),
        None, *(o.data_ptr() for o in out),
        ws.data_ptr(), ws.numel(), err.data_ptr(), _lib.stream_handle()), "k3")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for o, k in zip(out, ("ro", "jx", "jy", "jz")):
        close(N_(o[0]), getattr(cur, k)[0], 1e-12, "K3 " + k)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_stage_forms_match_separate_kernels(precision):
    """The fused first stage (K1 + K2 + K3 in one kernel) against the three
    kernels run separately, on a lattice whose particles are scattered so
    that every form of the fused gather and deposit runs: both particles of
    a thread in one cell, in neighbouring cells (the shared 6 x 6
    footprint), further apart, and outside the block's window (global
    atomics).  FP64 to 1e-12; mixed precision (FP32 gather, fixed-point
    deposit) to 1e-5 of the FP64 kernels, and bit-identical over two calls."""
    from lcodepy_b200.config import Config
    from lcodepy_b200.solver import CurrentSet, Plane2d3vPlasmaSolver
    cfg = Config({'geometry': '3d', 'window-width': 12.85, 'transverse-step': 0.1,
                  'xi-step': 0.1, 'window-length': 1.0, 'ion-model': 'background',
                  'plasma-particles-per-cell': 4, 'precision': precision, 'print-every': 0})
    cfg._adjust_config_values_3d()
    ps = Plane2d3vPlasmaSolver(cfg, DEV)
    ps.init_state(0.0)
    prev, full = ps.states
    N, h, n = ps.N, ps.h, prev.n_per_sort
    rng = np.random.default_rng(11)
    xi, yi = N_(prev.x_init), N_(prev.y_init)
    inner = (np.abs(xi) < ps.boundary - 12 * h) & (np.abs(yi) < ps.boundary - 12 * h)
    u = rng.random(n)
    mag = np.where(u < 0.4, 0.2, np.where(u < 0.9, 1.2, np.where(inner, 7.0, 1.2))) * h
    prev.x_offt.copy_(T(rng.uniform(-1, 1, n) * mag))
    prev.y_offt.copy_(T(rng.uniform(-1, 1, n) * mag))
    m = N_(prev.m)
    for k in ("px", "py", "pz"):    # |p| / m ~ 0.3: velocities up to ~0.7 c
        getattr(prev, k).copy_(T(rng.normal(0.0, 0.3, n) * m))
    F = ps.fields[0]
    F.buf.copy_(T(rng.uniform(-0.05, 0.05, (7, N, N))))

    def particles():
        return {k: N_(getattr(full, k)).copy() for k in ("x_offt", "y_offt", "px", "py", "pz", "q")}

    # the reference's three kernels, FP64 push, deposit in the stage's precision
    cs = CurrentSet(N, DEV)
    ps._move_wo_fields(prev, full)
    ps._move_smart(F, prev, full)
    ps._deposit(full, cs)
    torch.cuda.synchronize()
    sep_p, sep_c = particles(), N_(cs.buf).copy()
    assert int(ps.err.item()) == 0
    runs = []
    for _ in range(2):
        cf = CurrentSet(N, DEV)
        ps._move_deposit(F, prev, full, cf, True)
        torch.cuda.synchronize()
        runs.append((particles(), N_(cf.buf).copy()))
    assert int(ps.err.item()) == 0
    rel = 1e-12 if precision == "fp64" else 1e-5
    fus_p, fus_c = runs[0]
    for k in sep_p:
        close(fus_p[k], sep_p[k], rel, "fused " + k)
    for i, k in enumerate(("ro", "jx", "jy", "jz")):
        close(fus_c[i], sep_c[i], rel, "fused " + k)
    if precision == "mixed":
        for k in fus_p:
            np.testing.assert_array_equal(runs[1][0][k], fus_p[k])
        np.testing.assert_array_equal(runs[1][1], fus_c)


def test_declustering_filter_vs_reference(golden):
    """The noise filter's two kernels with the Gaussian average between them
    (cuFFT) against the reference's filter applied to the same seeded
    electron arrays (kat_noise_filter.npz)."""
    d = golden("kat_noise_filter.npz")
    L = _lib.load()
    n = d["x_offt"].shape[0]
    st = _lib.stream_handle()
    b = torch.zeros(4, n, n, dtype=torch.float64, device=DEV)
    xo, yo = T(d["x_offt"]), T(d["y_offt"])
    _lib.check(L.lcb_declustering_inhomogeneity(n, xo.data_ptr(), yo.data_ptr(),
                                                b[0].data_ptr(), b[1].data_ptr(), st), "inhom")
    f = torch.fft.fftfreq(n, dtype=torch.float64, device=DEV)
    g = torch.exp(-2 * np.pi ** 2 * float(d["declustering_averaging"]) ** 2 * f * f)
    b[2:4].copy_(torch.fft.ifft2(torch.fft.fft2(b[0:2]) * (g[:, None] * g[None, :])).real)
    px, py = T(d["px"]), T(d["py"])
    px0, py0 = px.clone(), py.clone()
    prev = [T(d["dx_chaotic_prev"]), T(d["dy_chaotic_prev"])]
    out = [torch.zeros(n, n, dtype=torch.float64, device=DEV) for _ in range(2)]
    a = _lib.DeclusteringArgs()
    a.n, a.xi_step = n, float(d["dxi"])
    a.force, a.damping = float(d["declustering_force"]), float(d["damping_declustering"])
    a.limit = float(d["declustering_limit"])
    a.dx_inhom, a.dy_inhom, a.dx_average, a.dy_average = (b[k].data_ptr() for k in range(4))
    a.dx_chaotic_prev, a.dy_chaotic_prev = prev[0].data_ptr(), prev[1].data_ptr()
    a.px, a.py = px.data_ptr(), py.data_ptr()
    a.dx_chaotic, a.dy_chaotic = out[0].data_ptr(), out[1].data_ptr()
    _lib.check(L.lcb_declustering_apply(C.byref(a), st), "apply")
    torch.cuda.synchronize()
    close(N_(out[0]), d["out_dx_chaotic"], 1e-12, "dx_chaotic")
    close(N_(out[1]), d["out_dy_chaotic"], 1e-12, "dy_chaotic")
    close(N_(px), d["out_px"], 1e-12, "px")
    close(N_(py), d["out_py"], 1e-12, "py")
    # the kicks themselves (a small change of px, py), to 1e-9 of their size
    close(N_(px - px0), d["out_px"] - d["px"], 1e-9, "px kick")
    close(N_(py - py0), d["out_py"] - d["py"], 1e-9, "py kick")


def _fields_args(d, precision, ops, outs, ws):
    N = int(d["N"])
    keep = []

    def t(a):
        x = T(a)
        keep.append(x)
        return x.data_ptr()
    a = _lib.ComputeFieldsArgs()
    a.grid_steps, a.h, a.xi_step = N, float(d["h"]), float(d["dxi"])
    a.subtraction_coeff, a.precision = float(d["sub"]), precision
    a.operators = ops.ptr
    for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")):
        a.fields.f[i] = t(d["in_" + k])
        a.fields_prev.f[i] = t(d["prev_" + k])
        a.out_full.f[i] = outs[0][i].data_ptr()
        a.out_half.f[i] = outs[1][i].data_ptr()
    a.currents_prev = _lib.Currents4(*(t(d["cp_" + k]) for k in ("ro", "jx", "jy", "jz")), 2)
    a.currents_full = _lib.Currents4(*(t(d["cf_" + k]) for k in ("ro", "jx", "jy", "jz")), 2)
    a.rho_beam_full, a.rho_beam_prev = t(d["rb_full"]), t(d["rb_prev"])
    a.rho_beam_divisor = 1.0
    a.workspace, a.workspace_bytes = ws.data_ptr(), ws.numel()
    return a, keep


@pytest.mark.parametrize("precision,rel", [(_lib.LCB_PREC_FP64, 1e-11),
                                           (_lib.LCB_PREC_MIXED, 3e-5)])
def test_compute_fields(golden, precision, rel):
    d = golden("kat_fields.npz")
    L = _lib.load()
    N = int(d["N"])
    ops = FieldOperators(N, float(d["h"]), float(d["sub"]), DEV,
                         precision == _lib.LCB_PREC_MIXED)
    outs = [torch.full((7, N, N), 3.0, dtype=torch.float64, device=DEV) for _ in range(2)]
    ws = torch.empty(L.lcb_compute_fields_workspace_bytes(N, precision), dtype=torch.uint8,
                     device=DEV)
    a, keep = _fields_args(d, precision, ops, outs, ws)
    _lib.check(L.lcb_compute_fields(C.byref(a), _lib.stream_handle()), "compute_fields")
    torch.cuda.synchronize()
    for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")):
        close(N_(outs[0][i]), d["full_" + k], rel, "full " + k)
        close(N_(outs[1][i]), d["half_" + k], rel, "half " + k)


@pytest.mark.parametrize("precision,rel", [(_lib.LCB_PREC_FP64, 1e-11),
                                           (_lib.LCB_PREC_MIXED, 3e-5)])
@pytest.mark.parametrize("N", [33, 129, 257, 513])
def test_compute_fields_sizes_vs_oracle(N, precision, rel):
    """Random currents at several grid sizes, up to the production grid 513
    (every tiling of the tensor-core waves: 32- and 64-wide tiles, eight and
    four slices, the stage counts of each grid)."""
    L = _lib.load()
    h, dxi = 0.05, 0.05
    rng = np.random.default_rng(N)
    p = O.Params(N=N, h=h, dxi=dxi, sub_coeff=1 + dxi, boundary=0)
    consts = O.Consts(None, O.dirichlet_matrix(N, h), O.mixed_matrix(N, h, 1 + dxi),
                      O.neumann_matrix(N, h))

    def cur():
        a = np.zeros((2, N, N))
        a[:, 3:-3, 3:-3] = rng.normal(0, 1, (2, N - 6, N - 6))
        return a
    cp = O.Currents(cur(), cur(), cur(), cur())
    cf = O.Currents(cur(), cur(), cur(), cur())
    F = O.Fields(*(rng.normal(0, 1, (N, N)) for _ in range(7)))
    Fp = O.Fields(*(rng.normal(0, 1, (N, N)) for _ in range(7)))
    for f in (F, Fp):  # fields vanish on the walls, as the solver produces them
        for k in ("Ex", "Ey", "Ez", "Bx", "By", "Phi"):
            getattr(f, k)[[0, -1], :] = 0
            getattr(f, k)[:, [0, -1]] = 0
    rbf, rbp = rng.normal(0, 1, (N, N)), rng.normal(0, 1, (N, N))
    full, half = O.compute_fields(p, F, Fp, consts, rbf, rbp, cp, cf)
    d = {"N": N, "h": h, "dxi": dxi, "sub": 1 + dxi, "rb_full": rbf, "rb_prev": rbp}
    for k in ("ro", "jx", "jy", "jz"):
        d["cp_" + k], d["cf_" + k] = getattr(cp, k), getattr(cf, k)
    for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi"):
        d["in_" + k], d["prev_" + k] = getattr(F, k), getattr(Fp, k)
    ops = FieldOperators(N, h, 1 + dxi, DEV, precision == _lib.LCB_PREC_MIXED)
    outs = [torch.zeros((7, N, N), dtype=torch.float64, device=DEV) for _ in range(2)]
    ws = torch.empty(L.lcb_compute_fields_workspace_bytes(N, precision), dtype=torch.uint8,
                     device=DEV)
    a, keep = _fields_args(d, precision, ops, outs, ws)
    _lib.check(L.lcb_compute_fields(C.byref(a), _lib.stream_handle()), "compute_fields")
    torch.cuda.synchronize()
    for i, k in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")):
        close(N_(outs[0][i]), getattr(full, k), rel, f"N={N} full {k}")
        close(N_(outs[1][i]), getattr(half, k), rel, f"N={N} half {k}")


def test_beam_deposit_and_substepping(kat):
    d = kat
    L = _lib.load()
    N, h, dxi = int(d["N"]), float(d["h"]), float(d["dxi"])
    x, y, xi, q = (T(d[k]) for k in ("b_x", "b_y", "b_xi", "b_q"))
    r0 = torch.zeros(N, N, dtype=torch.float64, device=DEV)
    r1 = torch.zeros_like(r0)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    _lib.check(L.lcb_beam_deposit(x.numel(), N, h, dxi, int(d["b_layer"]), x.data_ptr(),
                                  y.data_ptr(), xi.data_ptr(), q.data_ptr(), r0.data_ptr(),
                                  r1.data_ptr(), err.data_ptr(), _lib.stream_handle()), "k4")
    qm, pz = T(d["k6_qm"]), T(d["k6_pz"])
    dt = torch.zeros_like(qm)
    rs = torch.zeros(qm.numel(), dtype=torch.int64, device=DEV)
    _lib.check(L.lcb_beam_substepping(qm.numel(), qm.data_ptr(), pz.data_ptr(), 2.0, 1.0,
                                      dt.data_ptr(), rs.data_ptr(), _lib.stream_handle()), "k6")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    close(N_(r0), d["k4_ro0"], 1e-12, "K4 ro0")
    close(N_(r1), d["k4_ro1"], 1e-12, "K4 ro1")
    np.testing.assert_array_equal(N_(dt), d["k6_dt"])
    np.testing.assert_array_equal(N_(rs), (1.0 / d["k6_dt"]).astype(np.int64))


def test_beam_move_vs_oracle():
    """Substepped Higuera-Cary push of a layer against the oracle restatement,
    including particles that fall to the next layer and particles lost at the
    wall."""
    L = _lib.load()
    N, h, dxi = 65, 0.05, 0.05
    p = O.Params(N=N, h=h, dxi=dxi, sub_coeff=1, boundary=0)
    rng = np.random.default_rng(11)
    n = 3000
    layer = 9
    b = O.Beam(xi=rng.uniform(-(layer) * dxi, -(layer - 1) * dxi, n),
               x=rng.normal(0, 0.5, n), y=rng.normal(0, 0.5, n),
               px=rng.normal(0, 5, n), py=rng.normal(0, 5, n),
               pz=rng.choice([-50.0, 0.3, 20.0, 1000.0], n),
               q_m=rng.choice([-1.0, 1.0, 1 / 1836.0], n), q_norm=np.ones(n),
               id=np.arange(1, n + 1, dtype=np.int64), dt=np.zeros(n),
               remaining_steps=np.zeros(n, np.int64))
    b.x[:20] = 1.4  # near / beyond the loss radius
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    Fk = O.Fields(*(0.3 * np.sin(0.2 * (i + 1) * X + 0.1 * Y) for i in range(6)), np.zeros((N, N)))
    Fk1 = O.Fields(*(0.3 * np.cos(0.15 * (i + 1) * Y - 0.1 * X) for i in range(6)), np.zeros((N, N)))
    g = {k: T(getattr(b, k)) for k in ("xi", "x", "y", "px", "py", "pz", "q_m")}
    g["id"] = T(b.id, torch.int64)
    g["dt"] = torch.zeros(n, dtype=torch.float64, device=DEV)
    g["rs"] = torch.zeros(n, dtype=torch.int64, device=DEV)
    fell_size = 200
    rs0 = rng.integers(1, 4, fell_size)
    dt0 = 1.0 / rs0
    b.remaining_steps[n - fell_size:] = rs0
    b.dt[n - fell_size:] = dt0
    g["rs"][n - fell_size:] = T(rs0, torch.int64)
    g["dt"][n - fell_size:] = T(dt0)
    lost, moved, fell = O.move_beam_layer(p, b, fell_size, layer, Fk, Fk1, 1.0, 2.0)
    _lib.check(L.lcb_beam_substepping(n - fell_size, g["q_m"].data_ptr(), g["pz"].data_ptr(),
                                      2.0, 1.0, g["dt"].data_ptr(), g["rs"].data_ptr(),
                                      _lib.stream_handle()), "k6")
    fk = [T(getattr(Fk, k)) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")]
    fk1 = [T(getattr(Fk1, k)) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")]
    s0, s1 = _lib.Fields7(), _lib.Fields7()
    for i in range(7):
        s0.f[i], s1.f[i] = fk[i].data_ptr(), fk1[i].data_ptr()
    flags = torch.zeros(n, dtype=torch.uint8, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    R = h * N / 2
    _lib.check(L.lcb_beam_move(n, dxi, max(0.9 * R, R - 1), layer - 1, h, N,
                               g["q_m"].data_ptr(), g["dt"].data_ptr(), s0, s1,
                               g["rs"].data_ptr(), g["id"].data_ptr(), g["x"].data_ptr(),
                               g["y"].data_ptr(), g["xi"].data_ptr(), g["px"].data_ptr(),
                               g["py"].data_ptr(), g["pz"].data_ptr(), flags.data_ptr(),
                               err.data_ptr(), _lib.stream_handle()), "k5")
    torch.cuda.synchronize()
    fl = N_(flags)
    for sel, ref in ((fl & 1, lost), (fl & 2, moved), (fl & 4, fell)):
        idx = np.nonzero(sel)[0]
        np.testing.assert_array_equal(N_(g["id"])[idx], ref.id)
        for k in ("x", "y", "xi", "px", "py", "pz"):
            close(N_(g[k])[idx], getattr(ref, k), 1e-11, k)
    assert lost.size > 0 and moved.size > 0 and fell.size > 0


def _op_layout(N, mixed=False):
    n = N - 2
    se, so, ce, co = (n + 1) // 2, (n - 1) // 2, (N + 1) // 2, (N - 1) // 2
    shapes = [(se, se), (so, so), (se, se), (so, so), (ce, ce), (co, co), (ce, ce), (co, co),
              (n, n), (n, N), (N, n), (N, N)]
    offs, lds, o = [], [], 0
    for i, (r, c) in enumerate(shapes):
        # transform blocks: even row stride (FP64), or four tiled int8 slice planes
        ld = c
        offs.append(o)
        lds.append(ld)
        words = _plane_bytes(i, r, c) if i < 8 else r * ld
        o += (words + 31) // 32 * 32
    return shapes, offs, lds


def _tiles(x, t):
    return (x + t - 1) // t


def _a_role(i):
    return i in (0, 1, 4, 5)   # SE SO CE CO: left operators


def _plane_bytes(i, r, c):
    if _a_role(i):
        return _tiles(r, 128) * _tiles(c, 32) * 4096
    return _tiles(r, 32) * _tiles(c, 64) * 2048


def _tile_offsets(i, r, c, ns, k):
    """Byte offset of slice k of every element (row, col) of a tiled block
    (the ns slices of a tile are stored back to back)."""
    R, Cc = np.meshgrid(np.arange(r), np.arange(c), indexing="ij")
    if _a_role(i):
        KT = _tiles(c, 32)
        return ((((R >> 7) * KT + (Cc >> 5)) * ns + k) << 12) + ((R & 127) >> 3) * 256 + \
            ((Cc & 31) >> 4) * 128 + (R & 7) * 16 + (Cc & 15)
    KT = _tiles(r, 32)
    return ((((Cc >> 6) * KT + (R >> 5)) * ns + k) << 11) + ((Cc & 63) >> 4) * 512 + \
        ((R & 31) >> 3) * 128 + (R & 7) * 16 + (Cc & 15)


@pytest.mark.parametrize("N,mixed", [(33, False), (129, False), (65, True)])
def test_field_operators_build(N, mixed):
    """Device-built folded DST-I/DCT-I blocks and solver matrices against numpy."""
    from scipy import fft as sfft
    h, c = 0.05, 1.05
    ops = FieldOperators(N, h, c, DEV, mixed)
    torch.cuda.synchronize()
    dt = np.float32 if mixed else np.float64
    buf = ops.buf.cpu().numpy().view(dt)
    n = N - 2
    S = sfft.dst(np.eye(n), type=1, axis=0)   # column j = DST-I of e_j
    Cm = sfft.dct(np.eye(N), type=1, axis=0)
    blocks = [S[0::2, :(n + 1) // 2], S[1::2, :(n - 1) // 2]]
    blocks += [blocks[0].T, blocks[1].T]
    cb = [Cm[0::2, :(N + 1) // 2], Cm[1::2, :(N - 1) // 2]]
    blocks += cb + [cb[0].T, cb[1].T]
    blocks += [O.dirichlet_matrix(N, h), O.mixed_matrix(N, h, c), O.mixed_matrix(N, h, c).T,
               O.neumann_matrix(N, h)]
    shapes, offs, lds = _op_layout(N, mixed)
    rel = 1e-6 if mixed else 1e-13
    raw = ops.buf.cpu().numpy().view(np.uint8)
    ns = 4 if mixed else 8          # slices per element = bytes per element
    for i, (ref, shp, off, ld) in enumerate(zip(blocks, shapes, offs, lds)):
        if i < 8:
            # ns int8 slices per element in tiles, x = 2 sum_k s_k 2^-(6 + 7 k)
            plane = _plane_bytes(i, *shp)
            blk = raw[ns * off:ns * off + ns * plane].view(np.int8)
            planes = [blk[_tile_offsets(i, *shp, ns, k)].astype(np.float64) for k in range(ns)]
            got = 2 * sum(p * 2.0 ** -(6 + 7 * k) for k, p in enumerate(planes))
            # FP32 rounding of the value, then exact slices (mixed); FP64
            rel_b = 2.0 ** -23 if mixed else 1e-15
        else:
            got = buf[off:off + shp[0] * ld].reshape(shp[0], ld)[:, :shp[1]]
            rel_b = rel
        close(got.astype(np.float64), ref, rel_b, f"operator block {i}")


@pytest.mark.parametrize("tag", ["t1", "t5"])
def test_beam_move_vs_reference_kernel(golden, tag):
    """lcb_beam_substepping + lcb_beam_move against the reference's own GPU
    kernels (calculate_substepping_step and move_beam_cupy, compiled for the
    host from the reference's sources: tests/golden/make_ref_kernel_golden.py)
    on a layer with particles that stay, fall to the next layer and are lost."""
    d = golden("kat_ref_beam.npz")
    L = _lib.load()
    N, h, dxi, layer, fell_size, time_step, sub_e = d[f"{tag}_params"]
    N, layer, fell_size = int(N), int(layer), int(fell_size)
    g = {k: T(d[f"{tag}_in_{k}"]) for k in ("xi", "x", "y", "px", "py", "pz", "q_m", "dt")}
    g["id"] = T(d[f"{tag}_in_id"], torch.int64)
    g["rs"] = T(d[f"{tag}_in_remaining_steps"], torch.int64)
    n = g["x"].numel()
    _lib.check(L.lcb_beam_substepping(n - fell_size, g["q_m"].data_ptr(), g["pz"].data_ptr(),
                                      float(sub_e), float(time_step), g["dt"].data_ptr(),
                                      g["rs"].data_ptr(), _lib.stream_handle()), "k6")
    keys = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")
    fk = [T(d[f"{tag}_fk_{k}"]) for k in keys] + [torch.zeros(N, N, dtype=torch.float64, device=DEV)]
    fk1 = [T(d[f"{tag}_fk1_{k}"]) for k in keys] + [torch.zeros(N, N, dtype=torch.float64, device=DEV)]
    s0, s1 = _lib.Fields7(), _lib.Fields7()
    for i in range(7):
        s0.f[i], s1.f[i] = fk[i].data_ptr(), fk1[i].data_ptr()
    flags = torch.zeros(n, dtype=torch.uint8, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    R = h * N / 2
    _lib.check(L.lcb_beam_move(n, float(dxi), max(0.9 * R, R - 1), layer - 1, float(h), N,
                               g["q_m"].data_ptr(), g["dt"].data_ptr(), s0, s1,
                               g["rs"].data_ptr(), g["id"].data_ptr(), g["x"].data_ptr(),
                               g["y"].data_ptr(), g["xi"].data_ptr(), g["px"].data_ptr(),
                               g["py"].data_ptr(), g["pz"].data_ptr(), flags.data_ptr(),
                               err.data_ptr(), _lib.stream_handle()), "k5")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    fl = N_(flags)
    np.testing.assert_array_equal((fl & 1) != 0, d[f"{tag}_lost"])
    np.testing.assert_array_equal((fl & 2) != 0, d[f"{tag}_moved"])
    np.testing.assert_array_equal((fl & 4) != 0, d[f"{tag}_fell"])
    np.testing.assert_array_equal(N_(g["id"]), d[f"{tag}_out_id"])
    np.testing.assert_array_equal(N_(g["rs"]), d[f"{tag}_out_remaining_steps"])
    np.testing.assert_array_equal(N_(g["dt"]), d[f"{tag}_out_dt"])
    for k in ("x", "y", "xi", "px", "py", "pz"):
        close(N_(g[k]), d[f"{tag}_out_{k}"], 1e-11, k)


def test_beam_deposit_vs_reference_kernel(golden):
    """lcb_beam_deposit against the reference's deposit_beam_cupy (compiled
    for the host from the reference's sources)."""
    d = golden("kat_ref_beam.npz")
    L = _lib.load()
    N, h, dxi, layer = d["dep_params"]
    N, layer = int(N), int(layer)
    x, y, xi, q = (T(d[k]) for k in ("dep_x", "dep_y", "dep_xi", "dep_q"))
    r0 = T(d["dep_ro0_in"])
    r1 = torch.zeros(N, N, dtype=torch.float64, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    _lib.check(L.lcb_beam_deposit(x.numel(), N, float(h), float(dxi), layer, x.data_ptr(),
                                  y.data_ptr(), xi.data_ptr(), q.data_ptr(), r0.data_ptr(),
                                  r1.data_ptr(), err.data_ptr(), _lib.stream_handle()), "k4")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    close(N_(r0), d["dep_ro0"], 1e-12, "ro0")
    close(N_(r1), d["dep_ro1"], 1e-12, "ro1")
