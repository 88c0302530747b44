"""The oracle's particle loops against the reference's own GPU kernel bodies
(the CuPy ElementwiseKernel strings of lcode/beam3d and lcode/plasma3d,
compiled for the host by oracle/ref_kernels.py from the reference checkout).

This pins the oracle's beam pusher to the Higuera-Cary kernel the drop-in
replaces (lcode/beam3d/move.py:139-276): the reference's CPU pusher is a
different algorithm, and CuPy cannot run here, so the kernel body itself is
the only reference artefact for it.  The plasma kernels K1/K2/K3 and the beam
deposit / substepping are checked the same way (they are also pinned by the
numba known answers in tests/golden/kat_kernels.npz).

Both sides run serially in FP64 without FMA contraction.  The oracle's beam
kernels restate the GPU kernels in their operation order, so they are
compared bit for bit.  The oracle's plasma kernels follow the reference's
numba kernels (pinned by the reference's golden runs), which sum gamma in
another order than the CuPy strings (m^2 + pz^2 + px^2 + py^2 against
m^2 + px^2 + py^2 + pz^2); they are compared within 1e-13 of the largest
element."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_kernels as R

pytestmark = pytest.mark.skipif(not R.available(),
                                reason="reference checkout (LCODE_REFERENCE) not present")


def _fields(N, seed):
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    a = 0.2 + 0.05 * seed
    return O.Fields(*(0.3 * np.sin(a * (i + 1) * X + 0.1 * Y + seed) for i in range(6)),
                    np.zeros((N, N)))


def _layer(rng, n, layer, dxi):
    """A beam layer with particles that stay (moved), fall to the next layer
    (slow pz), and hit the loss radius (placed near the wall)."""
    b = O.Beam(xi=rng.uniform(-layer * dxi, -(layer - 1) * dxi, n),
               x=rng.normal(0, 0.5, n), y=rng.normal(0, 0.5, n),
               px=rng.normal(0, 5, n), py=rng.normal(0, 5, n),
               pz=rng.choice([-50.0, 0.3, 20.0, 1000.0], n),
               q_m=rng.choice([-1.0, 1.0, 1 / 1836.0, -0.3], n), q_norm=rng.uniform(0.5, 1.5, n),
               id=np.arange(1, n + 1, dtype=np.int64), dt=np.zeros(n),
               remaining_steps=np.zeros(n, np.int64))
    b.x[:20] = 1.4
    return b


@pytest.mark.parametrize("seed,time_step", [(0, 1.0), (1, 5.0), (2, 0.25)])
def test_beam_push_matches_reference_kernel(seed, time_step):
    N, h, dxi = 65, 0.05, 0.05
    p = O.Params(N=N, h=h, dxi=dxi, sub_coeff=1, boundary=0)
    rng = np.random.default_rng(100 + seed)
    n, layer, fell_size = 4000, 9, 300
    b = _layer(rng, n, layer, dxi)
    rs0 = rng.integers(1, 4, fell_size)
    b.remaining_steps[n - fell_size:] = rs0
    b.dt[n - fell_size:] = time_step / rs0
    Fk, Fk1 = _fields(N, seed), _fields(N, seed + 7)

    # the reference: substepping of the particles that did not fall from the
    # previous layer (beam_calculator.py:97-114), then move_beam_cupy
    r = {k: getattr(b, k).copy() for k in ("x", "y", "xi", "px", "py", "pz", "q_m", "id",
                                           "dt", "remaining_steps")}
    size = n - fell_size
    dt1 = R.substepping(r["q_m"][:size].copy(), r["pz"][:size].copy(), 2.0)
    r["dt"][:size] = dt1 * time_step
    r["remaining_steps"][:size] = (1.0 / dt1).astype(np.int64)
    R_ = h * N / 2
    keys6 = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")
    lost, moved, fell = R.move_beam(dxi, max(0.9 * R_, R_ - 1), layer - 1, h, N, r["q_m"],
                                    r["dt"], [getattr(Fk, k) for k in keys6],
                                    [getattr(Fk1, k) for k in keys6], r["remaining_steps"],
                                    r["id"], r["x"], r["y"], r["xi"], r["px"], r["py"], r["pz"])
    assert lost.sum() > 0 and moved.sum() > 0 and fell.sum() > 0

    o_lost, o_moved, o_fell = O.move_beam_layer(p, b, fell_size, layer, Fk, Fk1, time_step, 2.0)
    for sel, ob in ((lost, o_lost), (moved, o_moved), (fell, o_fell)):
        np.testing.assert_array_equal(r["id"][sel], ob.id)
        for k in ("x", "y", "xi", "px", "py", "pz", "dt", "remaining_steps"):
            np.testing.assert_array_equal(r[k][sel], getattr(ob, k), err_msg=k)


def test_beam_deposit_matches_reference_kernel():
    N, h, dxi, layer = 65, 0.05, 0.05, 7
    rng = np.random.default_rng(5)
    n = 5000
    x, y = rng.normal(0, 0.4, n), rng.normal(0, 0.4, n)
    xi = rng.uniform(-layer * dxi - dxi, -layer * dxi, n)
    q = rng.uniform(-1, 1, n)
    ro0, ro1 = rng.normal(0, 1, (N, N)), np.zeros((N, N))
    r0, r1 = ro0.copy(), ro1.copy()
    # beam3d/weights.py:152-163: xi_loc and x_h, y_h as the caller forms them
    xi_loc = (-dxi * layer - xi) / dxi
    R.deposit_beam(N, x / h + 0.5, y / h + 0.5, xi_loc, q, r0, r1)
    b = O.Beam(xi=xi, x=x, y=y, px=np.zeros(n), py=np.zeros(n), pz=np.zeros(n),
               q_m=np.ones(n), q_norm=q, id=np.arange(n), dt=np.zeros(n),
               remaining_steps=np.zeros(n, np.int64))
    O.deposit_beam(O.Params(N=N, h=h, dxi=dxi, sub_coeff=1, boundary=0), layer, b, ro0, ro1)
    np.testing.assert_array_equal(r0, ro0)
    np.testing.assert_array_equal(r1, ro1)


def _plasma(rng, N, h, boundary):
    Ns = N - 30
    g = O.plasma_grid(Ns, h, 2)
    y0 = np.ascontiguousarray(np.broadcast_to(g, (g.size, g.size)))
    x0 = np.ascontiguousarray(y0.T)
    sh = x0.shape
    xo = np.clip(x0 + rng.uniform(-0.3, 0.3, sh), -boundary * 1.05, boundary * 1.05) - x0
    yo = np.clip(y0 + rng.uniform(-0.3, 0.3, sh), -boundary * 1.05, boundary * 1.05) - y0
    return O.Sort(x0, y0, xo, yo, rng.normal(0, 0.3, sh), rng.normal(0, 0.3, sh),
                  rng.normal(0, 0.3, sh), np.full(sh, -h * h / 4), np.full(sh, h * h / 4))


def _close(a, b, what, rel=1e-13):
    err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    assert err <= rel, f"{what}: {err:.2e}"


def test_plasma_kernels_match_reference_kernels():
    N, h, dxi = 65, 0.05, 0.05
    p = O.Params(N=N, h=h, dxi=dxi, sub_coeff=1, boundary=h * (N / 2 - 10))
    rng = np.random.default_rng(9)
    prev = _plasma(rng, N, h, p.boundary)
    F = _fields(N, 3)
    keys6 = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")

    # K1: move_wo_fields_cupy on a copy (move.py:331-349)
    full_o = O.move_wo_fields(p, prev)
    full_r = prev.copy()
    R.move_wo_fields(dxi, full_r.m, full_r.x_offt, full_r.y_offt, full_r.px, full_r.py,
                     full_r.pz)
    for k in ("x_offt", "y_offt"):
        _close(getattr(full_r, k), getattr(full_o, k), "K1 " + k)

    # K2: move_smart_cupy, reading and writing the full arrays (move.py:351-381)
    O.move_smart(p, F, prev, full_o)
    R.move_smart(dxi, p.boundary, h, N, [getattr(F, k) for k in keys6], prev.x_init,
                 prev.y_init, prev.x_offt, prev.y_offt, prev.px, prev.py, prev.pz, full_r.m,
                 full_r.q, full_r.x_offt, full_r.y_offt, full_r.px, full_r.py, full_r.pz)
    assert ((full_r.px == 0) & (prev.px != 0)).any()   # some particles reflected at the wall
    np.testing.assert_array_equal(full_r.q, full_o.q)
    for k in ("x_offt", "y_offt", "px", "py", "pz"):
        _close(getattr(full_r, k), getattr(full_o, k), "K2 " + k)

    # K3: deposit_plasma_cupy with x_h, y_h formed as weights.py:270-273 forms them
    cur = O.Currents.zeros(N)
    O.deposit_sort(p, full_o, cur, 0)
    ro, jx, jy, jz = (np.zeros((N, N)) for _ in range(4))
    R.deposit_plasma(N, h, np.ascontiguousarray((full_r.x_init + full_r.x_offt) / h + 0.5),
                     np.ascontiguousarray((full_r.y_init + full_r.y_offt) / h + 0.5),
                     full_r.px, full_r.py, full_r.pz, full_r.q, full_r.m, ro, jx, jy, jz)
    for a, k in ((ro, "ro"), (jx, "jx"), (jy, "jy"), (jz, "jz")):
        _close(a, getattr(cur, k)[0], "K3 " + k)
