"""CPU oracle for the quasistatic 3D xi step -- TEST INFRASTRUCTURE ONLY.

This module restates the reference lcodePy 3D algorithm (FP64) on the CPU:
particle loops in C (``lcb_oracle.c``, loaded through ctypes) and the host
logic and field transforms in numpy/scipy.  It is the checker for the CUDA
product: only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline arm may import it.  The product package never imports it.

Every function cites the reference routine it follows (paths relative to the
lcodePy project root).  The field transforms use ``scipy.fft`` DST-I / DCT-I,
the same unnormalised transforms the reference takes from ``scipy.fftpack``
(``lcode/plasma3d/fields.py:16-31``).

Parity of this oracle is pinned against the reference's own golden states
``tests/integration/data/3D_test1.npz`` and ``3D_beam_evol.npz`` and against
fixtures produced by running the reference here (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np
from scipy import fft as sfft

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblcb_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> str:
    """Compile lcb_oracle.c into liblcb_oracle.so next to it (gcc, OpenMP)."""
    src = os.path.join(_HERE, "lcb_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or \
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
             "-fno-fast-math", "-o", _LIB_PATH, src, "-lm"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_oob_count.restype = ctypes.c_int64
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.int64:
        return a.ctypes.data_as(_i64p)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_u8p)
    raise TypeError(a.dtype)


def num_threads() -> int:
    return int(lib().orc_num_threads())


# --------------------------------------------------------------------------
# Config arithmetic (lcode/config/config.py)
# --------------------------------------------------------------------------

def _factor(n):
    out, d = [], 2
    while n > 1:
        while n % d == 0:
            out.append(d)
            n //= d
        d += 1
    return out


def good_size(n: int) -> bool:
    """FFTW-friendly odd size test, lcode/config/config.py:239-258."""
    fs = _factor(n - 1)
    return (all(f in (2, 3, 4, 5, 7, 11, 13) for f in fs)
            and fs.count(11) + fs.count(13) < 2 and n % 2 == 1)


def grid_steps_for(window_width: float, h: float) -> int:
    """window-width-steps after the 3D adjustment, config.py:185-220
    (the half-width is doubled, then snapped to the closest good size)."""
    est = int(2 * window_width / h)
    lo = max(est - 100, 0)
    cands = np.array([a for a in range(lo, est + 100) if good_size(a)])
    return int(cands[np.abs(cands - est).argmin()])


# --------------------------------------------------------------------------
# Solver matrices (lcode/plasma3d/initialization.py:15-67)
# --------------------------------------------------------------------------

def _lam(k, N, h):
    return 4 / h ** 2 * np.sin(k * np.pi / (2 * (N - 1))) ** 2


def dirichlet_matrix(N, h):
    lam = _lam(np.arange(1, N - 1), N, h)
    return 1 / (lam[:, None] + lam[None, :]) / (2 * (N - 1)) ** 2


def mixed_matrix(N, h, c):
    li = _lam(np.arange(1, N - 1), N, h)
    lj = _lam(np.arange(N), N, h)
    return 1 / (li[:, None] + lj[None, :] + c) / (2 * (N - 1)) ** 2


def neumann_matrix(N, h):
    lam = _lam(np.arange(N), N, h)
    with np.errstate(divide="ignore"):
        mul = 1 / (lam[:, None] + lam[None, :])
    mul[0, 0] = 0
    return mul / (2 * (N - 1)) ** 2


# --------------------------------------------------------------------------
# Plasma initial state (lcode/plasma3d/initialization.py:72-135,278-414,
# lcode/plasma3d/profile.py) -- uniform profile only in the oracle.
# --------------------------------------------------------------------------

def plasma_grid(steps, h, fineness):
    """Particle lattice coordinates, initialization.py:72-104."""
    step = h / fineness
    if fineness % 2:
        right = np.arange(steps // 2 * fineness) * step
        left = -right[:0:-1]
    else:
        right = (0.5 + np.arange(steps // 2 * fineness)) * step
        left = -right[::-1]
    return np.concatenate([left, right])


@dataclass
class Sort:
    x_init: np.ndarray
    y_init: np.ndarray
    x_offt: np.ndarray
    y_offt: np.ndarray
    px: np.ndarray
    py: np.ndarray
    pz: np.ndarray
    q: np.ndarray
    m: np.ndarray

    def copy(self) -> "Sort":
        return Sort(*(getattr(self, f).copy() for f in self.__dataclass_fields__))


@dataclass
class Params:
    N: int
    h: float
    dxi: float
    sub_coeff: float
    boundary: float
    ion_model: str = "background"


@dataclass
class Fields:
    Ex: np.ndarray
    Ey: np.ndarray
    Ez: np.ndarray
    Bx: np.ndarray
    By: np.ndarray
    Bz: np.ndarray
    Phi: np.ndarray

    @staticmethod
    def zeros(N):
        return Fields(*(np.zeros((N, N)) for _ in range(7)))

    def copy(self):
        return Fields(*(getattr(self, f).copy() for f in self.__dataclass_fields__))


@dataclass
class Currents:
    ro: np.ndarray
    jx: np.ndarray
    jy: np.ndarray
    jz: np.ndarray

    @staticmethod
    def zeros(N):
        return Currents(*(np.zeros((2, N, N)) for _ in range(4)))


@dataclass
class Consts:
    ro_initial: np.ndarray
    dirichlet: np.ndarray
    mixed: np.ndarray
    neumann: np.ndarray


def make_params(window_width, h, dxi, bound_padding=10, sub_coeff=1,
                ion_model="background") -> Params:
    """Parameters as the reference's 3D config adjustment leaves them,
    config.py:185-196: the subtraction coefficient becomes 1 + dxi only when
    its string form is exactly '1' (so 1.0 stays 1.0)."""
    N = grid_steps_for(window_width, h)
    c = 1 + dxi if str(sub_coeff) == "1" else float(sub_coeff)
    return Params(N=N, h=h, dxi=dxi, sub_coeff=c,
                  boundary=h * (N / 2 - bound_padding), ion_model=ion_model)


def init_plasma(p: Params, ppc=4, plasma_padding=15, ion_mass=1836.0):
    """Uniform cold plasma, initialization.py:278-414 (legacy uniform shape).
    Returns (sorts list, consts); sort 0 is electrons, sort 1 (mobile ions)."""
    f = int(round(np.sqrt(ppc)))
    g = plasma_grid(p.N - 2 * plasma_padding, p.h, f)
    Ns = len(g)
    y_init = np.ascontiguousarray(np.broadcast_to(g, (Ns, Ns)))
    x_init = np.ascontiguousarray(y_init.T)
    q = np.ones((Ns, Ns)) * -1 / f ** 2 * p.h ** 2
    m = np.ones((Ns, Ns)) * 1 / f ** 2 * p.h ** 2
    z = lambda: np.zeros((Ns, Ns))
    el = Sort(x_init, y_init, z(), z(), z(), z(), z(), q, m)
    ro0 = Currents.zeros(p.N)
    deposit_sort(p, el, ro0, 0)
    consts = Consts(ro_initial=-ro0.ro[0].copy(),
                    dirichlet=dirichlet_matrix(p.N, p.h),
                    mixed=mixed_matrix(p.N, p.h, p.sub_coeff),
                    neumann=neumann_matrix(p.N, p.h))
    sorts = [el]
    if p.ion_model == "mobile":
        sorts.append(Sort(x_init.copy(), y_init.copy(), z(), z(), z(), z(), z(),
                          -q.copy(), ion_mass * m.copy()))
    return sorts, consts


# --------------------------------------------------------------------------
# Particle kernels (C)
# --------------------------------------------------------------------------

def move_wo_fields(p: Params, s: Sort):
    """Copy then free-stream, plasma3d/move.py:331-349."""
    f = s.copy()
    lib().orc_move_wo_fields(ctypes.c_int64(f.m.size), ctypes.c_double(p.dxi),
                             _p(f.m), _p(f.x_offt), _p(f.y_offt), _p(f.px),
                             _p(f.py), _p(f.pz))
    return f


def move_smart(p: Params, F: Fields, prev: Sort, full: Sort):
    """K2 on one sort, plasma3d/move.py:351-381 (in-place on `full`)."""
    lib().orc_move_smart(
        ctypes.c_int64(prev.m.size), ctypes.c_double(p.dxi),
        ctypes.c_double(p.boundary), ctypes.c_double(p.h), ctypes.c_int(p.N),
        _p(F.Ex), _p(F.Ey), _p(F.Ez), _p(F.Bx), _p(F.By), _p(F.Bz),
        _p(prev.x_init), _p(prev.y_init), _p(prev.x_offt), _p(prev.y_offt),
        _p(prev.px), _p(prev.py), _p(prev.pz), _p(full.m), _p(full.q),
        _p(full.x_offt), _p(full.y_offt), _p(full.px), _p(full.py), _p(full.pz))


def deposit_sort(p: Params, s: Sort, cur: Currents, column: int):
    """K3 for one sort into column `column`, plasma3d/weights.py:249-285."""
    lib().orc_deposit_plasma(
        ctypes.c_int64(s.m.size), ctypes.c_int(p.N), ctypes.c_double(p.h),
        _p(s.x_init), _p(s.y_init), _p(s.x_offt), _p(s.y_offt),
        _p(s.px), _p(s.py), _p(s.pz), _p(s.q), _p(s.m),
        _p(cur.ro[column]), _p(cur.jx[column]), _p(cur.jy[column]),
        _p(cur.jz[column]))


def compute_rhoj(p: Params, sorts, consts: Consts) -> Currents:
    """plasma3d/rhoj.py:11-20."""
    cur = Currents.zeros(p.N)
    for col, s in enumerate(sorts):
        deposit_sort(p, s, cur, col)
    if p.ion_model == "background":
        cur.ro[1] = consts.ro_initial
    return cur


# --------------------------------------------------------------------------
# Field solver (plasma3d/fields.py)
# --------------------------------------------------------------------------

def dst2d(a):
    return sfft.dstn(a, type=1)


def dct2d(a):
    return sfft.dctn(a, type=1)


def mix2d(a):
    """DST-I along axis 0, DCT-I along axis 1, zero row on each side,
    fields.py:19-31."""
    out = sfft.dct(sfft.dst(a, type=1, axis=0), type=1, axis=1)
    return np.pad(out, ((1, 1), (0, 0)))


def _dx_dy(a, h):
    dx, dy = np.zeros_like(a), np.zeros_like(a)
    dx[1:-1, 1:-1] = a[2:, 1:-1] - a[:-2, 1:-1]
    dy[1:-1, 1:-1] = a[1:-1, 2:] - a[1:-1, :-2]
    return dx / (h * 2), dy / (h * 2)


def compute_fields(p: Params, F: Fields, Fprev: Fields, consts: Consts,
                   rb_full, rb_prev, cprev: Currents, cfull: Currents):
    """fields.py:276-322 (with calculate_* at :112-266)."""
    h = p.h
    cf = {k: getattr(cfull, k).sum(axis=0) for k in ("ro", "jx", "jy", "jz")}
    cp = {k: getattr(cprev, k).sum(axis=0) for k in ("ro", "jx", "jy", "jz")}
    ro_half = (cf["ro"] + rb_full + cp["ro"] + rb_prev) / 2
    jz_half = (cf["jz"] + rb_full + cp["jz"] + rb_prev) / 2
    dro_dx, dro_dy = _dx_dy(ro_half, h)
    djz_dx, djz_dy = _dx_dy(jz_half, h)
    djx_dxi = (cp["jx"] - cf["jx"]) / p.dxi
    djy_dxi = (cp["jy"] - cf["jy"]) / p.dxi
    c = p.sub_coeff
    Ex_rhs = -(dro_dx - djx_dxi - c * F.Ex)
    Ey_rhs = -(dro_dy - djy_dxi - c * F.Ey)
    Bx_rhs = +(djz_dy - djy_dxi + c * F.Bx)
    By_rhs = -(djz_dx - djx_dxi - c * F.By)
    M = consts.mixed
    Ey = mix2d(M * mix2d(Ey_rhs[1:-1, :])[1:-1, :])
    Bx = mix2d(M * mix2d(Bx_rhs[1:-1, :])[1:-1, :])
    By = np.ascontiguousarray(mix2d(M * mix2d(By_rhs.T[1:-1, :])[1:-1, :]).T)
    Ex = np.ascontiguousarray(mix2d(M * mix2d(Ex_rhs.T[1:-1, :])[1:-1, :]).T)

    jx, jy = cf["jx"], cf["jy"]
    rhs = -((jx[2:, 1:-1] - jx[:-2, 1:-1]) + (jy[1:-1, 2:] - jy[1:-1, :-2])) / (h * 2)
    Ez = np.pad(dst2d(dst2d(rhs) * consts.dirichlet), 1)

    djx_dy = np.pad(jx[1:-1, 2:] - jx[1:-1, :-2], 1)
    djy_dx = np.pad(jy[2:, 1:-1] - jy[:-2, 1:-1], 1)
    rhs = -(djx_dy - djy_dx) / (h * 2)
    Bz = dct2d(dct2d(rhs) * consts.neumann)
    Bz -= Bz.mean()

    Phi = np.pad(dst2d(dst2d((cf["ro"] - cf["jz"])[1:-1, 1:-1]) * consts.dirichlet), 1)

    full = Fields(2 * Ex - Fprev.Ex, 2 * Ey - Fprev.Ey, Ez,
                  2 * Bx - Fprev.Bx, 2 * By - Fprev.By, Bz, Phi)
    half = Fields(Ex, Ey, (Ez + Fprev.Ez) / 2, Bx, By, (Bz + Fprev.Bz) / 2, Phi)
    return full, half


def step_dxi(p: Params, sorts, F: Fields, cur: Currents, consts: Consts,
             rb_full, rb_prev):
    """Predictor-corrector, plasma3d/solver.py:25-78 (no noise filter)."""
    full = [move_wo_fields(p, s) for s in sorts]
    for s, f in zip(sorts, full):
        move_smart(p, F, s, f)
    cfull = compute_rhoj(p, full, consts)
    _, half = compute_fields(p, F, F, consts, rb_full, rb_prev, cur, cfull)
    for s, f in zip(sorts, full):
        move_smart(p, half, s, f)
    cfull = compute_rhoj(p, full, consts)
    Ffull, half = compute_fields(p, half, F, consts, rb_full, rb_prev, cur, cfull)
    for s, f in zip(sorts, full):
        move_smart(p, half, s, f)
    cfull = compute_rhoj(p, full, consts)
    return full, Ffull, cfull


# --------------------------------------------------------------------------
# Beam (beam3d/*)
# --------------------------------------------------------------------------

BEAM_KEYS = ("xi", "x", "y", "px", "py", "pz", "q_m", "q_norm", "id")


@dataclass
class Beam:
    """SoA beam, beam3d/data.py:21-178."""
    xi: np.ndarray = field(default_factory=lambda: np.zeros(0))
    x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    px: np.ndarray = field(default_factory=lambda: np.zeros(0))
    py: np.ndarray = field(default_factory=lambda: np.zeros(0))
    pz: np.ndarray = field(default_factory=lambda: np.zeros(0))
    q_m: np.ndarray = field(default_factory=lambda: np.zeros(0))
    q_norm: np.ndarray = field(default_factory=lambda: np.zeros(0))
    id: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    dt: np.ndarray = field(default_factory=lambda: np.zeros(0))
    remaining_steps: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))

    @staticmethod
    def from_array(arr) -> "Beam":
        b = Beam(**{k: np.array(arr[k], dtype=np.int64 if k == "id" else np.float64)
                    for k in BEAM_KEYS})
        b.dt = np.zeros(b.id.size)
        b.remaining_steps = np.zeros(b.id.size, np.int64)
        return b

    @property
    def size(self):
        return self.id.size

    def take(self, sel) -> "Beam":
        return Beam(**{k: np.ascontiguousarray(getattr(self, k)[sel])
                       for k in self.__dataclass_fields__})

    def sorted(self) -> "Beam":
        return self.take(np.argsort(-self.xi))

    def append(self, other: "Beam") -> "Beam":
        return Beam(**{k: np.concatenate((getattr(self, k), getattr(other, k)))
                       for k in self.__dataclass_fields__})


def deposit_beam(p: Params, layer_idx: int, b: Beam, ro0, ro1):
    """beam3d/weights.py:152-163."""
    if b.size == 0:
        return
    lib().orc_deposit_beam(ctypes.c_int64(b.size), ctypes.c_int(p.N),
                           ctypes.c_double(p.h), ctypes.c_double(p.dxi),
                           ctypes.c_int64(layer_idx), _p(b.x), _p(b.y), _p(b.xi),
                           _p(b.q_norm), _p(ro0), _p(ro1))


def move_beam_layer(p: Params, b: Beam, fell_size: int, xi_i: int,
                    F_k: Fields, F_k1: Fields, time_step: float,
                    substep_energy: float):
    """beam3d/beam_calculator.py:97-134 with the GPU pusher move.py:155-273.
    Returns (lost, moved, fell) layers."""
    n = b.size
    if n == 0:
        e = Beam()
        return e, e, e
    size = n - fell_size
    if size > 0:
        dt = np.empty(size)
        rs = np.empty(size, np.int64)
        lib().orc_beam_substepping(ctypes.c_int64(size), _p(b.q_m[:size].copy()),
                                   _p(b.pz[:size].copy()), ctypes.c_double(substep_energy),
                                   ctypes.c_double(time_step), _p(dt), _p(rs))
        b.dt[:size] = dt
        b.remaining_steps[:size] = rs
    R = p.h * p.N / 2
    r_max = max(0.9 * R, R - 1)
    flags = np.zeros(n, np.uint8)
    lib().orc_move_beam(
        ctypes.c_int64(n), ctypes.c_double(p.dxi), ctypes.c_double(r_max),
        ctypes.c_int64(xi_i - 1), ctypes.c_double(p.h), ctypes.c_int(p.N),
        _p(b.q_m), _p(b.dt),
        _p(F_k.Ex), _p(F_k.Ey), _p(F_k.Ez), _p(F_k.Bx), _p(F_k.By), _p(F_k.Bz),
        _p(F_k1.Ex), _p(F_k1.Ey), _p(F_k1.Ez), _p(F_k1.Bx), _p(F_k1.By), _p(F_k1.Bz),
        _p(b.remaining_steps), _p(b.id), _p(b.x), _p(b.y), _p(b.xi),
        _p(b.px), _p(b.py), _p(b.pz), _p(flags))
    return b.take((flags & 1) != 0), b.take((flags & 2) != 0), b.take((flags & 4) != 0)


def layer_length(beam: Beam, head: int, layer_idx: int, dxi: float) -> int:
    """Number of particles to cut for layer `layer_idx`,
    beam3d/beam_io.py:29-47 (count of remaining xi in [-(i+1)dxi, -i dxi))."""
    xi = beam.xi[head:]
    if xi.size == 0:
        return 0
    xi_min = -dxi * layer_idx
    xi_max = -dxi * (layer_idx + 1)
    return int(np.sum((xi_max <= xi) * (xi < xi_min)))


# --------------------------------------------------------------------------
# xi loop (push_solvers/push_solver.py:215-286)
# --------------------------------------------------------------------------

def step_dt(p: Params, sorts, F: Fields, cur: Currents, consts: Consts,
            xi_steps: int, beam: Beam | None = None, rigid=None,
            time_step=1.0, substep_energy=2.0, record=None):
    """One time step of the xi loop.  Either `beam` (sorted Beam, non-rigid)
    or `rigid` (callable fn(xp, xi, x_grid, y_grid)) drives the plasma.
    `record(xi_i, sorts, F, cur, rho_beam)` is called after each xi step.
    Returns (sorts, F, cur, drain Beam or None)."""
    N = p.N
    rb_prev = np.zeros((N, N))
    grid = (np.arange(N) - N // 2) * p.h
    xg, yg = np.meshgrid(grid, grid)
    rho_layout = np.zeros((N, N))
    head = 0
    to_move = Beam()
    fell_size = 0
    drain = Beam()
    for xi_i in range(0, xi_steps + 1):
        if rigid is not None:
            rb_full = rigid(np, -xi_i * p.dxi, xg, yg)
        else:
            L = layer_length(beam, head, xi_i, p.dxi)
            layer = beam.take(slice(head, head + L))
            head += L
            new = np.zeros((N, N))
            if layer.size:
                deposit_beam(p, xi_i, layer, rho_layout, new)
            rho_layout, rb_full = new, rho_layout
            rb_full /= p.h ** 2
        F_prev = F.copy()
        sorts, F, cur = step_dxi(p, sorts, F, cur, consts, rb_full, rb_prev)
        if rigid is None:
            lost, moved, fell = move_beam_layer(p, to_move, fell_size, xi_i,
                                                F_prev, F, time_step, substep_energy)
            to_move = layer.append(fell)
            fell_size = fell.size
            if moved.size:
                drain = drain.append(moved)
        rb_prev = rb_full.copy()
        if record is not None:
            record(xi_i, sorts, F, cur, rb_full)
    return sorts, F, cur, (None if rigid is not None else drain)
