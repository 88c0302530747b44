"""lcb_compute_fields_noalloc: the field solver for callers that cannot
allocate device memory (a host code that only receives device pointers from
another framework's pool, or a binding with no CUDA allocator), so cannot
hand lcb_compute_fields a workspace.  Its scratch is a fixed device array
inside liblcb.so.

Checked through the C ABI against lcb_compute_fields with a caller workspace,
on two calls in a row (the second call finds the first call's data in the
shared array), in FP64 and in mixed precision, up to the largest grid whose
scratch fits the array (283 and 427), at the tolerances the other
compute_fields tests use; grids beyond the array are rejected.  Kept in a
file of its own, collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs CUDA", allow_module_level=True)

from lcodepy_b200 import _lib  # noqa: E402
from lcodepy_b200.plasma3d import FieldOperators  # noqa: E402

DEV = torch.device("cuda")
# the compute_fields tolerances of tests/test_gpu_kernels.py, per precision
REL = {_lib.LCB_PREC_FP64: 1e-11, _lib.LCB_PREC_MIXED: 3e-5}
# the largest grid whose scratch fits the fixed array, per precision
LIMIT = {_lib.LCB_PREC_FP64: 283, _lib.LCB_PREC_MIXED: 427}


def _inputs(N, seed):
    rng = np.random.default_rng(seed)

    def cur():
        a = np.zeros((2, N, N))
        a[:, 3:-3, 3:-3] = rng.normal(0, 1, (2, N - 6, N - 6))
        return torch.tensor(a, device=DEV)

    def fld():
        f = rng.normal(0, 1, (7, N, N))
        f[:, [0, -1], :] = 0
        f[:, :, [0, -1]] = 0
        return torch.tensor(f, device=DEV)
    return dict(cp=[cur() for _ in range(4)], cf=[cur() for _ in range(4)],
                F=fld(), Fp=fld(), rbf=torch.tensor(rng.normal(0, 1, (N, N)), device=DEV),
                rbp=torch.tensor(rng.normal(0, 1, (N, N)), device=DEV))


def _args(N, h, dxi, ops, inp, out_full, out_half, ws=None, precision=0):
    a = _lib.ComputeFieldsArgs()
    a.grid_steps, a.h, a.xi_step, a.subtraction_coeff = N, h, dxi, 1 + dxi
    a.precision = precision
    a.operators = ops.ptr
    for i in range(7):
        a.fields.f[i] = inp["F"][i].data_ptr()
        a.fields_prev.f[i] = inp["Fp"][i].data_ptr()
        a.out_full.f[i] = out_full[i].data_ptr()
        a.out_half.f[i] = out_half[i].data_ptr()
    a.currents_prev = _lib.Currents4(*(t.data_ptr() for t in inp["cp"]), 2)
    a.currents_full = _lib.Currents4(*(t.data_ptr() for t in inp["cf"]), 2)
    a.rho_beam_full, a.rho_beam_prev = inp["rbf"].data_ptr(), inp["rbp"].data_ptr()
    a.rho_beam_divisor = 1.0
    if ws is not None:
        a.workspace, a.workspace_bytes = ws.data_ptr(), ws.numel()
    return a


def _rel(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision,N", [(_lib.LCB_PREC_FP64, 129), (_lib.LCB_PREC_FP64, 257),
                                         (_lib.LCB_PREC_FP64, 283), (_lib.LCB_PREC_MIXED, 129),
                                         (_lib.LCB_PREC_MIXED, 427)])
def test_noalloc_matches_workspace_entry_point_twice(precision, N):
    L = _lib.load()
    h, dxi = 0.05, 0.05
    assert L.lcb_compute_fields_workspace_bytes(LIMIT[precision], precision) <= \
        _lib.LCB_NOALLOC_FIELDS_SCRATCH_BYTES < \
        L.lcb_compute_fields_workspace_bytes(LIMIT[precision] + 2, precision)
    ops = FieldOperators(N, h, 1 + dxi, DEV, precision == _lib.LCB_PREC_MIXED)
    for call, seed in enumerate((N, N + 1)):  # two calls in a row, different inputs
        inp = _inputs(N, seed)
        ref_full = torch.zeros(7, N, N, dtype=torch.float64, device=DEV)
        ref_half = torch.zeros_like(ref_full)
        ws = torch.empty(L.lcb_compute_fields_workspace_bytes(N, precision), dtype=torch.uint8,
                         device=DEV)
        a = _args(N, h, dxi, ops, inp, ref_full, ref_half, ws, precision)
        _lib.check(L.lcb_compute_fields(C.byref(a), _lib.stream_handle()), "compute_fields")
        got_full = torch.full((7, N, N), 5.0, dtype=torch.float64, device=DEV)
        got_half = torch.full((7, N, N), 5.0, dtype=torch.float64, device=DEV)
        b = _args(N, h, dxi, ops, inp, got_full, got_half, None, precision)  # no workspace
        _lib.check(L.lcb_compute_fields_noalloc(C.byref(b), _lib.stream_handle()),
                   "compute_fields_noalloc")
        torch.cuda.synchronize()
        for i in range(7):
            assert _rel(got_full[i], ref_full[i]) <= REL[precision], (call, i, "full")
            assert _rel(got_half[i], ref_half[i]) <= REL[precision], (call, i, "half")


@pytest.mark.parametrize("precision", [_lib.LCB_PREC_FP64, _lib.LCB_PREC_MIXED])
def test_noalloc_rejects_grids_beyond_its_scratch(precision):
    L = _lib.load()
    for N in (LIMIT[precision] + 2, 513):
        a = _lib.ComputeFieldsArgs()
        a.grid_steps, a.precision = N, precision
        rc = L.lcb_compute_fields_noalloc(C.byref(a), _lib.stream_handle())
        assert rc == 1
        msg = L.lcb_last_error().decode()
        assert str(N) in msg and "scratch" in msg
