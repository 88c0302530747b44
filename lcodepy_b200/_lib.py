"""ctypes binding of liblcb.so (include/lcb.h).

The library is the product's compute path: there is no fallback.  Loading
fails loudly when the shared object is missing (build it with
``python -m lcodepy_b200.build``) or when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblcb.so")

LCB_OK = 0
LCB_PREC_FP64 = 0
LCB_PREC_MIXED = 1
# size of the fixed device scratch array of lcb_compute_fields_noalloc (lcb.h)
LCB_NOALLOC_FIELDS_SCRATCH_BYTES = 16 << 20
DEVERR_PLASMA_STENCIL = 1
DEVERR_BEAM_STENCIL = 2
DEVERR_CAPACITY = 4
DEVERR_FIXED_RANGE = 8

_vp = C.c_void_p
_i64 = C.c_int64
_d = C.c_double
_i = C.c_int


class LcbError(RuntimeError):
    """A liblcb call returned an error status."""


class Fields7(C.Structure):
    _fields_ = [("f", _vp * 7)]


class Currents4(C.Structure):
    _fields_ = [("ro", _vp), ("jx", _vp), ("jy", _vp), ("jz", _vp), ("n_planes", _i)]


class PlasmaParticles(C.Structure):
    _fields_ = [(n, _vp) for n in ("x_init", "y_init", "x_offt", "y_offt", "px", "py",
                                   "pz", "q", "m")]


class MoveDepositArgs(C.Structure):
    _fields_ = [
        ("n_per_sort", _i64), ("n_sorts", _i), ("particles_side", _i), ("grid_steps", _i),
        ("precision", _i), ("first", _i), ("lattice_fineness", _i),
        ("xi_step", _d), ("boundary", _d), ("h", _d), ("fields", _vp * 6),
        ("prev", PlasmaParticles), ("full", PlasmaParticles), ("ro_initial", _vp),
        ("ro", _vp), ("jx", _vp), ("jy", _vp), ("jz", _vp),
        ("workspace", _vp), ("workspace_bytes", C.c_size_t), ("err", _vp)]


class BeamSoA(C.Structure):
    _fields_ = [(n, _vp) for n in ("xi", "x", "y", "px", "py", "pz", "q_m", "q_norm",
                                   "id", "dt", "remaining_steps")]


class BeamStepArgs(C.Structure):
    _fields_ = [
        ("grid_steps", _i), ("h", _d), ("xi_step", _d), ("r_max", _d),
        ("substep_energy", _d), ("time_step", _d), ("layer_idx", _i64),
        ("layout_idx", _i64),
        ("source", BeamSoA), ("layout_begin", _i64), ("layout_end", _i64),
        ("move_begin", _i64), ("move_end", _i64),
        ("fell_in", BeamSoA), ("fell_in_count", _vp),
        ("fell_out", BeamSoA), ("fell_out_count", _vp), ("fell_capacity", _i64),
        ("drain", BeamSoA), ("drain_count", _vp), ("drain_capacity", _i64),
        ("lost", BeamSoA), ("lost_count", _vp), ("lost_capacity", _i64),
        ("stage", BeamSoA), ("stage_flags", _vp), ("stage_capacity", _i64),
        ("ro0", _vp), ("ro1", _vp), ("fields_k", _vp), ("fields_k1", _vp), ("err", _vp)]


class ComputeFieldsArgs(C.Structure):
    _fields_ = [
        ("grid_steps", _i), ("h", _d), ("xi_step", _d), ("subtraction_coeff", _d),
        ("precision", _i), ("operators", _vp), ("fields", Fields7),
        ("fields_prev", Fields7), ("currents_prev", Currents4),
        ("currents_full", Currents4), ("rho_beam_full", _vp), ("rho_beam_prev", _vp),
        ("rho_beam_divisor", _d), ("out_full", Fields7), ("out_half", Fields7),
        ("workspace", _vp), ("workspace_bytes", C.c_size_t)]


class DeclusteringArgs(C.Structure):
    _fields_ = [
        ("n", _i), ("xi_step", _d), ("force", _d), ("damping", _d), ("limit", _d),
        ("dx_inhom", _vp), ("dy_inhom", _vp), ("dx_average", _vp), ("dy_average", _vp),
        ("dx_chaotic_prev", _vp), ("dy_chaotic_prev", _vp), ("px", _vp), ("py", _vp),
        ("dx_chaotic", _vp), ("dy_chaotic", _vp)]


_SIGS = {
    "lcb_last_error": (C.c_char_p, []),
    "lcb_version": (_i, []),
    "lcb_launch_count": (_i64, []),
    "lcb_plasma_move_wo_fields": (_i, [_i64, _d] + [_vp] * 13 + [_vp]),
    "lcb_plasma_move_smart": (_i, [_i64, _d, _d, _d, _i] + [_vp] * 20 + [_vp, _vp]),
    "lcb_plasma_deposit": (_i, [_i64, _i, _i, _d, _i, _i] + [_vp] * 14 +
                           [_vp, C.c_size_t, _vp, _vp]),
    "lcb_plasma_deposit_workspace_bytes": (C.c_size_t, [_i, _i]),
    "lcb_plasma_move_deposit": (_i, [C.POINTER(MoveDepositArgs), _vp]),
    "lcb_field_operators_bytes": (C.c_size_t, [_i, _i]),
    "lcb_field_operators_build": (_i, [_i, _d, _d, _i, _vp, C.c_size_t, _vp]),
    "lcb_compute_fields": (_i, [C.POINTER(ComputeFieldsArgs), _vp]),
    "lcb_compute_fields_workspace_bytes": (C.c_size_t, [_i, _i]),
    "lcb_compute_fields_noalloc": (_i, [C.POINTER(ComputeFieldsArgs), _vp]),
    "lcb_wave_kernel_choice": (_i, [_i, _i]),
    "lcb_beam_deposit": (_i, [_i64, _i, _d, _d, _i64] + [_vp] * 6 + [_vp, _vp]),
    "lcb_beam_substepping": (_i, [_i64, _vp, _vp, _d, _d, _vp, _vp, _vp]),
    "lcb_beam_step": (_i, [C.POINTER(BeamStepArgs), _vp]),
    "lcb_rigid_gaussian": (_i, [_i, _d, _d, _d, _d, _d, _i64, _vp, _vp, _vp, _vp]),
    "lcb_record_axis": (_i, [_vp, _i, _vp, _vp, _i64, _vp]),
    "lcb_declustering_inhomogeneity": (_i, [_i, _vp, _vp, _vp, _vp, _vp]),
    "lcb_declustering_apply": (_i, [C.POINTER(DeclusteringArgs), _vp]),
    "lcb_beam_move": (_i, [_i64, _d, _d, _i64, _d, _i, _vp, _vp,
                           C.POINTER(Fields7), C.POINTER(Fields7)] + [_vp] * 9 + [_vp, _vp]),
}

_lib = None


def load():
    """Load liblcb.so once; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m lcodepy_b200.build` "
                "(this package has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGS)


def check(rc: int, what: str):
    if rc != LCB_OK:
        msg = load().lcb_last_error().decode(errors="replace")
        raise LcbError(f"{what} failed (status {rc}): {msg}")


_replayed = 0


def add_replayed(n: int):
    """Count kernel launches made by replaying captured CUDA graphs (the
    library's own counter sees each kernel once, at capture)."""
    global _replayed
    _replayed += n


def launch_count() -> int:
    """liblcb kernel launches so far, direct and through graph replays."""
    return int(load().lcb_launch_count()) + _replayed


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(stream=None) -> int | None:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
