"""The reference's own GPU kernels, compiled for the host -- TEST INFRASTRUCTURE ONLY.

lcodePy's GPU path is CuPy ``ElementwiseKernel`` objects: the per-particle
bodies are C strings inside the Python sources.  CuPy cannot run here, but the
bodies are plain C over ``i``, so this recipe reads them out of the reference
checkout, wraps each one in a host loop over ``i`` (``T = double``, serial,
so ``atomicAdd`` is a plain add in particle order) and compiles the result
with g++ into ``oracle/_ref/libref_kernels.so``.  Nothing is copied into the
repository: the generated source and the library live in ``oracle/_ref/``,
which git ignores.

Kernels built (paths relative to the lcodePy project root):

- ``move_beam_cupy``         lcode/beam3d/move.py:139-276 (Higuera-Cary push)
- ``deposit_beam_cupy``      lcode/beam3d/weights.py:108-138
- ``substepping``            lcode/beam3d/beam_calculator.py:28-46
- ``move_smart_cupy``        lcode/plasma3d/move.py:169-289
- ``move_wo_fields_cupy``    lcode/plasma3d/move.py:292-313
- ``deposit_plasma_cupy``    lcode/plasma3d/weights.py:151-190

with the ``weight1_cupy`` / ``weight4_cupy`` preambles of
lcode/beam3d/weights.py:70-103 and lcode/plasma3d/weights.py:127-148.

The checkout is found through the ``LCODE_REFERENCE`` environment variable
(default ``/root/reference``).  Only ``tests/`` and the golden-fixture
scripts use this module.
"""
from __future__ import annotations

import ast
import ctypes
import os
import re
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(_HERE, "_ref")
LIB_PATH = os.path.join(OUT_DIR, "libref_kernels.so")
SRC_PATH = os.path.join(OUT_DIR, "ref_kernels.cpp")


def reference_root() -> str:
    return os.environ.get("LCODE_REFERENCE", "/root/reference")


# (exported C name, source file, factory function, name of the Python preamble
# strings the kernel uses)
KERNELS = [
    ("move_beam", "lcode/beam3d/move.py", "get_move_beam_particles_kernel_cupy"),
    ("deposit_beam", "lcode/beam3d/weights.py", "get_deposit_beam_cupy"),
    ("substepping", "lcode/beam3d/beam_calculator.py", "get_beam_substepping_step_cupy"),
    ("move_smart", "lcode/plasma3d/move.py", "get_move_smart_kernel_cupy"),
    ("move_wo_fields", "lcode/plasma3d/move.py", "get_move_wo_fields_kernel_cupy"),
    ("deposit_plasma", "lcode/plasma3d/weights.py", "get_deposit_plasma_cupy"),
]


def _module_strings(tree):
    """Module-level `NAME = "..."` string assignments (the preambles)."""
    out = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Constant) \
                and isinstance(node.value.value, str):
            for t in node.targets:
                if isinstance(t, ast.Name):
                    out[t.id] = node.value.value
    return out


def _eval_str(node, names):
    if isinstance(node, ast.Constant) and isinstance(node.value, str):
        return node.value
    if isinstance(node, ast.Name):
        return names[node.id]
    if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Add):
        return _eval_str(node.left, names) + _eval_str(node.right, names)
    raise ValueError(f"cannot evaluate {ast.dump(node)}")


def extract(path: str, factory: str) -> dict:
    """The ElementwiseKernel arguments (in_params, out_params, operation,
    preamble) inside `factory` of the reference file `path`."""
    with open(path) as f:
        tree = ast.parse(f.read())
    names = _module_strings(tree)
    # preambles imported from a sibling module (beam3d/move.py imports them)
    for node in tree.body:
        if isinstance(node, ast.ImportFrom) and node.module and node.level >= 1:
            sib = os.path.join(os.path.dirname(path), node.module.split(".")[-1] + ".py")
            if os.path.exists(sib):
                with open(sib) as f:
                    names.update(_module_strings(ast.parse(f.read())))
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == factory:
            for sub in ast.walk(node):
                if isinstance(sub, ast.Call) and getattr(sub.func, "attr", "") == "ElementwiseKernel":
                    kw = {k.arg: k.value for k in sub.keywords}
                    pos = list(sub.args)
                    res = {}
                    for j, key in enumerate(("in_params", "out_params", "operation")):
                        node_ = kw.get(key, pos[j] if j < len(pos) else None)
                        res[key] = _eval_str(node_, names)
                    res["preamble"] = _eval_str(kw["preamble"], names) if "preamble" in kw else ""
                    return res
    raise LookupError(f"{factory} not found in {path}")


_CTYPE = {"T": "T", "float64": "double", "int64": "int64_t", "bool": "bool", "int32": "int32_t"}


def _params(spec: str):
    """[(raw, type, name)] from a CuPy parameter list."""
    out = []
    for item in spec.replace("\n", " ").split(","):
        toks = item.split()
        if not toks:
            continue
        raw = toks[0] == "raw"
        if raw:
            toks = toks[1:]
        out.append((raw, toks[0], toks[1]))
    return out


def generate(root: str | None = None) -> str:
    """C++ source with one `extern "C" ref_<name>(n, params...)` per kernel."""
    root = root or reference_root()
    parts = ["// generated from the reference checkout by oracle/ref_kernels.py; not committed",
             "#include <cmath>", "#include <cstdint>", "#include <cstddef>",
             "using namespace std;", "#define __device__", "typedef double T;",
             "static inline double atomicAdd(double *a, double v) "
             "{ double o = *a; *a = o + v; return o; }"]
    seen_pre = set()
    for cname, rel, factory in KERNELS:
        k = extract(os.path.join(root, rel), factory)
        pre = k["preamble"]
        # one definition per weight function across kernels
        blocks = re.split(r"(?=__device__ inline)", pre)
        for b in blocks:
            m = re.search(r"inline T (\w+)\(", b)
            if m and m.group(1) not in seen_pre:
                seen_pre.add(m.group(1))
                parts.append(b)
        ins, outs = _params(k["in_params"]), _params(k["out_params"])
        sig, binds = ["int64_t n_"], []
        for is_out, plist in ((False, ins), (True, outs)):
            for raw, ty, name in plist:
                cty = _CTYPE[ty]
                if raw:
                    sig.append(f"{cty} *{name}")
                elif ty == "float64" and not is_out:   # a scalar argument
                    sig.append(f"double {name}")
                else:   # an element-wise array argument: bound to element i
                    sig.append(f"{cty} *{name}_arr_")
                    binds.append(f"{cty} &{name} = {name}_arr_[i];")
        parts.append(f'extern "C" void ref_{cname}({", ".join(sig)})\n{{\n'
                     f"    for (ptrdiff_t i = 0; i < n_; ++i) {{\n        "
                     + "\n        ".join(binds) + "\n        {\n"
                     + k["operation"] + "\n        }\n    }\n}\n")
    return "\n".join(parts)


def build(force: bool = False) -> str:
    """Generate and compile oracle/_ref/libref_kernels.so; needs the
    reference checkout unless the library is already built."""
    if os.path.exists(LIB_PATH) and not force:
        return LIB_PATH
    root = reference_root()
    if not os.path.isdir(os.path.join(root, "lcode")):
        raise FileNotFoundError(f"reference checkout not found at {root} (set LCODE_REFERENCE)")
    os.makedirs(OUT_DIR, exist_ok=True)
    src = generate(root)
    with open(SRC_PATH, "w") as f:
        f.write(src)
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off",
                           "-fno-fast-math", "-w", "-o", tmp, SRC_PATH])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH) or os.path.isdir(os.path.join(reference_root(), "lcode"))


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
    return _lib


def _ptr(a):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def move_beam(xi_step, r_max, layer_idx, h, grid_steps, q_m, dt, fields_k, fields_k1,
              remaining_steps, id_, x, y, xi, px, py, pz):
    """move_beam_cupy over a layer, in place; returns (lost, moved, fell)
    boolean arrays.  fields_* are (Ex, Ey, Ez, Bx, By, Bz) N x N arrays."""
    n = q_m.size
    lost, moved, fell = (np.zeros(n, np.bool_) for _ in range(3))
    D = ctypes.c_double
    lib().ref_move_beam(ctypes.c_int64(n), D(xi_step), D(r_max), D(layer_idx), D(h),
                        D(grid_steps), _ptr(q_m), _ptr(dt),
                        *(_ptr(f) for f in fields_k), *(_ptr(f) for f in fields_k1),
                        _ptr(remaining_steps), _ptr(id_), _ptr(x), _ptr(y), _ptr(xi),
                        _ptr(px), _ptr(py), _ptr(pz), _ptr(lost), _ptr(moved), _ptr(fell))
    return lost, moved, fell


def substepping(q_m, pz, substep_energy):
    """calculate_substepping_step with dt starting at 1 (the reference's
    beam_substepping_step), returns dt."""
    dt = np.ones(q_m.size)
    lib().ref_substepping(ctypes.c_int64(q_m.size), _ptr(q_m), _ptr(pz),
                          ctypes.c_double(substep_energy), _ptr(dt))
    return dt


def deposit_beam(grid_steps, x_h, y_h, xi_loc, q, ro0, ro1):
    lib().ref_deposit_beam(ctypes.c_int64(x_h.size), ctypes.c_double(grid_steps), _ptr(x_h),
                           _ptr(y_h), _ptr(xi_loc), _ptr(q), _ptr(ro0), _ptr(ro1))


def move_smart(xi_step, boundary, h, grid_steps, fields, x_init, y_init, xo_prev, yo_prev,
               px_prev, py_prev, pz_prev, m, q, xo_full, yo_full, px_full, py_full, pz_full):
    D = ctypes.c_double
    lib().ref_move_smart(ctypes.c_int64(q.size), D(xi_step), D(boundary), D(h), D(grid_steps),
                         *(_ptr(f) for f in fields), _ptr(x_init), _ptr(y_init),
                         _ptr(xo_prev), _ptr(yo_prev), _ptr(px_prev), _ptr(py_prev),
                         _ptr(pz_prev), _ptr(m), _ptr(q), _ptr(xo_full), _ptr(yo_full),
                         _ptr(px_full), _ptr(py_full), _ptr(pz_full))


def move_wo_fields(xi_step, m, x_offt, y_offt, px, py, pz):
    lib().ref_move_wo_fields(ctypes.c_int64(m.size), ctypes.c_double(xi_step), _ptr(m),
                             _ptr(x_offt), _ptr(y_offt), _ptr(px), _ptr(py), _ptr(pz))


def deposit_plasma(grid_steps, h, x_h, y_h, px, py, pz, q, m, ro, jx, jy, jz):
    lib().ref_deposit_plasma(ctypes.c_int64(q.size), ctypes.c_double(grid_steps),
                             ctypes.c_double(h), _ptr(x_h), _ptr(y_h), _ptr(px), _ptr(py),
                             _ptr(pz), _ptr(q), _ptr(m), _ptr(ro), _ptr(jx), _ptr(jy), _ptr(jz))
