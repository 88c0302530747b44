"""Plasma state files: what the reference's Simulation loads when
``external_plasmastate`` is set (lcode/plasma3d/initialization.py:417-460,
lcode/simulation.py:154-165).

The file is an npz with

- the field planes ``Ex Ey Ez Bx By Bz Phi`` (N x N),
- the currents ``ro jx jy jz`` (2 x N x N: plasma sort, background plane),
- per sort (``electrons``, and ``ions`` with mobile ions) a record array of
  the lattice shape (Ns x Ns) with the fields ``x_init y_init q m x_offt
  y_offt px py pz dx_chaotic dy_chaotic dx_chaotic_perp dy_chaotic_perp``
  (plain float64 records, so ``numpy.load`` reads it without pickling),
- optionally ``rho_initial`` (N x N, the background charge) and
  ``xi_plasma_layer`` (the xi of the stored layer; the run continues from the
  next one).

``save_plasmastate`` writes it from host or device arrays, so a run can be
checkpointed at any xi layer (for instance from a diagnostic's
``after_step_dxi``) and resumed with ``Simulation.external_plasmastate``.
"""
from __future__ import annotations

import numpy as np

FIELD_KEYS = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Phi")
CURRENT_KEYS = ("ro", "jx", "jy", "jz")
PARTICLE_RECORD = ("x_init", "y_init", "q", "m", "x_offt", "y_offt", "px", "py", "pz",
                   "dx_chaotic", "dy_chaotic", "dx_chaotic_perp", "dy_chaotic_perp")


def _host(a) -> np.ndarray:
    """A host array from a tensor, a DeviceArray (``.get()``) or an array."""
    if hasattr(a, "get") and not isinstance(a, dict):
        return np.asarray(a.get())
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def save_plasmastate(path, particles: dict, fields, currents, ro_initial=None,
                     xi_plasma_layer=None):
    """Write a plasma state file.  ``particles`` maps sort names to objects
    with the particle arrays as attributes (missing chaotic displacements are
    written as zeros); ``fields`` and ``currents`` have the planes as
    attributes."""
    data = {k: _host(getattr(fields, k)) for k in FIELD_KEYS}
    data.update({k: _host(getattr(currents, k)) for k in CURRENT_KEYS})
    for sort, p in particles.items():
        shape = _host(p.x_init).shape
        rec = np.zeros(shape, dtype=[(k, "f8") for k in PARTICLE_RECORD])
        for k in PARTICLE_RECORD:
            if hasattr(p, k):
                rec[k] = _host(getattr(p, k))
        data[sort] = rec
    if ro_initial is not None:
        data["rho_initial"] = _host(ro_initial)
    if xi_plasma_layer is not None:
        data["xi_plasma_layer"] = np.array(float(xi_plasma_layer))
    np.savez_compressed(path, **data)


def load_plasmastate(path, sorts) -> dict:
    """Read a plasma state file into host arrays: ``fields`` and
    ``currents`` dicts, ``particles`` {sort: {name: (Ns, Ns) array}},
    ``rho_initial`` (or None) and ``xi_plasma_layer`` (or None)."""
    with np.load(path) as z:
        out = {"fields": {k: np.array(z[k], dtype=np.float64) for k in FIELD_KEYS},
               "currents": {k: np.array(z[k], dtype=np.float64) for k in CURRENT_KEYS},
               "particles": {}, "rho_initial": None, "xi_plasma_layer": None}
        for sort in sorts:
            if sort not in z.files:
                raise KeyError(f"plasma state {path} has no '{sort}' particles")
            rec = z[sort]
            out["particles"][sort] = {k: np.array(rec[k], dtype=np.float64)
                                      for k in rec.dtype.names}
        if "rho_initial" in z.files:
            out["rho_initial"] = np.array(z["rho_initial"], dtype=np.float64)
        if "xi_plasma_layer" in z.files:
            out["xi_plasma_layer"] = float(np.asarray(z["xi_plasma_layer"]).ravel()[0])
    return out
