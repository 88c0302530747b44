"""Plasma state files (the format the reference's Simulation loads with
external_plasmastate): write/read round trip on the host, and the reference
loader's own indexing (state[sort][name], float(state['xi_plasma_layer']))."""
import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lcodepy_b200.data import Arrays  # noqa: E402
from lcodepy_b200.plasma_state import (CURRENT_KEYS, FIELD_KEYS, PARTICLE_RECORD,  # noqa: E402
                                       load_plasmastate, save_plasmastate)


def _state(rng, N=9, Ns=6):
    fields = types.SimpleNamespace(**{k: torch.as_tensor(rng.standard_normal((N, N))) for k in FIELD_KEYS})
    currents = types.SimpleNamespace(**{k: torch.as_tensor(rng.standard_normal((2, N, N)))
                                        for k in CURRENT_KEYS})
    el = Arrays(torch, **{k: torch.as_tensor(rng.standard_normal((Ns, Ns)))
                          for k in ("x_init", "y_init", "q", "m", "x_offt", "y_offt", "px", "py", "pz")})
    return fields, currents, {"electrons": el.wrapped()}


def test_round_trip_and_reference_indexing(tmp_path):
    rng = np.random.default_rng(3)
    fields, currents, parts = _state(rng)
    ro0 = rng.standard_normal((9, 9))
    path = tmp_path / "plasmastate.npz"
    save_plasmastate(path, parts, fields, currents, ro_initial=ro0, xi_plasma_layer=-0.35)
    # the reference loader's accesses, without pickling
    with np.load(path) as z:
        assert z["electrons"]["x_init"].shape == (6, 6)
        assert set(z["electrons"].dtype.names) == set(PARTICLE_RECORD)
        assert float(z["xi_plasma_layer"]) == -0.35
        assert np.array_equal(z["Ez"], fields.Ez.numpy())
    st = load_plasmastate(path, ("electrons",))
    for k in FIELD_KEYS:
        assert np.array_equal(st["fields"][k], getattr(fields, k).numpy())
    for k in CURRENT_KEYS:
        assert np.array_equal(st["currents"][k], getattr(currents, k).numpy())
    for k in ("x_init", "px", "q", "m"):
        assert np.array_equal(st["particles"]["electrons"][k], parts["electrons"].__dict__[k].get())
    assert not st["particles"]["electrons"]["dx_chaotic"].any()
    assert np.array_equal(st["rho_initial"], ro0)
    assert st["xi_plasma_layer"] == -0.35


def test_missing_sort_is_an_error(tmp_path):
    rng = np.random.default_rng(4)
    fields, currents, parts = _state(rng)
    path = tmp_path / "s.npz"
    save_plasmastate(path, parts, fields, currents)
    with pytest.raises(KeyError):
        load_plasmastate(path, ("electrons", "ions"))
    assert load_plasmastate(path, ("electrons",))["xi_plasma_layer"] is None
