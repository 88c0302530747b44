"""Device-recorded diagnostics against the reference's FXiDiag / SliceDiag /
ParticlesDiag output files (tests/golden/diag_golden.npz, made by
make_diag_golden.py from the same seeded inputs).  Runs on CPU tensors and,
marked gpu, on CUDA tensors (the recording the drop-in Simulation does on
the device)."""
import os
import sys
import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_diag_golden import CASES, CONFIG, PARTICLE_KEYS, StubDrain, diag_steps, walk  # noqa: E402

from lcodepy_b200 import diagnostics as D  # noqa: E402
from lcodepy_b200.config import Config  # noqa: E402
from lcodepy_b200.data import Arrays, DeviceArray  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "diag_golden.npz"))


def _ns(dev, **kw):
    return types.SimpleNamespace(**{k: DeviceArray(torch.as_tensor(v, device=dev))
                                    for k, v in kw.items()})


DEVICES = ["cpu", pytest.param("cuda", marks=pytest.mark.gpu)]


@pytest.mark.parametrize("dev", DEVICES)
@pytest.mark.parametrize("case,cls,kw", CASES, ids=[c[0] for c in CASES])
def test_diagnostic_files_match_reference(tmp_path, monkeypatch, case, cls, kw, dev):
    if dev == "cuda" and not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    monkeypatch.chdir(tmp_path)
    cfg = Config(dict(CONFIG))
    cfg._adjust_config_values_3d()
    N = cfg.getint('window-width-steps')
    assert N == int(GOLD['N'])
    d = getattr(D, cls)(**kw)
    d.pull_config(cfg)
    last_t = None
    drain = StubDrain()
    for t, xi, f in diag_steps(N):
        if last_t is not None and t != last_t:
            d.dump(last_t, xi, particles, None, None, drain)
        last_t = t
        fields = _ns(dev, **{n: f[n] for n in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi')})
        currents = _ns(dev, ro=f['ro'])
        # what the drop-in Simulation hands to diagnostics: wrapped Arrays
        particles = {'electrons': Arrays(torch, **{n: torch.as_tensor(f[n], device=dev)
                                                   for n in PARTICLE_KEYS}).wrapped()}
        d.after_step_dxi(t, xi, particles, fields, currents,
                         DeviceArray(torch.as_tensor(f['rho_beam'], device=dev)))
    d.dump(last_t, 0.0, particles, None, None, drain)
    sub = tmp_path / 'diagnostics' / kw['directory_name']
    want = sorted({k.split('|')[1] for k in GOLD.files if k.startswith(case + '|')})
    assert walk(sub) == want
    for fn in want:
        with np.load(sub / fn) as z:
            keys = sorted(k.split('|')[2] for k in GOLD.files if k.startswith(f'{case}|{fn}|'))
            assert sorted(z.files) == keys, fn
            for k in keys:
                ref = GOLD[f'{case}|{fn}|{k}']
                assert z[k].shape == ref.shape and z[k].dtype == ref.dtype, (fn, k)
                if k == 'Sf':   # a reduction: summation order differs
                    np.testing.assert_allclose(z[k], ref, rtol=1e-12)
                else:
                    np.testing.assert_array_equal(z[k], ref)
