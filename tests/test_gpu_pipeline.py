"""The time-step pipeline end to end on the GPU: two ranks (processes on
one GPU, gloo with host-staged chunks; no kernel waits on the other rank)
run three time steps of a non-rigid beam -- rank 0 the steps 0 and 2, rank
1 the step 1, each streaming its moved beam to the other during its xi loop
-- and the last step equals the single-process run."""
import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs CUDA", allow_module_level=True)
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_STEPS = 3
BEAM = {'current': -0.5, 'particles_in_layer': 300,
        'default': {'length': 1.2, 'energy': 5.0, 'angspread': 1e-2}}


def _config():
    return {'geometry': '3d', 'processing-unit-type': 'gpu',
            'window-width': 3.2, 'transverse-step': 0.05,
            'window-length': 1.5, 'xi-step': 0.05, 'time-limit': N_STEPS, 'time-step': 5.0,
            'ion-model': 'background', 'plasma-particles-per-cell': 4, 'print-every': 0,
            'pipeline-chunk-steps': 4}


def _result(sim):
    ps = sim.push_solver
    _, fields, _ = ps._plasmastate
    beam = sim.beam_drain.beam_slice()
    order = np.argsort(beam.id.cpu().numpy())
    return {"ez": ps.ez_axis.cpu().numpy(), "Ez": fields.Ez.cpu().numpy(),
            "beam_id": beam.id.cpu().numpy()[order], "beam_pz": beam.pz.cpu().numpy()[order]}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from lcodepy_b200 import Simulation
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    sim = Simulation(config=_config(), beam_parameters=BEAM, runas_filename='')
    sim.step(N_STEPS)
    if (N_STEPS - 1) % ws == rank:
        out["last"] = _result(sim)
        out["rank"] = rank
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_pipeline_equals_single_process():
    from lcodepy_b200 import Simulation
    sim = Simulation(config=_config(), beam_parameters=BEAM, runas_filename='')
    sim.step(N_STEPS)
    want = _result(sim)
    del sim
    torch.cuda.synchronize()
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        got = dict(out["last"])
        assert out["rank"] == 0
    np.testing.assert_array_equal(got["beam_id"], want["beam_id"])
    for k in ("ez", "Ez", "beam_pz"):
        err = np.abs(got[k] - want[k]).max() / max(np.abs(want[k]).max(), 1e-300)
        assert err < 1e-10, (k, err)
    assert np.abs(want["ez"]).max() > 0
