"""The time-step pipeline's beam stream (lcodepy_b200/pipeline.py) on gloo
ranks on the CPU: a drain streamed in chunks of complete xi layers arrives
as the same sorted beam and the same layer slices that BeamSource cuts from
the whole beam (lcode/mpi/beam_io.py:6-118 semantics: time step t + 1 reads
what time step t moved)."""
import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DXI = 0.05
N_LAYERS = 60


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _beam(seed, n=3000):
    """A moved beam as the device drain holds it: grouped by xi layer in
    layer order, unsorted inside a layer, some layers empty."""
    from lcodepy_b200.beam3d import BeamParticles
    rng = np.random.default_rng(seed)
    xi = -rng.uniform(0.3, N_LAYERS - 3, n) * DXI
    xi[rng.random(n) < 0.1] = -7.5 * DXI        # a dense layer
    layer = np.floor(-xi / DXI).astype(np.int64)
    order = np.lexsort((rng.random(n), layer))  # by layer, shuffled inside
    b = BeamParticles(torch.device("cpu"), n)
    b.xi = torch.tensor(xi[order])
    for k in ("x", "y", "px", "py", "pz", "q_m", "q_norm", "dt"):
        setattr(b, k, torch.tensor(rng.normal(size=n)))
    b.id = torch.tensor(rng.permutation(n) + 1, dtype=torch.int64)
    b.remaining_steps = torch.tensor(rng.integers(0, 9, n), dtype=torch.int64)
    return b, layer[order]


class _Calc:
    """What StreamingDrain reads from the beam calculator: the drain buffer
    and its device counter after xi step i (layers below i complete)."""

    def __init__(self, beam, layer):
        self.drain = beam
        self.layer = layer
        self.counts = torch.zeros(4, dtype=torch.int64)

    def at(self, i):
        self.counts[2] = int(np.searchsorted(self.layer, i, side="left"))
        return self


def _send(transport, beam, layer, dst, chunk):
    from lcodepy_b200.config import Config
    from lcodepy_b200.pipeline import StreamingDrain
    cfg = Config({'xi-step': DXI})
    drain = StreamingDrain(cfg, transport, dst, chunk, torch.device("cpu"))
    calc = _Calc(beam, layer)
    for i in range(N_LAYERS):
        drain.after_xi_step(i, calc.at(i))
    drain.push_beam_layer(beam)


def _receive(transport, src, capacity):
    from lcodepy_b200.config import Config
    from lcodepy_b200.pipeline import StreamingSource
    cfg = Config({'xi-step': DXI})
    s = StreamingSource(cfg, transport, src, capacity)
    bounds = {i: s.layer_bounds(i) for i in range(N_LAYERS + 2)}
    s.finish()
    return s, bounds


def _expected(beam):
    from lcodepy_b200.beam3d import BeamSource
    from lcodepy_b200.config import Config
    src = BeamSource(Config({'xi-step': DXI}), beam.take(slice(None)), torch.device("cpu"))
    return src.beam, src.all_layer_bounds()


def _rank(rank, ws, port, chunk, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from lcodepy_b200.pipeline import BeamTransport
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    tr = BeamTransport(torch.device("cpu"))
    beam, layer = _beam(11)
    if rank == 0:                       # time step 0: streams what it moved
        _send(tr, beam, layer, 1, chunk)
    else:                               # time steps 1 .. ws-1: receive, pass on
        s, bounds = _receive(tr, rank - 1, beam.size)
        want_beam, want_bounds = _expected(beam)
        ok = s.filled == beam.size
        for k in beam._all():
            ok &= bool(torch.equal(getattr(s.beam, k)[:s.filled], getattr(want_beam, k)))
        ok &= all(bounds[i] == want_bounds.get(i, (bounds[i][0], bounds[i][0]))
                  for i in range(N_LAYERS + 2))
        out[rank] = ok
        if rank + 1 < ws:               # the next rank gets the same beam
            got = s.beam.take(slice(0, s.filled))
            lay = np.floor(-got.xi.numpy() / DXI).astype(np.int64)
            _send(tr, got, lay, rank + 1, chunk)
    tr.wait()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("ws,chunk", [(2, 1), (2, 7), (3, 16)])
def test_streamed_beam_equals_the_whole_beam(ws, chunk):
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(ws, port, chunk, out), nprocs=ws, join=True)
        assert dict(out) == {r: True for r in range(1, ws)}


def test_steps_of_rank_follow_the_reference():
    """transport.py:50-52: steps_per_node and the round-robin assignment."""
    from lcodepy_b200.pipeline import steps_of_rank
    for n, w in ((10, 3), (2, 4), (7, 7)):
        got = [steps_of_rank(n, r, w) for r in range(w)]
        assert sorted(t for g in got for t in g) == list(range(n))
        for r in range(w):
            assert len(got[r]) == n // w + (1 if n % w > r else 0)
