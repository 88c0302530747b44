"""Time-step pipeline over ranks: the reference's MPI beam transport
(lcode/mpi/transport.py:13-62, lcode/mpi/beam_io.py:6-118) on
torch.distributed.

With W ranks, rank r computes the time steps r, r + W, r + 2W, ... (the
reference's ``steps_per_node`` and ``current_time`` arithmetic).  Time step
t + 1 needs the beam that time step t moved, and it needs it layer by layer:
its xi loop lays out layer i + 1 at xi step i.  So rank r streams its moved
beam to rank (r + 1) mod W while its own xi loop runs, and the next rank
starts its time step as soon as the first layers have arrived.

The moved beam of a time step (the drain of the device beam step) is
ordered by xi layer: xi step i appends the particles that end in layer
i - 1, and a beam particle's xi only decreases, so after xi step i the
layers below i are complete.  ``StreamingDrain`` sends the drain in chunks
of complete layers (every ``chunk_steps`` xi steps and at the end of the
time step); ``StreamingSource`` appends the chunks into a fixed device
buffer, sorts each chunk by xi (stable, descending, as ``BeamSource`` sorts
the whole beam: a chunk holds whole layers, so the result is the same
order), and computes each layer's slice with the same head-cut rule as
``BeamSource.all_layer_bounds`` once the layers up to it are complete.  The
result of a pipelined run is the result of the single-process run.

A chunk is one header (particles, layers complete, last-chunk flag; int64)
and one payload tensor (the particle arrays stacked as float64, the integer
ones bit-cast), sent with point-to-point ``torch.distributed`` calls: NCCL
over NVLink between GPUs, or gloo through host copies (``staged``).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .beam3d import BeamDrain, BeamParticles

_INT_KEYS = ("id", "remaining_steps")


def steps_of_rank(n_steps: int, rank: int, world: int):
    """The global time steps that ``rank`` computes (transport.py:50-52)."""
    return list(range(rank, n_steps, world))


def _keys():
    return BeamParticles(torch.device("cpu"))._all()


class BeamTransport:
    """Chunks of beam particles between ranks of a process group."""

    def __init__(self, device, group=None, staged: bool | None = None):
        self.device = device
        self.group = group
        backend = dist.get_backend(group)
        self.staged = (backend != "nccl") if staged is None else staged
        self.pending = []

    def _wire(self, t: torch.Tensor) -> torch.Tensor:
        return t.cpu() if self.staged else t

    def _wire_device(self):
        """Where received tensors land: host memory when staged."""
        return torch.device("cpu") if self.staged else self.device

    def send(self, dst: int, beam: BeamParticles, complete: int, last: bool):
        n = beam.size
        header = torch.tensor([n, complete, int(last)], dtype=torch.int64,
                              device=self._wire_device())
        cols = []
        for k in _keys():
            a = getattr(beam, k)
            cols.append(a.view(torch.float64) if k in _INT_KEYS else a)
        payload = (torch.stack(cols) if n else
                   torch.zeros(len(cols), 0, dtype=torch.float64, device=self.device))
        h, p = self._wire(header), self._wire(payload.contiguous())
        # kept alive until the time step's sends have completed
        self.pending.append((dist.isend(h, dst, group=self.group), h))
        if n:
            self.pending.append((dist.isend(p, dst, group=self.group), p))

    def recv(self, src: int):
        """(BeamParticles on the device, layers complete, last chunk)."""
        header = torch.zeros(3, dtype=torch.int64, device=self._wire_device())
        dist.recv(header, src, group=self.group)
        n, complete, last = (int(v) for v in header.tolist())
        keys = _keys()
        b = BeamParticles(self.device)
        if n:
            payload = torch.empty(len(keys), n, dtype=torch.float64, device=self._wire_device())
            dist.recv(payload, src, group=self.group)
            payload = payload.to(self.device)
            for j, k in enumerate(keys):
                col = payload[j].contiguous()
                setattr(b, k, col.view(torch.int64) if k in _INT_KEYS else col)
        return b, complete, bool(last)

    def wait(self):
        for work, _ in self.pending:
            work.wait()
        self.pending.clear()


class StreamingSource:
    """The beam of a time step as it arrives from the previous rank, with the
    ``BeamSource`` interface the beam calculator uses (``beam``,
    ``layer_bounds``); ``layer_bounds(i)`` waits for the chunks that
    complete layer i."""

    streaming = True

    def __init__(self, config, transport: BeamTransport, src: int, capacity: int):
        self.dxi = config.getfloat('xi-step')
        self.transport, self.src = transport, src
        self.beam = BeamParticles(transport.device, capacity)
        self.capacity = capacity
        self.filled = 0
        self.neg_xi = np.empty(capacity, dtype=np.float64)   # host copy, sorted ascending
        self.complete = 0          # layers 0 .. complete-1 have arrived
        self.last = False
        self.bounds = {}
        self.head = 0
        self.next_layer = 0

    def _n_ge(self, v):
        return int(np.searchsorted(self.neg_xi[:self.filled], -v, side='right'))

    def _receive(self):
        b, complete, last = self.transport.recv(self.src)
        n = b.size
        if self.filled + n > self.capacity:
            raise RuntimeError(f"beam stream overflow: {self.filled + n} > {self.capacity}")
        if n:
            b.xi_sorted()
            for k in b._all():
                getattr(self.beam, k)[self.filled:self.filled + n].copy_(getattr(b, k))
            self.neg_xi[self.filled:self.filled + n] = (-b.xi).cpu().numpy()
            self.filled += n
        self.complete = max(self.complete, complete)
        self.last = last

    def _cut(self, i):
        # BeamSource.layer_bounds: count the layer's particles in the
        # complete prefix, then cut that many from the head
        xi_min, xi_max = -self.dxi * i, -self.dxi * (i + 1)
        lo = max(self._n_ge(xi_min), self.head)
        hi = max(self._n_ge(xi_max), self.head)
        a = self.head
        self.head += hi - lo
        return a, self.head

    def layer_bounds(self, i):
        while self.next_layer <= i:
            while not self.last and self.complete <= self.next_layer:
                self._receive()
            self.bounds[self.next_layer] = self._cut(self.next_layer)
            self.next_layer += 1
        return self.bounds[i]

    def finish(self):
        """Receive whatever is still in flight (the end of the stream)."""
        while not self.last:
            self._receive()


class StreamingDrain(BeamDrain):
    """The drain of a time step that streams its moved beam to the next rank:
    every ``chunk_steps`` xi steps the newly drained particles (complete
    layers) go out, the rest when the time step ends."""

    def __init__(self, config, transport: BeamTransport, dst: int, chunk_steps: int = 32,
                 device=None):
        super().__init__(config, device)
        # the previous time step's stream has been received by now (the next
        # rank consumed it during its own time step)
        transport.wait()
        self.transport, self.dst = transport, dst
        self.chunk_steps = max(1, int(chunk_steps))
        self.sent = 0

    def after_xi_step(self, xi_i: int, bc):
        """Called after the beam step of xi step ``xi_i``: layers below xi_i
        are complete in the calculator's drain buffer."""
        if (xi_i + 1) % self.chunk_steps:
            return
        n = int(bc.counts[2].item())     # one device read per chunk
        self.transport.send(self.dst, bc.drain.take(slice(self.sent, n)), xi_i, False)
        self.sent = n

    def push_beam_layer(self, layer: BeamParticles):
        # the whole moved beam of the time step (push_solver calls this once);
        # the sends complete while the next rank runs: the transport waits
        # for them when this rank starts its next streaming time step
        super().push_beam_layer(layer)
        rest = layer.take(slice(self.sent, None))
        self.transport.send(self.dst, rest, 1 << 62, True)
        self.sent = layer.size
