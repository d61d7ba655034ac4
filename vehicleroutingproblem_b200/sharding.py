"""One ant colony split over several GPUs (one process per GPU).

The reference runs one colony on one device (src/cuda/aco_cuda.cu:316-420):
every epoch all m ants are built, the iteration best is chosen
(aco_cuda.cu:349-366) and the pheromone matrix is evaporated and deposited
with the iteration and global best (aco_cuda.cu:385-396).  Split over N
devices, each rank builds m ants of its own with the pheromone matrix
replicated, and the only exchange is the choice of the iteration best:

    rank r:  shard_construct  -> packet (its best ant: cost, global ant id,
                                 ant-steps, route), int32 words on the device
             all-gather       -> N packets on every rank (NCCL)
             shard_update     -> the same winner on every rank (lowest cost,
                                 then lowest global ant id), the same
                                 bookkeeping, evaporation and deposits

Random draws are keyed by the global ant id (rank * m + local ant), so N
ranks with m ants run exactly the epochs of one GPU with N * m ants.  The
pheromone matrices stay identical without ever being sent; one epoch moves
N packets of 4 (n + 3K + 6) bytes.

The packet helpers below restate the device packet format on the host; they
decode packets and are what the multi-process CPU tests drive.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N

DBL_MAX = np.finfo(np.float64).max
INT_MAX = 0x7FFFFFFF


def packet_ints(n: int, K: int) -> int:
    """Packet length in int32 words (device: shard_packet_ints)."""
    return (6 + K + n + 2 * K + 3) & ~3


@dataclass
class Packet:
    cost: float
    found: bool
    global_ant: int
    steps: int
    lens: np.ndarray
    nodes: np.ndarray


def encode_packet(n: int, K: int, found: bool, cost: float, global_ant: int, steps: int,
                  lens=None, nodes=None) -> np.ndarray:
    """Packet words of one rank's best ant, as k_shard_pack writes them."""
    pk = np.zeros(packet_ints(n, K), np.int32)
    c = np.array([cost if found else DBL_MAX], np.float64).view(np.int32)
    pk[0], pk[1] = c[0], c[1]
    pk[2] = 1 if found else 0
    pk[3] = global_ant if found else INT_MAX
    s = np.array([steps], np.uint64).view(np.int32)
    pk[4], pk[5] = s[0], s[1]
    if found:
        lens = np.asarray(lens, np.int32)
        nodes = np.asarray(nodes, np.int32)
        pk[6:6 + K] = lens
        pk[6 + K:6 + K + int(lens.sum())] = nodes[:int(lens.sum())]
    return pk


def decode_packet(pk: np.ndarray, n: int, K: int) -> Packet:
    pk = np.asarray(pk, np.int32)
    cost = float(pk[0:2].copy().view(np.float64)[0])
    steps = int(pk[4:6].copy().view(np.uint64)[0])
    lens = pk[6:6 + K].copy()
    found = bool(pk[2])
    total = int(lens.sum()) if found else 0
    return Packet(cost, found, int(pk[3]), steps, lens, pk[6 + K:6 + K + total].copy())


def select_winner(packets: Sequence[Packet]) -> Optional[int]:
    """Index of the winning packet (k_shard_select): lowest cost, then
    lowest global ant id; None when no rank found a feasible ant."""
    best = None
    for i, p in enumerate(packets):
        if not p.found:
            continue
        q = packets[best] if best is not None else None
        if q is None or p.cost < q.cost or (p.cost == q.cost and p.global_ant < q.global_ant):
            best = i
    return best


def split_instances(work: Sequence[float], world: int) -> List[List[int]]:
    """The batched form over `world` GPUs: instance indices per rank, the
    instances being independent (no collective, only the results are
    gathered).  Largest work first to the rank with the least work so far
    (ties to the lower rank); each rank's list in ascending order.  The work
    of an instance is m (n + K) ant-steps per epoch, so with equal m, n + K."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda j: (-float(work[j]), j)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += float(work[i])
    return [sorted(p) for p in parts]


def exchange(send, recv, group=None) -> None:
    """All-gather of the packets in rank order: send (P words) -> recv
    (world * P words), torch tensors on the process group's device."""
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        dist.all_gather_into_tensor(recv, send, group=group)
        return
    world = dist.get_world_size(group)
    parts = list(recv.view(world, -1).unbind(0))
    gathered = [p.clone() for p in parts]
    dist.all_gather(gathered, send, group=group)
    for dst, src in zip(parts, gathered):
        dst.copy_(src)


class ShardedColony:
    """This rank's part of a colony split over the process group's ranks.

    Each rank holds an aco_b200 context on its GPU with `ants` ants and
    ant_base = rank * ants; work is queued on one CUDA stream, the packet
    all-gather included, so an epoch costs the host no synchronisation.
    Over NCCL (graphs=True, the default there) whole epochs, the all-gather
    included, are recorded once into CUDA graphs of 1 and `chunk` epochs
    and replayed, so an epoch is one graph launch instead of five kernel
    launches, two event waits and a collective call; the graphs are
    re-recorded when a set-up changes the launch arguments
    (Context.graph_generation) and released by close(), which must come
    before the process group is destroyed.
    """

    CHUNK = 16

    def __init__(self, inst, ants: int, device: int, group=None, stream=None,
                 graphs: Optional[bool] = None, **params):
        import torch
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = torch.device("cuda", device)
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        self.ants = ants
        if graphs is None:
            graphs = dist.get_backend(group) == "nccl"
        self.use_graphs = bool(graphs)
        self._graphs = {}
        self._warm = False  # one eager epoch since construction (NCCL set up)
        self.ctx = N.Context(device)
        self.ctx.set_stream(self.stream.cuda_stream)
        self.send = self.recv = None
        self.setup(inst, **params)

    def setup(self, inst, **params) -> None:
        """(Re)starts the colony on an instance; the context's device buffers
        and the packet buffers are reused when the sizes are unchanged."""
        import torch
        params = dict(params)
        self.timeout_seconds = float(params.pop("timeout_seconds", 0.0) or 0.0)
        self.ctx.setup_instance(inst, ants=self.ants, ant_base=self.rank * self.ants,
                                timeout_seconds=0.0, **params)
        P = self.ctx.shard_packet_ints()
        if self.send is None or self.send.numel() != P:
            self.send = torch.zeros(P, dtype=torch.int32, device=self.device)
            self.recv = torch.zeros(self.world * P, dtype=torch.int32, device=self.device)
        self._t0 = time.monotonic()

    def close(self) -> None:
        self._graphs.clear()
        self.ctx.close()

    def _enqueue_eager(self, epochs: int) -> None:
        import torch
        with torch.cuda.stream(self.stream):
            for _ in range(epochs):
                self.ctx.shard_construct(self.send.data_ptr())
                exchange(self.send, self.recv, self.group)
                self.ctx.shard_update(self.recv.data_ptr(), self.world)

    def _graph(self, epochs: int):
        """The recorded graph of `epochs` epochs for the current launch
        arguments (recorded on first use)."""
        import torch
        key = (self.ctx.graph_generation(), self.send.data_ptr(), self.recv.data_ptr(), epochs)
        g = self._graphs.get(key)
        if g is None:
            self._graphs = {k: v for k, v in self._graphs.items() if k[:3] == key[:3]}
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=self.stream, capture_error_mode="thread_local"):
                self._enqueue_eager(epochs)
            self._graphs[key] = g
        return g

    def enqueue_epochs(self, epochs: int) -> None:
        import torch
        if not self.use_graphs or not self._warm:
            if epochs > 0:
                self._enqueue_eager(1)
                self._warm = True
                self.enqueue_epochs(epochs - 1)
            return
        with torch.cuda.stream(self.stream):
            for _ in range(epochs // self.CHUNK):
                self._graph(self.CHUNK).replay()
            for _ in range(epochs % self.CHUNK):
                self._graph(1).replay()

    def enqueue_epoch(self) -> None:
        self.enqueue_epochs(1)

    def run(self, max_epochs: int, chunk: int = 16) -> N.State:
        """Runs up to max_epochs epochs, stopping on the device stop rules
        (identical on every rank) or on the host timeout (agreed by an
        all-reduce so every rank stops after the same epoch)."""
        import torch
        import torch.distributed as dist
        done = 0
        st = self.ctx.state()
        while done < max_epochs and not st.stopped:
            c = min(chunk, max_epochs - done)
            self.enqueue_epochs(c)
            done += c
            st = self.ctx.state()  # synchronises the stream
            timed_out = (self.timeout_seconds > 0 and
                         time.monotonic() - self._t0 > self.timeout_seconds)
            with torch.cuda.stream(self.stream):
                flags = torch.tensor([1 if timed_out else 0, 1 if st.error else 0],
                                     dtype=torch.int32, device=self.device)
                dist.all_reduce(flags, op=dist.ReduceOp.MAX, group=self.group)
            self.stream.synchronize()
            if flags[1].item():
                raise N.AcoError(N.ACO_ERR_BACKEND, "device error flag on a rank")
            if flags[0].item():
                break
        return st

    def state(self) -> N.State:
        return self.ctx.state()

    def best(self):
        return self.ctx.best()

    def tau(self) -> np.ndarray:
        return self.ctx.tau()

    def packets(self) -> List[Packet]:
        """The last exchanged packets, decoded (host copy)."""
        self.stream.synchronize()
        P = self.send.numel()
        r = self.recv.cpu().numpy()
        return [decode_packet(r[i * P:(i + 1) * P], self.ctx.n, self.ctx.K)
                for i in range(self.world)]
