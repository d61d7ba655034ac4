"""A colony split over devices (aco_b200_shard_*) equals one colony with all
the ants.  One GPU stands in for the devices: two contexts with ant_base 0
and m exchange their packets through a device buffer, epoch by epoch, and
must follow one context with 2m ants exactly (pheromone, state, best)."""
import contextlib
import datetime

import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I
from vehicleroutingproblem_b200 import sharding as S

pytestmark = pytest.mark.gpu

CASES = {
    "u150_unit": (lambda: I.uniform_instance(150, 4, 771, demand_max=1), 24, 16),
    "u300_demand": (lambda: I.uniform_instance(300, 6, 772), 32, 24),
    "c500_demand": (lambda: I.clustered_instance(500, 9, 773), 20, 32),
}


def _setup(N, inst, k, m, ant_base, stream, seed=99, **kw):
    ctx = N.Context(0)
    ctx.set_stream(stream.cuda_stream)
    ctx.setup_instance(inst, ants=m, cand_k=k, seed=seed, ant_base=ant_base, **kw)
    return ctx


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_shards_equal_one_colony(native, name):
    import torch
    make, k, m = CASES[name]
    inst = make()
    n, K = inst.n, inst.vehicles
    s = torch.cuda.Stream()
    whole = _setup(native, inst, k, 2 * m, 0, s)
    parts = [_setup(native, inst, k, m, r * m, s) for r in range(2)]
    P = parts[0].shard_packet_ints()
    assert P == S.packet_ints(n, K)
    send = [torch.zeros(P, dtype=torch.int32, device="cuda") for _ in parts]
    recv = torch.zeros(2 * P, dtype=torch.int32, device="cuda")
    ranks_won = set()
    for e in range(10):
        for c, b in zip(parts, send):
            c.shard_construct(b.data_ptr())
        with torch.cuda.stream(s):
            recv[:P].copy_(send[0])
            recv[P:].copy_(send[1])
        for c in parts:
            c.shard_update(recv.data_ptr(), 2)
        whole.enqueue_epochs(1)
        s.synchronize()
        # the packets hold each half's best ant, with the ant-steps
        nodes, lens, cost, feas, steps, _ = whole.ants()
        pk = [S.decode_packet(recv[r * P:(r + 1) * P].cpu().numpy(), n, K) for r in range(2)]
        for r in range(2):
            sl = slice(r * m, (r + 1) * m)
            c = np.where(feas[sl] != 0, cost[sl], np.inf)
            assert pk[r].steps == int(steps[sl].sum())
            assert pk[r].found == bool(np.isfinite(c).any())
            if pk[r].found:
                b = int(np.argmin(c))
                assert pk[r].global_ant == r * m + b and pk[r].cost == c[b]
                assert np.array_equal(pk[r].lens, lens[r * m + b])
                assert np.array_equal(pk[r].nodes, nodes[r * m + b][: int(lens[r * m + b].sum())])
        sw = whole.state()
        wi = S.select_winner(pk)
        if wi is not None:
            ranks_won.add(wi)
            assert sw.best_ant == pk[wi].global_ant
        t = whole.tau()
        for c in parts:
            st = c.state()
            assert (st.epochs, st.found, st.best_ant, st.iter_since_best, st.improved) == \
                (sw.epochs, sw.found, sw.best_ant, sw.iter_since_best, sw.improved)
            assert st.global_best == sw.global_best and st.iter_best == sw.iter_best
            assert st.dep_iter == sw.dep_iter and st.dep_global == sw.dep_global
            assert st.total_steps == sw.total_steps and st.error == 0
            assert np.array_equal(c.tau(), t)
            bn, bl, bc = c.best()
            wn, wl, wc = whole.best()
            assert bc == wc and np.array_equal(bl, wl) and np.array_equal(bn, wn)
    assert ranks_won == {0, 1}
    for c in parts + [whole]:
        c.close()


def test_stop_rules_agree_across_shards(native):
    """Stagnation stops every shard after the same epoch as the whole colony;
    the epochs queued after it are skipped."""
    import torch
    inst = I.uniform_instance(120, 3, 774)
    s = torch.cuda.Stream()
    whole = _setup(native, inst, 16, 32, 0, s, stagnation_epochs=3)
    st_w = whole.run(400)
    assert st_w.stopped and st_w.epochs < 400
    parts = [_setup(native, inst, 16, 16, r * 16, s, stagnation_epochs=3) for r in range(2)]
    P = parts[0].shard_packet_ints()
    send = [torch.zeros(P, dtype=torch.int32, device="cuda") for _ in parts]
    recv = torch.zeros(2 * P, dtype=torch.int32, device="cuda")
    for e in range(st_w.epochs + 5):
        for c, b in zip(parts, send):
            c.shard_construct(b.data_ptr())
        with torch.cuda.stream(s):
            recv[:P].copy_(send[0])
            recv[P:].copy_(send[1])
        for c in parts:
            c.shard_update(recv.data_ptr(), 2)
    s.synchronize()
    for c in parts:
        st = c.state()
        assert st.stopped and st.epochs == st_w.epochs
        assert st.global_best == st_w.global_best
        assert np.array_equal(c.tau(), whole.tau())
        c.close()
    whole.close()


def _unservable():
    # customer 60 needs 61 of a capacity of 60: no ant is ever feasible
    rs = np.random.RandomState(5)
    pts = [(500, 500)] + [tuple(rs.randint(0, 1001, 2)) for _ in range(60)]
    x = np.array([p[0] for p in pts], np.float32)
    y = np.array([p[1] for p in pts], np.float32)
    d = np.array([0] + [5] * 59 + [61], np.int32)
    return I.Instance("big", x, y, d, 6, 60)


def test_shards_without_a_feasible_ant(native):
    """No rank has a feasible ant: the select kernel leaves the pheromone and
    the best alone and keeps the same bookkeeping as one colony."""
    import torch
    inst = _unservable()
    s = torch.cuda.Stream()
    whole = _setup(native, inst, 8, 16, 0, s)
    parts = [_setup(native, inst, 8, 8, r * 8, s) for r in range(2)]
    t0 = whole.tau()
    P = parts[0].shard_packet_ints()
    send = [torch.zeros(P, dtype=torch.int32, device="cuda") for _ in parts]
    recv = torch.zeros(2 * P, dtype=torch.int32, device="cuda")
    for e in range(6):
        for c, b in zip(parts, send):
            c.shard_construct(b.data_ptr())
        with torch.cuda.stream(s):
            recv[:P].copy_(send[0])
            recv[P:].copy_(send[1])
        for c in parts:
            c.shard_update(recv.data_ptr(), 2)
        whole.enqueue_epochs(1)
    s.synchronize()
    sw = whole.state()
    assert sw.epochs == 6 and not sw.found and sw.iter_since_best == 6
    for c in parts + [whole]:
        st = c.state()
        assert (st.epochs, st.found, st.iter_since_best, st.total_steps, st.error) == \
            (sw.epochs, sw.found, sw.iter_since_best, sw.total_steps, 0)
        assert np.array_equal(c.tau(), t0)
        nodes, lens, cost = c.best()
        assert cost == float("inf") and nodes.size == 0
        c.close()


@contextlib.contextmanager
def _nccl_world_one():
    import os
    import socket
    import torch
    import torch.distributed as dist
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0),
                            timeout=datetime.timedelta(seconds=60))
    try:
        yield
    finally:
        dist.destroy_process_group()


def _same_colony(a, b):
    sa, sb = a.state(), b.state()
    assert (sa.epochs, sa.found, sa.best_ant, sa.iter_since_best, sa.total_steps, sa.error) == \
        (sb.epochs, sb.found, sb.best_ant, sb.iter_since_best, sb.total_steps, 0)
    assert sa.global_best == sb.global_best and sa.iter_best == sb.iter_best
    assert np.array_equal(a.tau(), b.tau())
    (an, al, ac), (bn, bl, bc) = a.best(), b.best()
    assert ac == bc and np.array_equal(al, bl) and np.array_equal(an, bn)


def test_sharded_colony_graphs_follow_eager_epochs(native):
    """Epochs replayed from the recorded graphs (1 and 16 epochs, the NCCL
    all-gather inside) equal epochs launched one call at a time, and a set-up
    with other sizes re-records them."""
    import torch
    with _nccl_world_one():
        inst = I.uniform_instance(200, 5, 776)
        a = S.ShardedColony(inst, 48, 0, cand_k=16, seed=7, graphs=True)
        b = S.ShardedColony(inst, 48, 0, cand_k=16, seed=7, graphs=False)
        try:
            for e in (1, 16, 3, 17):
                a.enqueue_epochs(e)
                a.stream.synchronize()
                b.enqueue_epochs(e)
                b.stream.synchronize()
                _same_colony(a, b)
            assert len(a._graphs) == 2 and not b._graphs
            g0 = a.ctx.graph_generation()
            inst2 = I.uniform_instance(260, 6, 777)
            for c in (a, b):
                c.setup(inst2, cand_k=16, seed=8)
            assert a.ctx.graph_generation() != g0
            a.enqueue_epochs(18)
            a.stream.synchronize()
            b.enqueue_epochs(18)
            b.stream.synchronize()
            _same_colony(a, b)
            assert a.state().epochs == 18 and len(a._graphs) == 2
        finally:
            a.close()
            b.close()
        torch.cuda.synchronize()


def test_sharded_colony_over_nccl_world_one(native):
    """ShardedColony through a real NCCL process group (one rank) follows the
    plain context epoch for epoch."""
    import torch
    inst = I.uniform_instance(200, 5, 775)
    with _nccl_world_one():
        col = S.ShardedColony(inst, 48, 0, cand_k=16, seed=5)
        st = col.run(37, chunk=16)
        ref = _setup(native, inst, 16, 48, 0, torch.cuda.Stream(), seed=5)
        st_r = ref.run(37)
        assert st.epochs == st_r.epochs == 37
        assert st.global_best == st_r.global_best and st.total_steps == st_r.total_steps
        assert np.array_equal(col.tau(), ref.tau())
        pk = col.packets()
        assert len(pk) == 1 and pk[0].found and pk[0].global_ant == st_r.best_ant
        col.close()
        ref.close()
