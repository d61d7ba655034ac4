"""CPU tests of the split-colony protocol (vehicleroutingproblem_b200.sharding).

Two gloo ranks each build their half of the ants with the oracle, exchange
their best-ant packets through sharding.exchange, pick the winner with
sharding.select_winner and update their pheromone copies.  Epoch by epoch
both ranks must hold the winner and the pheromone matrix of one colony with
all the ants (the oracle run in this process)."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I
from vehicleroutingproblem_b200 import sharding as S

N_CUST, K_VEH, K_CAND, SEED, EPOCHS = 60, 3, 12, 4242, 5


def _instance():
    return I.uniform_instance(N_CUST, K_VEH, 9031, demand_max=40)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Colony:
    """The oracle's epoch for a set of global ant ids on one pheromone copy."""

    def __init__(self, O, inst):
        self.O, self.inst = O, inst
        self.P = O.params()
        self.A, self.lut, thr = O.tables()
        self.cand = O.knn(inst.x, inst.y, K_CAND)
        self.lvl = O.levels(inst.x, inst.y, self.cand, K_CAND, thr)
        self.tau = np.full((inst.n + 1) ** 2, self.P["q_tau0"], np.uint8)
        self.gbest, self.gnodes, self.glens = np.inf, None, None

    def construct(self, epoch, ants):
        O, inst = self.O, self.inst
        w = O.weights(inst.n, K_CAND, self.cand, self.lvl, self.tau, self.A, self.lut)
        return [(a, O.construct_ant(inst.x, inst.y, inst.demand, inst.vehicles, inst.capacity,
                                    K_CAND, self.cand, w, SEED, epoch, a)) for a in ants]

    @staticmethod
    def local_best(res):
        """First minimum over ascending ant ids (the device's argmin)."""
        best = None
        for a, r in res:
            if r[0] and (best is None or r[3] < best[1][3]):
                best = (a, r)
        return best

    def update(self, cost, nodes, lens):
        """Bookkeeping deposit amounts, evaporation and the two deposits."""
        if cost is None:
            return
        O, P = self.O, self.P
        Qs = np.float32(100.0)
        dep_i = np.float32(np.float32(0.3) * Qs) / np.float32(cost)
        if cost < self.gbest:
            self.gbest, self.gnodes, self.glens = cost, nodes, lens
        dep_g = np.float32(np.float32(0.7) * Qs) / np.float32(self.gbest)
        t = O.evaporate(self.tau, P["q_evap_delta"])
        t = O.deposit(t, self.inst.n, nodes, lens, float(dep_i), P["log_tau_min"],
                      P["log_tau_step"])
        self.tau = O.deposit(t, self.inst.n, self.gnodes, self.glens, float(dep_g),
                             P["log_tau_min"], P["log_tau_step"])


def _rank_worker(rank, world, port, m, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        inst = _instance()
        col = _Colony(O, inst)
        n, K = inst.n, inst.vehicles
        Pn = S.packet_ints(n, K)
        winners, taus = [], []
        for e in range(EPOCHS):
            res = col.construct(e, range(rank * m, (rank + 1) * m))
            lb = col.local_best(res)
            steps = sum(r[4] for _, r in res)
            if lb is None:
                pk = S.encode_packet(n, K, False, 0.0, 0, steps)
            else:
                a, r = lb
                pk = S.encode_packet(n, K, True, r[3], a, steps, r[2], r[1])
            send = torch.from_numpy(pk)
            recv = torch.zeros(world * Pn, dtype=torch.int32)
            S.exchange(send, recv)
            packets = [S.decode_packet(recv[i * Pn:(i + 1) * Pn].numpy(), n, K)
                       for i in range(world)]
            wi = S.select_winner(packets)
            if wi is None:
                winners.append((-1, np.inf, sum(p.steps for p in packets)))
                col.update(None, None, None)
            else:
                p = packets[wi]
                winners.append((p.global_ant, p.cost, sum(q.steps for q in packets)))
                col.update(p.cost, p.nodes, p.lens)
            taus.append(col.tau.copy())
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), winners=np.array(winners),
                 taus=np.array(taus))
    finally:
        dist.destroy_process_group()


def test_packet_round_trip_and_winner_rule():
    n, K = 10, 2
    nodes = np.array([0, 3, 1, 0, 0, 2, 4, 5, 6, 7, 8, 9, 10, 0], np.int32)
    lens = np.array([4, 10], np.int32)
    pk = S.encode_packet(n, K, True, 123.5, 77, (1 << 33) + 5, lens, nodes)
    assert pk.size == S.packet_ints(n, K) and pk.size % 4 == 0
    p = S.decode_packet(pk, n, K)
    assert p.found and p.cost == 123.5 and p.global_ant == 77 and p.steps == (1 << 33) + 5
    assert np.array_equal(p.lens, lens) and np.array_equal(p.nodes, nodes)
    none = S.decode_packet(S.encode_packet(n, K, False, 0.0, 0, 9), n, K)
    assert not none.found and none.steps == 9 and none.nodes.size == 0
    mk = lambda c, a: S.decode_packet(S.encode_packet(n, K, True, c, a, 0, lens, nodes), n, K)
    # lowest cost wins; equal costs go to the lowest global ant, whatever the rank order
    assert S.select_winner([mk(5.0, 3), mk(4.0, 9), none]) == 1
    assert S.select_winner([mk(4.0, 9), mk(4.0, 3)]) == 1
    assert S.select_winner([mk(4.0, 3), mk(4.0, 9)]) == 0
    assert S.select_winner([none, none]) is None


@pytest.mark.timeout(300)
def test_two_gloo_ranks_equal_one_colony(oracle_mod, tmp_path):
    import torch.multiprocessing as mp
    m, world = 10, 2
    mp.spawn(_rank_worker, args=(world, _free_port(), m, str(tmp_path)), nprocs=world,
             join=True)
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    assert np.array_equal(r0["winners"], r1["winners"])
    assert np.array_equal(r0["taus"], r1["taus"])
    # both ranks' ants win some epoch, so the exchange decides something
    assert {int(w) // m for w in r0["winners"][:, 0] if w >= 0} == {0, 1}

    col = _Colony(oracle_mod, _instance())
    found_any = False
    for e in range(EPOCHS):
        res = col.construct(e, range(world * m))
        lb = col.local_best(res)
        steps = sum(r[4] for _, r in res)
        w = r0["winners"][e]
        assert w[2] == steps
        if lb is None:
            assert w[0] == -1
            col.update(None, None, None)
        else:
            found_any = True
            a, r = lb
            assert (int(w[0]), float(w[1])) == (a, r[3])
            col.update(r[3], r[1], r[2])
        assert np.array_equal(r0["taus"][e], col.tau)
    assert found_any


def _leaving_worker(rank, world, port, out_dir):
    import time
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=5))
    n, K = 10, 2
    P = S.packet_ints(n, K)
    send = torch.from_numpy(S.encode_packet(n, K, False, 0.0, 0, rank))
    recv = torch.zeros(world * P, dtype=torch.int32)
    S.exchange(send, recv)  # epoch 1: both ranks
    if rank == 1:
        os._exit(0)  # leaves between epochs, with no collective in flight
    t0 = time.monotonic()
    try:
        S.exchange(send, recv)  # epoch 2: the peer is gone
        outcome = "no error"
    except Exception as exc:  # the process group reports the lost rank
        outcome = "error: " + type(exc).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write(f"{outcome}\n{time.monotonic() - t0:.3f}\n")
    os._exit(0)


@pytest.mark.timeout(120)
def test_lost_rank_is_reported_not_waited_for(tmp_path):
    """A rank that leaves between epochs: the other rank's next packet
    exchange ends with an error within the process group's timeout."""
    import torch.multiprocessing as mp
    mp.spawn(_leaving_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    outcome, secs = (tmp_path / "rank0.txt").read_text().splitlines()[:2]
    assert outcome.startswith("error"), outcome
    assert float(secs) < 30.0


def test_split_instances_balances_work():
    """The batched form's split over ranks: every instance once, the ranks'
    work within one instance's work of each other, deterministic."""
    insts = I.batched_instances(512, 30000)
    work = [x.n + x.vehicles for x in insts]
    for world in (1, 2, 3, 8):
        parts = S.split_instances(work, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(insts)))
        loads = [sum(work[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(work)
        assert parts == S.split_instances(work, world)
    assert S.split_instances([5, 3, 3, 1], 2) == [[0, 3], [1, 2]]
    with pytest.raises(ValueError):
        S.split_instances(work, 0)
