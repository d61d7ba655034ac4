"""Learned heuristic prior: training set, training and time-to-cost.

The pipeline the prior is built with:

1. elite routes -- the plain ACO itself solves the training instances
   (`elite_solutions`: all of them in one batched persistent launch);
2. training set -- every row an elite route leaves through a candidate edge
   becomes an example: the depot row with the route's first customer, and
   both directions of every customer-customer arc (`Prior.set_dataset`);
3. training -- softmax cross-entropy of the MLP's scores over each row's
   candidate slots against the elite successor, Adam, on the tensor cores
   (`Prior.train`);
4. use -- `Context.apply_prior(prior, gamma)` replaces the eta levels of an
   instance by the learned ones; the plain levels stay the fallback;
5. judgement -- `time_to_cost`: on held-out instances, the time the learned
   prior needs to reach the plain solver's final cost (+0.5%), FP64 costs,
   against the time the plain solver needs.
"""
from __future__ import annotations

import time
from typing import Dict, Optional, Sequence

import numpy as np

from . import _native as N
from . import instances as I


def elite_solutions(instances: Sequence[I.Instance], ants: int = 64, cand_k: int = 16,
                    epochs: int = 150, seed: int = 7, device: int = 0):
    """Best solution of a plain ACO run per instance (batched solver):
    a list of (nodes, lens, cost)."""
    with N.Batch(device) as b:
        b.setup(list(instances), ants=ants, cand_k=cand_k, seed=seed, epochs=epochs)
        b.autotune(trial_epochs=2)
        b.solve()
        out = []
        for i in range(len(instances)):
            nodes, lens, cost, _ = b.best(i)
            out.append((nodes, lens, cost))
    return out


def train_prior(prior: "N.Prior", instances, solutions, epochs: int = 8, batch: int = 4096,
                lr: float = 2e-3, seed: int = 11, cand_k: int = 32):
    """Builds the training set from (nodes, lens[, cost]) solutions and trains
    the prior; returns (examples, per-epoch losses, seconds)."""
    sols = [(s[0], s[1]) for s in solutions]
    t0 = time.perf_counter()
    count = prior.set_dataset(list(instances), sols, cand_k=cand_k)
    losses = prior.train(epochs, batch=batch, lr=lr, seed=seed)
    return count, losses, time.perf_counter() - t0


def convergence(inst: I.Instance, epochs: int, prior: Optional["N.Prior"] = None,
                gamma: float = 1.0, ants: int = 256, cand_k: int = 32, seed: int = 1234,
                device: int = 0):
    """Best cost after every epoch, the device time (s) at every epoch (from
    the first epoch's start) and the seconds spent applying the prior."""
    import torch
    s = torch.cuda.Stream(device)
    with N.Context(device) as c:
        c.set_stream(s.cuda_stream)
        c.setup_instance(inst, ants=ants, cand_k=cand_k, seed=seed, fixed_epochs=epochs)
        t_prior = 0.0
        if prior is not None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            c.apply_prior(prior, gamma)
            e1.record(s)
            e1.synchronize()
            t_prior = e0.elapsed_time(e1) / 1e3
        _, recs = c.run(epochs, want_records=True)
    best = np.array([r.global_best for r in recs], np.float64)
    t = np.array([r.elapsed_ns for r in recs], np.float64) * 1e-9
    return best, t, t_prior


def time_to_cost(heldout: Sequence[I.Instance], prior: "N.Prior", gamma: float = 1.0,
                 epochs: int = 300, ants: int = 256, cand_k: int = 32, tol: float = 0.005,
                 seed: int = 1234, device: int = 0) -> Dict:
    """Per held-out instance: the plain solver's final cost C after `epochs`
    epochs, the target (1 + tol) C, and the time each solver first reaches
    it (the learned one pays its inference time too).  An instance the
    learned prior does not bring to the target counts as its whole run plus
    one epoch."""
    rows = []
    for j, inst in enumerate(heldout):
        bp, tp, _ = convergence(inst, epochs, None, gamma, ants, cand_k, seed + j, device)
        bl, tl, t_inf = convergence(inst, epochs, prior, gamma, ants, cand_k, seed + j, device)
        target = bp[-1] * (1.0 + tol)
        ip = int(np.argmax(bp <= target))
        hit = bool((bl <= target).any())
        il = int(np.argmax(bl <= target)) if hit else len(bl)
        per_epoch = tl[-1] / len(tl)
        time_l = (tl[il] if hit else tl[-1] + per_epoch) + t_inf
        rows.append(dict(plain_cost=float(bp[-1]), learned_cost=float(bl[-1]),
                         plain_epochs=ip + 1, learned_epochs=il + 1, learned_hit=hit,
                         plain_s=float(tp[ip]), learned_s=float(time_l), prior_s=t_inf))
    ratio = np.array([r["learned_s"] / r["plain_s"] for r in rows])
    return {
        "instances": len(rows),
        "epochs": epochs,
        "target": f"plain final cost x {1 + tol}",
        "time_ratio_median": float(np.median(ratio)),
        "time_ratio_mean": float(np.mean(ratio)),
        "time_ratio_of_sums": float(sum(r["learned_s"] for r in rows) /
                                    sum(r["plain_s"] for r in rows)),
        "hit_rate": float(np.mean([r["learned_hit"] for r in rows])),
        "final_cost_ratio_mean": float(np.mean([r["learned_cost"] / r["plain_cost"]
                                                for r in rows])),
        "prior_inference_s_mean": float(np.mean([r["prior_s"] for r in rows])),
        "rows": rows,
    }
