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
5. evaluation -- `time_to_cost`: on held-out instances, the time the learned
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
                    epochs: int = 150, seed: int = 7, device: int = 0, beta: float = 2.0):
    """Best solution of a plain ACO run per instance (batched solver):
    a list of (nodes, lens, cost)."""
    with N.Batch(device) as b:
        b.setup(list(instances), ants=ants, cand_k=cand_k, seed=seed, epochs=epochs, beta=beta)
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
                device: int = 0, beta: float = 2.0, residual: bool = False):
    """Best cost after every epoch, the device time (s) at every epoch (from
    the first epoch's start) and the seconds spent applying the prior
    (residual: its levels added to the plain eta^beta levels)."""
    import torch
    s = torch.cuda.Stream(device)
    with N.Context(device) as c:
        c.set_stream(s.cuda_stream)
        c.setup_instance(inst, ants=ants, cand_k=cand_k, seed=seed, fixed_epochs=epochs,
                         beta=beta)
        t_prior = 0.0
        if prior is not None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            c.apply_prior(prior, gamma, residual=residual)
            e1.record(s)
            e1.synchronize()
            t_prior = e0.elapsed_time(e1) / 1e3
        _, recs = c.run(epochs, want_records=True)
    best = np.array([r.global_best for r in recs], np.float64)
    t = np.array([r.elapsed_ns for r in recs], np.float64) * 1e-9
    return best, t, t_prior


def _time_to(best, t, target, extra=0.0):
    """(epochs, seconds, hit) to the first epoch at or below target; a run
    that never gets there counts as its whole run plus one epoch."""
    hit = bool((best <= target).any())
    i = int(np.argmax(best <= target)) if hit else len(best)
    sec = (t[i] if hit else t[-1] + t[-1] / len(t)) + extra
    return i + 1, float(sec), hit


def time_to_cost(heldout: Sequence[I.Instance], prior: "N.Prior", gamma: float = 1.0,
                 epochs: int = 300, ants: int = 256, cand_k: int = 32, tol: float = 0.005,
                 seed: int = 1234, device: int = 0, control_beta: Optional[float] = None,
                 residual_beta: Optional[float] = None) -> Dict:
    """Per held-out instance: the plain solver's final cost C after `epochs`
    epochs, the target (1 + tol) C, and the time each solver first reaches
    it (the learned one pays its inference time too).  control_beta: also
    the plain solver with eta^control_beta (a sharper hand-set heuristic)
    against the same target.  residual_beta: the learned levels are added to
    the plain eta^residual_beta levels instead of replacing the plain ones."""
    rows = []
    for j, inst in enumerate(heldout):
        bp, tp, _ = convergence(inst, epochs, None, gamma, ants, cand_k, seed + j, device)
        if residual_beta is None:
            bl, tl, t_inf = convergence(inst, epochs, prior, gamma, ants, cand_k, seed + j, device)
        else:
            bl, tl, t_inf = convergence(inst, epochs, prior, gamma, ants, cand_k, seed + j, device,
                                        beta=residual_beta, residual=True)
        target = bp[-1] * (1.0 + tol)
        ep, sp, _ = _time_to(bp, tp, target)
        el, sl, hit = _time_to(bl, tl, target, t_inf)
        row = dict(plain_cost=float(bp[-1]), learned_cost=float(bl[-1]),
                   plain_epochs=ep, learned_epochs=el, learned_hit=hit,
                   plain_s=sp, learned_s=sl, prior_s=t_inf)
        if control_beta is not None:
            bc, tc, _ = convergence(inst, epochs, None, gamma, ants, cand_k, seed + j, device,
                                    beta=control_beta)
            ec, sc, hc = _time_to(bc, tc, target)
            row.update(control_cost=float(bc[-1]), control_epochs=ec, control_s=sc,
                       control_hit=hc)
        rows.append(row)
    ratio = np.array([r["learned_s"] / r["plain_s"] for r in rows])
    out = {
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
    if control_beta is not None:
        out["control"] = {
            "beta": control_beta,
            "time_ratio_of_sums": float(sum(r["control_s"] for r in rows) /
                                        sum(r["plain_s"] for r in rows)),
            "hit_rate": float(np.mean([r["control_hit"] for r in rows])),
            "final_cost_ratio_mean": float(np.mean([r["control_cost"] / r["plain_cost"]
                                                    for r in rows])),
            "learned_vs_control_final_cost_mean": float(np.mean(
                [r["learned_cost"] / r["control_cost"] for r in rows])),
        }
    return out


def final_costs(instances: Sequence[I.Instance], epochs: int = 300, prior=None,
                gamma: float = 1.0, residual: bool = False, beta: float = 2.0,
                ants: int = 256, cand_k: int = 32, seed: int = 100, device: int = 0):
    """Best cost after `epochs` epochs per instance (seed + index)."""
    import torch
    out = []
    for j, inst in enumerate(instances):
        s = torch.cuda.Stream(device)
        with N.Context(device) as c:
            c.set_stream(s.cuda_stream)
            c.setup_instance(inst, ants=ants, cand_k=cand_k, seed=seed + j, fixed_epochs=epochs,
                             beta=beta)
            if prior is not None:
                c.apply_prior(prior, gamma, residual=residual)
            out.append(c.run(epochs).global_best)
    return np.array(out)


def ablation(train: int = 2048, val: int = 12, epochs: int = 300, device: int = 0):
    """Final cost relative to the plain solver (beta = 2) on validation
    instances (n=1000, K=8, seeds 60000..): the plain solver with sharper
    hand-set eta^beta, and priors trained on elite routes of the plain solver
    at beta 2 and 8, their levels replacing (pure) or added to (residual,
    on plain levels of beta 2, 5 or 8) the plain levels.  Yields one dict
    per configuration."""
    tr = I.prior_training_instances(train)
    vs = [I.uniform_instance(1000, 8, 60000 + i) for i in range(val)]
    base = final_costs(vs, epochs, device=device)

    def row(tag, costs, **kw):
        r = costs / base
        return dict(config=tag, mean=float(r.mean()), min=float(r.min()), max=float(r.max()), **kw)

    for b in (5.0, 8.0, 12.0):
        yield row(f"plain beta={b:g}", final_costs(vs, epochs, beta=b, device=device))
    for eb in (2.0, 8.0):
        sols = elite_solutions(tr, epochs=120, beta=eb, device=device)
        with N.Prior(device, seed=1) as pr:
            count = pr.set_dataset(tr, [(x[0], x[1]) for x in sols], cand_k=32)
            losses = pr.train(10, batch=4096, lr=2e-3, seed=11)
            info = dict(elite_beta=eb, examples=count, loss=[float(losses[0]), float(losses[-1])])
            for g in (1.0, 2.0, 4.0):
                yield row(f"learned (elites beta={eb:g}) pure gamma={g:g}",
                          final_costs(vs, epochs, pr, g, device=device), **info)
            for g in (0.5, 1.0, 2.0):
                for pb in (2.0, 5.0, 8.0):
                    yield row(f"learned (elites beta={eb:g}) residual gamma={g:g} beta={pb:g}",
                              final_costs(vs, epochs, pr, g, True, pb, device=device), **info)


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned prior tools")
    ap.add_argument("command", choices=["ablation"])
    ap.add_argument("--train", type=int, default=2048)
    ap.add_argument("--val", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=300)
    a = ap.parse_args()
    for r in ablation(a.train, a.val, a.epochs):
        print(json.dumps(r), flush=True)
