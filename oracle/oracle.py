"""ctypes front end of the oracle (test infrastructure only).

Loads ``oracle/liboracle.so`` (own C restatement, always built) and, when
present, ``oracle/_ref/libseqref.so`` (the reference's own seq construct code
driven with recorded draws).  Only tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
SEQREF_PATH = os.path.join(REF_DIR, "libseqref.so")

J_LEVELS = 4095          # threshold table length
REL_MAX = 255

_lib = None
_ref = None


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def build() -> None:
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, u32, f32, f64, i64 = C.c_void_p, C.c_int, C.c_uint32, C.c_float, C.c_double, C.c_int64
        L.orc_philox4x32_10.argtypes = [vp, vp, vp]
        L.orc_draw24.argtypes = [u32, u32, u32, u32, u32]
        L.orc_draw24.restype = u32
        L.orc_params.argtypes = [f64, f64, vp, vp, vp, vp]
        L.orc_tables.argtypes = [f64, f64, f32, vp, vp, vp, i32]
        L.orc_level.argtypes = [f32, vp, i32]
        L.orc_level.restype = C.c_uint16
        L.orc_knn.argtypes = [i32, i32, vp, vp, vp]
        L.orc_levels.argtypes = [i32, i32, vp, vp, vp, vp, i32, vp]
        L.orc_weights.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp]
        L.orc_route_cost.argtypes = [vp, vp, vp, vp, i32]
        L.orc_route_cost.restype = f64
        L.orc_construct_ant.argtypes = [i32, i32, i32, i64, vp, vp, vp, vp, vp,
                                        u32, u32, u32, u32, vp, vp, vp, vp, vp]
        L.orc_construct_ant.restype = i32
        L.orc_construct_ant_rule.argtypes = [i32, i32, i32, i64, vp, vp, vp, vp, vp,
                                             u32, u32, u32, u32, i32, vp, vp,
                                             vp, vp, vp, vp, vp]
        L.orc_construct_ant_rule.restype = i32
        L.orc_depot_rel.argtypes = [i32, i32, vp, vp, vp, vp, vp, C.c_int32, vp]
        L.orc_evaporate.argtypes = [vp, C.c_uint64, C.c_uint8, C.c_uint8]
        L.orc_deposit_level.argtypes = [C.c_uint8, f32, f32, f32, C.c_uint8, C.c_uint8]
        L.orc_deposit_level.restype = C.c_uint8
        L.orc_deposit.argtypes = [vp, i32, vp, vp, i32, f32, f32, f32, C.c_uint8, C.c_uint8]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(SEQREF_PATH)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(SEQREF_PATH)
        vp, i32 = C.c_void_p, C.c_int
        R.seqref_construct_ant.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp]
        R.seqref_construct_ant.restype = i32
        R.seqref_construct_ants.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, i32, vp, i32,
                                            vp, vp, vp, vp]
        R.seqref_construct_ants.restype = i32
        R.seqref_solution_cost.argtypes = [i32, i32, vp, vp, vp, vp]
        R.seqref_solution_cost.restype = C.c_double
        R.seqref_validate.argtypes = [i32, i32, vp, vp]
        R.seqref_validate.restype = i32
        _ref = R
    return _ref


# --------------------------------------------------------------------------

def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def draw24(seed, epoch, ant, stream, d) -> int:
    return int(lib().orc_draw24(seed, epoch, ant, stream, d))


def draws(seed, epoch, ant, stream, count) -> np.ndarray:
    return np.array([draw24(seed, epoch, ant, stream, d) for d in range(count)],
                    dtype=np.uint32)


def params(rho=0.5, tau0=1.0):
    lmin, step = C.c_float(), C.c_float()
    delta, q0 = C.c_uint8(), C.c_uint8()
    lib().orc_params(rho, tau0, C.byref(lmin), C.byref(step), C.byref(delta), C.byref(q0))
    return dict(log_tau_min=lmin.value, log_tau_step=step.value,
                q_evap_delta=delta.value, q_tau0=q0.value, q_tau_min=0, q_tau_max=255)


def tables(alpha=1.0, beta=2.0, log_tau_step=None):
    if log_tau_step is None:
        log_tau_step = params()["log_tau_step"]
    A = np.zeros(256, dtype=np.int32)
    lut = np.zeros(256, dtype=np.uint32)
    thr = np.zeros(J_LEVELS, dtype=np.float32)
    lib().orc_tables(alpha, beta, log_tau_step, _p(A), _p(lut), _p(thr), J_LEVELS)
    return A, lut, thr


def knn(x, y, k) -> np.ndarray:
    n = len(x) - 1
    cand = np.zeros((n + 1) * k, dtype=np.int32)
    lib().orc_knn(n, k, _p(np.ascontiguousarray(x, np.float32)),
                  _p(np.ascontiguousarray(y, np.float32)), _p(cand))
    return cand


def levels(x, y, cand, k, thr) -> np.ndarray:
    n = len(x) - 1
    lvl = np.zeros((n + 1) * k, dtype=np.uint16)
    lib().orc_levels(n, k, _p(np.ascontiguousarray(x, np.float32)),
                     _p(np.ascontiguousarray(y, np.float32)),
                     _p(np.ascontiguousarray(cand, np.int32)), _p(thr), len(thr), _p(lvl))
    return lvl


def weights(n, k, cand, lvl, tau, A, lut) -> np.ndarray:
    w = np.zeros((n + 1) * k, dtype=np.uint32)
    lib().orc_weights(n, k, _p(np.ascontiguousarray(cand, np.int32)),
                      _p(np.ascontiguousarray(lvl, np.uint16)),
                      _p(np.ascontiguousarray(tau, np.uint8)), _p(A), _p(lut), _p(w))
    return w


def depot_rel(n, k, cand, lvl, tau, A, lvl0, e_dep) -> np.ndarray:
    """Depot-close levels of the reference-CUDA depot rule, per row."""
    out = np.zeros(n + 1, dtype=np.int32)
    lib().orc_depot_rel(n, k, _p(np.ascontiguousarray(cand, np.int32)),
                        _p(np.ascontiguousarray(lvl, np.uint16)),
                        _p(np.ascontiguousarray(tau, np.uint8)),
                        _p(np.ascontiguousarray(A, np.int32)),
                        _p(np.ascontiguousarray(lvl0, np.uint16)), int(e_dep), _p(out))
    return out


def construct_ant(inst_x, inst_y, demand, K, cap, k, cand, w, seed, epoch, ant,
                  stream=0, rule=0, rdep=None, lut=None):
    """Returns (feasible, nodes, lens, cost, steps, draws_used).  rule 1 is
    the reference-CUDA depot rule (needs rdep and the weight LUT)."""
    n = len(inst_x) - 1
    nodes = np.zeros(n + 2 * K, dtype=np.int32)
    lens = np.zeros(K, dtype=np.int32)
    cost = C.c_double()
    steps = C.c_int32()
    used = C.c_uint32()
    dem = None if demand is None else np.ascontiguousarray(demand, np.int32)
    if rule == 0:
        feas = lib().orc_construct_ant(
            n, K, k, int(cap), _p(np.ascontiguousarray(inst_x, np.float32)),
            _p(np.ascontiguousarray(inst_y, np.float32)), _p(dem),
            _p(np.ascontiguousarray(cand, np.int32)), _p(np.ascontiguousarray(w, np.uint32)),
            seed, epoch, ant, stream, _p(nodes), _p(lens), C.byref(cost), C.byref(steps),
            C.byref(used))
    else:
        feas = lib().orc_construct_ant_rule(
            n, K, k, int(cap), _p(np.ascontiguousarray(inst_x, np.float32)),
            _p(np.ascontiguousarray(inst_y, np.float32)), _p(dem),
            _p(np.ascontiguousarray(cand, np.int32)), _p(np.ascontiguousarray(w, np.uint32)),
            seed, epoch, ant, stream, int(rule), _p(np.ascontiguousarray(rdep, np.int32)),
            _p(np.ascontiguousarray(lut, np.uint32)), _p(nodes), _p(lens), C.byref(cost),
            C.byref(steps), C.byref(used))
    total = int(lens.sum())
    return bool(feas), nodes[:total].copy(), lens, cost.value, steps.value, used.value


def route_cost(x, y, nodes, lens) -> float:
    return lib().orc_route_cost(_p(np.ascontiguousarray(x, np.float32)),
                                _p(np.ascontiguousarray(y, np.float32)),
                                _p(np.ascontiguousarray(nodes, np.int32)),
                                _p(np.ascontiguousarray(lens, np.int32)), len(lens))


def evaporate(tau: np.ndarray, delta: int, q_min: int = 0) -> np.ndarray:
    t = np.ascontiguousarray(tau, np.uint8).copy()
    lib().orc_evaporate(_p(t), t.size, delta, q_min)
    return t


def deposit(tau: np.ndarray, n, nodes, lens, dep, log_min, log_step, q_min=0,
            q_max=255) -> np.ndarray:
    t = np.ascontiguousarray(tau, np.uint8).copy()
    lib().orc_deposit(_p(t), n, _p(np.ascontiguousarray(nodes, np.int32)),
                      _p(np.ascontiguousarray(lens, np.int32)), len(lens), dep,
                      log_min, log_step, q_min, q_max)
    return t


# --------------------------------------------------------------------------
# The reference's own code (oracle/_ref), when built.
# --------------------------------------------------------------------------

def ref_construct_ants(x, y, K, cap, k, cand, w, draw_streams):
    """The reference's build_ant_solution for every row of draw_streams
    (m x n_draws recorded draws), one distance matrix for all ants.
    Returns [(nodes, lens, cost, used)] per ant."""
    n = len(x) - 1
    d = np.ascontiguousarray(draw_streams, np.uint32)
    m, nd = d.shape
    nodes = np.zeros((m, n + 2 * K), dtype=np.int32)
    lens = np.zeros((m, K), dtype=np.int32)
    cost = np.zeros(m, dtype=np.float64)
    used = np.zeros(m, dtype=np.int32)
    rc = ref().seqref_construct_ants(
        n, K, int(cap), k, _p(np.ascontiguousarray(x, np.float32)),
        _p(np.ascontiguousarray(y, np.float32)), _p(np.ascontiguousarray(cand, np.int32)),
        _p(np.ascontiguousarray(w, np.uint32)), m, _p(d), nd, _p(nodes), _p(lens), _p(cost),
        _p(used))
    if rc < 0:
        raise RuntimeError(f"seqref_construct_ants failed ({rc})")
    return [(nodes[a, : int(lens[a].sum())].copy(), lens[a].copy(), float(cost[a]),
             int(used[a])) for a in range(m)]


def ref_construct_ant(x, y, K, cap, k, cand, w, draw_stream):
    n = len(x) - 1
    nodes = np.zeros(n + 2 * K, dtype=np.int32)
    lens = np.zeros(K, dtype=np.int32)
    cost = C.c_double()
    d = np.ascontiguousarray(draw_stream, np.uint32)
    used = ref().seqref_construct_ant(
        n, K, int(cap), k, _p(np.ascontiguousarray(x, np.float32)),
        _p(np.ascontiguousarray(y, np.float32)), _p(np.ascontiguousarray(cand, np.int32)),
        _p(np.ascontiguousarray(w, np.uint32)), _p(d), len(d), _p(nodes), _p(lens),
        C.byref(cost))
    if used < 0:
        raise RuntimeError(f"seqref_construct_ant failed ({used})")
    total = int(lens.sum())
    return nodes[:total].copy(), lens, cost.value, used


def ref_validate(n, K, nodes, lens) -> bool:
    return bool(ref().seqref_validate(n, K, _p(np.ascontiguousarray(nodes, np.int32)),
                                      _p(np.ascontiguousarray(lens, np.int32))))


def ref_cost(x, y, nodes, lens) -> float:
    n = len(x) - 1
    return ref().seqref_solution_cost(n, len(lens), _p(np.ascontiguousarray(x, np.float32)),
                                      _p(np.ascontiguousarray(y, np.float32)),
                                      _p(np.ascontiguousarray(nodes, np.int32)),
                                      _p(np.ascontiguousarray(lens, np.int32)))


def seq_pheromone_update(tau, n, it_nodes, it_lens, d_it, gb_nodes, gb_lens, d_gb, rho,
                         tau_min, tau_max, reset, tau0) -> np.ndarray:
    """The sequential path's FP64 pheromone update (src/seq/aco_sequential.c:
    829-886) on an (n+1)^2 row-major matrix: evaporation of every i != j by
    (1 - rho); both directions of every arc of the iteration best, then of
    the global best (gb_nodes None to skip), arc by arc in route order; the
    MMAS clamp of every i != j; the 0.5 tau + 0.5 tau0 reset when `reset`.
    numpy's float64 element-wise operations are single IEEE operations in
    this order, as the reference's loops are."""
    t = np.array(tau, dtype=np.float64).reshape(n + 1, n + 1).copy()
    off = ~np.eye(n + 1, dtype=bool)
    t[off] = t[off] * (1.0 - rho)
    for nodes, lens, d in ((it_nodes, it_lens, d_it), (gb_nodes, gb_lens, d_gb)):
        if nodes is None:
            continue
        nodes = np.asarray(nodes, np.int64)
        e = 0
        for ln in lens:
            for q in range(int(ln) - 1):
                u, v = nodes[e + q], nodes[e + q + 1]
                t[u, v] += d
                t[v, u] += d
            e += int(ln)
    x = t[off]
    x = np.where(x < tau_min, tau_min, np.where(x > tau_max, tau_max, x))
    if reset:
        x = 0.5 * x + 0.5 * tau0
    t[off] = x
    return t.ravel()
