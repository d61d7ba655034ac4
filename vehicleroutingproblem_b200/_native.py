"""ctypes binding of the C ABI in ``include/aco_b200.h``.

The shared library ``libaco_b200.so`` is built in-tree (``make lib`` or
``__graft_entry__.build()``).  There is no fallback: if the library is missing
or no CUDA device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Tuple

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libaco_b200.so")

ACO_OK = 0
ACO_ERR_INVALID_INPUT = 1
ACO_ERR_ALLOCATION = 2
ACO_ERR_NO_SOLUTION = 3
ACO_ERR_BACKEND = 4

LAYOUT_AUTO, LAYOUT_SMEM_WEIGHTS, LAYOUT_SMEM_PACKED, LAYOUT_GLOBAL = -1, 0, 1, 2
N_THRESHOLDS = 4095

# Every symbol include/aco_b200.h and include/aco.h declare.
EXPORTED = [
    "aco_b200_create", "aco_b200_destroy", "aco_b200_set_stream", "aco_b200_setup",
    "aco_b200_run", "aco_b200_enqueue_epochs", "aco_b200_synchronize",
    "aco_b200_get_best", "aco_b200_get_state", "aco_b200_get_dims", "aco_b200_get_plan",
    "aco_b200_get_tau", "aco_b200_set_tau", "aco_b200_get_candidates", "aco_b200_get_tier",
    "aco_b200_get_tier2",
    "aco_b200_get_tables", "aco_b200_get_weights", "aco_b200_construct",
    "aco_b200_get_ants", "aco_b200_evaporate_deposit", "aco_b200_build_info",
    "aco_b200_profile_epochs", "aco_b200_profile_update", "aco_b200_evaporate_deposit_noalloc",
    "aco_b200_seq_update_scratch_bytes", "aco_b200_seq_pheromone_update",
    "aco_b200_batch_create", "aco_b200_batch_destroy", "aco_b200_batch_setup",
    "aco_b200_batch_set_stream",
    "aco_b200_batch_set_tuning", "aco_b200_batch_get_tuning", "aco_b200_batch_autotune",
    "aco_b200_batch_set_cand_k", "aco_b200_batch_get_cand_k", "aco_b200_batch_autotune_k",
    "aco_b200_batch_solve", "aco_b200_batch_enqueue", "aco_b200_batch_synchronize",
    "aco_b200_batch_get", "aco_b200_batch_get_costs", "aco_b200_batch_get_all",
    "aco_b200_shard_packet_ints", "aco_b200_shard_construct", "aco_b200_shard_update",
    "aco_b200_graph_generation",
    "aco_b200_get_depot_tables", "aco_b200_debug_inject", "aco_b200_construct_with_draws",
    "aco_b200_prior_create", "aco_b200_prior_destroy", "aco_b200_prior_set_stream",
    "aco_b200_prior_init", "aco_b200_prior_set_params", "aco_b200_prior_get_params",
    "aco_b200_prior_load", "aco_b200_prior_save", "aco_b200_prior_set_dataset",
    "aco_b200_prior_train", "aco_b200_prior_gradient", "aco_b200_prior_num_examples",
    "aco_b200_prior_get_examples", "aco_b200_prior_get_rows", "aco_b200_apply_prior",
    "aco_b200_batch_apply_prior", "aco_b200_apply_prior_mode",
    "aco_status_string", "aco_vrp_cuda_with_capacity", "aco_vrp_cuda_with_demands",
    "solution_create", "solution_free", "solution_reset", "solution_copy",
    "solution_cost", "route_append", "solution_validate",
    "vrp_load_tsplib_euc2d_coords", "vrp_load_tsplib_euc2d_coords_demands",
    "aco_runtime_config_defaults", "aco_runtime_config_load_env",
    "aco_parse_min_rel_improvement_percent", "cli_parse_int_arg",
    "cli_parse_uint_arg", "cli_print_solution_routes", "cli_print_solution_cost",
    "cli_validate_solution_or_report",
]


class AcoError(RuntimeError):
    def __init__(self, status: int, where: str):
        names = {1: "invalid input", 2: "allocation failure", 3: "no solution",
                 4: "backend failure"}
        super().__init__(f"{where}: {names.get(status, 'status %d' % status)}")
        self.status = status


class Problem(C.Structure):
    _fields_ = [("n", C.c_int), ("K", C.c_int), ("capacity", C.c_longlong),
                ("ants", C.c_int), ("cand_k", C.c_int),
                ("x", C.c_void_p), ("y", C.c_void_p), ("demand", C.c_void_p),
                ("alpha", C.c_double), ("beta", C.c_double), ("rho", C.c_double),
                ("tau0", C.c_double), ("Q", C.c_double), ("seed", C.c_uint),
                ("stagnation_epochs", C.c_int), ("fixed_epochs", C.c_int),
                ("min_rel_improvement", C.c_double), ("timeout_seconds", C.c_double),
                ("ant_base", C.c_int), ("depot_rule", C.c_int)]


class State(C.Structure):
    _fields_ = [("epochs", C.c_int), ("iter_since_best", C.c_int),
                ("stopped", C.c_int), ("stop_reason", C.c_int), ("found", C.c_int),
                ("improved", C.c_int), ("best_ant", C.c_int), ("error", C.c_int),
                ("global_best", C.c_double), ("iter_best", C.c_double),
                ("dep_iter", C.c_float), ("dep_global", C.c_float),
                ("total_steps", C.c_ulonglong)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class EpochRecord(C.Structure):
    _fields_ = [("epoch", C.c_int), ("iter_since_best", C.c_int),
                ("improved", C.c_int), ("found", C.c_int),
                ("global_best", C.c_double), ("elapsed_ns", C.c_ulonglong)]


_lib = None


def library_path() -> str:
    return LIB_PATH


def load():
    """Loads libaco_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make lib` (or "
            "__graft_entry__.build()); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
    sigs = {
        "aco_b200_create": [vp, i32], "aco_b200_destroy": [vp],
        "aco_b200_set_stream": [vp, vp], "aco_b200_setup": [vp, vp],
        "aco_b200_run": [vp, i32, vp, vp, i32, vp],
        "aco_b200_enqueue_epochs": [vp, i32], "aco_b200_synchronize": [vp],
        "aco_b200_get_best": [vp, vp, vp, vp], "aco_b200_get_state": [vp, vp],
        "aco_b200_get_dims": [vp, vp, vp, vp, vp], "aco_b200_get_plan": [vp, vp],
        "aco_b200_get_tau": [vp, vp], "aco_b200_set_tau": [vp, vp],
        "aco_b200_get_candidates": [vp, vp, vp], "aco_b200_get_tier": [vp, vp],
        "aco_b200_get_tier2": [vp, vp],
        "aco_b200_get_tables": [vp, vp, vp, vp, i32],
        "aco_b200_get_weights": [vp, vp], "aco_b200_construct": [vp, i32, i32],
        "aco_b200_get_ants": [vp, vp, vp, vp, vp, vp, vp],
        "aco_b200_evaporate_deposit": [vp, i32, f32, vp, vp, f32],
        "aco_b200_profile_epochs": [vp, i32, vp],
        "aco_b200_profile_update": [vp, i32, vp],
        "aco_b200_batch_create": [vp, i32], "aco_b200_batch_destroy": [vp],
        "aco_b200_batch_set_stream": [vp, vp],
        "aco_b200_batch_setup": [vp, vp], "aco_b200_batch_set_tuning": [vp, vp],
        "aco_b200_batch_get_tuning": [vp, vp],
        "aco_b200_batch_autotune": [vp, i32, vp, vp, i32, vp],
        "aco_b200_batch_set_cand_k": [vp, i32], "aco_b200_batch_get_cand_k": [vp, vp],
        "aco_b200_batch_autotune_k": [vp, i32, vp, i32, C.c_double, vp, vp, vp, vp, vp, vp,
                                      i32, vp],
        "aco_b200_batch_solve": [vp], "aco_b200_batch_enqueue": [vp],
        "aco_b200_batch_synchronize": [vp],
        "aco_b200_batch_get": [vp, i32, vp, vp, vp, vp],
        "aco_b200_batch_get_all": [vp, vp, vp, vp],
        "aco_b200_batch_get_costs": [vp, vp, vp, vp],
        "aco_b200_shard_packet_ints": [vp], "aco_b200_shard_construct": [vp, vp],
        "aco_b200_shard_update": [vp, vp, i32], "aco_b200_graph_generation": [vp],
        "aco_b200_get_depot_tables": [vp, vp, vp, vp],
        "aco_b200_debug_inject": [vp, i32, i32],
        "aco_b200_construct_with_draws": [vp, vp, i32],
        "aco_b200_prior_create": [vp, i32], "aco_b200_prior_destroy": [vp],
        "aco_b200_prior_set_stream": [vp, vp], "aco_b200_prior_init": [vp, C.c_uint],
        "aco_b200_prior_set_params": [vp, vp, i32], "aco_b200_prior_get_params": [vp, vp, i32],
        "aco_b200_prior_load": [vp, C.c_char_p], "aco_b200_prior_save": [vp, C.c_char_p],
        "aco_b200_prior_set_dataset": [vp, vp, vp],
        "aco_b200_prior_train": [vp, i32, i32, f32, C.c_uint, vp],
        "aco_b200_prior_gradient": [vp, vp, i32, vp, vp],
        "aco_b200_prior_get_examples": [vp, vp, C.c_longlong],
        "aco_b200_prior_get_rows": [vp, C.c_longlong, i32, vp, vp, vp],
        "aco_b200_apply_prior": [vp, vp, f32],
        "aco_b200_apply_prior_mode": [vp, vp, f32, i32],
        "aco_b200_batch_apply_prior": [vp, vp, f32],
    }
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i32
    L.aco_b200_seq_update_scratch_bytes.argtypes = [i32]
    L.aco_b200_seq_update_scratch_bytes.restype = C.c_size_t
    f64 = C.c_double
    L.aco_b200_seq_pheromone_update.argtypes = [vp, i32, i32, vp, vp, f64, vp, vp, f64, f64,
                                                f64, f64, i32, f64, vp, vp]
    L.aco_b200_seq_pheromone_update.restype = i32
    L.aco_b200_prior_num_examples.argtypes = [vp]
    L.aco_b200_prior_num_examples.restype = C.c_longlong
    L.aco_b200_build_info.restype = C.c_char_p
    L.aco_status_string.restype = C.c_char_p
    L.aco_status_string.argtypes = [i32]
    _lib = L
    return L


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc: int, where: str) -> None:
    if rc != ACO_OK:
        raise AcoError(rc, where)


class Context:
    """One instance on one GPU (aco_b200_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        self._h = C.c_void_p()
        _check(self._lib.aco_b200_create(C.byref(self._h), device), "aco_b200_create")
        self._keep = []
        self.n = self.K = self.k = self.m = 0

    def close(self):
        if self._h:
            self._lib.aco_b200_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle: int) -> None:
        _check(self._lib.aco_b200_set_stream(self._h, C.c_void_p(stream_handle)),
               "aco_b200_set_stream")

    def setup(self, x, y, K: int, capacity: int, demand=None, ants: int = 256,
              cand_k: int = 0, alpha=1.0, beta=2.0, rho=0.5, tau0=1.0, Q=1.0,
              seed: int = 1234, stagnation_epochs: int = 0, fixed_epochs: int = 0,
              min_rel_improvement: float = 1e-3, timeout_seconds: float = 0.0,
              ant_base: int = 0, depot_rule: int = 0):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        d = None if demand is None else np.ascontiguousarray(demand, np.int32)
        self._keep = [x, y, d]
        p = Problem(n=len(x) - 1, K=K, capacity=int(capacity), ants=ants, cand_k=cand_k,
                    x=_p(x).value, y=_p(y).value, demand=None if d is None else _p(d).value,
                    alpha=alpha, beta=beta, rho=rho, tau0=tau0, Q=Q, seed=seed & 0xffffffff,
                    stagnation_epochs=stagnation_epochs, fixed_epochs=fixed_epochs,
                    min_rel_improvement=min_rel_improvement, timeout_seconds=timeout_seconds,
                    ant_base=ant_base, depot_rule=depot_rule)
        _check(self._lib.aco_b200_setup(self._h, C.byref(p)), "aco_b200_setup")
        n, K_, k, m = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(self._lib.aco_b200_get_dims(self._h, C.byref(n), C.byref(K_), C.byref(k),
                                            C.byref(m)), "aco_b200_get_dims")
        self.n, self.K, self.k, self.m = n.value, K_.value, k.value, m.value
        return self

    def plan(self) -> dict:
        """Launch shape of the construction (ants per block, table layout,
        register bitmap words per lane, shared memory bytes)."""
        out = np.zeros(4, np.int32)
        _check(self._lib.aco_b200_get_plan(self._h, _p(out)), "aco_b200_get_plan")
        return {"wpb": int(out[0]), "layout": int(out[1]), "vreg": int(out[2]),
                "smem": int(out[3])}

    def setup_instance(self, inst, **kw):
        demand = None if inst.is_unit_demand() else inst.demand
        return self.setup(inst.x, inst.y, inst.vehicles, inst.capacity, demand=demand, **kw)

    def run(self, max_epochs: int, want_records: bool = False):
        st = State()
        recs = (EpochRecord * max(1, max_epochs))() if want_records else None
        nrec = C.c_int(0)
        _check(self._lib.aco_b200_run(self._h, max_epochs, C.byref(st),
                                      recs, max_epochs if want_records else 0,
                                      C.byref(nrec)), "aco_b200_run")
        if want_records:
            return st, [recs[i] for i in range(nrec.value)]
        return st

    def enqueue_epochs(self, epochs: int) -> None:
        _check(self._lib.aco_b200_enqueue_epochs(self._h, epochs), "aco_b200_enqueue_epochs")

    def profile_epochs(self, epochs: int) -> np.ndarray:
        """Per-kernel device ms summed over `epochs` epochs, the kernels run
        one after another: [weights, construct, evaporate, best+deposit]."""
        ms = np.zeros(4, np.float32)
        _check(self._lib.aco_b200_profile_epochs(self._h, epochs, _p(ms)),
               "aco_b200_profile_epochs")
        return ms

    def profile_update(self, launches: int) -> float:
        """Mean device ms of one launch of the pheromone evaporation sweep
        (2 (n+1)^2 bytes read + written), timed alone over `launches`."""
        ms = np.zeros(1, np.float32)
        _check(self._lib.aco_b200_profile_update(self._h, launches, _p(ms)),
               "aco_b200_profile_update")
        return float(ms[0])

    def synchronize(self) -> None:
        _check(self._lib.aco_b200_synchronize(self._h), "aco_b200_synchronize")

    def state(self) -> State:
        st = State()
        _check(self._lib.aco_b200_get_state(self._h, C.byref(st)), "aco_b200_get_state")
        return st

    def best(self) -> Tuple[np.ndarray, np.ndarray, float]:
        nodes = np.zeros(self.n + 2 * self.K, np.int32)
        lens = np.zeros(self.K, np.int32)
        cost = C.c_double()
        rc = self._lib.aco_b200_get_best(self._h, _p(nodes), _p(lens), C.byref(cost))
        if rc == ACO_ERR_NO_SOLUTION:
            return nodes[:0], lens, float("inf")
        _check(rc, "aco_b200_get_best")
        return nodes[: int(lens.sum())].copy(), lens, cost.value

    def tau(self) -> np.ndarray:
        t = np.zeros((self.n + 1) * (self.n + 1), np.uint8)
        _check(self._lib.aco_b200_get_tau(self._h, _p(t)), "aco_b200_get_tau")
        return t

    def set_tau(self, tau: np.ndarray) -> None:
        t = np.ascontiguousarray(tau, np.uint8)
        assert t.size == (self.n + 1) ** 2
        _check(self._lib.aco_b200_set_tau(self._h, _p(t)), "aco_b200_set_tau")

    def candidates(self) -> Tuple[np.ndarray, np.ndarray]:
        cnt = (self.n + 1) * self.k
        cand = np.zeros(cnt, np.int32)
        lvl = np.zeros(cnt, np.uint16)
        _check(self._lib.aco_b200_get_candidates(self._h, _p(cand), _p(lvl)),
               "aco_b200_get_candidates")
        return cand, lvl

    def tier(self) -> np.ndarray:
        """Neighbours of ranks k+1 .. k+64 of every node ([(n+1) 64], 0 = empty)."""
        t = np.zeros((self.n + 1) * 64, np.uint16)
        _check(self._lib.aco_b200_get_tier(self._h, _p(t)), "aco_b200_get_tier")
        return t

    def tier2(self) -> np.ndarray:
        """Neighbours of ranks k+65 .. k+256 ([(n+1) 192], 0 = empty; n >= 1500)."""
        t = np.zeros((self.n + 1) * 192, np.uint16)
        _check(self._lib.aco_b200_get_tier2(self._h, _p(t)), "aco_b200_get_tier2")
        return t

    def tables(self):
        A = np.zeros(256, np.int32)
        lut = np.zeros(256, np.uint32)
        thr = np.zeros(N_THRESHOLDS, np.float32)
        _check(self._lib.aco_b200_get_tables(self._h, _p(A), _p(lut), _p(thr), N_THRESHOLDS),
               "aco_b200_get_tables")
        return A, lut, thr

    def weights(self) -> np.ndarray:
        w = np.zeros((self.n + 1) * self.k, np.uint32)
        _check(self._lib.aco_b200_get_weights(self._h, _p(w)), "aco_b200_get_weights")
        return w

    def debug_inject(self, what: int, value: int) -> None:
        """Fault-injection test hook (aco_b200_debug_inject): what 1 fails the
        value-th device allocation of the next set-up; what 2 makes the
        construct kernel's staging wait run out (value 1) or not (0)."""
        _check(self._lib.aco_b200_debug_inject(self._h, what, value), "aco_b200_debug_inject")

    def depot_tables(self):
        """Reference-CUDA depot rule: (lvl0 [n+1], rdep [n+1] of the last
        weights pass, e_dep)."""
        lvl0 = np.zeros(self.n + 1, np.uint16)
        rdep = np.zeros(self.n + 1, np.int32)
        e = C.c_int()
        _check(self._lib.aco_b200_get_depot_tables(self._h, _p(lvl0), _p(rdep), C.byref(e)),
               "aco_b200_get_depot_tables")
        return lvl0, rdep, e.value

    def construct_with_draws(self, draws) -> None:
        """One construct pass on recorded draws [m][per_ant] (24-bit values)."""
        d = np.ascontiguousarray(draws, np.uint32)
        assert d.ndim == 2 and d.shape[0] == self.m
        _check(self._lib.aco_b200_construct_with_draws(self._h, _p(d), d.shape[1]),
               "aco_b200_construct_with_draws")

    def construct(self, epoch: int, layout: int = LAYOUT_AUTO) -> None:
        _check(self._lib.aco_b200_construct(self._h, epoch, layout), "aco_b200_construct")

    def ants(self):
        R = self.n + 2 * self.K
        nodes = np.zeros(self.m * R, np.int32)
        lens = np.zeros(self.m * self.K, np.int32)
        cost = np.zeros(self.m, np.float64)
        feas = np.zeros(self.m, np.int32)
        steps = np.zeros(self.m, np.int32)
        draws = np.zeros(self.m, np.uint32)
        _check(self._lib.aco_b200_get_ants(self._h, _p(nodes), _p(lens), _p(cost), _p(feas),
                                           _p(steps), _p(draws)), "aco_b200_get_ants")
        return (nodes.reshape(self.m, R), lens.reshape(self.m, self.K), cost, feas, steps,
                draws)

    def evaporate_deposit(self, best_ant: int, dep_iter: float, gbest_nodes=None,
                          gbest_lens=None, dep_global: float = 0.0) -> None:
        gn = None if gbest_nodes is None else np.ascontiguousarray(gbest_nodes, np.int32)
        gl = None if gbest_lens is None else np.ascontiguousarray(gbest_lens, np.int32)
        _check(self._lib.aco_b200_evaporate_deposit(self._h, best_ant, dep_iter, _p(gn),
                                                    _p(gl), dep_global),
               "aco_b200_evaporate_deposit")

    # --- colony split over several devices (aco_b200_shard_*) -------------

    def shard_packet_ints(self) -> int:
        P = self._lib.aco_b200_shard_packet_ints(self._h)
        if P < 0:
            raise AcoError(ACO_ERR_INVALID_INPUT, "aco_b200_shard_packet_ints")
        return P

    def graph_generation(self) -> int:
        """Changes whenever a set-up changes the arguments the context's
        launches are recorded with; graphs recorded around its launches are
        re-recorded when it does."""
        return int(self._lib.aco_b200_graph_generation(self._h))

    def shard_construct(self, d_send: int) -> None:
        """Enqueues weights, construction and the packet of this device's best
        ant into the device buffer at address d_send."""
        _check(self._lib.aco_b200_shard_construct(self._h, C.c_void_p(d_send)),
               "aco_b200_shard_construct")

    def shard_update(self, d_recv: int, world: int) -> None:
        """Enqueues winner selection over `world` gathered packets at device
        address d_recv, bookkeeping, evaporation and deposits."""
        _check(self._lib.aco_b200_shard_update(self._h, C.c_void_p(d_recv), world),
               "aco_b200_shard_update")

    def apply_prior(self, prior: Optional["Prior"], gamma: float = 1.0,
                    residual: bool = False) -> None:
        """Learned eta levels from `prior` (None or gamma <= 0: plain levels);
        residual: added to the plain levels instead of replacing them."""
        _check(self._lib.aco_b200_apply_prior_mode(self._h, prior._h if prior else None, gamma,
                                                   1 if residual else 0),
               "aco_b200_apply_prior_mode")


PRIOR_PARAMS = 4801


class PriorDataset(C.Structure):
    _fields_ = [("count", C.c_int), ("n", C.c_void_p), ("K", C.c_void_p),
                ("capacity", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p),
                ("demand", C.c_void_p), ("nodes", C.c_void_p), ("lens", C.c_void_p),
                ("cand_k", C.c_int)]


class Prior:
    """Learned heuristic prior (aco_b200_prior): MLP parameters, training set,
    tensor-core training and inference."""

    def __init__(self, device: int = 0, seed: Optional[int] = None):
        self._lib = load()
        self._h = C.c_void_p()
        _check(self._lib.aco_b200_prior_create(C.byref(self._h), device), "aco_b200_prior_create")
        if seed is not None:
            self.init(seed)

    def close(self):
        if self._h:
            self._lib.aco_b200_prior_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init(self, seed: int) -> None:
        _check(self._lib.aco_b200_prior_init(self._h, seed & 0xffffffff), "aco_b200_prior_init")

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == PRIOR_PARAMS
        _check(self._lib.aco_b200_prior_set_params(self._h, _p(p), PRIOR_PARAMS),
               "aco_b200_prior_set_params")

    def params(self) -> np.ndarray:
        p = np.zeros(PRIOR_PARAMS, np.float32)
        _check(self._lib.aco_b200_prior_get_params(self._h, _p(p), PRIOR_PARAMS),
               "aco_b200_prior_get_params")
        return p

    def save(self, path: str) -> None:
        _check(self._lib.aco_b200_prior_save(self._h, path.encode()), "aco_b200_prior_save")

    def load(self, path: str) -> None:
        _check(self._lib.aco_b200_prior_load(self._h, path.encode()), "aco_b200_prior_load")

    def set_dataset(self, instances, solutions, cand_k: int = 32) -> int:
        """instances: list of Instance; solutions: list of (nodes, lens) in
        compact form.  Returns the number of training examples."""
        n = np.array([x.n for x in instances], np.int32)
        K = np.array([x.vehicles for x in instances], np.int32)
        cap = np.array([x.capacity for x in instances], np.int64)
        xs = np.concatenate([x.x for x in instances]).astype(np.float32)
        ys = np.concatenate([x.y for x in instances]).astype(np.float32)
        dem = np.concatenate([x.demand for x in instances]).astype(np.int32)
        nodes = np.concatenate([np.asarray(s[0], np.int32) for s in solutions])
        lens = np.concatenate([np.asarray(s[1], np.int32) for s in solutions])
        keep = [n, K, cap, xs, ys, dem, nodes, lens]
        d = PriorDataset(count=len(instances), n=_p(n).value, K=_p(K).value, capacity=_p(cap).value,
                         x=_p(xs).value, y=_p(ys).value, demand=_p(dem).value,
                         nodes=_p(nodes).value, lens=_p(lens).value, cand_k=cand_k)
        cnt = C.c_longlong()
        _check(self._lib.aco_b200_prior_set_dataset(self._h, C.byref(d), C.byref(cnt)),
               "aco_b200_prior_set_dataset")
        del keep
        return cnt.value

    def num_examples(self) -> int:
        return int(self._lib.aco_b200_prior_num_examples(self._h))

    def examples(self) -> np.ndarray:
        cnt = self.num_examples()
        e = np.zeros(2 * max(cnt, 1), np.int32)
        _check(self._lib.aco_b200_prior_get_examples(self._h, _p(e), cnt),
               "aco_b200_prior_get_examples")
        return e[: 2 * cnt].reshape(cnt, 2)

    def rows(self, first: int, count: int, scores: bool = False):
        """(features [count][32][8] BF16 bit patterns, kv [count],
        scores [count][32] or None)."""
        f = np.zeros(count * 32 * 8, np.uint16)
        kv = np.zeros(count, np.uint8)
        sc = np.zeros(count * 32, np.float32) if scores else None
        _check(self._lib.aco_b200_prior_get_rows(self._h, first, count, _p(f), _p(kv), _p(sc)),
               "aco_b200_prior_get_rows")
        return f.reshape(count, 32, 8), kv, None if sc is None else sc.reshape(count, 32)

    def gradient(self, example_ids):
        ids = np.ascontiguousarray(example_ids, np.int32)
        g = np.zeros(PRIOR_PARAMS, np.float32)
        loss = C.c_float()
        _check(self._lib.aco_b200_prior_gradient(self._h, _p(ids), len(ids), _p(g),
                                                 C.byref(loss)), "aco_b200_prior_gradient")
        return float(loss.value), g

    def train(self, epochs: int, batch: int = 2048, lr: float = 1e-3, seed: int = 0):
        losses = np.zeros(max(epochs, 1), np.float32)
        _check(self._lib.aco_b200_prior_train(self._h, epochs, batch, lr, seed & 0xffffffff,
                                              _p(losses)), "aco_b200_prior_train")
        return losses[:epochs]


class BatchProblem(C.Structure):
    _fields_ = [("count", C.c_int), ("n", C.c_void_p), ("K", C.c_void_p),
                ("capacity", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p),
                ("demand", C.c_void_p), ("ants", C.c_int), ("cand_k", C.c_int),
                ("alpha", C.c_double), ("beta", C.c_double), ("rho", C.c_double),
                ("tau0", C.c_double), ("Q", C.c_double), ("seed", C.c_uint),
                ("epochs", C.c_int), ("stagnation_epochs", C.c_int),
                ("min_rel_improvement", C.c_double)]


class BatchTuning(C.Structure):
    _fields_ = [("lanes_per_ant", C.c_int), ("ants_per_block", C.c_int), ("order", C.c_int)]

    def as_tuple(self):
        return (self.lanes_per_ant, self.ants_per_block, self.order)


class Batch:
    """Many instances in one persistent launch (aco_b200_batch)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        self._h = C.c_void_p()
        _check(self._lib.aco_b200_batch_create(C.byref(self._h), device), "aco_b200_batch_create")
        self.count = 0
        self.instances = []

    def close(self):
        if self._h:
            self._lib.aco_b200_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def setup(self, instances, ants=64, cand_k=16, seed=1234, epochs=300,
              stagnation_epochs=0, alpha=1.0, beta=2.0, rho=0.5, tau0=1.0, Q=1.0,
              min_rel_improvement=1e-3):
        ns = np.array([i.n for i in instances], np.int32)
        Ks = np.array([i.vehicles for i in instances], np.int32)
        caps = np.array([i.capacity for i in instances], np.int64)
        x = np.concatenate([i.x for i in instances]).astype(np.float32)
        y = np.concatenate([i.y for i in instances]).astype(np.float32)
        unit = all(i.is_unit_demand() for i in instances)
        d = None if unit else np.concatenate([i.demand for i in instances]).astype(np.int32)
        self._keep = [ns, Ks, caps, x, y, d]
        p = BatchProblem(count=len(instances), n=_p(ns).value, K=_p(Ks).value,
                         capacity=_p(caps).value, x=_p(x).value, y=_p(y).value,
                         demand=None if d is None else _p(d).value, ants=ants, cand_k=cand_k,
                         alpha=alpha, beta=beta, rho=rho, tau0=tau0, Q=Q,
                         seed=seed & 0xffffffff, epochs=epochs,
                         stagnation_epochs=stagnation_epochs,
                         min_rel_improvement=min_rel_improvement)
        _check(self._lib.aco_b200_batch_setup(self._h, C.byref(p)), "aco_b200_batch_setup")
        self.count = len(instances)
        self.instances = list(instances)
        return self

    def set_stream(self, stream_handle: int) -> None:
        _check(self._lib.aco_b200_batch_set_stream(self._h, C.c_void_p(stream_handle)),
               "aco_b200_batch_set_stream")

    def set_tuning(self, lanes_per_ant, ants_per_block, order=1):
        t = BatchTuning(lanes_per_ant, ants_per_block, order)
        _check(self._lib.aco_b200_batch_set_tuning(self._h, C.byref(t)),
               "aco_b200_batch_set_tuning")

    def tuning(self):
        t = BatchTuning()
        _check(self._lib.aco_b200_batch_get_tuning(self._h, C.byref(t)),
               "aco_b200_batch_get_tuning")
        return t.as_tuple()

    def autotune(self, trial_epochs=3):
        t = BatchTuning()
        ms = np.zeros(16, np.float32)
        nt = C.c_int()
        _check(self._lib.aco_b200_batch_autotune(self._h, trial_epochs, C.byref(t), _p(ms), 16,
                                                 C.byref(nt)), "aco_b200_batch_autotune")
        return t.as_tuple(), ms[: nt.value].copy()

    def set_cand_k(self, k: int) -> None:
        _check(self._lib.aco_b200_batch_set_cand_k(self._h, k), "aco_b200_batch_set_cand_k")

    def cand_k(self) -> int:
        k = C.c_int()
        _check(self._lib.aco_b200_batch_get_cand_k(self._h, C.byref(k)),
               "aco_b200_batch_get_cand_k")
        return k.value

    def autotune_k(self, ks=(16, 20, 32), quality_tol=0.005, trial_epochs=3):
        """Candidate-list length, then launch shape (aco_b200_batch_autotune_k):
        returns (k, shape, per-length {k: (solve ms, mean cost, solved)},
        shape trial ms)."""
        kk = np.array(ks, np.int32)
        t = BatchTuning()
        ck = C.c_int()
        kms = np.zeros(len(ks), np.float64)
        kcost = np.zeros(len(ks), np.float64)
        kfeas = np.zeros(len(ks), np.int32)
        ms = np.zeros(16, np.float32)
        nt = C.c_int()
        _check(self._lib.aco_b200_batch_autotune_k(
            self._h, trial_epochs, _p(kk), len(ks), quality_tol, C.byref(t), C.byref(ck),
            _p(kms), _p(kcost), _p(kfeas), _p(ms), 16, C.byref(nt)), "aco_b200_batch_autotune_k")
        per = {int(k): (float(kms[i]), float(kcost[i]), int(kfeas[i])) for i, k in enumerate(ks)}
        return ck.value, t.as_tuple(), per, ms[: nt.value].copy()

    def solve(self):
        _check(self._lib.aco_b200_batch_solve(self._h), "aco_b200_batch_solve")

    def enqueue(self):
        _check(self._lib.aco_b200_batch_enqueue(self._h), "aco_b200_batch_enqueue")

    def synchronize(self):
        _check(self._lib.aco_b200_batch_synchronize(self._h), "aco_b200_batch_synchronize")

    def best(self, i):
        inst = self.instances[i]
        nodes = np.zeros(inst.n + 2 * inst.vehicles, np.int32)
        lens = np.zeros(inst.vehicles, np.int32)
        cost = C.c_double()
        ep = C.c_int()
        rc = self._lib.aco_b200_batch_get(self._h, i, _p(nodes), _p(lens), C.byref(cost),
                                          C.byref(ep))
        if rc == ACO_ERR_NO_SOLUTION:
            return nodes[:0], lens, float("inf"), ep.value
        _check(rc, "aco_b200_batch_get")
        return nodes[: int(lens.sum())].copy(), lens, cost.value, ep.value

    def best_all(self):
        """Best solution of every instance, read in three copies: a list of
        (nodes, lens, cost) as best() returns them (nodes empty and cost inf
        where no ant was feasible)."""
        insts = self.instances
        slot = np.array([i.n + 2 * i.vehicles for i in insts], np.int64)
        kv = np.array([i.vehicles for i in insts], np.int64)
        nodes = np.zeros(int(slot.sum()), np.int32)
        lens = np.zeros(int(kv.sum()), np.int32)
        costs = np.zeros(len(insts), np.float64)
        _check(self._lib.aco_b200_batch_get_all(self._h, _p(nodes), _p(lens), _p(costs)),
               "aco_b200_batch_get_all")
        out = []
        no = np.concatenate([[0], np.cumsum(slot)])
        lo = np.concatenate([[0], np.cumsum(kv)])
        for i in range(len(insts)):
            ln = lens[lo[i]:lo[i + 1]].copy()
            c = float(costs[i])
            if c >= np.finfo(np.float64).max:
                out.append((nodes[:0].copy(), ln, float("inf")))
            else:
                out.append((nodes[no[i]:no[i] + int(ln.sum())].copy(), ln, c))
        return out

    def apply_prior(self, prior: Optional[Prior], gamma: float = 1.0) -> None:
        _check(self._lib.aco_b200_batch_apply_prior(self._h, prior._h if prior else None, gamma),
               "aco_b200_batch_apply_prior")

    def costs(self):
        c = np.zeros(self.count, np.float64)
        e = np.zeros(self.count, np.int32)
        s = np.zeros(self.count, np.uint64)
        _check(self._lib.aco_b200_batch_get_costs(self._h, _p(c), _p(e), _p(s)),
               "aco_b200_batch_get_costs")
        return c, e, s


def build_info() -> str:
    return load().aco_b200_build_info().decode()


def split_routes(nodes: np.ndarray, lens: np.ndarray) -> List[List[int]]:
    out, off = [], 0
    for ln in lens:
        out.append([int(v) for v in nodes[off:off + int(ln)]])
        off += int(ln)
    return out
