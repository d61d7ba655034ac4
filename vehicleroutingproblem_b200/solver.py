"""Python mirror of the reference's solver interface for the GPU hot path.

``aco_vrp_cuda_with_capacity`` / ``aco_vrp_cuda_with_demands`` call the
library's C entry points of the same names (reference:
src/cuda/aco_cuda.cu:188-192) with a ``Solution`` created by the library's
``solution_create`` and return ``(status, routes, cost)``; routes are the K
node lists including both depots, as in the reference's ``Solution``.
``solve`` is the context-based form (include/aco_b200.h) used by the tests
and the benchmark.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

import numpy as np

from . import _native
from .instances import Instance


class _Route(C.Structure):
    _fields_ = [("nodes", C.POINTER(C.c_int)), ("len", C.c_int), ("cap", C.c_int)]


class _Solution(C.Structure):
    _fields_ = [("routes", C.POINTER(_Route)), ("K", C.c_int), ("route_cap", C.c_int),
                ("nodes_storage", C.POINTER(C.c_int))]


def _bind(L):
    if getattr(L, "_solver_bound", False):
        return L
    L.solution_create.restype = C.POINTER(_Solution)
    L.solution_create.argtypes = [C.c_int, C.c_int]
    L.solution_free.argtypes = [C.POINTER(_Solution)]
    L.solution_validate.argtypes = [C.POINTER(_Solution), C.c_int, C.c_int, C.c_char_p,
                                    C.c_size_t]
    L.solution_validate.restype = C.c_bool
    f = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    tail = [C.c_double] * 5 + [C.c_uint, C.POINTER(_Solution), C.POINTER(C.c_double)]
    L.aco_vrp_cuda_with_capacity.argtypes = f + tail
    L.aco_vrp_cuda_with_capacity.restype = C.c_int
    L.aco_vrp_cuda_with_demands.argtypes = f + [C.c_void_p] + tail
    L.aco_vrp_cuda_with_demands.restype = C.c_int
    L._solver_bound = True
    return L


def _routes(sol) -> List[List[int]]:
    s = sol.contents
    return [[s.routes[v].nodes[t] for t in range(s.routes[v].len)] for v in range(s.K)]


def aco_vrp_cuda_with_capacity(n: int, K: int, capacity: int, m: int, x, y,
                               alpha=1.0, beta=2.0, rho=0.5, tau0=1.0, Q=1.0,
                               seed: int = 1234) -> Tuple[int, List[List[int]], float]:
    L = _bind(_native.load())
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.ascontiguousarray(y, np.float32)
    sol = L.solution_create(K, n)
    if not sol:
        return _native.ACO_ERR_ALLOCATION, [], float("inf")
    cost = C.c_double(0.0)
    try:
        rc = L.aco_vrp_cuda_with_capacity(n, K, capacity, m, xs.ctypes.data, ys.ctypes.data,
                                          alpha, beta, rho, tau0, Q, seed & 0xffffffff, sol,
                                          C.byref(cost))
        routes = _routes(sol) if rc == 0 else []
    finally:
        L.solution_free(sol)
    return rc, routes, cost.value


def aco_vrp_cuda_with_demands(n: int, K: int, capacity: int, m: int, x, y, demand,
                              alpha=1.0, beta=2.0, rho=0.5, tau0=1.0, Q=1.0,
                              seed: int = 1234) -> Tuple[int, List[List[int]], float]:
    L = _bind(_native.load())
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.ascontiguousarray(y, np.float32)
    ds = np.ascontiguousarray(demand, np.int32)
    sol = L.solution_create(K, n)
    if not sol:
        return _native.ACO_ERR_ALLOCATION, [], float("inf")
    cost = C.c_double(0.0)
    try:
        rc = L.aco_vrp_cuda_with_demands(n, K, capacity, m, xs.ctypes.data, ys.ctypes.data,
                                         ds.ctypes.data, alpha, beta, rho, tau0, Q,
                                         seed & 0xffffffff, sol, C.byref(cost))
        routes = _routes(sol) if rc == 0 else []
    finally:
        L.solution_free(sol)
    return rc, routes, cost.value


def solve(inst: Instance, ants: int = 256, epochs: int = 200, seed: int = 1234,
          cand_k: int = 0, stagnation_epochs: int = 0, device: int = 0,
          **params) -> Tuple[List[List[int]], float, _native.State]:
    """Runs up to ``epochs`` epochs (fewer if the stagnation rule fires)."""
    with _native.Context(device) as ctx:
        ctx.setup_instance(inst, ants=ants, cand_k=cand_k, seed=seed,
                           stagnation_epochs=stagnation_epochs, fixed_epochs=epochs, **params)
        st = ctx.run(epochs)
        nodes, lens, cost = ctx.best()
        return _native.split_routes(nodes, lens), cost, st
