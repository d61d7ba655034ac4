"""B200-native (sm_100a) ACO hot path for the Capacitated Vehicle Routing Problem.

Drop-in for the GPU path of JustCh3cco-19/VehicleRoutingProblem: warp-per-ant
route construction over shared-memory candidate tables with an exact integer
roulette, and streaming evaporation/deposit on the log-quantized pheromone
matrix.  The compute path is CUDA C++ behind a C ABI (include/aco_b200.h,
libaco_b200.so); this package is its Python front end.
"""
from . import instances  # noqa: F401

__all__ = ["instances", "native", "solver"]


def native():
    from . import _native
    return _native
