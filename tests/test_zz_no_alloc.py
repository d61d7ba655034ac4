"""The allocation-free evaporate + deposit entry point.

aco_b200_evaporate_deposit_noalloc serves callers that may not allocate
device memory while they run (applications that own all device memory and
hand plugins only their own buffers, real-time loops that cannot afford
cudaMalloc's synchronisation or its failure under memory pressure).  Here its
output is compared with the context-based aco_b200_evaporate_deposit, which
allocates its buffers at set-up, on the same inputs, bit for bit (the
tolerance of every pheromone test), for two calls in a row; the caller-owned
device buffers of the test come from torch.  The file sorts last so that a
run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu


def _entry():
    L = _native.load()
    f = L.aco_b200_evaporate_deposit_noalloc
    vp = C.c_void_p
    f.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_float, vp, vp, C.c_float, C.c_double, vp]
    f.restype = C.c_int
    return f


def _at_capacity():
    """4096 routes, the most the fixed scratch holds: 4500 unit-demand
    customers, at most 2 per vehicle, so the early vehicles stay empty and
    the last route offset is the scratch's last word."""
    base = I.uniform_instance(4500, 4096, 908).unit_twin()
    return I.Instance("noalloc_cap", base.x, base.y, base.demand, 4096, 2), 4, 8


@pytest.mark.parametrize("case", ["n300_K6", "K4096"])
@pytest.mark.parametrize("with_global", [True, False])
def test_no_alloc_matches_context_entry_point(with_global, case):
    import torch
    noalloc = _entry()
    if case == "K4096":
        inst, ants, k = _at_capacity()
    else:
        inst, ants, k = I.uniform_instance(300, 6, 907), 16, 20
    n, K = inst.n, inst.vehicles
    with _native.Context(0) as ctx:
        ctx.setup_instance(inst, ants=ants, cand_k=k, seed=11)
        tau0 = np.random.RandomState(5).randint(0, 256, size=(n + 1) ** 2).astype(np.uint8)
        ctx.set_tau(tau0)
        ctx.construct(0)
        nodes, lens, cost, feas, _, _ = ctx.ants()
        best = int(np.argmin(np.where(feas > 0, cost, np.inf)))
        other = (best + 5) % ctx.m
        it_nodes, it_lens = nodes[best][: lens[best].sum()], lens[best]
        gb_nodes, gb_lens = nodes[other][: lens[other].sum()], lens[other]
        dep_i = float(np.float32(30.0) / np.float32(cost[best]))
        dep_g = float(np.float32(70.0) / np.float32(cost[other]))

        # Existing entry point (context-owned device buffers), two calls.
        ctx.set_tau(tau0)
        expected = []
        for _ in range(2):
            if with_global:
                ctx.evaporate_deposit(best, dep_i, gb_nodes, gb_lens, dep_g)
            else:
                ctx.evaporate_deposit(best, dep_i)
            expected.append(ctx.tau())

    # Allocation-free entry point on caller-owned device buffers, two calls.
    d_tau = torch.from_numpy(tau0.copy()).cuda()
    d_in = torch.from_numpy(it_nodes.astype(np.int32)).cuda()
    d_il = torch.from_numpy(it_lens.astype(np.int32)).cuda()
    d_gn = torch.from_numpy(gb_nodes.astype(np.int32)).cuda()
    d_gl = torch.from_numpy(gb_lens.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rc = noalloc(d_tau.data_ptr(), n, K, d_in.data_ptr(), d_il.data_ptr(), dep_i,
                     d_gn.data_ptr() if with_global else None,
                     d_gl.data_ptr() if with_global else None, dep_g, 0.5, stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(d_tau.cpu().numpy(), expected[call]), f"call {call + 1}"


def test_no_alloc_rejects_what_its_scratch_cannot_hold():
    import torch
    noalloc = _entry()
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    # More routes than the fixed scratch holds: rejected before any launch.
    assert noalloc(buf.data_ptr(), 5, 5000, buf.data_ptr(), buf.data_ptr(), 1.0, None, None,
                   0.0, 0.5, None) == _native.ACO_ERR_INVALID_INPUT
    # A pheromone buffer that is not 16-byte aligned: rejected.
    assert noalloc(buf.data_ptr() + 4, 5, 2, buf.data_ptr(), buf.data_ptr(), 1.0, None, None,
                   0.0, 0.5, None) == _native.ACO_ERR_INVALID_INPUT
