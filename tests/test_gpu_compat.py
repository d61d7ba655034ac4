"""GPU tests of the drop-in kernel header (include/aco_cuda_kernels.h).

The launch_* functions of libaco_b200.so are run on the reference's buffer
layouts and compared byte-for-byte with the reference's own kernels
(oracle/_ref/librefcuda.so, built from its sources); the drop-in construct is
compared route-for-route with the oracle; and the reference's own host solver
and CLI, linked against libaco_b200.so in place of its kernel file
(oracle/_ref/aco_vrp_cuda_refhost.out), solve instances end to end.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFCUDA = os.path.join(ROOT, "oracle", "_ref", "librefcuda.so")
REFHOST = os.path.join(ROOT, "oracle", "_ref", "aco_vrp_cuda_refhost.out")
need_ref = pytest.mark.skipif(not os.path.exists(REFCUDA), reason="oracle/_ref not built")


class CudaParams(C.Structure):
    _fields_ = [("n", C.c_int), ("K", C.c_int), ("m", C.c_int), ("cap", C.c_int),
                ("cand_k", C.c_int), ("route_max_len", C.c_int),
                ("alpha", C.c_float), ("beta", C.c_float), ("rho", C.c_float),
                ("tau0", C.c_float), ("Q", C.c_float), ("tau_min", C.c_float),
                ("tau_max", C.c_float), ("log_tau_min", C.c_float),
                ("log_tau_step", C.c_float), ("q_tau_min", C.c_uint8),
                ("q_tau_max", C.c_uint8), ("q_evap_delta", C.c_uint8),
                ("visited_l1_words", C.c_int), ("visited_l2_words", C.c_int),
                ("visited_row_stride", C.c_size_t), ("depot_close_weight", C.c_float)]


class AntSummary(C.Structure):
    _fields_ = [("feasible", C.c_int), ("unvisited_count", C.c_int), ("cost", C.c_float)]


def mangled(lib_path, name):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True,
                         text=True).stdout
    for line in out.splitlines():
        sym = line.split()[-1]
        if re.match(rf"_Z\d+{name}P", sym):
            return sym
    raise KeyError(name)


@pytest.fixture(scope="module")
def ours():
    L = _native.load()
    path = _native.library_path()
    vp, i32, u8, f32 = C.c_void_p, C.c_int, C.c_uint8, C.c_float
    sig = {
        "launch_init_tau": [vp, i32, u8],
        "launch_evaporate_tau": [vp, i32, u8, u8],
        "launch_build_candidate_lists": [vp, vp, vp, CudaParams],
        "launch_reset_ant_state": [vp, vp, vp, vp, vp, vp, CudaParams, C.c_uint],
        "launch_construct_solutions": [vp] * 11 + [CudaParams],
        "launch_deposit_solution": [vp, vp, vp, f32, i32, CudaParams],
        "launch_deposit_flat_solution": [vp, vp, vp, f32, CudaParams],
    }
    fns = {}
    for name, args in sig.items():
        f = getattr(L, mangled(path, name))
        f.argtypes = args
        f.restype = None
        fns[name] = f
    return fns


@pytest.fixture(scope="module")
def ref():
    R = C.CDLL(REFCUDA)
    vp = C.c_void_p
    for fn, args in {"refcuda_init_tau": [vp, C.c_int, C.c_uint8],
                     "refcuda_evaporate": [vp, C.c_int, C.c_uint8, C.c_uint8],
                     "refcuda_build_candidates": [vp, vp, vp, vp],
                     "refcuda_deposit_solution": [vp, vp, vp, C.c_float, C.c_int, vp],
                     "refcuda_deposit_flat": [vp, vp, vp, C.c_float, vp]}.items():
        getattr(R, fn).argtypes = args
        getattr(R, fn).restype = C.c_int
    return R


def params_for(inst, k, m, cap=None):
    P = __import__("oracle.oracle", fromlist=["params"]).params()
    n = inst.n
    l1 = (n + 64) // 64
    return CudaParams(n=n, K=inst.vehicles, m=m, cap=cap or inst.capacity, cand_k=k,
                      route_max_len=inst.vehicles * (n + 1), alpha=1.0, beta=2.0, rho=0.5,
                      tau0=1.0, Q=100.0, tau_min=1e-4, tau_max=100.0,
                      log_tau_min=P["log_tau_min"], log_tau_step=P["log_tau_step"],
                      q_tau_min=0, q_tau_max=255, q_evap_delta=P["q_evap_delta"],
                      visited_l1_words=l1, visited_l2_words=(l1 + 63) // 64,
                      visited_row_stride=((l1 * 8 + 127) // 128) * 128, depot_close_weight=2.0)


def sync():
    import torch
    torch.cuda.synchronize()


@need_ref
@pytest.mark.parametrize("n,offset", [(1000, 0), (301, 3), (10, 1)])
def test_init_and_evaporate_match_reference(ours, ref, n, offset):
    import torch
    total = (n + 1) ** 2
    rs = np.random.RandomState(n)
    src = torch.from_numpy(rs.randint(0, 256, size=total).astype(np.uint8)).cuda()
    a = torch.zeros(total + 32, dtype=torch.uint8, device="cuda")
    b = torch.zeros(total + 32, dtype=torch.uint8, device="cuda")
    for delta, qmin in [(13, 0), (40, 7), (250, 30)]:
        a[offset:offset + total] = src
        b[offset:offset + total] = src
        ours["launch_evaporate_tau"](a.data_ptr() + offset, n, delta, qmin)
        sync()
        assert ref.refcuda_evaporate(b.data_ptr() + offset, n, delta, qmin) == 0
        assert torch.equal(a, b)
    ours["launch_init_tau"](a.data_ptr() + offset, n, 170)
    sync()
    assert ref.refcuda_init_tau(b.data_ptr() + offset, n, 170) == 0
    assert torch.equal(a, b)


@need_ref
@pytest.mark.parametrize("name,k", [("u500", 32), ("c700", 20), ("tiny", 5)])
def test_candidate_lists_match_reference(ours, ref, name, k):
    import torch
    inst = {"u500": lambda: I.uniform_instance(500, 6, 701),
            "c700": lambda: I.clustered_instance(700, 8, 702),
            "tiny": lambda: I.uniform_instance(5, 2, 703)}[name]()
    k = min(k, inst.n)
    prm = params_for(inst, k, 8)
    xy = torch.tensor(np.stack([inst.x, inst.y], 1).ravel(), dtype=torch.float32, device="cuda")
    cnt = (inst.n + 1) * k
    ia, ib = (torch.zeros(cnt, dtype=torch.int32, device="cuda") for _ in range(2))
    ea, eb = (torch.zeros(cnt, dtype=torch.float32, device="cuda") for _ in range(2))
    ours["launch_build_candidate_lists"](xy.data_ptr(), ia.data_ptr(), ea.data_ptr(), prm)
    sync()
    assert ref.refcuda_build_candidates(xy.data_ptr(), ib.data_ptr(), eb.data_ptr(),
                                        C.byref(prm)) == 0
    assert torch.equal(ia, ib)
    assert torch.equal(ea.view(torch.int32), eb.view(torch.int32))


def _random_solution(n, K, rs):
    while True:
        nodes, lens = _random_split(n, K, rs)
        if lens.max() <= n + 1:  # the reference's flat buffer holds n+1 per route
            return nodes, lens


def _random_split(n, K, rs):
    perm = rs.permutation(np.arange(1, n + 1))
    cuts = np.sort(rs.choice(np.arange(0, n + 1), size=K - 1, replace=True))
    parts = np.split(perm, cuts)
    nodes, lens = [], []
    for p in parts:
        nodes += [0] + list(p) + [0]
        lens.append(len(p) + 2)
    return np.array(nodes, np.int32), np.array(lens, np.int32)


@need_ref
@pytest.mark.parametrize("n,K,seed", [(300, 6, 1), (200, 12, 2), (40, 9, 3)])
def test_deposits_match_reference(ours, ref, n, K, seed):
    """Random route sets, including empty and one-customer routes."""
    import torch
    rs = np.random.RandomState(seed)
    nodes, lens = _random_solution(n, K, rs)
    inst = I.uniform_instance(n, K, 800 + seed).unit_twin()
    prm = params_for(inst, 16, 1)
    tau0 = rs.randint(0, 256, size=(n + 1) ** 2).astype(np.uint8)
    seq = [0]
    off = 0
    for L in lens:
        seq += list(nodes[off + 1: off + L])
        off += L
    steps = torch.tensor(seq, dtype=torch.int32, device="cuda")
    dl = torch.from_numpy(lens).cuda()
    flat = np.zeros(K * (n + 1), np.int32)
    off = 0
    for v, L in enumerate(lens):
        flat[v * (n + 1): v * (n + 1) + L] = nodes[off: off + L]
        off += L
    dflat = torch.from_numpy(flat).cuda()
    a = torch.from_numpy(tau0).cuda()
    b = torch.from_numpy(tau0).cuda()
    ours["launch_deposit_solution"](a.data_ptr(), steps.data_ptr(), dl.data_ptr(), 0.37, 0, prm)
    ours["launch_deposit_flat_solution"](a.data_ptr(), dflat.data_ptr(), dl.data_ptr(), 1.9, prm)
    sync()
    assert ref.refcuda_deposit_solution(b.data_ptr(), steps.data_ptr(), dl.data_ptr(), 0.37, 0,
                                        C.byref(prm)) == 0
    assert ref.refcuda_deposit_flat(b.data_ptr(), dflat.data_ptr(), dl.data_ptr(), 1.9,
                                    C.byref(prm)) == 0
    ga, gb = a.cpu().numpy(), b.cpu().numpy()
    if (lens == 2).sum() >= 2:  # the reference races on the depot loop cell
        ga, gb = ga[1:], gb[1:]
    assert np.array_equal(ga, gb)


@pytest.mark.parametrize("name", ["u200", "smoke_like", "n1000_twin"])
def test_dropin_construct_matches_oracle(ours, oracle_mod, name):
    import torch
    O = oracle_mod
    inst = {"u200": lambda: I.uniform_instance(200, 4, 711).unit_twin(),
            "smoke_like": lambda: I.uniform_instance(8, 2, 712).unit_twin(),
            "n1000_twin": lambda: I.workload_n1000().unit_twin()}[name]()
    n, K = inst.n, inst.vehicles
    k, m = min(32, n), 24
    prm = params_for(inst, k, m)
    xy = torch.tensor(np.stack([inst.x, inst.y], 1).ravel(), dtype=torch.float32, device="cuda")
    cand = torch.zeros((n + 1) * k, dtype=torch.int32, device="cuda")
    eta = torch.zeros((n + 1) * k, dtype=torch.float32, device="cuda")
    tau_np = np.random.RandomState(4).randint(0, 256, size=(n + 1) ** 2).astype(np.uint8)
    tau = torch.from_numpy(tau_np).cuda()
    routes = torch.zeros((K * (n + 1) + 1) * m, dtype=torch.int32, device="cuda")
    lens = torch.zeros(m * K, dtype=torch.int32, device="cuda")
    l1 = torch.zeros(m * prm.visited_row_stride // 8, dtype=torch.int64, device="cuda")
    l2 = torch.zeros(m * prm.visited_l2_words, dtype=torch.int64, device="cuda")
    rng = torch.zeros(m, dtype=torch.int32, device="cuda")
    summ = torch.zeros(m * 3, dtype=torch.int32, device="cuda")
    stats = torch.zeros(10, dtype=torch.int64, device="cuda")
    ours["launch_build_candidate_lists"](xy.data_ptr(), cand.data_ptr(), eta.data_ptr(), prm)
    ours["launch_reset_ant_state"](routes.data_ptr(), lens.data_ptr(), l1.data_ptr(),
                                   l2.data_ptr(), rng.data_ptr(), summ.data_ptr(), prm, 1234 + 5)
    ours["launch_construct_solutions"](xy.data_ptr(), tau.data_ptr(), cand.data_ptr(),
                                       eta.data_ptr(), routes.data_ptr(), lens.data_ptr(),
                                       l1.data_ptr(), l2.data_ptr(), rng.data_ptr(),
                                       summ.data_ptr(), stats.data_ptr(), prm)
    sync()
    A, lut, thr = O.tables()
    c_np = cand.cpu().numpy()
    w = O.weights(n, k, c_np, O.levels(inst.x, inst.y, c_np, k, thr), tau_np, A, lut)
    R = routes.cpu().numpy().reshape(-1, m)
    Ls = lens.cpu().numpy().reshape(m, K)
    S = summ.cpu().numpy().reshape(m, 3)
    keys = rng.cpu().numpy().view(np.uint32)
    for a in range(m):
        assert keys[a] == ((1234 + 5) ^ ((1664525 * (a + 1)) & 0xffffffff))
        f, on, ol, oc, _, _ = O.construct_ant(inst.x, inst.y, None, K, inst.capacity, k, c_np,
                                              w, int(keys[a]), 0, a, stream=0xC0FA)
        assert np.array_equal(Ls[a], ol)
        seq = [0]
        off = 0
        for L in ol:
            seq += list(on[off + 1: off + L])
            off += L
        assert np.array_equal(R[: len(seq), a], seq)
        assert S[a, 0] == int(f) and S[a, 1] == 0
        assert np.float32(S[a].view(np.float32)[2]) == np.float32(oc)


@pytest.mark.skipif(not os.path.exists(REFHOST), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", ["smoke", "u300"])
def test_reference_host_solver_on_these_kernels(tmp_path, case):
    from tests.test_boundary import SMOKE
    p = tmp_path / "inst.vrp"
    if case == "smoke":
        p.write_text(SMOKE)
        K, n = 2, 8
    else:
        inst = I.uniform_instance(300, 5, 721).unit_twin()
        I.write_vrp(inst, str(p))
        K, n = 5, 300
    env = dict(os.environ, ACO_SOLVER_STAGNATION_EPOCHS="15", ACO_SOLVER_TIMEOUT_SECONDS="20")
    r = subprocess.run(["timeout", "120", REFHOST, str(p), str(K), "64", "7"],
                       capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr[-500:]
    assert "CUDA Solver starting" in r.stdout
    routes = [[int(v) for v in l.split(":")[1].split()] for l in r.stdout.splitlines()
              if l.startswith("Route ")]
    assert len(routes) == K and sorted(v for rr in routes for v in rr) == list(range(1, n + 1))
    assert re.search(r"^best cost: [0-9.]+$", r.stdout, re.M)
