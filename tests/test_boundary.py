"""CPU tests of the drop-in boundary: the C ABI library loads and exports every
declared symbol, the CLI argument contract, the TSPLIB parser, the
environment configuration and the instance generator.  No GPU compute."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "aco_vrp_cuda.out")


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h") or h == "aco_api.h":
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        for m in re.finditer(r"ACO_API\s+[\w\s\*]*?\b(\w+)\s*\(", text):
            names.add(m.group(1))
        for m in re.finditer(r"__global__\s+void\s+(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-DC", "--defined-only", path], capture_output=True,
                         text=True).stdout
    names = set()
    for line in out.splitlines():
        parts = line.split(" T ")
        if len(parts) == 2:
            names.add(parts[1].split("(")[0])
    return names


def test_library_exports_every_declared_symbol(native):
    L = native.load()
    names = declared_symbols()
    assert len(names) >= 54  # C ABI + reference-compatible C API + kernel header
    missing = sorted(names - exported_symbols(native.library_path()))
    assert not missing, missing
    c_names = [s for s in names if not s.startswith(("kernel_", "launch_"))]
    assert all(hasattr(L, s) for s in c_names)
    assert set(native.EXPORTED) <= names


def test_library_hides_internal_symbols(native):
    exported = {n for n in exported_symbols(native.library_path())
                if not n.startswith("__device_stub__")}  # host stubs of exported kernels
    assert exported <= declared_symbols() | {"_init", "_fini"}, exported - declared_symbols()


def test_status_strings(native):
    L = native.load()
    assert [L.aco_status_string(i).decode() for i in range(5)] == [
        "ok", "invalid input", "allocation failure", "no solution", "backend failure"]


def test_context_without_gpu_fails_loudly(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.AcoError):
        native.Context(0)


@pytest.mark.parametrize("args", [[], ["x.vrp", "2"], ["x.vrp", "-1", "4"], ["x.vrp", "2", "a"],
                                  ["x.vrp", "2", "4", "5", "6"], ["x.vrp", "0", "4"],
                                  ["x.vrp", "2", "4", "notanumber"]])
def test_cli_usage_errors(args):
    r = subprocess.run([CLI] + args, capture_output=True, text=True)
    assert r.returncode == 1 and "usage:" in r.stderr and r.stdout == ""


def _write(tmp_path, text, name="inst.vrp"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


SMOKE = """NAME : smoke
TYPE : CVRP
DIMENSION : 9
VEHICLES : 2
EDGE_WEIGHT_TYPE : EUC_2D
CAPACITY : 5
NODE_COORD_SECTION
1 50 50
2 10 10
3 20 10
4 10 20
5 20 20
6 80 80
7 90 80
8 80 90
9 90 90
DEMAND_SECTION
1 0
2 1
3 1
4 1
5 1
6 1
7 1
8 1
9 1
DEPOT_SECTION
1
-1
EOF
"""


def _load(native, path, demands=False):
    L = native.load()
    n = C.c_int()
    x, y, d = C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_int)()

    class Meta(C.Structure):
        _fields_ = [("vehicles", C.c_int), ("capacity", C.c_int)]
    meta = Meta()
    if demands:
        rc = L.vrp_load_tsplib_euc2d_coords_demands(path.encode(), C.byref(n), C.byref(x),
                                                    C.byref(y), C.byref(d), C.byref(meta))
    else:
        rc = L.vrp_load_tsplib_euc2d_coords(path.encode(), C.byref(n), C.byref(x), C.byref(y),
                                            C.byref(meta))
    if rc != 0:
        return rc, None
    xs = [x[i] for i in range(n.value + 1)]
    ds = [d[i] for i in range(n.value + 1)] if demands else None
    return rc, (n.value, xs, ds, meta.vehicles, meta.capacity)


def test_parser_reference_format(native, tmp_path):
    rc, (n, xs, _, K, cap) = _load(native, _write(tmp_path, SMOKE))
    assert rc == 0 and n == 8 and K == 2 and cap == 5 and xs[0] == 50.0 and xs[8] == 90.0


def test_parser_rejects_what_the_reference_rejects(native, tmp_path):
    bad_demand = SMOKE.replace("3 1\n", "3 2\n", 1)
    assert _load(native, _write(tmp_path, bad_demand, "a.vrp"))[0] == 1
    # the demand loader accepts it
    rc, (n, _, ds, _, _) = _load(native, _write(tmp_path, bad_demand, "b.vrp"), demands=True)
    assert rc == 0 and ds[2] == 2
    no_veh = SMOKE.replace("VEHICLES : 2\n", "")
    assert _load(native, _write(tmp_path, no_veh, "c.vrp"))[0] == 1
    depot = SMOKE.replace("1 0\n", "1 3\n", 1)
    assert _load(native, _write(tmp_path, depot, "d.vrp"), demands=True)[0] == 1
    truncated = SMOKE.split("DEMAND_SECTION")[0]
    assert _load(native, _write(tmp_path, truncated, "e.vrp"))[0] == 1
    nodim = SMOKE.replace("DIMENSION : 9\n", "")
    assert _load(native, _write(tmp_path, nodim, "f.vrp"))[0] == 1
    assert _load(native, str(tmp_path / "missing.vrp"))[0] == 1


def test_depot_section(native, tmp_path):
    """DEPOT_SECTION naming node 1 is accepted; any other depot is refused by
    both readers (every solver here, like the reference, has node 1 as depot)."""
    base = SMOKE.split("EOF")[0].rstrip("\n") + "\n"
    ok = base + "DEPOT_SECTION\n1\n-1\nEOF\n"
    rc, (n, *_rest) = _load(native, _write(tmp_path, ok, "g.vrp"), demands=True)
    assert rc == 0 and n == 8
    assert I.read_vrp(_write(tmp_path, ok, "g2.vrp")).n == 8
    other = base + "DEPOT_SECTION\n3\n-1\nEOF\n"
    assert _load(native, _write(tmp_path, other, "h.vrp"), demands=True)[0] == 1
    with pytest.raises(ValueError):
        I.read_vrp(_write(tmp_path, other, "h2.vrp"))


def test_cli_rejects_vehicle_mismatch(tmp_path):
    p = _write(tmp_path, SMOKE)
    r = subprocess.run([CLI, p, "3", "4"], capture_output=True, text=True)
    assert r.returncode == 1 and "VEHICLES mismatch" in r.stderr


def test_config_env(native, monkeypatch):
    L = native.load()

    class Cfg(C.Structure):
        _fields_ = [("timeout_seconds", C.c_double), ("stagnation_epochs", C.c_int),
                    ("min_rel_improvement", C.c_double), ("fixed_epochs", C.c_int),
                    ("candidate_k", C.c_int), ("ants", C.c_int), ("seed", C.c_uint),
                    ("progress_interval_seconds", C.c_double)]
    for k in ("ACO_SOLVER_TIMEOUT_SECONDS", "ACO_SOLVER_STAGNATION_EPOCHS",
              "ACO_SOLVER_MIN_REL_IMPROVEMENT", "ACO_SOLVER_FIXED_EPOCHS",
              "ACO_SOLVER_PROGRESS_INTERVAL_SECONDS", "ACO_CUDA_CANDIDATE_K"):
        monkeypatch.delenv(k, raising=False)
    c = Cfg()
    L.aco_runtime_config_load_env(C.byref(c))
    assert (c.timeout_seconds, c.stagnation_epochs, c.min_rel_improvement, c.fixed_epochs,
            c.progress_interval_seconds, c.seed) == (0.0, 0, 1e-3, 0, 10.0, 1234)
    monkeypatch.setenv("ACO_SOLVER_TIMEOUT_SECONDS", "2.5")
    monkeypatch.setenv("ACO_SOLVER_STAGNATION_EPOCHS", "80")
    monkeypatch.setenv("ACO_SOLVER_MIN_REL_IMPROVEMENT", "10")   # percent
    monkeypatch.setenv("ACO_SOLVER_FIXED_EPOCHS", "-3")
    monkeypatch.setenv("ACO_CUDA_CANDIDATE_K", "16")
    L.aco_runtime_config_load_env(C.byref(c))
    assert c.timeout_seconds == 2.5 and c.stagnation_epochs == 80
    assert abs(c.min_rel_improvement - 0.1) < 1e-15 and c.fixed_epochs == 0
    assert c.candidate_k == 16
    monkeypatch.setenv("ACO_SOLVER_MIN_REL_IMPROVEMENT", "-1")
    L.aco_runtime_config_load_env(C.byref(c))
    assert c.min_rel_improvement == 1e-3


def test_generator_is_seeded_and_shaped():
    a, b = I.workload_n1000(), I.workload_n1000()
    assert np.array_equal(a.x, b.x) and np.array_equal(a.demand, b.demand)
    assert a.n == 1000 and a.vehicles == 8 and a.x[0] == 500 and a.y[0] == 500
    assert a.demand[0] == 0 and 1 <= a.demand[1:].min() and a.demand[1:].max() <= 100
    assert a.capacity == int(np.ceil(a.demand.sum() / (0.9 * 8)))
    assert np.all((a.x >= 0) & (a.x <= 1000)) and np.all(a.x == np.round(a.x))
    s = I.workload_small()
    assert s.n == 100 and s.vehicles == 4 and s.demand[1:].max() <= 30
    c = I.workload_clustered2000()
    assert c.n == 2000 and c.vehicles == 16 and np.all((c.x >= 0) & (c.x <= 1000))
    batch = I.batched_instances(16)
    assert all(50 <= b.n <= 500 and b.vehicles == int(np.ceil(b.n / 60)) for b in batch)
    t = a.unit_twin()
    assert t.is_unit_demand() and t.capacity == int(np.ceil(1000 / (0.9 * 8)))


def test_tsplib_round_trip(tmp_path, native):
    inst = I.uniform_instance(50, 3, 5)
    p = str(tmp_path / "u.vrp")
    I.write_vrp(inst, p)
    back = I.read_vrp(p)
    assert np.array_equal(back.x, inst.x) and np.array_equal(back.demand, inst.demand)
    assert back.vehicles == 3 and back.capacity == inst.capacity
    rc, (n, xs, ds, K, cap) = _load(native, p, demands=True)
    assert rc == 0 and n == 50 and ds == list(inst.demand) and cap == inst.capacity
