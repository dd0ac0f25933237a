"""Host-side invariants of the cluster-synchronous triangular-solve plan
(slot lifetimes, level order, records), checked by tests/cpp/cluster_plan_check.cpp
compiled against the library's setup code, on the unit cube and on the same
mesh with randomly relabelled nodes (irregular levels, long-lived values)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "atlas-flexmesh_b200", "csrc")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("plan") / "cluster_plan_check")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-fopenmp", "-I", CSRC, "-o", out,
                    os.path.join(ROOT, "tests", "cpp", "cluster_plan_check.cpp"),
                    os.path.join(CSRC, "fm_setup.cpp")], check=True, timeout=300)
    return out


@pytest.mark.parametrize("N,seed", [(4, 0), (12, 0), (24, 0), (6, 7), (12, 11)])
def test_cluster_plan_invariants(exe, N, seed):
    r = subprocess.run([exe, str(N), str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
