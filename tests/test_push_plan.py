"""Host-side invariants of the push triangular-solve plans (slot ownership,
level order, records, push lists, deadlock freedom of the warp-pair
schedule), checked by tests/cpp/push_plan_check.cpp compiled against the
library's setup code, on the unit cube and on the same mesh with relabelled
nodes (irregular levels, long-lived values)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "atlas-flexmesh_b200", "csrc")


@pytest.fixture(scope="module")
def push_exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("push") / "push_plan_check")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", CSRC, "-o", out,
                    os.path.join(ROOT, "tests", "cpp", "push_plan_check.cpp"),
                    os.path.join(CSRC, "fm_setup.cpp")], check=True, timeout=300)
    return out


# (N, relabelling seed (> 0: random ids, which the plan refuses where a side
# holds more than 16 neighbours; < 0: shuffled inside blocks of 8), clusters,
# CTAs per cluster (8, and 9 as the solves use on B200), block (0: chosen),
# slot limit); N = 1 leaves most CTAs
# without nodes, 3 clusters give uneven slabs, the last case forces the plan
# past the block sizes whose slots overflow
@pytest.mark.parametrize("N,seed,ncl,cs,block,limit", [
    (4, 0, 16, 8, 0, 1 << 20), (12, 0, 16, 8, 0, 1 << 20), (24, 0, 16, 8, 0, 1 << 20),
    (6, 7, 16, 8, 0, 1 << 20), (12, -11, 3, 8, 0, 1 << 20), (1, 0, 16, 8, 0, 1 << 20),
    (2, 5, 4, 2, 0, 1 << 20), (12, 0, 16, 8, 65, 1 << 20), (12, 0, 4, 8, 0, 300),
    (10, -3, 15, 8, 0, 1 << 20), (12, 0, 15, 9, 0, 1 << 20), (10, -3, 15, 9, 0, 1 << 20),
    (24, 0, 15, 9, 0, 5909), (1, 0, 15, 9, 0, 1 << 20)])
def test_push_plan_invariants(push_exe, N, seed, ncl, cs, block, limit):
    r = subprocess.run([push_exe, str(N), str(seed), str(ncl), str(cs), str(block), str(limit)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
