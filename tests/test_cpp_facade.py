"""The C++ drop-in header (include/flexmesh_b200.hpp) compiles and links
against the library (CPU), and a reference-style C++ caller reproduces the
oracle's Newton solution and the Poisson PCG answer on the GPU."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "atlas-flexmesh_b200", "flexmesh_b200")


def build(tmp_path):
    exe = str(tmp_path / "facade_demo")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp"), "-L", LIBDIR,
                    "-lflexmesh_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_facade_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_facade_newton_matches_oracle(tmp_path):
    import oracle as O
    from flexmesh_b200 import configs

    exe = build(tmp_path)
    out = str(tmp_path / "u.bin")
    subprocess.run([exe, out, "4"], check=True, timeout=600)
    data = np.fromfile(out, np.float64)
    u, meta = data[:-3], data[-3:]
    P = configs.small_block(4)
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    uo, st, nps, _ = O.newton(P.xyz, P.conn, mu, lam, P.nu, rp, ci,
                              O.slot_map(P.n_nodes, P.conn, rp, ci), P.mask, P.bc_value,
                              P.n_steps, rtol=1e-10, inner_tol=1e-12,
                              active=(P.elem_volume >= 1e-30).astype(np.uint8))
    assert st == 0
    assert np.linalg.norm(u - uo) <= 1e-10 * np.linalg.norm(uo)
    assert int(meta[0]) == int(nps.sum())
    assert meta[2] < 1e-6
