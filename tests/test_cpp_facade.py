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


REF_DEMO = os.path.join(ROOT, "oracle", "_ref", "ref_types_demo")


def test_reference_types_demo_compiles():
    """The drop-in compiles against the reference's own headers and types
    (oracle/Makefile refdemo; needs the reference checkout at build time)."""
    ref_root = os.environ.get("FLEXMESH_REF_ROOT", "/root/reference")
    if not os.path.isdir(os.path.join(ref_root, "FEM")):
        pytest.skip("no reference checkout to compile against")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "refdemo",
                    f"REF_ROOT={ref_root}"], check=True, timeout=600)
    assert os.path.exists(REF_DEMO)


@pytest.mark.gpu
def test_reference_types_drop_in_matches_oracle(tmp_path):
    """atlas::fem::MeshTopology / BoundaryConditions / NeoHookeanMaterial /
    LoadStep / NewtonSolverConfig / SparseCSR / ProblemDescriptor passed
    unchanged to flexmesh_b200::NonlinearNewtonSolver, assemble_global_threadlocal
    and pcg_solve_ilu0: Newton matches the oracle run with the same options
    (Armijo with (1 - 0.1 alpha), 10 trials), the assembly and the PCG match
    the reference's own functions run on the CPU in the same program."""
    import oracle as O
    from flexmesh_b200 import configs

    if not os.path.exists(REF_DEMO):
        pytest.skip("oracle/_ref/ref_types_demo was not built (no reference checkout)")
    out = str(tmp_path / "u.bin")
    subprocess.run([REF_DEMO, out, "4"], check=True, timeout=600)
    data = np.fromfile(out, np.float64)
    u, meta = data[:-6], data[-6:]
    P = configs.small_block(4)
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    uo, st, nps, _, _ = O.newton_ex(P.xyz, P.conn, mu, lam, P.nu, rp, ci,
                                    O.slot_map(P.n_nodes, P.conn, rp, ci), P.mask, P.bc_value,
                                    P.n_steps, rtol=1e-10, inner_tol=1e-12, max_newton=200,
                                    line_search=10, ls_c=0.1, diverge_growth=10.0,
                                    active=(P.elem_volume >= 1e-30).astype(np.uint8))
    assert st == 0
    assert np.linalg.norm(u - uo) <= 1e-10 * np.linalg.norm(uo)
    assert int(meta[0]) == int(nps.sum())
    assert meta[1] <= 1e-13 and meta[2] <= 1e-13  # K, f vs the reference's assembly
    assert abs(meta[3] - meta[4]) <= 1 and meta[5] <= 1e-10  # PCG vs the reference's
