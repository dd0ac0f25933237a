"""The C oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref) and, where the reference build
is present, against the reference directly.  CPU only."""
import numpy as np
import pytest

import oracle as O


def test_element_matches_reference(golden):
    for t in range(golden["in_elem_x"].shape[0]):
        K, f = O.element(golden["in_elem_x"][t], golden["in_elem_u"][t], golden["in_elem_E"][t], 0.3)
        assert np.array_equal(K, golden["ref_elem_K"][t])
        assert np.array_equal(f, golden["ref_elem_f"][t])


@pytest.mark.parametrize("N", [2, 4])
def test_mesh_and_patterns_bitwise(golden, N):
    p = f"n{N}_"
    xyz, conn = O.unit_cube(N)
    assert np.array_equal(xyz, golden[p + "ref_xyz"])
    assert np.array_equal(conn, golden[p + "ref_conn"])
    assert np.array_equal(O.volumes(xyz, conn), golden[p + "ref_vol"])
    ptr, data = O.node_to_elem(xyz.size // 3, conn)
    assert np.array_equal(ptr, golden[p + "ref_n2e_ptr"])
    assert np.array_equal(data, golden[p + "ref_n2e"])
    rp, ci = O.pattern(xyz.size // 3, conn, "reference")
    assert np.array_equal(rp, golden[p + "ref_row_ptr"])
    assert np.array_equal(ci, golden[p + "ref_col_idx"])
    rps, cis = O.pattern(xyz.size // 3, conn, "solve")
    assert np.array_equal(rps, rp)
    assert np.array_equal(cis, golden[p + "orc_solve_col_idx"])


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("pat", ["refpat", "solvepat"])
@pytest.mark.parametrize("utag", ["u0", "useed"])
def test_assembly_bitwise(golden, N, pat, utag):
    p = f"n{N}_"
    xyz, conn, vol = golden[p + "ref_xyz"], golden[p + "ref_conn"], golden[p + "ref_vol"]
    rp = golden[p + "ref_row_ptr"]
    ci = golden[p + "ref_col_idx"] if pat == "refpat" else golden[p + "orc_solve_col_idx"]
    u = golden[p + "in_u"] if utag == "useed" else np.zeros(xyz.size)
    ne = conn.size // 4
    mu, lam = O.lame(1.0, 0.3)
    slot = O.slot_map(xyz.size // 3, conn, rp, ci)
    K, f = O.assemble(xyz, conn, np.full(ne, mu), np.full(ne, lam), 0.3, u, slot, ci.size,
                      (vol >= 1e-30).astype(np.uint8))
    assert np.array_equal(K, golden[p + f"ref_K_{pat}_{utag}"])
    assert np.array_equal(f, golden[p + f"ref_f_{pat}_{utag}"])
    if utag == "useed":
        _, fr = O.assemble(xyz, conn, np.full(ne, mu), np.full(ne, lam), 0.3, u,
                           active=(vol >= 1e-30).astype(np.uint8))
        assert np.array_equal(fr, golden[p + "ref_fres_useed"])


@pytest.mark.parametrize("N", [2, 4])
def test_ilu0_trsv_pcg_bitwise(golden, N):
    p = f"n{N}_"
    rp, ci = golden[p + "ref_row_ptr"], golden[p + "orc_solve_col_idx"]
    K = golden[p + "in_Kbc"]
    LU, d, _ = O.ilu0(rp, ci, K)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    lo, up = ci < rows, ci > rows
    assert np.array_equal(LU[lo], golden[p + "ref_ilu_L"][lo])
    assert np.array_equal(LU[up], golden[p + "ref_ilu_U"][up])
    assert np.array_equal(d, golden[p + "ref_ilu_diag"])
    # the reference's schedule is natural order: level[i] == i
    assert np.array_equal(golden[p + "ref_ilu_level"], np.arange(rp.size - 1))
    y = O.ilu0_apply(rp, ci, LU, d, golden[p + "in_r"])
    assert np.array_equal(y, golden[p + "ref_ilu_solve"])
    x, it, _ = O.pcg_ilu0(rp, ci, K, golden[p + "in_Rbc"], tol=1e-12, max_iter=1000)
    assert it == int(golden[p + "ref_pcg_iters"][0])
    assert np.array_equal(x, golden[p + "ref_pcg_x"])


@pytest.mark.parametrize("g", [8, 32])
def test_poisson_known_answer(golden, g):
    rp, ci, val, b, xe = O.poisson(g)
    assert np.array_equal(rp, golden[f"poisson{g}_rp"]) and np.array_equal(ci, golden[f"poisson{g}_ci"])
    assert np.array_equal(val, golden[f"poisson{g}_val"]) and np.array_equal(b, golden[f"poisson{g}_b"])
    x, it, _ = O.pcg_ilu0(rp, ci, val, b, tol=1e-10, max_iter=4000)
    assert it == int(golden[f"poisson{g}_ref_iters"][0])
    assert np.array_equal(x, golden[f"poisson{g}_ref_x"])
    res = np.linalg.norm(b - O.spmv(rp, ci, val, x)) / np.linalg.norm(b)
    assert res <= 1e-8
    if g == 32:
        assert it == 27


def test_levels_are_true_depths(golden):
    rp, ci = golden["n4_ref_row_ptr"], golden["n4_orc_solve_col_idx"]
    fp, fr, bp, br = O.levels(rp, ci)
    n = rp.size - 1
    depth = np.empty(n, np.int64)
    for lv in range(fp.size - 1):
        depth[fr[fp[lv]:fp[lv + 1]]] = lv
    for i in range(n):
        cols = ci[rp[i]:rp[i + 1]]
        lower = cols[cols < i]
        assert depth[i] == (0 if lower.size == 0 else 1 + depth[lower].max())
    assert fp.size - 1 == 18 * 4  # 18 N DOF levels on the unit cube


@pytest.mark.skipif(not O.have_reference(), reason="reference build absent")
def test_oracle_vs_reference_n8():
    import ctypes as C

    R = O.ref()
    xyz, conn = O.unit_cube(8)
    nn = xyz.size // 3
    rp, ci = O.pattern(nn, conn, "solve")
    vol = O.volumes(xyz, conn)
    rng = np.random.default_rng(8)
    u = 0.02 * rng.standard_normal(3 * nn)
    K1, f1 = np.zeros(ci.size), np.zeros(3 * nn)
    R.ref_assemble(nn, xyz, conn.size // 4, conn, vol, 1.0, 0.3, u, rp, ci, K1, f1, 1)
    mu, lam = O.lame(1.0, 0.3)
    ne = conn.size // 4
    K2, f2 = O.assemble(xyz, conn, np.full(ne, mu), np.full(ne, lam), 0.3, u,
                        O.slot_map(nn, conn, rp, ci), ci.size, (vol >= 1e-30).astype(np.uint8))
    assert np.array_equal(K1, K2) and np.array_equal(f1, f2)
