"""GPU parity: the CUDA path (through the C ABI) against the reference's own
outputs (golden fixtures from oracle/_ref) and the C oracle.

Bars: integer structures (patterns, slot maps, level sets) bit-exact; FP64
values within the stated normwise tolerances; Newton displacements within
1e-10 relative of the oracle; mixed precision within 1e-8 of FP64.
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# element K/f on random, poorly shaped tets, normwise max-relative: the
# kernel evaluates the Mandel stress as mu (C - I) + lam lnJ I, the reference
# as C S with C^-1, whose own rounding grows with cond(C)
TOL_ELEM = 1e-12
TOL_ASM = 1e-13    # assembled K.val / f_int, normwise max-relative
TOL_ILU = 1e-12    # L, U multipliers and pivots, normwise max-relative
TOL_U = 1e-10      # Newton displacement vs oracle, relative 2-norm


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


@pytest.fixture(scope="module")
def fm():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def make_ctx(fm, xyz, conn, vol=None, E=1.0, nu=0.3, E_elem=None):
    ctx = fm.Context(0)
    ctx.set_mesh(xyz, conn, vol)
    ctx.set_material(E, nu, E_elem)
    return ctx


def test_elements_match_reference(fm, golden):
    x, u, E = golden["in_elem_x"], golden["in_elem_u"], golden["in_elem_E"]
    ctx = fm.Context(0)
    K, f = ctx.elements(cu(x), cu(u), cu(E), 0.3)
    K, f = K.cpu().numpy(), f.cpu().numpy()
    for t in range(x.shape[0]):
        assert rel(K[t], golden["ref_elem_K"][t]) <= TOL_ELEM
        assert rel(f[t], golden["ref_elem_f"][t]) <= TOL_ELEM


@pytest.mark.parametrize("N", [2, 4])
def test_patterns_and_slot_maps_bitwise(fm, golden, N):
    p = f"n{N}_"
    xyz, conn = golden[p + "ref_xyz"], golden[p + "ref_conn"]
    ctx = make_ctx(fm, xyz, conn)
    rp, ci, sm = ctx.build_pattern(fm.FM_PATTERN_REFERENCE, slot_map=True)
    assert np.array_equal(rp, golden[p + "ref_row_ptr"])
    assert np.array_equal(ci, golden[p + "ref_col_idx"])
    assert np.array_equal(sm, O.slot_map(xyz.size // 3, conn, rp, ci))
    rp2, ci2, sm2 = ctx.build_pattern(fm.FM_PATTERN_SOLVE, slot_map=True)
    assert np.array_equal(rp2, rp)
    assert np.array_equal(ci2, golden[p + "orc_solve_col_idx"])
    assert np.array_equal(sm2, O.slot_map(xyz.size // 3, conn, rp2, ci2))
    assert (sm2 >= 0).all()


@pytest.mark.parametrize("N", [4, 8])
def test_level_sets_bitwise(fm, N):
    xyz, conn = O.unit_cube(N)
    ctx = make_ctx(fm, xyz, conn)
    rp, ci, _ = ctx.build_pattern(fm.FM_PATTERN_SOLVE)
    got = ctx.levels()
    exp = O.levels(rp, ci)
    for g, e in zip(got, exp):
        assert np.array_equal(g, e)
    assert got[0].size - 1 == 18 * N


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("utag", ["u0", "useed"])
def test_assembly_matches_reference(fm, golden, N, utag):
    p = f"n{N}_"
    xyz, conn, vol = golden[p + "ref_xyz"], golden[p + "ref_conn"], golden[p + "ref_vol"]
    ctx = make_ctx(fm, xyz, conn, vol)
    u = golden[p + "in_u"] if utag == "useed" else np.zeros(xyz.size)
    K, f = ctx.assemble(cu(u))
    Kr, fr = golden[p + f"ref_K_solvepat_{utag}"], golden[p + f"ref_f_solvepat_{utag}"]
    assert rel(K.cpu().numpy(), Kr) <= TOL_ASM
    # f_int is a sum of cancelling element forces: compare on the element-force scale
    fe = np.abs(golden[p + "ref_fres_useed"]).max() if utag == "useed" else 1.0
    assert np.abs(f.cpu().numpy() - fr).max() <= TOL_ASM * max(fe, np.abs(fr).max(), 1e-300)
    # residual-only entry point
    fo = ctx.residual(cu(u)).cpu().numpy()
    assert np.array_equal(fo, f.cpu().numpy())
    # mixed: f_int stays FP64 and identical; K in FP32
    K32, f32 = ctx.assemble(cu(u), prec=fm.FM_MIXED)
    assert np.array_equal(f32.cpu().numpy(), f.cpu().numpy())
    assert rel(K32.cpu().numpy().astype(np.float64), Kr) <= 1e-6


@pytest.mark.parametrize("N", [2, 4])
def test_reference_pattern_assembly(fm, golden, N):
    p = f"n{N}_"
    xyz, conn, vol = golden[p + "ref_xyz"], golden[p + "ref_conn"], golden[p + "ref_vol"]
    ctx = make_ctx(fm, xyz, conn, vol)
    K, f = ctx.assemble_reference_pattern(cu(golden[p + "in_u"]))
    assert rel(K.cpu().numpy(), golden[p + "ref_K_refpat_useed"]) <= TOL_ASM
    fr = golden[p + "ref_f_refpat_useed"]
    assert np.abs(f.cpu().numpy() - fr).max() <= 1e-13 * np.abs(fr).max()


def test_assembly_deterministic_and_host_entry(fm):
    P_xyz, P_conn = O.unit_cube(8)
    ctx = make_ctx(fm, P_xyz, P_conn)
    u = 0.01 * np.random.default_rng(3).standard_normal(P_xyz.size)
    K1, f1 = ctx.assemble(cu(u))
    K2, f2 = ctx.assemble(cu(u))
    assert torch.equal(K1, K2) and torch.equal(f1, f2)
    Kh, fh = ctx.assemble_host(u)
    assert np.array_equal(Kh, K1.cpu().numpy()) and np.array_equal(fh, f1.cpu().numpy())


def test_assembly_n8_matches_oracle_with_bc(fm):
    from flexmesh_b200 import configs

    P = configs.small_block(8)
    ctx = make_ctx(fm, P.xyz, P.conn)
    ctx.set_bc(P.mask, P.bc_value)
    u = 0.01 * np.random.default_rng(5).standard_normal(P.xyz.size)
    K, f = ctx.assemble(cu(u), apply_bc=True)
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    Ko, fo = O.assemble(P.xyz, P.conn, mu, lam, P.nu, u, O.slot_map(P.n_nodes, P.conn, rp, ci),
                        ci.size)
    O.apply_bc(rp, ci, Ko, None, P.mask)
    assert rel(K.cpu().numpy(), Ko) <= TOL_ASM
    assert np.abs(f.cpu().numpy() - fo).max() <= TOL_ASM * 1e-1


@pytest.mark.parametrize("N", [2, 4])
def test_csr_ilu0_matches_reference(fm, golden, N):
    p = f"n{N}_"
    rp, ci, K = golden[p + "ref_row_ptr"], golden[p + "orc_solve_col_idx"], golden[p + "in_Kbc"]
    ctx = fm.Context(0)
    LU, d = ctx.csr_ilu0(rp, ci, K)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    lo, up = ci < rows, ci > rows
    assert rel(LU[lo], golden[p + "ref_ilu_L"][lo]) <= TOL_ILU
    assert rel(LU[up], golden[p + "ref_ilu_U"][up]) <= TOL_ILU
    assert rel(d, golden[p + "ref_ilu_diag"]) <= TOL_ILU
    # unsorted input columns give the same factors in the caller's order
    perm = np.concatenate([np.arange(rp[i], rp[i + 1])[::-1] for i in range(rp.size - 1)])
    LU2, d2 = ctx.csr_ilu0(rp, ci[perm], K[perm])
    assert np.array_equal(LU2, LU[perm]) and np.array_equal(d2, d)


@pytest.mark.parametrize("N", [2, 4])
def test_pcg_matches_reference(fm, golden, N):
    p = f"n{N}_"
    rp, ci, K = golden[p + "ref_row_ptr"], golden[p + "orc_solve_col_idx"], golden[p + "in_Kbc"]
    ctx = fm.Context(0)
    x, it, rr = ctx.csr_pcg_ilu0(rp, ci, K, golden[p + "in_Rbc"], tol=1e-12, max_iter=1000)
    assert it == int(golden[p + "ref_pcg_iters"][0])
    xr = golden[p + "ref_pcg_x"]
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)


@pytest.mark.parametrize("g", [8, 32])
def test_poisson_known_answer(fm, golden, g):
    rp, ci, val, b = (golden[f"poisson{g}_rp"], golden[f"poisson{g}_ci"], golden[f"poisson{g}_val"],
                      golden[f"poisson{g}_b"])
    ctx = fm.Context(0)
    x, it, rr = ctx.csr_pcg_ilu0(rp, ci, val, b, tol=1e-10, max_iter=4000)
    assert it == int(golden[f"poisson{g}_ref_iters"][0])
    xr = golden[f"poisson{g}_ref_x"]
    assert np.linalg.norm(x - xr) <= 1e-10 * np.linalg.norm(xr)
    res = np.linalg.norm(b - O.spmv(rp, ci, val, x)) / np.linalg.norm(b)
    assert res <= 1e-8


def test_context_ilu_pcg_matches_oracle(fm):
    from flexmesh_b200 import configs

    P = configs.small_block(6)
    ctx = make_ctx(fm, P.xyz, P.conn)
    ctx.set_bc(P.mask, P.bc_value)
    u = 0.01 * np.random.default_rng(7).standard_normal(P.xyz.size)
    u[P.mask == 1] = 0.0
    ctx.assemble_into_context(cu(u), apply_bc=True)
    ctx.ilu0()
    LU, d = ctx.get_ilu0()
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    Ko, fo = O.assemble(P.xyz, P.conn, mu, lam, P.nu, u, O.slot_map(P.n_nodes, P.conn, rp, ci),
                        ci.size)
    Ro = -fo
    O.apply_bc(rp, ci, Ko, Ro, P.mask)
    LUo, do, _ = O.ilu0(rp, ci, Ko)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    off = ci != rows
    assert rel(LU[off], LUo[off]) <= TOL_ILU and rel(d, do) <= TOL_ILU
    # one preconditioner apply
    r = np.random.default_rng(9).standard_normal(P.xyz.size)
    y = ctx.ilu0_apply(cu(r)).cpu().numpy()
    yo = O.ilu0_apply(rp, ci, LUo, do, r)
    assert np.linalg.norm(y - yo) <= 1e-11 * np.linalg.norm(yo)
    x, it, rr = ctx.pcg(cu(Ro), tol=1e-12, max_iter=2000)
    xo, ito, _ = O.pcg_ilu0(rp, ci, Ko, Ro, tol=1e-12, max_iter=2000)
    assert abs(it - ito) <= 1
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)


@pytest.mark.parametrize("N", [4, 8])
def test_newton_small_matches_oracle(fm, N):
    """the small workload (E=1, nu=0.3, top u_z=-0.1 in 5 steps), node by node"""
    from flexmesh_b200 import configs

    P = configs.small_block(N)
    ctx = make_ctx(fm, P.xyz, P.conn)
    ctx.set_bc(P.mask, P.bc_value)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    counts = []
    for s in range(1, P.n_steps + 1):
        r = ctx.newton_step(u, s / P.n_steps, rtol=1e-10, inner_tol=1e-12)
        counts.append(r["newton_iters"])
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    uo, st, nps, pps = O.newton(P.xyz, P.conn, mu, lam, P.nu, rp, ci,
                                O.slot_map(P.n_nodes, P.conn, rp, ci), P.mask, P.bc_value,
                                P.n_steps, rtol=1e-10, inner_tol=1e-12)
    assert st == 0
    ug = u.cpu().numpy()
    assert np.linalg.norm(ug - uo) <= TOL_U * np.linalg.norm(uo)
    assert np.abs(ug - uo).max() <= TOL_U * np.abs(uo).max()
    assert counts == list(nps)


def test_mixed_precision_matches_fp64(fm):
    from flexmesh_b200 import configs

    P = configs.small_block(8)
    ctx = make_ctx(fm, P.xyz, P.conn)
    ctx.set_bc(P.mask, P.bc_value)
    u64 = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    r64 = ctx.newton_solve(u64, P.n_steps, rtol=1e-10, inner_tol=1e-12)
    u32 = torch.zeros_like(u64)
    r32 = ctx.newton_solve(u32, P.n_steps, rtol=1e-10, inner_tol=1e-4, prec=fm.FM_MIXED)
    err = (torch.linalg.norm(u32 - u64) / torch.linalg.norm(u64)).item()
    assert err <= 1e-8, (err, r64, r32)
    assert r32["pcg_iters"] < r64["pcg_iters"]


def test_line_search_accepts_full_steps(fm):
    from flexmesh_b200 import configs

    P = configs.small_block(4)
    ctx = make_ctx(fm, P.xyz, P.conn)
    ctx.set_bc(P.mask, P.bc_value)
    ua = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    ub = torch.zeros_like(ua)
    for s in range(1, P.n_steps + 1):
        ra = ctx.newton_step(ua, s / P.n_steps)
        rb = ctx.newton_step(ub, s / P.n_steps, line_search=10, ls_c=0.1)
        assert ra["newton_iters"] == rb["newton_iters"]
    assert torch.equal(ua, ub)
