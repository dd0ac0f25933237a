"""GPU parity on meshes without the unit cube's node numbering.

The unit cube's natural numbering gives short, regular dependency levels.
Relabelling its nodes at random keeps the same elements and physics but
gives the solver an irregular graph: long-lived dependencies, uneven level
widths, neighbours of a neighbour scattered over the node range.  That
exercises the host-built schedules and the ILU(0) column map beyond the
regular case.  The tiniest mesh (one hex) checks the degenerate schedules.
Bars as in test_gpu_parity.py.
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_ILU = 1e-12
TOL_U = 1e-10


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


def relabelled(N, seed):
    """small_block(N) with node i renamed perm[i]"""
    from flexmesh_b200 import configs

    P = configs.small_block(N)
    nn = P.n_nodes
    perm = np.random.default_rng(seed).permutation(nn)
    xyz = np.empty_like(P.xyz).reshape(-1, 3)
    xyz[perm] = P.xyz.reshape(-1, 3)
    conn = perm[P.conn.astype(np.int64)].astype(np.uint32)
    dof = (3 * perm[:, None] + np.arange(3)).reshape(-1)
    mask = np.empty_like(P.mask)
    val = np.empty_like(P.bc_value)
    mask[dof] = P.mask
    val[dof] = P.bc_value
    return P, xyz.reshape(-1), conn, mask, val


@pytest.mark.parametrize("seed", [3, 17])
def test_relabelled_ilu_apply_pcg_match_oracle(fm, seed):
    P, xyz, conn, mask, val = relabelled(5, seed)
    ctx = fm.Context(0)
    ctx.set_mesh(xyz, conn, P.elem_volume)
    ctx.set_material(1.0, P.nu)
    ctx.set_bc(mask, val)
    u = 0.01 * np.random.default_rng(seed).standard_normal(xyz.size)
    u[mask == 1] = 0.0
    ctx.assemble_into_context(cu(u), apply_bc=True)
    ctx.ilu0()
    LU, d = ctx.get_ilu0()
    rp, ci = O.pattern(P.n_nodes, conn, "solve")
    mu, lam = P.lame()
    act = (P.elem_volume >= 1e-30).astype(np.uint8)
    Ko, fo = O.assemble(xyz, conn, mu, lam, P.nu, u, O.slot_map(P.n_nodes, conn, rp, ci),
                        ci.size, act)
    Ro = -fo
    O.apply_bc(rp, ci, Ko, Ro, mask)
    LUo, do, _ = O.ilu0(rp, ci, Ko)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    off = ci != rows
    assert rel(LU[off], LUo[off]) <= TOL_ILU and rel(d, do) <= TOL_ILU
    r = np.random.default_rng(seed + 1).standard_normal(xyz.size)
    y = ctx.ilu0_apply(cu(r))
    yo = O.ilu0_apply(rp, ci, LUo, do, r)
    assert np.linalg.norm(y.cpu().numpy() - yo) <= 1e-11 * np.linalg.norm(yo)
    x, it, _ = ctx.pcg(cu(Ro), tol=1e-12, max_iter=2000)
    xo, ito, _ = O.pcg_ilu0(rp, ci, Ko, Ro, tol=1e-12, max_iter=2000)
    assert abs(it - ito) <= 1
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-10 * np.linalg.norm(xo)
    # mixed precision factors and solves on the same graph
    ctx.assemble_into_context(cu(u), prec=fm.FM_MIXED, apply_bc=True)
    ctx.ilu0(fm.FM_MIXED)
    x32, _, rr32 = ctx.pcg(cu(Ro), tol=1e-5, max_iter=2000, prec=fm.FM_MIXED)
    assert rr32 < 1e-5
    assert np.linalg.norm(x32.cpu().numpy() - xo) <= 1e-3 * np.linalg.norm(xo)


def test_relabelled_newton_matches_oracle(fm):
    P, xyz, conn, mask, val = relabelled(4, 5)
    ctx = fm.Context(0)
    ctx.set_mesh(xyz, conn, P.elem_volume)
    ctx.set_material(1.0, P.nu)
    ctx.set_bc(mask, val)
    u = torch.zeros(xyz.size, dtype=torch.float64, device="cuda")
    counts = []
    for s in range(1, P.n_steps + 1):
        r = ctx.newton_step(u, s / P.n_steps, rtol=1e-10, inner_tol=1e-12)
        counts.append(r["newton_iters"])
    rp, ci = O.pattern(P.n_nodes, conn, "solve")
    mu, lam = P.lame()
    uo, st, nps, _ = O.newton(xyz, conn, mu, lam, P.nu, rp, ci,
                              O.slot_map(P.n_nodes, conn, rp, ci), mask, val, P.n_steps,
                              rtol=1e-10, inner_tol=1e-12)
    assert st == 0
    ug = u.cpu().numpy()
    assert np.linalg.norm(ug - uo) <= TOL_U * np.linalg.norm(uo)
    assert counts == list(nps)


def test_single_hex_mesh(fm):
    """N = 1: 8 nodes, 6 tets (one a sliver), every node on the top or bottom face"""
    from flexmesh_b200 import configs

    P = configs.small_block(1)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn, P.elem_volume)
    ctx.set_material(1.0, P.nu)
    ctx.set_bc(P.mask, P.bc_value)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    for s in range(1, P.n_steps + 1):
        ctx.newton_step(u, s / P.n_steps, rtol=1e-10, inner_tol=1e-12)
    ug = u.cpu().numpy()
    assert np.isfinite(ug).all()
    assert np.allclose(ug[P.mask == 1], P.bc_value[P.mask == 1], rtol=0, atol=1e-15)
