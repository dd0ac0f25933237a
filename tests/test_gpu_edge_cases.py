"""Edge cases of the C ABI on the GPU: meshes the library refuses, and
right-hand sides and load levels that leave nothing to solve.

- An empty mesh (no nodes or no tets) and connectivity that names a node
  outside the mesh are refused with FM_ERR_ARG; the context takes a valid
  mesh afterwards.
- PCG on b = 0 takes the reference's early exit (||b - A x0|| < tol * 1e-3,
  FEM/adaptive_fem_engine.hpp:1296-1298): zero iterations, x = 0, as the
  oracle's restatement of pcg_solve_ilu0 gives.
- A Newton load step at load 0 from u = 0 has R = 0 from the start: it
  returns after zero Newton iterations with u unchanged, in both precisions.
- Every tet skipped (stored volume 0, as the 6-tet split's slivers are):
  the tangent has no element contribution; with every DOF prescribed the
  eliminated system is the identity and PCG returns b.
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FM_ERR_ARG = 1


@pytest.fixture(scope="module")
def fm():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def test_empty_and_out_of_range_meshes_are_refused(fm):
    from flexmesh_b200 import configs

    ctx = fm.Context(0)
    with pytest.raises(fm.FMError) as e:
        ctx.set_mesh(np.zeros(3), np.zeros(0, np.uint32))
    assert e.value.status == FM_ERR_ARG
    P = configs.small_block(2)
    bad = P.conn.copy()
    bad[5] = P.n_nodes  # one past the last node
    with pytest.raises(fm.FMError) as e:
        ctx.set_mesh(P.xyz, bad)
    assert e.value.status == FM_ERR_ARG and "out of range" in str(e.value)
    ctx.set_mesh(P.xyz, P.conn)
    assert ctx.n_nodes == P.n_nodes


def small_ctx(fm, N=4):
    from flexmesh_b200 import configs

    P = configs.small_block(N)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn)
    ctx.set_material(P.E, P.nu)
    ctx.set_bc(P.mask, P.bc_value)
    return ctx, P


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pcg_on_zero_rhs_exits_early(fm, prec):
    p = fm.FM_FP64 if prec == "fp64" else fm.FM_MIXED
    ctx, P = small_ctx(fm)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    ctx.assemble_into_context(u, prec=p, apply_bc=True)
    ctx.ilu0(p)
    b = torch.zeros_like(u)
    x, it, _ = ctx.pcg(b, tol=1e-10, max_iter=100, prec=p)
    assert it == 0 and not torch.any(x != 0)
    # the oracle's pcg_solve_ilu0 restatement takes the same exit
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    K, _ = O.assemble(P.xyz, P.conn, mu, lam, P.nu, np.zeros(P.xyz.size),
                      O.slot_map(P.n_nodes, P.conn, rp, ci), ci.size)
    xo, ito = O.pcg_ilu0(rp, ci, K, np.zeros(P.xyz.size), tol=1e-10, max_iter=100)[:2]
    assert ito == 0 and not np.any(xo)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_newton_at_zero_load_does_nothing(fm, prec):
    p = fm.FM_FP64 if prec == "fp64" else fm.FM_MIXED
    ctx, P = small_ctx(fm)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    r = ctx.newton_step_cfg(u, 0.0, prec=p)
    assert r["status"] == 0 and r["newton_iters"] == 0
    assert not torch.any(u != 0)


def test_all_tets_skipped_leaves_identity_rows(fm):
    from flexmesh_b200 import configs

    P = configs.small_block(2)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn, np.zeros(P.n_elems))  # every stored volume 0
    ctx.set_material(P.E, P.nu)
    mask = np.ones(P.xyz.size, np.uint8)  # every DOF prescribed
    ctx.set_bc(mask, np.zeros(P.xyz.size))
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    K, f = ctx.assemble(u)
    assert not torch.any(f != 0)
    ctx.assemble_into_context(u, apply_bc=True)
    ctx.ilu0()
    b = torch.as_tensor(np.random.default_rng(1).standard_normal(P.xyz.size), device="cuda")
    x, it, _ = ctx.pcg(b, tol=1e-12, max_iter=10)
    assert it <= 1 and torch.allclose(x, b, rtol=0, atol=1e-14)
