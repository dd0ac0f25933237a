"""The slab-partitioned push solves (fm_trsv_push.cu, the default path)
against the grid-wide pipelined solves (fm_trsv.cu, FM_TRSV_PATH=pipe).

Both walk the same node-block factors with the same per-node arithmetic
(lane k owns neighbour k, the same butterfly, the same finish), so every
result must be bit-identical: the preconditioner apply, PCG in FP64 and in
mixed precision, and Newton load steps.  The pipelined path is the one the
oracle parity tests pin.  Meshes: the unit-cube block, the same block with
nodes relabelled at random inside blocks of 8 ids (irregular levels and
slots), and a single hex (most CTAs own no node).  A block relabelled at
random over all ids has nodes with up to 18 neighbours on one side; the
push solves give a node half a warp (at most 16), so there the context
keeps the pipelined solves, which is checked too.  The path is
chosen when the mesh is set, so the environment variable is set around
fm_set_mesh only; the profiler's kernel count shows which path ran (three
kernels per fused apply, four in place).
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def block(N, seed):
    """small_block(N), nodes renamed by a seeded permutation: over all ids
    (seed > 0) or inside blocks of 8 consecutive ids (seed < 0)"""
    from flexmesh_b200 import configs

    P = configs.small_block(N)
    if not seed:
        return P, P.xyz, P.conn, P.mask, P.bc_value
    nn = P.n_nodes
    rng = np.random.default_rng(abs(seed))
    if seed > 0:
        perm = rng.permutation(nn)
    else:
        perm = np.arange(nn)
        for b in range(0, nn, 8):
            perm[b:b + 8] = b + rng.permutation(min(8, nn - b))
    xyz = np.empty_like(P.xyz).reshape(-1, 3)
    xyz[perm] = P.xyz.reshape(-1, 3)
    conn = perm[P.conn.astype(np.int64)].astype(np.uint32)
    dof = (3 * perm[:, None] + np.arange(3)).reshape(-1)
    mask = np.empty_like(P.mask)
    val = np.empty_like(P.bc_value)
    mask[dof] = P.mask
    val[dof] = P.bc_value
    return P, xyz.reshape(-1), conn, mask, val


def context(fm, monkeypatch, mesh, push):
    P, xyz, conn, mask, val = mesh
    monkeypatch.setenv("FM_TRSV_PATH", "push" if push else "pipe")
    ctx = fm.Context(0)
    ctx.set_mesh(xyz, conn, P.elem_volume)
    monkeypatch.delenv("FM_TRSV_PATH", raising=False)
    ctx.set_material(1.0, P.nu)
    ctx.set_bc(mask, val)
    return ctx


def trsv_kernels(ctx, fn):
    ctx.profile_enable(True)
    out = fn()
    prof = ctx.profile_read()["trsv"]
    ctx.profile_enable(False)
    return out, prof["kernels"], prof["calls"]


@pytest.mark.parametrize("N,seed", [(6, 0), (12, 0), (5, -3), (8, -17)])
def test_push_apply_and_pcg_bitwise(fm, monkeypatch, N, seed):
    mesh = block(N, seed)
    xyz = mesh[1]
    u = 0.01 * np.random.default_rng(abs(seed) + 1).standard_normal(xyz.size)
    u[mesh[3] == 1] = 0.0
    r = cu(np.random.default_rng(abs(seed) + 2).standard_normal(xyz.size))
    res = {}
    for push in (False, True):
        ctx = context(fm, monkeypatch, mesh, push)
        ctx.assemble_into_context(cu(u), apply_bc=True)
        ctx.ilu0()
        y, kern, calls = trsv_kernels(ctx, lambda: ctx.ilu0_apply(r))
        assert calls == 1 and kern == (3 if push else 4)
        b = cu(np.random.default_rng(abs(seed) + 3).standard_normal(xyz.size))
        x, it, rr = ctx.pcg(b, tol=1e-10, max_iter=2000)
        ctx.assemble_into_context(cu(u), prec=fm.FM_MIXED, apply_bc=True)
        ctx.ilu0(fm.FM_MIXED)
        x32, it32, rr32 = ctx.pcg(b, tol=1e-6, max_iter=2000, prec=fm.FM_MIXED)
        assert ctx.flags() & fm.FLAG_TIMEOUT == 0
        res[push] = (y, x, it, rr, x32, it32, rr32)
    (y0, x0, i0, r0, xm0, im0, rm0), (y1, x1, i1, r1, xm1, im1, rm1) = res[False], res[True]
    assert torch.equal(y0, y1)
    assert i0 == i1 and r0 == r1 and torch.equal(x0, x1)
    assert im0 == im1 and rm0 == rm1 and torch.equal(xm0, xm1)
    assert rm1 < 1e-6 and r1 < 1e-10


def test_push_declines_high_valence(fm, monkeypatch):
    """random relabelling: a side with more than 16 neighbours keeps the
    pipelined solves (four kernels per apply) with the same results"""
    mesh = block(5, 3)
    u = np.zeros(mesh[1].size)
    r = cu(np.random.default_rng(9).standard_normal(mesh[1].size))
    ys = []
    for push in (False, True):
        ctx = context(fm, monkeypatch, mesh, push)
        ctx.assemble_into_context(cu(u), apply_bc=True)
        ctx.ilu0()
        y, kern, calls = trsv_kernels(ctx, lambda: ctx.ilu0_apply(r))
        assert calls == 1 and kern == 4
        ys.append(y)
    assert torch.equal(ys[0], ys[1])


def test_push_in_place_apply(fm, monkeypatch):
    """r and y the same buffer: the forward solve still reads r, so y is
    filled only after it (four kernels)"""
    mesh = block(7, 0)
    ctx = context(fm, monkeypatch, mesh, True)
    u = np.zeros(mesh[1].size)
    ctx.assemble_into_context(cu(u), apply_bc=True)
    ctx.ilu0()
    r = cu(np.random.default_rng(5).standard_normal(mesh[1].size))
    ref = ctx.ilu0_apply(r)
    buf = r.clone()
    ptr = C.c_void_p(buf.data_ptr())

    def in_place():
        st = fm.lib().fm_ilu0_apply(ctx._h, ptr, ptr)
        assert st == 0
        torch.cuda.synchronize()
        return buf

    out, kern, calls = trsv_kernels(ctx, in_place)
    assert calls == 1 and kern == 4
    assert torch.equal(out, ref)


@pytest.mark.parametrize("N,seed,mixed", [(8, 0, False), (4, -5, False), (1, 0, False),
                                          (12, 0, True)])
def test_push_newton_bitwise(fm, monkeypatch, N, seed, mixed):
    mesh = block(N, seed)
    P = mesh[0]
    out = {}
    for push in (False, True):
        ctx = context(fm, monkeypatch, mesh, push)
        u = torch.zeros(mesh[1].size, dtype=torch.float64, device="cuda")
        counts = []
        for s in range(1, min(P.n_steps, 3) + 1):
            if mixed:
                rep = ctx.newton_step(u, s / P.n_steps, rtol=1e-10, inner_tol=0.2,
                                      max_newton=400, prec=fm.FM_MIXED)
            else:
                rep = ctx.newton_step(u, s / P.n_steps, rtol=1e-10, inner_tol=1e-12)
            counts.append((rep["newton_iters"], rep.get("pcg_iters")))
        assert ctx.flags() & fm.FLAG_TIMEOUT == 0
        out[push] = (u, counts)
    assert out[False][1] == out[True][1]
    assert torch.equal(out[False][0], out[True][0])
    assert bool(torch.isfinite(out[True][0]).all())
