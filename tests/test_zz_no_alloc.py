"""fm_ilu0_apply_noalloc against fm_ilu0_apply on the same factorization.

The no-alloc entry point serves callers that must not allocate device
memory during a call (their HBM belongs to another allocator, or they
cannot take cudaFree's device-wide synchronization): it keeps its
intermediate vector and status word in a library-owned static device array
instead of context buffers.  Both entry points run the same node-block
solves on the same LU, so the outputs must be bit-identical.  Two no-alloc
calls in a row check that the shared scratch carries nothing from one call
into the next.  This file is collected last, so it runs both alone and
after every other GPU test in one process.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MAX_DOFS = 1 << 20  # FM_NOALLOC_MAX_DOFS in include/fm_api.h
FM_ERR_LIMITS = 9


@pytest.fixture(scope="module")
def fm():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


@pytest.mark.parametrize("N,path", [(6, "push"), (12, "push"), (6, "pipe")])
def test_noalloc_apply_matches_ilu0_apply(fm, monkeypatch, N, path):
    """path: the triangular solves the context plans at fm_set_mesh (the
    slab-partitioned push solves, or the grid-wide pipelined ones that
    meshes beyond the push plan's limits use); the static scratch serves both"""
    from flexmesh_b200 import configs

    P = configs.small_block(N)
    monkeypatch.setenv("FM_TRSV_PATH", path)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn)
    monkeypatch.delenv("FM_TRSV_PATH", raising=False)
    ctx.set_material(1.0, P.nu)
    ctx.set_bc(P.mask, P.bc_value)
    u = 0.01 * np.random.default_rng(3).standard_normal(P.xyz.size)
    u[P.mask == 1] = 0.0
    ctx.assemble_into_context(cu(u), apply_bc=True)
    ctx.ilu0()
    rng = np.random.default_rng(11)
    r1 = cu(rng.standard_normal(P.xyz.size))
    r2 = cu(rng.standard_normal(P.xyz.size))
    ref1 = ctx.ilu0_apply(r1)
    ref2 = ctx.ilu0_apply(r2)
    y = torch.full_like(r1, float("nan"))
    ctx.ilu0_apply_noalloc(r1, y)
    assert torch.equal(y, ref1)
    # second call in a row: other right-hand side, same output buffer
    ctx.ilu0_apply_noalloc(r2, y)
    assert torch.equal(y, ref2)
    assert bool(torch.isfinite(y).all())


def test_noalloc_rejects_beyond_limit(fm):
    # unit cube N=70: 3 * 71^3 = 1,073,733 DOFs > 2^20
    xyz, conn = fm.unit_cube(70)
    assert xyz.size > MAX_DOFS
    ctx = fm.Context(0)
    ctx.set_mesh(xyz, conn)
    r = torch.zeros(xyz.size, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(r)
    with pytest.raises(fm.FMError) as exc:
        ctx.ilu0_apply_noalloc(r, y)
    assert exc.value.status == FM_ERR_LIMITS
    assert "scratch limit" in str(exc.value)
