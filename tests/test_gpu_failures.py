"""Failure detection on the GPU, in the forms that fault, trap or hang no GPU.

- A bounded wait runs out: a wait on a flag that nothing sets (fm_check_wait)
  and real solves under a tiny wait limit end with FM_ERR_TIMEOUT, never a
  hang, and the same context solves correctly afterwards.
- Host-side injection: a NaN planted in u gives FM_ERR_NONFINITE with the
  flags named in the error text; an element pushed through its opposite
  face raises FM_FLAG_INVERTED / FM_FLAG_J_CLAMPED with K and f still equal
  to the oracle's (the reference clamps ln J at J = 0.01,
  FEM/adaptive_fem_engine.hpp:102).
- A vanishing ILU(0) pivot gets the reference's +-1e-8 perturbation
  (FEM/adaptive_fem_engine.hpp:384-386) and raises FM_FLAG_PIVOT.
"""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FM_ERR_NONFINITE, FM_ERR_TIMEOUT = 4, 7


@pytest.fixture(scope="module")
def fm():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def small_ctx(fm, N=4):
    from flexmesh_b200 import configs

    P = configs.small_block(N)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn)
    ctx.set_material(P.E, P.nu)
    ctx.set_bc(P.mask, P.bc_value)
    return ctx, P


def pcg_once(ctx, P, u):
    ctx.assemble_into_context(u, apply_bc=True)
    ctx.ilu0()
    b = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    b[torch.as_tensor(P.mask == 0, device="cuda")] = 1.0
    return ctx.pcg(b, tol=1e-10, max_iter=500)


def test_wait_on_unset_flag_times_out_and_context_recovers(fm):
    ctx, P = small_ctx(fm)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    x_ref, it_ref, _ = pcg_once(ctx, P, u)
    ctx.set_wait_limit(4_000_000)  # about 2 ms at B200 clocks
    assert ctx.check_wait() == FM_ERR_TIMEOUT
    assert ctx.flags() & fm.FLAG_TIMEOUT
    # while the flag stands every wait gives up at once: the solve reports it
    with pytest.raises(fm.FMError) as e:
        pcg_once(ctx, P, u)
    assert e.value.status == FM_ERR_TIMEOUT
    ctx.clear_flags()
    ctx.set_wait_limit(0)
    x, it, _ = pcg_once(ctx, P, u)
    assert it == it_ref
    assert torch.equal(x, x_ref)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_tiny_wait_limit_on_real_solves_never_hangs(fm, prec):
    """A limit of 1024 cycles: the factorization's and the triangular
    solves' dependency waits may run out (FM_ERR_TIMEOUT) or all finish in
    time (FM_OK); either way the call returns, and with the default limit
    the context reproduces a fresh context's Newton step."""
    p = fm.FM_FP64 if prec == "fp64" else fm.FM_MIXED
    tol = 1e-12 if prec == "fp64" else 1e-4
    ctx0, P = small_ctx(fm, 6)
    u0 = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    r0 = ctx0.newton_step(u0, 1.0 / P.n_steps, inner_tol=tol, prec=p)
    ctx, _ = small_ctx(fm, 6)
    ctx.set_wait_limit(1024)
    u = torch.zeros_like(u0)
    statuses = set()
    for _ in range(3):
        try:
            ctx.newton_step(u.zero_(), 1.0 / P.n_steps, inner_tol=tol, prec=p)
            statuses.add(0)
        except fm.FMError as e:
            assert e.status == FM_ERR_TIMEOUT, str(e)
            statuses.add(FM_ERR_TIMEOUT)
            ctx.clear_flags()
    assert statuses <= {0, FM_ERR_TIMEOUT}
    ctx.set_wait_limit(0)
    ctx.clear_flags()
    r = ctx.newton_step(u.zero_(), 1.0 / P.n_steps, inner_tol=tol, prec=p)
    assert r["newton_iters"] == r0["newton_iters"]
    assert torch.equal(u, u0)


def test_nan_in_u_gives_nonfinite(fm):
    ctx, P = small_ctx(fm)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    free = np.nonzero(P.mask == 0)[0]
    u[int(free[len(free) // 2])] = float("nan")
    with pytest.raises(fm.FMError) as e:
        ctx.newton_step(u, 1.0 / P.n_steps)
    assert e.value.status == FM_ERR_NONFINITE
    assert "nonfinite" in str(e.value)
    assert ctx.flags() & fm.FLAG_NONFINITE
    # the context is usable again once the flags are cleared
    ctx.clear_flags()
    u.zero_()
    r = ctx.newton_step(u, 1.0 / P.n_steps)
    assert r["status"] == 0


def test_inverted_element_raises_flags_and_matches_oracle(fm):
    from flexmesh_b200 import configs

    P = configs.small_block(2)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn)
    ctx.set_material(P.E, P.nu)
    # push the centre node (1,1,1) through the tets around it: 7 tets end
    # up inverted, none within 0.1 of a singular F (near det F = 0 the
    # reference's guarded 3x3 inverse decides on rounding noise)
    X = P.xyz.reshape(-1, 3)
    c = int(np.argmin(np.abs(X - 0.5).sum(1)))
    u = np.zeros(P.xyz.size)
    u[3 * c: 3 * c + 3] = [0.7, 0.6, 0.55]
    ctx.clear_flags()
    K, f = ctx.assemble(cu(u))
    fl = ctx.flags()
    assert fl & fm.FLAG_INVERTED and fl & fm.FLAG_J_CLAMPED
    assert not fl & fm.FLAG_NONFINITE
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    mu, lam = P.lame()
    Ko, fo = O.assemble(P.xyz, P.conn, mu, lam, P.nu, u, O.slot_map(P.n_nodes, P.conn, rp, ci),
                        ci.size)
    K, f = K.cpu().numpy(), f.cpu().numpy()
    assert np.abs(K - Ko).max() <= 1e-12 * np.abs(Ko).max()
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()


def test_vanishing_pivot_is_perturbed_as_the_reference(fm):
    # row 1 eliminates to a zero pivot: 1 - (1/1) * 1 = 0 -> +1e-8
    rp = np.array([0, 2, 5, 7], np.uint32)
    ci = np.array([0, 1, 0, 1, 2, 1, 2], np.uint32)
    val = np.array([1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 2.0])
    ctx = fm.Context(0)
    ctx.clear_flags()
    LU, d = ctx.csr_ilu0(rp, ci, val)
    assert ctx.flags() & fm.FLAG_PIVOT
    LUo, do, npert = O.ilu0(rp, ci, val)
    assert npert == 1
    assert d[1] == 1e-8 and do[1] == 1e-8
    np.testing.assert_array_equal(d, do)
    np.testing.assert_array_equal(LU, LUo)
    R = O.ref()
    if R is not None:  # the reference's own factorize, where it was built
        Lr, Ur, dr = np.zeros(ci.size), np.zeros(ci.size), np.zeros(3)
        R.ref_ilu0(3, rp, ci, val, Lr, Ur, dr, None)
        np.testing.assert_array_equal(d, dr)


def test_flattened_element_takes_the_reference_guarded_inverse(fm):
    """A tet deformed flat (det F ~ 1e-16, det C below 1e-30): the reference's
    matrix_3x3_inv returns 1e30 I for C^-1 (FEM/adaptive_fem_engine.hpp:56-60)
    and the stress becomes (mu (1 - 1e30) + lam ln(0.01) 1e30) C; the
    element kernel reproduces it (oracle pinned to the reference)"""
    x = np.array([0.0, 0.0, 0.0, 1.0, 0.1, 0.0, 0.2, 1.0, 0.1, 0.1, 0.3, 1.0])
    y = x.copy()
    y[2::3] = 0.0  # every vertex moved into the plane z = 0
    u = y - x
    E, nu = 1.0, 0.3
    ctx = fm.Context(0)
    K, f = ctx.elements(cu(x.reshape(1, 12)), cu(u.reshape(1, 12)), cu(np.array([E])), nu)
    Ko, fo = O.element(x, u, E, nu)
    K, f = K.cpu().numpy().ravel(), f.cpu().numpy().ravel()
    assert np.abs(fo).max() > 1e20  # the guarded branch was taken
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
    assert np.abs(K - Ko).max() <= 1e-12 * np.abs(Ko).max()


def test_valence_beyond_the_kernels_limit_is_refused(fm):
    """a node shared by 40 tets (the kernels hold at most 32 incident tets
    and 32 neighbours per node): fm_set_mesh refuses with FM_ERR_LIMITS"""
    k = 40
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    ring = np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1)
    xyz = np.concatenate([[[0, 0, 0], [0, 0, 1]], ring]).reshape(-1)
    conn = np.array([[0, 1, 2 + i, 2 + (i + 1) % k] for i in range(k)], np.uint32).reshape(-1)
    ctx = fm.Context(0)
    with pytest.raises(fm.FMError) as e:
        ctx.set_mesh(xyz, conn)
    assert e.value.status == 9 and "valence" in str(e.value)
    # the context takes a valid mesh afterwards
    from flexmesh_b200 import configs

    P = configs.small_block(2)
    ctx.set_mesh(P.xyz, P.conn)
    assert ctx.n_nodes == P.n_nodes
