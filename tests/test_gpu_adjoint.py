"""GPU adjoint: the exact-Jacobian products and the adjoint gradients
through the C ABI against the oracle, against central finite differences of
complete GPU Newton solves (the 1e-6 bar), FP64 vs mixed precision, and the
torch.autograd entry point."""
import numpy as np
import pytest

import oracle as O
from test_oracle_adjoint import small_problem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def bc_top(xyz, uz=-0.05):
    z = xyz[2::3]
    mask = np.zeros(xyz.size, np.uint8)
    val = np.zeros(xyz.size)
    mask[np.repeat(z < 1e-12, 3)] = 1
    mask[2::3][z > 1 - 1e-12] = 1
    val[2::3][z > 1 - 1e-12] = uz
    top = np.nonzero(z > 1 - 1e-12)[0]
    sel = np.sort(np.concatenate([3 * top, 3 * top + 1]))
    return mask, val, sel


def lame_ctx(F, xyz, conn, mu, lam, act, mask=None, val=None):
    ctx = F.Context(0)
    vol = act.astype(np.float64)  # stored volume 0 -> skipped, 1 -> kept
    ctx.set_mesh(xyz, conn, vol)
    ctx.set_material_lame(mu, lam, 0.3)
    if mask is not None:
        ctx.set_bc(mask, val)
    return ctx


@pytest.mark.parametrize("transpose", [False, True])
def test_exact_apply_matches_oracle(F, transpose):
    xyz, conn, mu, lam, act = small_problem(N=4)
    ctx = lame_ctx(F, xyz, conn, mu, lam, act)
    rng = np.random.default_rng(5)
    u = 0.02 * rng.standard_normal(xyz.size)
    v = rng.standard_normal(xyz.size)
    y = ctx.exact_apply(cu(u), cu(v), transpose).cpu().numpy()
    yo = O.exact_apply(xyz, conn, mu, lam, u, v, transpose=transpose, active=act)
    assert np.linalg.norm(y - yo) <= 1e-12 * np.linalg.norm(yo)


def solve_gpu(ctx, n, steps=3, prec=0, inner=1e-13):
    u = torch.zeros(n, dtype=torch.float64, device="cuda")
    for s in range(1, steps + 1):
        ctx.newton_step(u, s / steps, rtol=1e-13, inner_tol=inner, max_newton=400, prec=prec)
    return u


def test_adjoint_matches_oracle_and_finite_differences(F):
    xyz, conn, mu, lam, act = small_problem(N=2)
    mask, val, sel = bc_top(xyz)
    ctx = lame_ctx(F, xyz, conn, mu, lam, act, mask, val)
    target = np.random.default_rng(9).standard_normal(sel.size) * 1e-3
    u = solve_gpu(ctx, xyz.size)
    g = torch.zeros_like(u)
    g[cu(sel)] = u[cu(sel)] - cu(target)
    gm, gl, w, sweeps, _ = ctx.adjoint(u, g, tol=1e-12, inner_tol=1e-12, want_w=True)
    gm, gl = gm.cpu().numpy(), gl.cpu().numpy()
    # oracle adjoint at the same state
    nn = xyz.size // 3
    rp, ci = O.pattern(nn, conn, "solve")
    slot = O.slot_map(nn, conn, rp, ci)
    uh = u.cpu().numpy()
    Kt, _ = O.assemble(xyz, conn, mu, lam, 0.3, uh, slot, ci.size, act)
    O.apply_bc(rp, ci, Kt, None, mask)
    wo, _ = O.adjoint(xyz, conn, mu, lam, rp, ci, Kt, mask, uh, g.cpu().numpy(), tol=1e-12,
                      active=act)
    gmo, glo = O.param_grads(xyz, conn, uh, wo, active=act)
    assert np.linalg.norm(gm - gmo) <= 1e-9 * np.linalg.norm(gmo)
    assert np.linalg.norm(gl - glo) <= 1e-9 * np.linalg.norm(glo)

    def loss(uu):
        return 0.5 * float(torch.sum((uu[cu(sel)] - cu(target)) ** 2))

    for e in np.nonzero(act)[0][::9][:4]:
        for name, arr, grad in (("mu", mu, gm), ("lam", lam, gl)):
            p = arr.copy()
            h = 1e-6 * p[e]
            res = []
            for sgn in (1.0, -1.0):
                p[e] = arr[e] + sgn * h
                ctx.set_material_lame(p if name == "mu" else mu, p if name == "lam" else lam, 0.3)
                res.append(loss(solve_gpu(ctx, xyz.size)))
            fd = (res[0] - res[1]) / (2 * h)
            assert abs(grad[e] - fd) <= 1e-6 * abs(fd), (name, e, grad[e], fd)
    ctx.set_material_lame(mu, lam, 0.3)


def test_mixed_adjoint_matches_fp64(F):
    xyz, conn, mu, lam, act = small_problem(N=4)
    mask, val, sel = bc_top(xyz)
    ctx = lame_ctx(F, xyz, conn, mu, lam, act, mask, val)
    u = solve_gpu(ctx, xyz.size)
    g = torch.zeros_like(u)
    g[cu(sel)] = u[cu(sel)]
    gm64, gl64, _, s64, p64 = ctx.adjoint(u, g, tol=1e-10, inner_tol=1e-12)
    gm32, gl32, _, s32, p32 = ctx.adjoint(u, g, tol=1e-10, inner_tol=0.1, prec=F.FM_MIXED)
    rel = lambda a, b: (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()
    assert rel(gm32, gm64) <= 1e-8 and rel(gl32, gl64) <= 1e-8
    assert p32 < p64


def test_autograd_entry_point(F):
    from flexmesh_b200.autograd import LameSolver, SolveSettings, newton_solve

    xyz, conn, mu, lam, act = small_problem(N=3)
    mask, val, sel = bc_top(xyz)
    solver = LameSolver(xyz, conn, mask, val, 0.3, SolveSettings(n_steps=3, rtol=1e-12,
                                                                  inner_tol=1e-12),
                        elem_volume=act.astype(np.float64))
    mu_t = torch.tensor(mu, dtype=torch.float64, device="cuda", requires_grad=True)
    lam_t = torch.tensor(lam, dtype=torch.float64, device="cuda", requires_grad=True)
    u = newton_solve(mu_t, lam_t, solver)
    selt = cu(sel)
    L = 0.5 * torch.sum(u[selt] ** 2)
    L.backward()
    g = torch.zeros_like(u)
    g[selt] = u.detach()[selt]
    gm, gl = solver.adjoint(u.detach(), g)
    assert torch.allclose(mu_t.grad, gm, rtol=0, atol=1e-14 + 1e-12 * gm.abs().max().item())
    assert torch.allclose(lam_t.grad, gl, rtol=0, atol=1e-14 + 1e-12 * gl.abs().max().item())
    assert solver.last["adjoint_sweeps"] > 0
