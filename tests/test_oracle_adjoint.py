"""CPU checks of the oracle's exact Jacobian and adjoint (new math: the
reference has no derivative code).  These pin the checker itself:
K_exact v against central differences of the reference-exact element force,
transpose consistency, parameter derivatives, and the full adjoint gradient
against central differences of complete Newton solves."""
import numpy as np
import pytest

import oracle as O


def small_problem(N=2, jitter=0.1, seed=3):
    xyz, conn = O.unit_cube(N)
    vol0 = O.volumes(xyz, conn)
    rng = np.random.default_rng(seed)
    s = N + 1
    idx = np.arange(xyz.size // 3)
    i, j, k = idx % s, (idx // s) % s, idx // (s * s)
    interior = (i > 0) & (i < N) & (j > 0) & (j < N) & (k > 0) & (k < N)
    X = xyz.reshape(-1, 3).copy()
    X[interior] += rng.uniform(-jitter / N, jitter / N, (interior.sum(), 3))
    ne = conn.size // 4
    mu = 0.38 * np.exp(0.3 * rng.standard_normal(ne))
    lam = 1.5 * mu
    act = (vol0 >= 1e-30).astype(np.uint8)
    return X.reshape(-1), conn, mu, lam, act


def test_exact_jacobian_matches_central_differences():
    xyz, conn, mu, lam, act = small_problem()
    rng = np.random.default_rng(1)
    u = 0.02 * rng.standard_normal(xyz.size)
    v = rng.standard_normal(xyz.size)
    Kv = O.exact_apply(xyz, conn, mu, lam, u, v, active=act)
    h = 1e-6
    _, fp = O.assemble(xyz, conn, mu, lam, 0.3, u + h * v, active=act)
    _, fm = O.assemble(xyz, conn, mu, lam, 0.3, u - h * v, active=act)
    fd = (fp - fm) / (2 * h)
    assert np.linalg.norm(Kv - fd) <= 1e-7 * np.linalg.norm(fd)


def test_exact_transpose_consistency():
    xyz, conn, mu, lam, act = small_problem(N=3)
    rng = np.random.default_rng(2)
    u = 0.02 * rng.standard_normal(xyz.size)
    v, w = rng.standard_normal(xyz.size), rng.standard_normal(xyz.size)
    Kv = O.exact_apply(xyz, conn, mu, lam, u, v, active=act)
    KTw = O.exact_apply(xyz, conn, mu, lam, u, w, transpose=True, active=act)
    assert abs(w @ Kv - KTw @ v) <= 1e-12 * abs(w @ Kv)
    # the jacobian is genuinely non-symmetric (the reference tangent is not it)
    KTv = O.exact_apply(xyz, conn, mu, lam, u, v, transpose=True, active=act)
    assert np.linalg.norm(KTv - Kv) > 1e-6 * np.linalg.norm(Kv)


def test_parameter_derivatives():
    xyz, conn, mu, lam, act = small_problem()
    rng = np.random.default_rng(4)
    u = 0.02 * rng.standard_normal(xyz.size)
    w = rng.standard_normal(xyz.size)
    gm, gl = O.param_grads(xyz, conn, u, w, active=act)
    for e in np.nonzero(act)[0][:6]:
        for arr, g in ((mu, gm), (lam, gl)):
            h = 1e-6 * arr[e]
            p = arr.copy()
            p[e] += h
            _, fp = O.assemble(xyz, conn, p if arr is mu else mu, p if arr is lam else lam, 0.3, u,
                               active=act)
            p[e] -= 2 * h
            _, fm = O.assemble(xyz, conn, p if arr is mu else mu, p if arr is lam else lam, 0.3, u,
                               active=act)
            fd = -(w @ (fp - fm)) / (2 * h)
            assert abs(g[e] - fd) <= 1e-6 * max(abs(fd), 1e-12), (e, g[e], fd)


def _solve(xyz, conn, mu, lam, rp, ci, slot, mask, val, act):
    u, st, nps, _ = O.newton(xyz, conn, mu, lam, 0.3, rp, ci, slot, mask, val, 3, rtol=1e-13,
                             inner_tol=1e-13, max_newton=400, active=act)
    assert st == 0
    return u


@pytest.mark.parametrize("which", ["mu", "lam"])
def test_adjoint_gradient_matches_full_solve_differences(which):
    xyz, conn, mu, lam, act = small_problem()
    nn = xyz.size // 3
    rp, ci = O.pattern(nn, conn, "solve")
    slot = O.slot_map(nn, conn, rp, ci)
    z = xyz[2::3]
    mask = np.zeros(xyz.size, np.uint8)
    val = np.zeros(xyz.size)
    mask[np.repeat(z < 1e-12, 3)] = 1
    mask[2::3][z > 1 - 1e-12] = 1
    val[2::3][z > 1 - 1e-12] = -0.05
    top = np.nonzero(z > 1 - 1e-12)[0]
    sel = np.sort(np.concatenate([3 * top, 3 * top + 1]))
    target = np.random.default_rng(9).standard_normal(sel.size) * 1e-3

    def loss(u):
        return 0.5 * np.sum((u[sel] - target) ** 2)

    u = _solve(xyz, conn, mu, lam, rp, ci, slot, mask, val, act)
    g = np.zeros_like(u)
    g[sel] = u[sel] - target
    Kt, _ = O.assemble(xyz, conn, mu, lam, 0.3, u, slot, ci.size, act)
    O.apply_bc(rp, ci, Kt, None, mask)
    w, sweeps = O.adjoint(xyz, conn, mu, lam, rp, ci, Kt, mask, u, g, tol=1e-12, active=act)
    assert sweeps >= 0
    gm, gl = O.param_grads(xyz, conn, u, w, active=act)
    grad = gm if which == "mu" else gl
    for e in np.nonzero(act)[0][::7][:5]:
        p = (mu if which == "mu" else lam).copy()
        h = 1e-6 * p[e]
        p[e] += h
        up = _solve(xyz, conn, p if which == "mu" else mu, p if which == "lam" else lam, rp, ci,
                    slot, mask, val, act)
        p[e] -= 2 * h
        um = _solve(xyz, conn, p if which == "mu" else mu, p if which == "lam" else lam, rp, ci,
                    slot, mask, val, act)
        fd = (loss(up) - loss(um)) / (2 * h)
        assert abs(grad[e] - fd) <= 1e-6 * abs(fd), (e, grad[e], fd)
