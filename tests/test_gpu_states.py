"""Element state update on the GPU (fm_element_states, the device form of
update_element_states_rigorous) against the oracle's restatement, which is
pinned bit for bit to the reference's sl3_retraction and
neo_hookean_response (tests/test_oracle_states.py).

Tolerances: F_sl3 entries within 1e-12 absolute (they are O(1)); stresses
within 1e-12 of the largest shear modulus, absolute (the Mandel stress is a
difference of O(mu) terms: matrix log/exp chains of ~100 FP64 operations,
FMA-contracted on the GPU); the det-violation count exact.  The split's
sliver tets, whose reference Jacobian is nearly singular under the node
jitter (their F_sl3 can overflow in the reference as here), are left out of
the comparison."""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import flexmesh_b200 as F

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return F


def block(fm, N=6):
    from flexmesh_b200 import configs

    P = configs.scaleup_block(N)
    ctx = fm.Context(0)
    ctx.set_mesh(P.xyz, P.conn, P.elem_volume)
    ctx.set_material(P.E, P.nu, P.E_elem)
    ctx.set_bc(P.mask, P.bc_value)
    return ctx, P


def det_violations(F):
    """the det monitor applied to an [E, 9] array of F_sl3: per row,
    |det - 1| > 1e-8 (rows with a non-finite entry never count)"""
    fin = np.isfinite(F).all(1)
    bad = np.zeros(F.shape[0], bool)
    bad[fin] = np.abs(np.linalg.det(F[fin].reshape(-1, 3, 3)) - 1.0) > 1e-8
    return bad, fin


@pytest.mark.parametrize("amp", [1e-9, 0.005, 0.02])
def test_element_states_match_oracle(fm, amp):
    """random nodal displacements of amp (h = 1/6; at 0.02 the smallest
    volume ratio of a non-sliver tet is 0.03)"""
    ctx, P = block(fm)
    rng = np.random.default_rng(3)
    u = amp * rng.standard_normal(P.xyz.size)
    F, S, (v, nf) = ctx.element_states(torch.as_tensor(u, device="cuda"), counts=True)
    mu, lam = P.lame()
    Fo, So, vo = O.element_states(P.xyz, P.conn, mu, lam, u)
    F, S = F.cpu().numpy(), S.cpu().numpy()
    ok = P.elem_volume >= 1e-30  # not a sliver of the split
    assert np.abs(F[ok] - Fo[ok]).max() <= 1e-12
    assert np.abs(S[ok] - So[ok]).max() <= 1e-12 * mu.max()
    # the monitor's verdict per non-sliver tet is the oracle's; the kernel's
    # total is the monitor applied to its own output (slivers included)
    bad, fin = det_violations(F)
    bad_o, _ = det_violations(Fo)
    assert np.array_equal(bad[ok], bad_o[ok])
    assert int(bad.sum()) <= v <= int(bad.sum()) + int((~fin).sum())
    assert nf == int((~np.isfinite(np.concatenate([F, S], 1))).any(1).sum())


def test_grossly_distorted_states_are_counted_not_raised(fm):
    """displacements of 0.15 on h = 1/6 invert hundreds of tets (volume
    ratios down to -17): the matrix log of such an F is ill-conditioned and
    its digits depend on rounding, so there is no oracle comparison; the
    call succeeds and its two counts are those of its own output"""
    ctx, P = block(fm)
    rng = np.random.default_rng(3)
    u = 0.15 * rng.standard_normal(P.xyz.size)
    F, S, (v, nf) = ctx.element_states(torch.as_tensor(u, device="cuda"), counts=True)
    F, S = F.cpu().numpy(), S.cpu().numpy()
    bad, fin = det_violations(F)
    # for these F the determinant's last digits depend on how it is formed
    # (numpy's LU here, the kernel's cofactor expansion): a tet right at
    # |det - 1| = 1e-8 may count on one side only
    slack = max(2, int(0.03 * bad.sum()))
    assert int(bad.sum()) - slack <= v <= int(bad.sum()) + int((~fin).sum()) + slack
    assert v > 0
    assert nf == int((~np.isfinite(np.concatenate([F, S], 1))).any(1).sum())


def test_states_follow_newton_iterations(fm):
    """attached to a Newton load step, the states are those of the final u"""
    ctx, P = block(fm)
    ne = P.n_elems
    F = torch.eye(3, dtype=torch.float64, device="cuda").reshape(1, 9).repeat(ne, 1).contiguous()
    S = torch.zeros(ne, 6, dtype=torch.float64, device="cuda")
    ctx.set_state_output(F, S)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    r = ctx.newton_step_cfg(u, 1.0 / P.n_steps, inner_tol=1e-12)
    assert r["status"] == 0
    prof = ctx.profile_read()
    assert prof["states"]["calls"] == r["newton_iters"]  # one update per update of u
    ctx.set_state_output(None, None)
    F2, S2, _ = ctx.element_states(u)
    assert torch.equal(F, F2) and torch.equal(S, S2)
