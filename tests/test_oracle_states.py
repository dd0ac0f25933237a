"""The oracle's element state update (sl3_retraction and the Neo-Hookean
response of update_element_states_rigorous) against the reference's own
functions compiled from its headers (oracle/_ref): bitwise on random
deformation gradients from near-identity (the series fast path) to large
strains (several Denman-Beavers square roots and Newton clean-ups)."""
import numpy as np
import pytest

import oracle as O


def ref_or_skip():
    R = O.ref()
    if R is None or not hasattr(R, "ref_sl3_retraction"):
        pytest.skip("oracle/_ref not built from the reference")
    return R


@pytest.mark.parametrize("scale", [1e-9, 1e-4, 0.05, 0.3, 0.8])
def test_sl3_retraction_bitwise_vs_reference(scale):
    R = ref_or_skip()
    rng = np.random.default_rng(int(scale * 1e9) % 1000)
    for _ in range(300):
        G = np.eye(3).reshape(9) + scale * rng.standard_normal(9)
        if np.linalg.det(G.reshape(3, 3)) <= 0.05:
            continue
        a = O.sl3_retraction(G)
        b = np.zeros(9)
        R.ref_sl3_retraction(G, b)
        np.testing.assert_array_equal(a, b)
        assert abs(np.linalg.det(a.reshape(3, 3)) - 1.0) < 1e-12


def test_nh_response_bitwise_vs_reference():
    R = ref_or_skip()
    rng = np.random.default_rng(7)
    E, nu = 1.3, 0.3
    mu, lam = O.lame(E, nu)
    for _ in range(200):
        F = np.eye(3).reshape(9) + 0.2 * rng.standard_normal(9)
        J = np.linalg.det(F.reshape(3, 3))
        a = O.nh_response(F, mu, lam, J)
        b = np.zeros(6)
        R.ref_nh_response(F, E, nu, J, b)
        np.testing.assert_array_equal(a, b)


def test_element_states_properties():
    """det F_sl3 = 1, u = 0 gives the identity and zero stress, and tets whose
    reference Jacobian is degenerate (the split's slivers) keep their state"""
    xyz, conn = O.unit_cube(3)
    ne = conn.size // 4
    mu, lam = np.full(ne, 0.4), np.full(ne, 0.6)
    u = np.zeros(xyz.size)
    F, S, v = O.element_states(xyz, conn, mu, lam, u)
    assert v == 0
    np.testing.assert_allclose(F, np.tile(np.eye(3).reshape(9), (ne, 1)), atol=1e-15)
    assert np.abs(S).max() < 1e-14
    u = 0.05 * np.sin(7 * xyz)
    F0 = np.full((ne, 9), 7.0)
    F, S, v = O.element_states(xyz, conn, mu, lam, u, F0=F0)
    vol = O.volumes(xyz, conn)
    sliver = vol < 1e-30
    assert sliver.any()
    assert (F[sliver] == 7.0).all()
    d = np.linalg.det(F[~sliver].reshape(-1, 3, 3))
    assert np.abs(d - 1).max() < 1e-12 and v == 0
