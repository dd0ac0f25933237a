"""Element colouring (fm_mesh_coloring, host) against the reference's own
MeshColoring::compute (FEM/adaptive_fem_engine.hpp:1549-1602, built in
oracle/_ref): the same colour of every tet, on the unit cube and on a
relabelled mesh; and a proper colouring (no two tets sharing a node alike)."""
import numpy as np
import pytest

import oracle as O


@pytest.fixture(scope="module")
def F():
    import flexmesh_b200 as F

    return F


def check_proper(conn, colors):
    c = conn.reshape(-1, 4)
    for n in np.unique(c):
        tets = np.nonzero((c == n).any(1))[0]
        assert np.unique(colors[tets]).size == tets.size


@pytest.mark.parametrize("N,perm_seed", [(2, None), (4, None), (3, 5)])
def test_coloring_matches_reference(F, N, perm_seed):
    xyz, conn = O.unit_cube(N)
    nn = xyz.size // 3
    if perm_seed is not None:  # relabel nodes and shuffle the tets
        rng = np.random.default_rng(perm_seed)
        p = rng.permutation(nn)
        conn = p[conn].astype(np.uint32)
        xyz = xyz.reshape(-1, 3)[np.argsort(p)].reshape(-1).copy()
        conn = conn.reshape(-1, 4)[rng.permutation(conn.size // 4)].reshape(-1).copy()
    colors, nc = F._lib.mesh_coloring(nn, conn)
    check_proper(conn, colors)
    assert nc == colors.max() + 1
    R = O.ref()
    if R is None or not hasattr(R, "ref_mesh_coloring"):
        pytest.skip("oracle/_ref not built from the reference")
    rc = np.zeros(conn.size // 4, np.uint32)
    rn = R.ref_mesh_coloring(nn, xyz, conn.size // 4, conn, O.volumes(xyz, conn), rc)
    np.testing.assert_array_equal(colors, rc)
    assert nc == rn
