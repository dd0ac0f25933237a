"""Restart files in the reference's CheckpointFile layout
(FEM/adaptive_fem_engine.hpp:1347-1452): files written by the reference's
own CheckpointFile::save (oracle/_ref) load through fm_checkpoint_load, a
file rewritten by fm_checkpoint_save from what was loaded is byte-identical
to the reference's, and the reference's CheckpointFile::load reads files
written here."""
import os

import numpy as np
import pytest

import oracle as O


def ref_or_skip():
    R = O.ref()
    if R is None or not hasattr(R, "ref_checkpoint_save"):
        pytest.skip("oracle/_ref not built from the reference")
    return R


@pytest.fixture(scope="module")
def F():
    import flexmesh_b200 as F

    return F


@pytest.mark.parametrize("N", [1, 3])
def test_reference_file_round_trip(F, tmp_path, N):
    R = ref_or_skip()
    nn = (N + 1) ** 3
    ne = 6 * N ** 3
    rng = np.random.default_rng(N)
    u = rng.standard_normal(3 * nn)
    Fs = rng.standard_normal(9 * ne)
    S = rng.standard_normal(6 * ne)
    ref_path = str(tmp_path / "ref.ckpt")
    assert R.ref_checkpoint_save(os.fsencode(ref_path), N, u, Fs, S, 7, 2) == 0
    ck = F._lib.load_checkpoint(ref_path)
    assert (ck["load_step"], ck["adapt_iter"]) == (7, 2)
    xyz, conn = F.unit_cube(N)
    np.testing.assert_array_equal(ck["xyz"], xyz)
    np.testing.assert_array_equal(ck["conn"], conn)
    np.testing.assert_array_equal(ck["u"], u)
    np.testing.assert_array_equal(ck["node_disp"], u)
    np.testing.assert_array_equal(ck["F"], Fs)
    np.testing.assert_array_equal(ck["stress"], S)
    vol = O.volumes(xyz, conn)
    np.testing.assert_array_equal(ck["volume"], vol)
    np.testing.assert_array_equal(ck["jacobian_det"], vol * 6.0)
    ours = str(tmp_path / "ours.ckpt")
    F._lib.save_checkpoint(ours, ck["xyz"], ck["conn"], ck["u"], ck["load_step"],
                           ck["adapt_iter"], **{k: ck[k] for k in (
                               "node_disp", "volume", "jacobian_det", "quality", "F", "stress",
                               "eps_plastic", "kappa", "gamma_p")})
    assert open(ours, "rb").read() == open(ref_path, "rb").read()


def test_reference_loads_our_file(F, tmp_path):
    R = ref_or_skip()
    import ctypes as C

    N = 2
    xyz, conn = F.unit_cube(N)
    ne, nd = conn.size // 4, xyz.size
    rng = np.random.default_rng(5)
    u = rng.standard_normal(nd)
    Fs = rng.standard_normal(9 * ne)
    path = str(tmp_path / "ours.ckpt")
    F._lib.save_checkpoint(path, xyz, conn, u, 3, 1, F=Fs, node_disp=u)
    sz = [C.c_uint32() for _ in range(5)]
    uo, Fo, So = np.zeros(nd), np.zeros(9 * ne), np.ones(6 * ne)
    assert R.ref_checkpoint_load(os.fsencode(path), *[C.byref(x) for x in sz], uo, Fo, So,
                                 nd, ne) == 0
    assert [x.value for x in sz] == [xyz.size // 3, ne, nd, 3, 1]
    np.testing.assert_array_equal(uo, u)
    np.testing.assert_array_equal(Fo, Fs)
    np.testing.assert_array_equal(So, 0.0)  # stress defaulted to ElementState's zeros


def test_defaults_and_errors(F, tmp_path):
    xyz, conn = F.unit_cube(1)
    path = str(tmp_path / "d.ckpt")
    F._lib.save_checkpoint(path, xyz, conn, np.zeros(xyz.size))
    ck = F._lib.load_checkpoint(path)
    np.testing.assert_array_equal(ck["F"].reshape(-1, 9), np.tile(np.eye(3).ravel(), (6, 1)))
    assert os.path.getsize(path) == 20 + 8 * 48 + 6 * 40 + 6 * 184 + 8 * 24
    with pytest.raises(F.FMError):
        F._lib.load_checkpoint(str(tmp_path / "missing.ckpt"))
