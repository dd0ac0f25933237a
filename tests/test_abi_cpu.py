"""CPU checks of the C ABI: the library loads, exports every function that
include/fm_api.h declares, and its host-only entry points agree with the
oracle.  No GPU calls."""
import os
import re

import numpy as np
import pytest

import oracle as O
from flexmesh_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^(?:fm_status|void)\s+(fm_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    decl = declared_functions()
    assert len(decl) >= 25
    missing = [n for n in sorted(decl) if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) == decl


@pytest.mark.parametrize("N", [1, 2, 5, 8])
def test_unit_cube_matches_oracle(N):
    xyz, conn = _lib.unit_cube(N)
    x2, c2 = O.unit_cube(N)
    assert np.array_equal(xyz, x2) and np.array_equal(conn, c2)


def test_unit_cube_rejects_bad_sizes():
    L = _lib.lib()
    import ctypes as C

    a, b = C.c_uint32(), C.c_uint32()
    assert L.fm_unit_cube_sizes(0, C.byref(a), C.byref(b)) == 1
    assert L.fm_unit_cube_sizes(-3, C.byref(a), C.byref(b)) == 1


def test_synthetic_configs_are_deterministic():
    from flexmesh_b200 import configs

    a = configs.scaleup_block(N=6)
    b = configs.scaleup_block(N=6)
    assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.E_elem, b.E_elem)
    # boundary nodes are not jittered; interior ones are, within 0.15 h
    x0, _ = _lib.unit_cube(6)
    d = np.abs(a.xyz - x0).reshape(-1, 3).max(axis=1)
    s = 7
    idx = np.arange(d.size)
    i, j, k = idx % s, (idx // s) % s, idx // (s * s)
    interior = (i > 0) & (i < 6) & (j > 0) & (j < 6) & (k > 0) & (k < 6)
    assert np.all(d[~interior] == 0) and np.all(d[interior] > 0)
    assert d.max() <= 0.15 / 6
    mask, val = configs.clamp_top_bc(a.xyz, -0.2)
    z = a.xyz[2::3]
    assert mask.reshape(-1, 3)[z == 0].all() and np.all(val[2::3][z == 1.0] == -0.2)
