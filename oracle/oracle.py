"""numpy/ctypes front end of the CPU checkers (TEST INFRASTRUCTURE).

Two libraries are wrapped:

* ``libfm_oracle.so`` -- the C restatement in ``fm_oracle.c`` (always built);
* ``_ref/libfm_ref.so`` -- the reference's own headers compiled by
  ``oracle/Makefile`` (optional: present where the reference checkout was
  available at build time, and it travels as a built file).

Only tests, the smoke check and the benchmark's CPU-baseline leg import this
module.  The product path never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORC_PATH = os.path.join(_HERE, "libfm_oracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libfm_ref.so")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def _opt(ptr_type):
    """ndpointer that also accepts None (NULL)."""

    class _Opt(ptr_type):
        @classmethod
        def from_param(cls, obj):
            if obj is None:
                return None
            return ptr_type.from_param(obj)

    return _Opt


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORC_PATH):
            raise RuntimeError(f"oracle library missing: run make -C {_HERE} oracle")
        L = C.CDLL(_ORC_PATH)
        u32, f64, i32 = C.c_uint32, C.c_double, C.c_int
        L.orc_unit_cube_sizes.argtypes = [i32, C.POINTER(u32), C.POINTER(u32)]
        L.orc_unit_cube.argtypes = [i32, _f64p, _u32p]
        L.orc_volumes.argtypes = [u32, _f64p, _u32p, _f64p]
        L.orc_node_to_elem.argtypes = [u32, u32, _u32p, _u32p, _u32p]
        L.orc_pattern_nnz.argtypes = [u32, u32, _u32p]
        L.orc_pattern_nnz.restype = C.c_uint64
        L.orc_pattern_reference.argtypes = [u32, u32, _u32p, _u32p, _u32p]
        L.orc_pattern_solve.argtypes = [u32, u32, _u32p, _u32p, _u32p]
        L.orc_slot_map.argtypes = [u32, u32, _u32p, _u32p, _u32p, _i32p]
        L.orc_lame.argtypes = [f64, f64, C.POINTER(f64), C.POINTER(f64)]
        L.orc_element.argtypes = [_f64p, _f64p, f64, f64, _f64p, _f64p]
        L.orc_element_lame.argtypes = [_f64p, _f64p, f64, f64, f64, _f64p, _f64p]
        L.orc_assemble.argtypes = [u32, u32, _f64p, _u32p, _opt(_u8p), _f64p, _f64p, f64,
                                   _f64p, _opt(_i32p), C.c_uint64, _opt(_f64p), _f64p]
        L.orc_apply_bc.argtypes = [u32, _u32p, _u32p, _f64p, _opt(_f64p), _u8p]
        L.orc_spmv.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p]
        L.orc_ilu0.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p]
        L.orc_ilu0.restype = i32
        L.orc_ilu0_apply.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p, _f64p, _f64p]
        L.orc_levels.argtypes = [u32, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p,
                                 C.POINTER(u32), C.POINTER(u32)]
        L.orc_pcg_ilu0.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p, f64, i32,
                                   C.POINTER(f64)]
        L.orc_pcg_ilu0.restype = i32
        L.orc_newton.argtypes = [u32, u32, _f64p, _u32p, _opt(_u8p), _f64p, _f64p, f64,
                                 _u32p, _u32p, _i32p, _u8p, _f64p, i32, f64, f64, i32, i32,
                                 _f64p, _opt(_i32p), _opt(_i32p)]
        L.orc_newton.restype = i32
        L.orc_newton_ex.argtypes = [u32, u32, _f64p, _u32p, _opt(_u8p), _f64p, _f64p, f64,
                                    _u32p, _u32p, _i32p, _u8p, _f64p, i32, i32, i32, f64, f64,
                                    f64, i32, i32, i32, f64, f64, i32, f64, _f64p,
                                    _opt(_i32p), _opt(_i32p), _opt(_f64p), i32,
                                    C.POINTER(i32)]
        L.orc_newton_ex.restype = i32
        L.orc_sl3_retraction.argtypes = [_f64p, _f64p]
        L.orc_nh_response.argtypes = [_f64p, f64, f64, f64, _f64p]
        L.orc_element_states.argtypes = [u32, u32, _f64p, _u32p, _f64p, _f64p, _f64p, _f64p,
                                         _f64p]
        L.orc_element_states.restype = u32
        L.orc_exact_apply.argtypes = [u32, u32, _f64p, _u32p, _opt(_u8p), _f64p, _f64p,
                                      _f64p, _f64p, _f64p, i32]
        L.orc_param_grads.argtypes = [u32, _f64p, _u32p, _opt(_u8p), _f64p, _f64p, _f64p, _f64p]
        L.orc_adjoint.argtypes = [u32, u32, _f64p, _u32p, _opt(_u8p), _f64p, _f64p, _u32p,
                                  _u32p, _f64p, _u8p, _f64p, _f64p, f64, f64, i32, i32, _f64p]
        L.orc_adjoint.restype = i32
        L.orc_poisson.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p]
        L.orc_poisson.restype = u32
        _lib = L
    return _lib


def have_reference() -> bool:
    return os.path.exists(_REF_PATH)


def ref():
    """The reference compiled from its own headers (None when not built)."""
    global _ref
    if _ref is None:
        if not have_reference():
            return None
        R = C.CDLL(_REF_PATH)
        u32, f64, i32, vp = C.c_uint32, C.c_double, C.c_int, C.c_void_p
        R.ref_mesh_new.argtypes = [i32]
        R.ref_mesh_new.restype = vp
        R.ref_mesh_free.argtypes = [vp]
        R.ref_mesh_sizes.argtypes = [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
        R.ref_mesh_get.argtypes = [vp, _f64p, _u32p, _f64p, _u32p, _u32p]
        R.ref_tet_volume.argtypes = [_f64p, _f64p, _f64p, _f64p]
        R.ref_tet_volume.restype = f64
        R.ref_pattern.argtypes = [u32, _f64p, u32, _u32p, _opt(_u32p), _opt(_u32p)]
        R.ref_pattern.restype = C.c_uint64
        R.ref_element.argtypes = [_f64p, _f64p, f64, f64, _f64p, _f64p]
        R.ref_assemble.argtypes = [u32, _f64p, u32, _u32p, _f64p, f64, f64, _f64p, _u32p, _u32p,
                                   _f64p, _f64p, i32]
        R.ref_residual.argtypes = [u32, _f64p, u32, _u32p, _f64p, f64, f64, _f64p, _f64p, i32]
        R.ref_assemble_slotmap.argtypes = [u32, _f64p, u32, _u32p, _f64p, _f64p, f64, _f64p,
                                           _i32p, C.c_uint64, _f64p, _f64p]
        R.ref_ilu0.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p, _f64p, _opt(_i32p)]
        R.ref_ilu0.restype = i32
        R.ref_ilu0_solve.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p]
        R.ref_pcg_ilu0.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p, f64, i32, i32]
        R.ref_pcg_ilu0.restype = i32
        R.ref_spmv.argtypes = [u32, _u32p, _u32p, _f64p, _f64p, _f64p]
        if hasattr(R, "ref_mesh_coloring"):
            R.ref_mesh_coloring.argtypes = [u32, _f64p, u32, _u32p, _f64p, _u32p]
            R.ref_mesh_coloring.restype = u32
        if hasattr(R, "ref_checkpoint_save"):
            R.ref_checkpoint_save.argtypes = [C.c_char_p, i32, _f64p, _opt(_f64p), _opt(_f64p),
                                              u32, u32]
            R.ref_checkpoint_save.restype = i32
            R.ref_checkpoint_load.argtypes = [C.c_char_p] + [C.POINTER(u32)] * 5 + [
                _opt(_f64p), _opt(_f64p), _opt(_f64p), u32, u32]
            R.ref_checkpoint_load.restype = i32
        if hasattr(R, "ref_sl3_retraction"):
            R.ref_sl3_retraction.argtypes = [_f64p, _f64p]
            R.ref_nh_response.argtypes = [_f64p, f64, f64, f64, _f64p]
        _ref = R
    return _ref


# ---------------------------------------------------------------------------
# oracle (C restatement) wrappers
# ---------------------------------------------------------------------------
def unit_cube(N: int):
    L = lib()
    nn, ne = C.c_uint32(), C.c_uint32()
    L.orc_unit_cube_sizes(N, C.byref(nn), C.byref(ne))
    xyz = np.zeros(3 * nn.value, np.float64)
    conn = np.zeros(4 * ne.value, np.uint32)
    L.orc_unit_cube(N, xyz, conn)
    return xyz, conn


def volumes(xyz, conn):
    v = np.zeros(conn.size // 4, np.float64)
    lib().orc_volumes(conn.size // 4, xyz, conn, v)
    return v


def node_to_elem(n_nodes, conn):
    ptr = np.zeros(n_nodes + 1, np.uint32)
    data = np.zeros(conn.size, np.uint32)
    lib().orc_node_to_elem(n_nodes, conn.size // 4, conn, ptr, data)
    return ptr, data


def pattern(n_nodes, conn, kind="solve"):
    L = lib()
    ne = conn.size // 4
    nnz = L.orc_pattern_nnz(n_nodes, ne, conn)
    rp = np.zeros(3 * n_nodes + 1, np.uint32)
    ci = np.zeros(nnz, np.uint32)
    if kind == "solve":
        L.orc_pattern_solve(n_nodes, ne, conn, rp, ci)
    elif kind == "reference":
        L.orc_pattern_reference(n_nodes, ne, conn, rp, ci)
    else:
        raise ValueError(kind)
    return rp, ci


def slot_map(n_nodes, conn, rp, ci):
    ne = conn.size // 4
    s = np.zeros(144 * ne, np.int32)
    lib().orc_slot_map(3 * n_nodes, ne, conn, rp, ci, s)
    return s


def lame(E, nu):
    mu, lam = C.c_double(), C.c_double()
    lib().orc_lame(E, nu, C.byref(mu), C.byref(lam))
    return mu.value, lam.value


def element(x12, u12, E, nu):
    K = np.zeros(144, np.float64)
    f = np.zeros(12, np.float64)
    lib().orc_element(np.ascontiguousarray(x12, np.float64), np.ascontiguousarray(u12, np.float64),
                      E, nu, K, f)
    return K, f


def element_lame(x12, u12, mu, lam, nu):
    K = np.zeros(144, np.float64)
    f = np.zeros(12, np.float64)
    lib().orc_element_lame(np.ascontiguousarray(x12, np.float64),
                           np.ascontiguousarray(u12, np.float64), mu, lam, nu, K, f)
    return K, f


def assemble(xyz, conn, mu_e, lam_e, nu, u, slot=None, nnz=0, active=None):
    nn = xyz.size // 3
    ne = conn.size // 4
    K = np.zeros(max(int(nnz), 1), np.float64) if slot is not None else None
    f = np.zeros(3 * nn, np.float64)
    lib().orc_assemble(nn, ne, xyz, conn, active, np.ascontiguousarray(mu_e, np.float64),
                       np.ascontiguousarray(lam_e, np.float64), nu, u, slot, int(nnz), K, f)
    return (K[:nnz] if K is not None else None), f


def apply_bc(rp, ci, K, R, mask):
    lib().orc_apply_bc(rp.size - 1, rp, ci, K, R, mask)


def spmv(rp, ci, val, x):
    y = np.zeros(rp.size - 1, np.float64)
    lib().orc_spmv(rp.size - 1, rp, ci, val, x, y)
    return y


def ilu0(rp, ci, val):
    n = rp.size - 1
    LU = np.zeros(ci.size, np.float64)
    d = np.zeros(n, np.float64)
    npert = lib().orc_ilu0(n, rp, ci, val, LU, d)
    return LU, d, npert


def ilu0_apply(rp, ci, LU, diag, r):
    n = rp.size - 1
    y = np.zeros(n, np.float64)
    w = np.zeros(n, np.float64)
    lib().orc_ilu0_apply(n, rp, ci, LU, diag, r, y, w)
    return y


def levels(rp, ci):
    n = rp.size - 1
    fp = np.zeros(n + 2, np.uint32)
    fr = np.zeros(max(n, 1), np.uint32)
    bp = np.zeros(n + 2, np.uint32)
    br = np.zeros(max(n, 1), np.uint32)
    nf, nb = C.c_uint32(), C.c_uint32()
    lib().orc_levels(n, rp, ci, fp, fr, bp, br, C.byref(nf), C.byref(nb))
    return fp[: nf.value + 1].copy(), fr[:n].copy(), bp[: nb.value + 1].copy(), br[:n].copy()


def pcg_ilu0(rp, ci, val, b, x0=None, tol=1e-10, max_iter=1000):
    n = rp.size - 1
    x = np.zeros(n, np.float64) if x0 is None else np.array(x0, np.float64)
    rr = C.c_double()
    it = lib().orc_pcg_ilu0(n, rp, ci, val, np.ascontiguousarray(b, np.float64), x, tol,
                            max_iter, C.byref(rr))
    return x, it, rr.value


def newton(xyz, conn, mu_e, lam_e, nu, rp, ci, slot, mask, bc_value, n_steps, rtol=1e-10,
           inner_tol=1e-12, max_newton=200, max_pcg=5000, u0=None, active=None):
    nn = xyz.size // 3
    ne = conn.size // 4
    u = np.zeros(3 * nn, np.float64) if u0 is None else np.array(u0, np.float64)
    nps = np.zeros(n_steps, np.int32)
    pps = np.zeros(n_steps, np.int32)
    st = lib().orc_newton(nn, ne, xyz, conn, active, np.ascontiguousarray(mu_e, np.float64),
                          np.ascontiguousarray(lam_e, np.float64), nu, rp, ci, slot, mask,
                          np.ascontiguousarray(bc_value, np.float64), n_steps, rtol, inner_tol,
                          max_newton, max_pcg, u, nps, pps)
    return u, st, nps, pps


def newton_ex(xyz, conn, mu_e, lam_e, nu, rp, ci, slot, mask, bc_value, n_steps, first_step=1,
              last_step=None, rtol=1e-10, inner_tol=1e-12, predictor_tol=0.0, max_newton=200,
              max_pcg=5000, line_search=0, ls_c=1e-4, diverge_rate=0.0, diverge_count=3,
              diverge_growth=0.0, u0=None, active=None, alpha_cap=100000):
    """orc_newton_ex: load steps first_step..last_step with the GPU path's
    Newton options; returns (u, status, newton per step, pcg per step,
    alpha of every Newton iteration)"""
    nn = xyz.size // 3
    ne = conn.size // 4
    last_step = n_steps if last_step is None else last_step
    k = last_step - first_step + 1
    u = np.zeros(3 * nn, np.float64) if u0 is None else np.array(u0, np.float64)
    nps = np.zeros(k, np.int32)
    pps = np.zeros(k, np.int32)
    al = np.zeros(alpha_cap, np.float64)
    na = C.c_int()
    st = lib().orc_newton_ex(nn, ne, xyz, conn, active, np.ascontiguousarray(mu_e, np.float64),
                             np.ascontiguousarray(lam_e, np.float64), nu, rp, ci, slot, mask,
                             np.ascontiguousarray(bc_value, np.float64), first_step, last_step,
                             n_steps, rtol, inner_tol, predictor_tol, max_newton, max_pcg,
                             line_search, ls_c, diverge_rate, diverge_count, diverge_growth, u,
                             nps, pps, al, alpha_cap, C.byref(na))
    return u, st, nps, pps, al[:min(na.value, alpha_cap)]


def sl3_retraction(G):
    out = np.zeros(9)
    lib().orc_sl3_retraction(np.ascontiguousarray(G, np.float64), out)
    return out


def nh_response(F, mu, lam, J):
    sig = np.zeros(6)
    lib().orc_nh_response(np.ascontiguousarray(F, np.float64), mu, lam, J, sig)
    return sig


def element_states(xyz, conn, mu_e, lam_e, u, F0=None, stress0=None):
    """orc_element_states: (F_sl3 [E, 9], stress [E, 6], det violations);
    untouched tets keep F0/stress0 (default identity / zero)"""
    ne = conn.size // 4
    F = (np.tile(np.eye(3).reshape(9), ne) if F0 is None else np.array(F0, np.float64)).ravel()
    S = np.zeros(6 * ne) if stress0 is None else np.array(stress0, np.float64).ravel()
    v = lib().orc_element_states(xyz.size // 3, ne, xyz, conn,
                                 np.ascontiguousarray(mu_e, np.float64),
                                 np.ascontiguousarray(lam_e, np.float64), u, F, S)
    return F.reshape(ne, 9), S.reshape(ne, 6), int(v)


def exact_apply(xyz, conn, mu_e, lam_e, u, v, transpose=False, active=None):
    nn = xyz.size // 3
    y = np.zeros(3 * nn, np.float64)
    lib().orc_exact_apply(nn, conn.size // 4, xyz, conn, active,
                          np.ascontiguousarray(mu_e, np.float64),
                          np.ascontiguousarray(lam_e, np.float64), u,
                          np.ascontiguousarray(v, np.float64), y, int(transpose))
    return y


def param_grads(xyz, conn, u, w, active=None):
    ne = conn.size // 4
    gm = np.zeros(ne, np.float64)
    gl = np.zeros(ne, np.float64)
    lib().orc_param_grads(ne, xyz, conn, active, u, np.ascontiguousarray(w, np.float64), gm, gl)
    return gm, gl


def adjoint(xyz, conn, mu_e, lam_e, rp, ci, Kt, mask, u, g, tol=1e-10, inner_tol=1e-12,
            max_sweeps=500, max_pcg=5000, active=None):
    nn = xyz.size // 3
    w = np.zeros(3 * nn, np.float64)
    sweeps = lib().orc_adjoint(nn, conn.size // 4, xyz, conn, active,
                               np.ascontiguousarray(mu_e, np.float64),
                               np.ascontiguousarray(lam_e, np.float64), rp, ci, Kt, mask, u,
                               np.ascontiguousarray(g, np.float64), tol, inner_tol, max_sweeps,
                               max_pcg, w)
    return w, sweeps


def poisson(g):
    n = g * g
    rp = np.zeros(n + 1, np.uint32)
    ci = np.zeros(5 * n, np.uint32)
    val = np.zeros(5 * n, np.float64)
    b = np.zeros(n, np.float64)
    xe = np.zeros(n, np.float64)
    nnz = lib().orc_poisson(g, rp, ci, val, b, xe)
    return rp, ci[:nnz].copy(), val[:nnz].copy(), b, xe
