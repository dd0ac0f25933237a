"""ctypes binding of libflexmesh_b200.so (the C ABI in include/fm_api.h).

Device arrays are torch CUDA tensors passed by data_ptr(); host arrays are
numpy.  There is no CPU fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libflexmesh_b200.so")

FM_FP64, FM_MIXED = 0, 1
FM_PATTERN_REFERENCE, FM_PATTERN_SOLVE = 0, 1
STATUS = {0: "FM_OK", 1: "FM_ERR_ARG", 2: "FM_ERR_CUDA", 3: "FM_ERR_OOM", 4: "FM_ERR_NONFINITE",
          5: "FM_ERR_ZERO_PIVOT", 6: "FM_ERR_INVERTED", 7: "FM_ERR_TIMEOUT",
          8: "FM_ERR_NOT_CONVERGED", 9: "FM_ERR_LIMITS", 10: "FM_ERR_DIVERGED"}
FM_ERR_NOT_CONVERGED, FM_ERR_DIVERGED = 8, 10
FLAG_NONFINITE, FLAG_INVERTED, FLAG_J_CLAMPED, FLAG_PIVOT, FLAG_TIMEOUT, FLAG_BREAKDOWN = (
    1, 2, 4, 8, 16, 32)

# every symbol include/fm_api.h declares (checked by the CPU tests)
EXPORTS = [
    "fm_create", "fm_destroy", "fm_last_error", "fm_get_flags", "fm_clear_flags", "fm_sizes",
    "fm_unit_cube_sizes", "fm_unit_cube", "fm_set_mesh", "fm_build_pattern", "fm_set_material",
    "fm_set_material_lame", "fm_set_bc", "fm_elements", "fm_assemble", "fm_assemble_host",
    "fm_residual", "fm_assemble_reference_pattern", "fm_levels", "fm_ilu0", "fm_get_ilu0",
    "fm_ilu0_apply", "fm_ilu0_apply_noalloc", "fm_spmv", "fm_pcg", "fm_csr_pcg_ilu0", "fm_newton_solve",
    "fm_exact_apply", "fm_adjoint", "fm_csr_ilu0", "fm_newton_step", "fm_newton_step_host",
    "fm_profile_enable", "fm_profile_read", "fm_newton_config_default", "fm_newton_step_cfg",
    "fm_newton_history", "fm_set_wait_limit", "fm_check_wait", "fm_newton_step_cfg_host",
    "fm_newton_solve_cfg", "fm_element_states", "fm_set_state_output", "fm_checkpoint_save",
    "fm_checkpoint_header", "fm_checkpoint_load", "fm_mesh_coloring",
]
PROF_KINDS = {0: "assemble", 1: "ilu0", 2: "trsv", 3: "spmv", 4: "vector", 5: "states"}


class Profile(C.Structure):
    _fields_ = [("ms", C.c_double * 8), ("calls", C.c_uint64 * 8), ("kernels", C.c_uint64 * 8)]


class NewtonConfig(C.Structure):
    """fm_newton_config (include/fm_api.h)"""
    _fields_ = [("newton_rtol", C.c_double), ("newton_atol", C.c_double),
                ("inner_tol", C.c_double), ("predictor_tol", C.c_double),
                ("inner_tol_min", C.c_double), ("max_newton", C.c_int), ("max_pcg", C.c_int),
                ("line_search", C.c_int), ("ls_c", C.c_double), ("diverge_rate", C.c_double),
                ("diverge_count", C.c_int), ("diverge_growth", C.c_double),
                ("precision", C.c_int), ("ilu_every", C.c_int), ("initial_guess", C.c_int)]


class NewtonResult(C.Structure):
    _fields_ = [("newton_iters", C.c_int), ("pcg_iters", C.c_int), ("backtracks", C.c_int),
                ("flags", C.c_uint32), ("rnorm0", C.c_double), ("rnorm", C.c_double),
                ("final_relres", C.c_double)]


class NewtonRecord(C.Structure):
    _fields_ = [("kind", C.c_int), ("pcg_iters", C.c_int), ("rnorm", C.c_double),
                ("alpha", C.c_double), ("inner_tol", C.c_double), ("flags", C.c_uint32),
                ("pad", C.c_uint32)]


class Checkpoint(C.Structure):
    """fm_checkpoint (include/fm_api.h): the reference's CheckpointFile layout"""
    _fields_ = [("load_step", C.c_uint32), ("adapt_iter", C.c_uint32), ("n_nodes", C.c_uint32),
                ("n_elems", C.c_uint32), ("n_dofs", C.c_uint32)] + [
        (name, C.c_void_p) for name in ("xyz", "node_disp", "conn", "volume", "jacobian_det",
                                         "quality", "F", "stress", "eps_plastic", "kappa",
                                         "gamma_p", "u")]


# checkpoint arrays: (name, dtype, entries per node / element / DOF)
_CK_ARRAYS = [("xyz", np.float64, "n", 3), ("node_disp", np.float64, "n", 3),
              ("conn", np.uint32, "e", 4), ("volume", np.float64, "e", 1),
              ("jacobian_det", np.float64, "e", 1), ("quality", np.float64, "e", 1),
              ("F", np.float64, "e", 9), ("stress", np.float64, "e", 6),
              ("eps_plastic", np.float64, "e", 6), ("kappa", np.float64, "e", 1),
              ("gamma_p", np.float64, "e", 1), ("u", np.float64, "d", 1)]


def mesh_coloring(n_nodes, conn):
    """fm_mesh_coloring: (colors per tet, colour count) of MeshColoring::compute"""
    conn = np.ascontiguousarray(conn, np.uint32)
    colors = np.zeros(conn.size // 4, np.uint32)
    nc = _u32()
    st = lib().fm_mesh_coloring(n_nodes, conn.size // 4, _hp(conn), _hp(colors), C.byref(nc))
    if st:
        raise FMError(st, "fm_mesh_coloring")
    return colors, nc.value


def save_checkpoint(path, xyz, conn, u, load_step=0, adapt_iter=0, **arrays):
    """fm_checkpoint_save: a restart file in the reference's CheckpointFile
    layout; arrays: node_disp, volume, jacobian_det, quality, F, stress,
    eps_plastic, kappa, gamma_p (host arrays; missing ones take the
    ElementState defaults / zeros)"""
    ck = Checkpoint()
    keep = {"xyz": np.ascontiguousarray(xyz, np.float64),
            "conn": np.ascontiguousarray(conn, np.uint32),
            "u": np.ascontiguousarray(u, np.float64)}
    for name, dt, _, _ in _CK_ARRAYS:
        if name in arrays and arrays[name] is not None:
            keep[name] = np.ascontiguousarray(arrays[name], dt)
    ck.load_step, ck.adapt_iter = load_step, adapt_iter
    ck.n_nodes, ck.n_elems, ck.n_dofs = keep["xyz"].size // 3, keep["conn"].size // 4, keep["u"].size
    for name, a in keep.items():
        setattr(ck, name, a.ctypes.data)
    st = lib().fm_checkpoint_save(os.fsencode(path), C.byref(ck))
    if st:
        raise FMError(st, f"fm_checkpoint_save: cannot write {path}")


def load_checkpoint(path):
    """fm_checkpoint_load: every array of a CheckpointFile-layout file"""
    ck = Checkpoint()
    st = lib().fm_checkpoint_header(os.fsencode(path), C.byref(ck))
    if st:
        raise FMError(st, f"fm_checkpoint_header: cannot read {path}")
    sizes = {"n": ck.n_nodes, "e": ck.n_elems, "d": ck.n_dofs}
    out = {}
    for name, dt, kind, k in _CK_ARRAYS:
        out[name] = np.zeros(sizes[kind] * k, dt)
        setattr(ck, name, out[name].ctypes.data)
    st = lib().fm_checkpoint_load(os.fsencode(path), C.byref(ck))
    if st:
        raise FMError(st, f"fm_checkpoint_load: cannot read {path}")
    out["load_step"], out["adapt_iter"] = ck.load_step, ck.adapt_iter
    return out


class FMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None
_vp, _u32, _i32, _f64, _u64 = C.c_void_p, C.c_uint32, C.c_int, C.c_double, C.c_uint64
_P = C.POINTER


def lib() -> C.CDLL:
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run python atlas-flexmesh_b200/build.py")
        L = C.CDLL(LIB_PATH)
        sig = {
            "fm_create": [_P(_vp), _i32, _vp],
            "fm_destroy": [_vp],
            "fm_last_error": [_vp, C.c_char_p, C.c_size_t],
            "fm_get_flags": [_vp, _P(_u32)],
            "fm_clear_flags": [_vp],
            "fm_sizes": [_vp, _P(_u32), _P(_u32), _P(_u32), _P(_u64)],
            "fm_unit_cube_sizes": [_i32, _P(_u32), _P(_u32)],
            "fm_unit_cube": [_i32, _vp, _vp],
            "fm_set_mesh": [_vp, _u32, _vp, _u32, _vp, _vp],
            "fm_build_pattern": [_vp, _i32, _vp, _vp, _vp],
            "fm_set_material": [_vp, _f64, _f64, _vp],
            "fm_set_material_lame": [_vp, _vp, _vp, _f64],
            "fm_set_bc": [_vp, _vp, _vp],
            "fm_elements": [_vp, _u32, _vp, _vp, _vp, _f64, _vp, _vp],
            "fm_assemble": [_vp, _vp, _vp, _vp, _i32, _i32],
            "fm_assemble_host": [_vp, _vp, _vp, _vp],
            "fm_residual": [_vp, _vp, _vp],
            "fm_assemble_reference_pattern": [_vp, _vp, _vp, _vp],
            "fm_levels": [_vp, _vp, _vp, _vp, _vp, _P(_u32), _P(_u32)],
            "fm_ilu0": [_vp, _i32],
            "fm_get_ilu0": [_vp, _vp, _vp],
            "fm_ilu0_apply": [_vp, _vp, _vp],
            "fm_ilu0_apply_noalloc": [_vp, _vp, _vp],
            "fm_spmv": [_vp, _vp, _vp],
            "fm_pcg": [_vp, _vp, _vp, _f64, _i32, _P(_i32), _P(_f64), _i32],
            "fm_csr_pcg_ilu0": [_vp, _u32, _vp, _vp, _vp, _vp, _vp, _f64, _i32, _P(_i32),
                                _P(_f64)],
            "fm_newton_solve": [_vp, _vp, _i32, _i32, _f64, _f64, _f64, _i32, _i32, _i32,
                                _P(_i32), _P(_i32), _P(_f64)],
            "fm_csr_ilu0": [_vp, _u32, _vp, _vp, _vp, _vp, _vp],
            "fm_newton_step": [_vp, _vp, _f64, _f64, _f64, _f64, _i32, _i32, _i32, _f64, _i32,
                               _P(_i32), _P(_i32), _P(_f64)],
            "fm_newton_step_host": [_vp, _vp, _f64, _f64, _f64, _f64, _i32, _i32, _i32, _f64,
                                    _i32, _P(_i32), _P(_i32), _P(_f64)],
            "fm_newton_config_default": [_P(NewtonConfig)],
            "fm_newton_step_cfg": [_vp, _vp, _f64, _P(NewtonConfig), _P(NewtonResult)],
            "fm_newton_history": [_vp, _P(NewtonRecord), _i32, _P(_i32)],
            "fm_newton_step_cfg_host": [_vp, _vp, _f64, _P(NewtonConfig), _P(NewtonResult)],
            "fm_newton_solve_cfg": [_vp, _vp, _i32, _i32, _P(NewtonConfig), _P(NewtonResult)],
            "fm_element_states": [_vp, _vp, _vp, _vp, _P(_u32), _P(_u32)],
            "fm_set_state_output": [_vp, _vp, _vp],
            "fm_checkpoint_save": [C.c_char_p, _P(Checkpoint)],
            "fm_checkpoint_header": [C.c_char_p, _P(Checkpoint)],
            "fm_checkpoint_load": [C.c_char_p, _P(Checkpoint)],
            "fm_mesh_coloring": [_u32, _u32, _vp, _vp, _P(_u32)],
            "fm_set_wait_limit": [_vp, _u64],
            "fm_check_wait": [_vp],
            "fm_profile_enable": [_vp, _i32],
            "fm_profile_read": [_vp, _P(Profile)],
            "fm_exact_apply": [_vp, _vp, _vp, _vp, _i32],
            "fm_adjoint": [_vp, _vp, _vp, _vp, _vp, _vp, _f64, _f64, _i32, _i32, _P(_i32),
                           _P(_i32)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = None if name == "fm_destroy" else _i32
        _lib = L
    return _lib


def _hp(a):
    """host pointer of a numpy array (or None)"""
    return None if a is None else a.ctypes.data_as(_vp)


def _dp(t):
    """device pointer of a torch CUDA tensor (or None)"""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return _vp(t.data_ptr())


def unit_cube(N: int):
    L = lib()
    nn, ne = _u32(), _u32()
    st = L.fm_unit_cube_sizes(N, C.byref(nn), C.byref(ne))
    if st:
        raise FMError(st, "fm_unit_cube_sizes")
    xyz = np.zeros(3 * nn.value, np.float64)
    conn = np.zeros(4 * ne.value, np.uint32)
    st = L.fm_unit_cube(N, _hp(xyz), _hp(conn))
    if st:
        raise FMError(st, "fm_unit_cube")
    return xyz, conn


class Context:
    """One fm_ctx: mesh, pattern, material, BCs and solver state on one GPU."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        self.torch = torch
        self.device = device
        self._h = _vp()
        # default: torch's current stream, so library work is ordered with the
        # torch copies/kernels that produce inputs and read results
        if stream is None:
            stream = torch.cuda.current_stream(device)
        h = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        # handle 0 is the legacy default stream; NULL would ask the library
        # for a private stream, so pass cudaStreamLegacy (0x1) instead
        s = _vp(h if h else 1)
        self.stream = stream
        self._check(lib().fm_create(C.byref(self._h), device, s), "fm_create")
        self.n_nodes = self.n_elems = self.n_dofs = self.nnz = 0

    # ------------------------------------------------------------------
    def _check(self, st, what):
        if st:
            buf = C.create_string_buffer(512)
            if self._h:
                lib().fm_last_error(self._h, buf, 512)
            raise FMError(st, f"{what}: {buf.value.decode(errors='replace')}")

    def close(self):
        if self._h:
            lib().fm_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def flags(self) -> int:
        f = _u32()
        self._check(lib().fm_get_flags(self._h, C.byref(f)), "fm_get_flags")
        return f.value

    def clear_flags(self):
        self._check(lib().fm_clear_flags(self._h), "fm_clear_flags")

    def set_wait_limit(self, cycles: int = 0):
        """bounded-wait limit of this context's kernels (SM cycles; 0: default)"""
        self._check(lib().fm_set_wait_limit(self._h, int(cycles)), "fm_set_wait_limit")

    def check_wait(self):
        """fm_check_wait: returns its status (FM_ERR_TIMEOUT = 7 expected)"""
        return lib().fm_check_wait(self._h)

    # ------------------------------------------------------------------
    def set_mesh(self, xyz, conn, elem_volume=None):
        xyz = np.ascontiguousarray(xyz, np.float64)
        conn = np.ascontiguousarray(conn, np.uint32)
        vol = None if elem_volume is None else np.ascontiguousarray(elem_volume, np.float64)
        self._check(lib().fm_set_mesh(self._h, xyz.size // 3, _hp(xyz), conn.size // 4,
                                      _hp(conn), _hp(vol)), "fm_set_mesh")
        nn, ne, nd, nz = _u32(), _u32(), _u32(), _u64()
        lib().fm_sizes(self._h, C.byref(nn), C.byref(ne), C.byref(nd), C.byref(nz))
        self.n_nodes, self.n_elems, self.n_dofs, self.nnz = nn.value, ne.value, nd.value, nz.value

    def build_pattern(self, kind=FM_PATTERN_SOLVE, slot_map=False):
        rp = np.zeros(self.n_dofs + 1, np.uint32)
        ci = np.zeros(self.nnz, np.uint32)
        sm = np.zeros(144 * self.n_elems, np.int32) if slot_map else None
        self._check(lib().fm_build_pattern(self._h, kind, _hp(rp), _hp(ci), _hp(sm)),
                    "fm_build_pattern")
        return rp, ci, sm

    def set_material(self, E, nu, E_elem=None):
        Ee = None if E_elem is None else np.ascontiguousarray(E_elem, np.float64)
        self._check(lib().fm_set_material(self._h, E, nu, _hp(Ee)), "fm_set_material")

    def set_material_lame(self, mu_e, lam_e, nu):
        mu = np.ascontiguousarray(mu_e, np.float64)
        lam = np.ascontiguousarray(lam_e, np.float64)
        self._check(lib().fm_set_material_lame(self._h, _hp(mu), _hp(lam), nu),
                    "fm_set_material_lame")

    def set_bc(self, mask, value=None):
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        v = None if value is None else np.ascontiguousarray(value, np.float64)
        self._check(lib().fm_set_bc(self._h, _hp(m), _hp(v)), "fm_set_bc")

    # ------------------------------------------------------------------ device calls
    def _zeros(self, n, dtype=None):
        t = self.torch
        return t.zeros(n, dtype=dtype or t.float64, device=f"cuda:{self.device}")

    def elements(self, x, u, E, nu):
        n = x.shape[0]
        K = self._zeros(144 * n)
        f = self._zeros(12 * n)
        self._check(lib().fm_elements(self._h, n, _dp(x), _dp(u), _dp(E), nu, _dp(K), _dp(f)),
                    "fm_elements")
        return K.view(n, 144), f.view(n, 12)

    def assemble(self, u, prec=FM_FP64, apply_bc=False, K=None, f=None):
        t = self.torch
        if K is None:
            K = self._zeros(self.nnz, t.float64 if prec == FM_FP64 else t.float32)
        if f is None:
            f = self._zeros(self.n_dofs)
        self._check(lib().fm_assemble(self._h, _dp(u), _dp(K), _dp(f), prec, int(apply_bc)),
                    "fm_assemble")
        return K, f

    def assemble_into_context(self, u, prec=FM_FP64, apply_bc=True, f=None):
        self._check(lib().fm_assemble(self._h, _dp(u), None, _dp(f), prec, int(apply_bc)),
                    "fm_assemble")

    def assemble_host(self, u_host):
        K = np.zeros(self.nnz, np.float64)
        f = np.zeros(self.n_dofs, np.float64)
        u = np.ascontiguousarray(u_host, np.float64)
        self._check(lib().fm_assemble_host(self._h, _hp(u), _hp(K), _hp(f)), "fm_assemble_host")
        return K, f

    def residual(self, u, f=None):
        if f is None:
            f = self._zeros(self.n_dofs)
        self._check(lib().fm_residual(self._h, _dp(u), _dp(f)), "fm_residual")
        return f

    def assemble_reference_pattern(self, u):
        K = self._zeros(self.nnz)
        f = self._zeros(self.n_dofs)
        self._check(lib().fm_assemble_reference_pattern(self._h, _dp(u), _dp(K), _dp(f)),
                    "fm_assemble_reference_pattern")
        return K, f

    def levels(self):
        n = self.n_dofs
        fp = np.zeros(n + 1, np.uint32)
        fr = np.zeros(n, np.uint32)
        bp = np.zeros(n + 1, np.uint32)
        br = np.zeros(n, np.uint32)
        nf, nb = _u32(), _u32()
        self._check(lib().fm_levels(self._h, _hp(fp), _hp(fr), _hp(bp), _hp(br), C.byref(nf),
                                    C.byref(nb)), "fm_levels")
        return fp[: nf.value + 1], fr, bp[: nb.value + 1], br

    def ilu0(self, prec=FM_FP64):
        self._check(lib().fm_ilu0(self._h, prec), "fm_ilu0")

    def get_ilu0(self):
        LU = np.zeros(self.nnz, np.float64)
        d = np.zeros(self.n_dofs, np.float64)
        self._check(lib().fm_get_ilu0(self._h, _hp(LU), _hp(d)), "fm_get_ilu0")
        return LU, d

    def ilu0_apply(self, r):
        y = self._zeros(self.n_dofs)
        self._check(lib().fm_ilu0_apply(self._h, _dp(r), _dp(y)), "fm_ilu0_apply")
        return y

    def ilu0_apply_noalloc(self, r, y):
        """fm_ilu0_apply into the caller's y without any allocation in the call
        (library-owned static scratch, at most 2**20 DOFs, one call at a time
        per device)."""
        self._check(lib().fm_ilu0_apply_noalloc(self._h, _dp(r), _dp(y)),
                    "fm_ilu0_apply_noalloc")
        return y

    def spmv(self, x):
        y = self._zeros(self.n_dofs)
        self._check(lib().fm_spmv(self._h, _dp(x), _dp(y)), "fm_spmv")
        return y

    def pcg(self, b, x=None, tol=1e-10, max_iter=1000, prec=FM_FP64):
        if x is None:
            x = self._zeros(self.n_dofs)
        it, rr = _i32(), _f64()
        self._check(lib().fm_pcg(self._h, _dp(b), _dp(x), tol, max_iter, C.byref(it),
                                 C.byref(rr), prec), "fm_pcg")
        return x, it.value, rr.value

    def csr_pcg_ilu0(self, row_ptr, col_idx, val, b, x0=None, tol=1e-10, max_iter=1000):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        v = np.ascontiguousarray(val, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        n = rp.size - 1
        x = np.zeros(n, np.float64) if x0 is None else np.array(x0, np.float64)
        it, rr = _i32(), _f64()
        self._check(lib().fm_csr_pcg_ilu0(self._h, n, _hp(rp), _hp(ci), _hp(v), _hp(bb), _hp(x),
                                          tol, max_iter, C.byref(it), C.byref(rr)),
                    "fm_csr_pcg_ilu0")
        return x, it.value, rr.value

    def newton_solve(self, u, n_steps, first_step=1, rtol=1e-10, atol=0.0, inner_tol=1e-12,
                     max_newton=200, max_pcg=5000, prec=FM_FP64, allow_not_converged=False):
        nit, pit, rel = _i32(), _i32(), _f64()
        st = lib().fm_newton_solve(self._h, _dp(u), first_step, n_steps, rtol, atol, inner_tol,
                                   max_newton, max_pcg, prec, C.byref(nit), C.byref(pit),
                                   C.byref(rel))
        if st and not (allow_not_converged and st == 8):
            self._check(st, "fm_newton_solve")
        return {"newton_iters": nit.value, "pcg_iters": pit.value, "final_relres": rel.value,
                "status": st}

    def csr_ilu0(self, row_ptr, col_idx, val):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        v = np.ascontiguousarray(val, np.float64)
        LU = np.zeros(ci.size, np.float64)
        d = np.zeros(rp.size - 1, np.float64)
        self._check(lib().fm_csr_ilu0(self._h, rp.size - 1, _hp(rp), _hp(ci), _hp(v), _hp(LU),
                                      _hp(d)), "fm_csr_ilu0")
        return LU, d

    def newton_step(self, u, load_frac, rtol=1e-10, atol=0.0, inner_tol=1e-12, max_newton=200,
                    max_pcg=5000, line_search=0, ls_c=0.1, prec=FM_FP64,
                    allow_not_converged=False):
        nit, pit, rel = _i32(), _i32(), _f64()
        st = lib().fm_newton_step(self._h, _dp(u), load_frac, rtol, atol, inner_tol, max_newton,
                                  max_pcg, line_search, ls_c, prec, C.byref(nit), C.byref(pit),
                                  C.byref(rel))
        if st and not (allow_not_converged and st == 8):
            self._check(st, "fm_newton_step")
        return {"newton_iters": nit.value, "pcg_iters": pit.value, "final_relres": rel.value,
                "status": st}

    def newton_step_host(self, u_host, load_frac, rtol=1e-10, atol=0.0, inner_tol=1e-12,
                         max_newton=200, max_pcg=5000, line_search=0, ls_c=0.1, prec=FM_FP64,
                         allow_not_converged=False):
        """u_host: contiguous float64 numpy array, updated in place"""
        assert u_host.dtype == np.float64 and u_host.flags.c_contiguous
        nit, pit, rel = _i32(), _i32(), _f64()
        st = lib().fm_newton_step_host(self._h, _hp(u_host), load_frac, rtol, atol, inner_tol,
                                       max_newton, max_pcg, line_search, ls_c, prec,
                                       C.byref(nit), C.byref(pit), C.byref(rel))
        if st and not (allow_not_converged and st == 8):
            self._check(st, "fm_newton_step_host")
        return {"newton_iters": nit.value, "pcg_iters": pit.value, "final_relres": rel.value,
                "status": st}

    @staticmethod
    def newton_config(**cfg):
        """an fm_newton_config: fm_newton_config_default's values with the
        given fields replaced (prec= is accepted for precision=)"""
        g = NewtonConfig()
        lib().fm_newton_config_default(C.byref(g))
        for k, v in cfg.items():
            if k == "prec":
                k = "precision"
            if k not in {f for f, _ in NewtonConfig._fields_}:
                raise TypeError(f"unknown Newton option {k}")
            setattr(g, k, v)
        return g

    def newton_step_cfg(self, u, load_frac, allow=(), **cfg):
        """fm_newton_step_cfg: cfg keys are fm_newton_config's fields (the
        rest keep fm_newton_config_default's values); statuses listed in
        `allow` are returned in the result instead of raised.  u: a CUDA
        tensor, or a float64 numpy array (the host-buffer call)"""
        g = self.newton_config(**cfg)
        r = NewtonResult()
        if isinstance(u, np.ndarray):
            assert u.dtype == np.float64 and u.flags.c_contiguous
            st = lib().fm_newton_step_cfg_host(self._h, _hp(u), load_frac, C.byref(g),
                                               C.byref(r))
        else:
            st = lib().fm_newton_step_cfg(self._h, _dp(u), load_frac, C.byref(g), C.byref(r))
        out = {f: getattr(r, f) for f, _ in NewtonResult._fields_}
        out["status"] = st
        if st and st not in allow:
            self._check(st, "fm_newton_step_cfg")
        if st:
            buf = C.create_string_buffer(512)
            lib().fm_last_error(self._h, buf, 512)
            out["error"] = buf.value.decode(errors="replace")
        return out

    def newton_solve_cfg(self, u, n_steps, first_step=1, allow=(), **cfg):
        """fm_newton_solve_cfg over load steps first_step..n_steps"""
        g = self.newton_config(**cfg)
        r = NewtonResult()
        st = lib().fm_newton_solve_cfg(self._h, _dp(u), first_step, n_steps, C.byref(g),
                                       C.byref(r))
        out = {f: getattr(r, f) for f, _ in NewtonResult._fields_}
        out["status"] = st
        if st and st not in allow:
            self._check(st, "fm_newton_solve_cfg")
        return out

    def element_states(self, u, F=None, stress=None, counts=False):
        """fm_element_states: (F_sl3 [E, 9], stress [E, 6], det violations);
        with counts=True the last item is (det violations, non-finite
        states).  F/stress default to ElementState's initial values
        (identity, zero)"""
        t = self.torch
        if F is None:
            F = t.eye(3, dtype=t.float64, device=f"cuda:{self.device}").reshape(1, 9).repeat(
                self.n_elems, 1).contiguous()
        if stress is None:
            stress = self._zeros(6 * self.n_elems).view(self.n_elems, 6)
        v, nf = _u32(), _u32()
        self._check(lib().fm_element_states(self._h, _dp(u), _dp(F), _dp(stress), C.byref(v),
                                            C.byref(nf)), "fm_element_states")
        return F, stress, ((v.value, nf.value) if counts else v.value)

    def set_state_output(self, F=None, stress=None):
        self._state_keep = (F, stress)  # the library holds the raw pointers
        self._check(lib().fm_set_state_output(self._h, _dp(F), _dp(stress)),
                    "fm_set_state_output")

    def newton_history(self):
        """per-solve records of the latest Newton call"""
        cnt = _i32()
        lib().fm_newton_history(self._h, None, 0, C.byref(cnt))
        recs = (NewtonRecord * max(cnt.value, 1))()
        self._check(lib().fm_newton_history(self._h, recs, cnt.value, C.byref(cnt)),
                    "fm_newton_history")
        return [{f: getattr(r, f) for f, _ in NewtonRecord._fields_ if f != "pad"}
                for r in recs[: cnt.value]]

    def profile_enable(self, on=True):
        self._check(lib().fm_profile_enable(self._h, int(on)), "fm_profile_enable")

    def profile_read(self):
        p = Profile()
        self._check(lib().fm_profile_read(self._h, C.byref(p)), "fm_profile_read")
        return {name: {"ms": p.ms[k], "calls": p.calls[k], "kernels": p.kernels[k]}
                for k, name in PROF_KINDS.items()}

    def exact_apply(self, u, v, transpose=False):
        y = self._zeros(self.n_dofs)
        self._check(lib().fm_exact_apply(self._h, _dp(u), _dp(v), _dp(y), int(transpose)),
                    "fm_exact_apply")
        return y

    def adjoint(self, u, dLdu, tol=1e-10, inner_tol=1e-12, max_sweeps=500, prec=FM_FP64,
                want_w=False):
        gm = self._zeros(self.n_elems)
        gl = self._zeros(self.n_elems)
        w = self._zeros(self.n_dofs) if want_w else None
        sw, pit = _i32(), _i32()
        self._check(lib().fm_adjoint(self._h, _dp(u), _dp(dLdu), _dp(gm), _dp(gl), _dp(w), tol,
                                     inner_tol, max_sweeps, prec, C.byref(sw), C.byref(pit)),
                    "fm_adjoint")
        return gm, gl, w, sw.value, pit.value
