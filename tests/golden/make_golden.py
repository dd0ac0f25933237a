"""Generate the golden fixtures in this directory from the REFERENCE itself.

Every array marked ``ref_*`` is produced by the reference's own functions,
compiled from its headers by ``oracle/Makefile`` into
``oracle/_ref/libfm_ref.so`` (mesh generator, CSR pattern builder,
element kernel, single-thread global assembly, ILU(0) factorize/solve,
PCG-ILU(0)).  Inputs (``in_*``) are seeded numpy draws stored alongside.
The only oracle-made arrays are the solve pattern (the reference's pattern
with its column fill fixed) and the Dirichlet mask, marked ``orc_*``; they
define the inputs on which the reference's ILU/PCG are run.

Run from the repository root:  python tests/golden/make_golden.py
(requires oracle/_ref/libfm_ref.so, i.e. the reference checkout at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def ref_mesh(R, N):
    h = R.ref_mesh_new(N)
    nn, ne, nl = C.c_uint32(), C.c_uint32(), C.c_uint32()
    R.ref_mesh_sizes(h, C.byref(nn), C.byref(ne), C.byref(nl))
    xyz = np.zeros(3 * nn.value)
    conn = np.zeros(4 * ne.value, np.uint32)
    vol = np.zeros(ne.value)
    p = np.zeros(nn.value + 1, np.uint32)
    d = np.zeros(nl.value, np.uint32)
    R.ref_mesh_get(h, xyz, conn, vol, p, d)
    R.ref_mesh_free(h)
    return xyz, conn, vol, p, d


def ref_pattern(R, xyz, conn):
    nn = xyz.size // 3
    nnz = R.ref_pattern(nn, xyz, conn.size // 4, conn, None, None)
    rp = np.zeros(3 * nn + 1, np.uint32)
    ci = np.zeros(nnz, np.uint32)
    R.ref_pattern(nn, xyz, conn.size // 4, conn, rp, ci)
    return rp, ci


def clamp_mask(xyz):
    """Bottom face z=0 clamped (xyz), top face z=1 u_z prescribed."""
    z = xyz[2::3]
    mask = np.zeros(xyz.size, np.uint8)
    mask[np.repeat(z < 1e-12, 3)] = 1
    mask[2::3][z > 1.0 - 1e-12] = 1
    return mask


def main():
    R = O.ref()
    if R is None:
        raise SystemExit("oracle/_ref/libfm_ref.so not built (needs the reference checkout)")
    out = {}
    rng = np.random.default_rng(20261203)
    # ---- element kernel on random tets ------------------------------------
    nel = 16
    x = rng.random((nel, 12))
    u = 0.05 * rng.standard_normal((nel, 12))
    Ks = np.zeros((nel, 144))
    fs = np.zeros((nel, 12))
    Es = 0.5 + rng.random(nel)
    for t in range(nel):
        R.ref_element(np.ascontiguousarray(x[t]), np.ascontiguousarray(u[t]), Es[t], 0.3, Ks[t],
                      fs[t])
    out.update(in_elem_x=x, in_elem_u=u, in_elem_E=Es, ref_elem_K=Ks, ref_elem_f=fs)
    for N in (2, 4):
        xyz, conn, vol, n2e_ptr, n2e = ref_mesh(R, N)
        nn, ne = xyz.size // 3, conn.size // 4
        rp, ci = ref_pattern(R, xyz, conn)
        rps, cis = O.pattern(nn, conn, "solve")
        uN = 0.02 * rng.standard_normal(3 * nn)
        p = f"n{N}_"
        out.update({p + "ref_xyz": xyz, p + "ref_conn": conn, p + "ref_vol": vol,
                    p + "ref_n2e_ptr": n2e_ptr, p + "ref_n2e": n2e, p + "ref_row_ptr": rp,
                    p + "ref_col_idx": ci, p + "orc_solve_col_idx": cis, p + "in_u": uN})
        for tag, cols in (("refpat", ci), ("solvepat", cis)):
            for utag, uu in (("u0", np.zeros(3 * nn)), ("useed", uN)):
                K = np.zeros(ci.size)
                f = np.zeros(3 * nn)
                R.ref_assemble(nn, xyz, ne, conn, vol, 1.0, 0.3, uu, rp, cols, K, f, 1)
                out[p + f"ref_K_{tag}_{utag}"] = K
                out[p + f"ref_f_{tag}_{utag}"] = f
        fr = np.zeros(3 * nn)
        R.ref_residual(nn, xyz, ne, conn, vol, 1.0, 0.3, uN, fr, 1)
        out[p + "ref_fres_useed"] = fr
        # Dirichlet-eliminated tangent at the seeded u -> ILU(0) and PCG
        mask = clamp_mask(xyz)
        K = out[p + "ref_K_solvepat_useed"].copy()
        Rv = -out[p + "ref_f_solvepat_useed"].copy()
        O.apply_bc(rp, cis, K, Rv, mask)
        Lv = np.zeros(ci.size)
        Uv = np.zeros(ci.size)
        dg = np.zeros(3 * nn)
        lev = np.zeros(3 * nn, np.int32)
        ml = R.ref_ilu0(3 * nn, rp, cis, K, Lv, Uv, dg, lev)
        r = rng.standard_normal(3 * nn)
        y = np.zeros(3 * nn)
        R.ref_ilu0_solve(3 * nn, rp, cis, K, r, y)
        xs = np.zeros(3 * nn)
        its = R.ref_pcg_ilu0(3 * nn, rp, cis, K, Rv, xs, 1e-12, 1000, 1)
        out.update({p + "orc_mask": mask, p + "in_Kbc": K, p + "in_Rbc": Rv,
                    p + "ref_ilu_L": Lv, p + "ref_ilu_U": Uv, p + "ref_ilu_diag": dg,
                    p + "ref_ilu_level": lev, p + "ref_ilu_maxlevel": np.array([ml]),
                    p + "in_r": r, p + "ref_ilu_solve": y, p + "ref_pcg_x": xs,
                    p + "ref_pcg_iters": np.array([its])})
    # ---- Poisson known-answer problem (TESTS/external_validation_runner.cpp)
    for g in (8, 32):
        rp, ci, val, b, xe = O.poisson(g)
        x0 = np.zeros(g * g)
        its = R.ref_pcg_ilu0(g * g, rp, ci, val, b, x0, 1e-10, 4000, 1)
        out.update({f"poisson{g}_rp": rp, f"poisson{g}_ci": ci, f"poisson{g}_val": val,
                    f"poisson{g}_b": b, f"poisson{g}_xexact": xe, f"poisson{g}_ref_x": x0,
                    f"poisson{g}_ref_iters": np.array([its])})
    path = os.path.join(HERE, "golden_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
