"""Single-kernel cases and the per-workload runs, for profiling and reports.

    python -m flexmesh_b200.cases trsv     --N 64 --prec mixed --applies 4
    python -m flexmesh_b200.cases ilu      --N 64 --prec fp64 --reps 2
    python -m flexmesh_b200.cases assemble --N 128 --prec fp64 --reps 5
    python -m flexmesh_b200.cases newton   --N 64 --levels 1 --inner-tol 0.2
    python -m flexmesh_b200.cases adjoint  --N 32 --fd 64
    python -m flexmesh_b200.cases incompressible --N 48

(with ``atlas-flexmesh_b200`` on ``PYTHONPATH``).  Every case prints one JSON
line.  ``trsv``, ``ilu`` and ``assemble`` are sized for ``ncu`` captures: one
context, a few launches of the kernel of interest after a short set-up, and
device timings from CUDA events on the context's stream.  ``adjoint`` and
``incompressible`` are the material-gradient check on the 32^3 block and the
near-incompressible 48^3 run (nu = 0.49, 20 load steps).

Algorithmic bytes per launch (what the roofline fractions count; schedule
records, neighbour lists and recomputation are not counted):
  assembly   24 E + 48 Nn + w nnz + 8 n       (conn + E_e, X and u, K, f_int)
  ILU(0)     (2w + 4) nnz + 4 (n + 1)
  solves     (w + 4)(nnz - n) + w n + 8 (n + 1) + 4 w n   (forward + backward)
with E tets, Nn nodes, n = 3 Nn DOFs, w = 8 (FP64) or 4 (FP32).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np
import torch

from . import _lib as L
from . import configs

PREC = {"fp64": L.FM_FP64, "mixed": L.FM_MIXED}


def hbm_peak():
    """measured copy bandwidth of this GPU pool (GB/s) when the repository
    carries MEASURED_PEAKS.json, else the fallback figure"""
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, "..", "..", "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bytes_assembly(E, Nn, nnz, w):
    return 24 * E + 48 * Nn + w * nnz + 8 * 3 * Nn


def bytes_ilu(nnz, n, w):
    return (2 * w + 4) * nnz + 4 * (n + 1)


def bytes_solves(nnz, n, w):
    return (w + 4) * (nnz - n) + w * n + 8 * (n + 1) + 4 * w * n


def problem_context(P, device=0):
    ctx = L.Context(device)
    ctx.set_mesh(P.xyz, P.conn, P.elem_volume)
    ctx.set_material(P.E, P.nu, P.E_elem)
    ctx.set_bc(P.mask, P.bc_value)
    return ctx


class Timer:
    """CUDA-event interval on the given stream"""

    def __init__(self, stream):
        self.s = stream
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)

    def __enter__(self):
        torch.cuda.synchronize()
        self.a.record(self.s)
        return self

    def __exit__(self, *exc):
        self.b.record(self.s)
        torch.cuda.synchronize()
        self.ms = self.a.elapsed_time(self.b)


def case_trsv(a):
    """Forward + backward solves of ILU(0) on the scale-up block's tangent
    at u = 0 (Dirichlet rows eliminated).  FP64 applies go through
    fm_ilu0_apply; FP32 ones through fm_pcg in mixed precision, whose
    iterations each make one apply (plus one SpMV and vector updates)."""
    P = configs.scaleup_block(a.N)
    ctx = problem_context(P)
    n = ctx.n_dofs
    u = torch.zeros(n, dtype=torch.float64, device="cuda")
    prec = PREC[a.prec]
    ctx.assemble_into_context(u, prec=prec, apply_bc=True)
    ctx.ilu0(prec)
    r = torch.as_tensor(np.random.default_rng(5).standard_normal(n), device="cuda")
    r[torch.as_tensor(P.mask, device="cuda") == 1] = 0.0
    ctx.profile_enable(True)
    with Timer(ctx.stream) as t:
        if prec == L.FM_FP64:
            for _ in range(a.applies):
                ctx.ilu0_apply(r)
        else:
            ctx.pcg(r, tol=1e-30, max_iter=max(a.applies - 1, 0), prec=prec)
    prof = ctx.profile_read()
    w = 8 if prec == L.FM_FP64 else 4
    p = prof["trsv"]
    per = p["ms"] / max(p["calls"], 1)
    B = bytes_solves(ctx.nnz, n, w)
    peak, kind = hbm_peak()
    return {"case": "trsv", "N": a.N, "prec": a.prec, "applies": p["calls"],
            "ms_per_apply": round(per, 4), "bytes_per_apply": B,
            "achieved_gbs": round(B / per / 1e6, 1), "peak_gbs": peak, "peak_kind": kind,
            "frac": round(B / per / 1e6 / peak, 4), "wall_ms": round(t.ms, 2),
            "spmv_ms_per_call": round(prof["spmv"]["ms"] / prof["spmv"]["calls"], 4)
            if prof.get("spmv", {}).get("calls") else None,
            "flags": ctx.flags()}


def case_ilu(a):
    """ILU(0) factorizations of the scale-up block's tangent at u = 0"""
    P = configs.scaleup_block(a.N)
    ctx = problem_context(P)
    n = ctx.n_dofs
    u = torch.zeros(n, dtype=torch.float64, device="cuda")
    prec = PREC[a.prec]
    ctx.assemble_into_context(u, prec=prec, apply_bc=True)
    ctx.profile_enable(True)
    for _ in range(a.reps):
        ctx.ilu0(prec)
    prof = ctx.profile_read()["ilu0"]
    w = 8 if prec == L.FM_FP64 else 4
    per = prof["ms"] / max(prof["calls"], 1)
    B = bytes_ilu(ctx.nnz, n, w)
    peak, kind = hbm_peak()
    return {"case": "ilu", "N": a.N, "prec": a.prec, "reps": prof["calls"],
            "ms_per_factorization": round(per, 3), "bytes": B,
            "achieved_gbs": round(B / per / 1e6, 1), "peak_gbs": peak, "peak_kind": kind,
            "frac": round(B / per / 1e6 / peak, 4), "flags": ctx.flags()}


def case_assemble(a):
    """One residual + tangent + CSR scatter of the assembly block (128^3 x 6
    tets: sinusoidal displacement, log-normal mu), timed per call.  The K of
    consecutive calls (2.9 GB FP64, 1.4 GB FP32 at N=128) exceeds the L2, so
    each call streams from HBM."""
    P = configs.assembly_block(a.N)
    ctx = problem_context(P)
    prec = PREC[a.prec]
    u = torch.as_tensor(P.meta["u"], device="cuda")
    f = torch.zeros_like(u)
    for _ in range(a.warmup):
        ctx.assemble_into_context(u, prec=prec, apply_bc=False, f=f)
    times = []
    for _ in range(a.reps):
        with Timer(ctx.stream) as t:
            ctx.assemble_into_context(u, prec=prec, apply_bc=False, f=f)
        times.append(t.ms)
    ms = float(np.median(times))
    w = 8 if prec == L.FM_FP64 else 4
    B = bytes_assembly(ctx.n_elems, ctx.n_nodes, ctx.nnz, w)
    peak, kind = hbm_peak()
    return {"case": "assemble", "N": a.N, "prec": a.prec, "tets": ctx.n_elems,
            "ms_median": round(ms, 3), "ms_min": round(min(times), 3),
            "tets_per_s": round(ctx.n_elems / ms * 1e3, 1), "bytes": B,
            "achieved_gbs": round(B / ms / 1e6, 1), "peak_gbs": peak, "peak_kind": kind,
            "frac": round(B / ms / 1e6 / peak, 4),
            "flags": ctx.flags()}


def _solve_path(ctx, n, n_steps, prec, inner_tol, rtol=1e-10, u0=None, steps=None,
                line_search=0, max_newton=400, allow_not_converged=False):
    u = torch.zeros(n, dtype=torch.float64, device="cuda") if u0 is None else u0.clone()
    newton, pcg, per_step = 0, 0, []
    for s in (steps if steps is not None else range(1, n_steps + 1)):
        r = ctx.newton_step(u, s / n_steps, rtol=rtol, inner_tol=inner_tol,
                            max_newton=max_newton, max_pcg=20000, line_search=line_search,
                            prec=prec, allow_not_converged=allow_not_converged)
        newton += r["newton_iters"]
        pcg += r["pcg_iters"]
        per_step.append((r["newton_iters"], r["pcg_iters"]))
    return u, newton, pcg, per_step


def case_newton(a):
    """Load levels 1 .. a.levels of the scale-up block in mixed precision
    with the engine's line search and the given inner tolerance, predictor
    tolerance, ILU(0) interval and initial-guess setting (bench.py's MIXED
    dict holds the benchmark's), timed and broken down by kernel class: a
    small, self-contained command for settings sweeps and launch lists."""
    P = configs.scaleup_block(a.N)
    ctx = problem_context(P)
    u = torch.zeros(P.xyz.size, dtype=torch.float64, device="cuda")
    cfg = dict(newton_rtol=1e-10, inner_tol=a.inner_tol, predictor_tol=a.predictor_tol,
               max_newton=400, max_pcg=20000, line_search=10, ls_c=1e-4, prec=L.FM_MIXED,
               ilu_every=a.ilu_every, initial_guess=a.initial_guess)
    ctx.profile_enable(True)
    levels = []
    with Timer(ctx.stream) as t:
        for lvl in range(1, a.levels + 1):
            r = ctx.newton_step_cfg(u, lvl / P.n_steps, **cfg)
            levels.append((lvl, r["newton_iters"], r["pcg_iters"], r["backtracks"]))
    prof = ctx.profile_read()
    if a.save_u:
        np.save(a.save_u, u.cpu().numpy())
    return {"case": "newton", "N": a.N, "levels": levels, "ms": round(t.ms, 1),
            "inner_tol": a.inner_tol, "predictor_tol": a.predictor_tol,
            "ilu_every": a.ilu_every, "initial_guess": a.initial_guess,
            "newton_total": sum(x[1] for x in levels), "pcg_total": sum(x[2] for x in levels),
            "profile_ms": {k: round(v["ms"], 1) for k, v in prof.items()},
            "launches": {k: v["kernels"] for k, v in prof.items()}}


def case_adjoint(a):
    """Material gradients of L = 1/2 |u_top(mu) - u*|^2 on the 32^3 block:
    u* from the 'true' log-normal mu (seed A), the model mu from seed B.
    FP64 and mixed adjoints against central finite differences
    (step a.fd_step times mu_e, lambda_e; 1e-6 by default) on a.fd seeded
    elements.  The finite
    differences re-solve from the converged state at full load (the
    material is hyperelastic, so the equilibrium does not depend on the
    path).  Those Newton iterations use the reference's tangent, which
    converges linearly (about 0.7 per iteration), so each perturbed solve
    runs a fixed a.fd_newton iterations (80: 0.7^80 ~ 4e-13 of the
    perturbation left); a fixed count keeps the two solves' rounding
    alike, and the mixed inner solve is enough because every iteration's
    residual is FP64.  The loss difference is formed as
    1/2 sum (a+ - a-)(a+ + a- - 2 u*), which keeps the cancellation of the
    two nearby losses out of the quotient."""
    P = configs.adjoint_block(a.N)
    nu = P.nu
    ctx = problem_context(P)
    n = ctx.n_dofs
    sel = torch.as_tensor(configs.top_face_xy_dofs(P.xyz), device="cuda")
    mu_m, lam_m = P.lame()
    Et = P.meta["E_true"]
    mu_t = Et / (2 * (1 + nu))
    lam_t = Et * nu / ((1 + nu) * (1 - 2 * nu))
    # target from the true field
    ctx.set_material_lame(mu_t, lam_t, nu)
    u_t, *_ = _solve_path(ctx, n, P.n_steps, L.FM_FP64, 1e-12, rtol=1e-12)
    target = u_t[sel].clone()
    ctx.set_material_lame(mu_m, lam_m, nu)
    t0 = time.perf_counter()
    u, nw, npcg, _ = _solve_path(ctx, n, P.n_steps, L.FM_FP64, 1e-12, rtol=1e-12)
    t_fwd = time.perf_counter() - t0

    def loss(uu):
        return 0.5 * float(torch.sum((uu[sel] - target) ** 2))

    g = torch.zeros_like(u)
    g[sel] = u[sel] - target
    res = {"case": "adjoint", "N": a.N, "tets": ctx.n_elems, "forward_s": round(t_fwd, 3),
           "forward_newton": nw, "forward_pcg": npcg, "loss": loss(u)}
    grads = {}
    for name, prec, inner in (("fp64", L.FM_FP64, 1e-12), ("mixed", L.FM_MIXED, 0.1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gm, gl, _, sweeps, pit = ctx.adjoint(u, g, tol=1e-11, inner_tol=inner, prec=prec)
        torch.cuda.synchronize()
        grads[name] = (gm.cpu().numpy(), gl.cpu().numpy())
        res[f"adjoint_{name}"] = {"s": round(time.perf_counter() - t0, 3), "sweeps": sweeps,
                                  "pcg": pit}
    g64, g32 = grads["fp64"], grads["mixed"]
    res["mixed_vs_fp64_rel"] = {
        "mu": float(np.linalg.norm(g32[0] - g64[0]) / np.linalg.norm(g64[0])),
        "lam": float(np.linalg.norm(g32[1] - g64[1]) / np.linalg.norm(g64[1]))}
    # central finite differences on seeded active elements
    active = np.nonzero(P.elem_volume >= 1e-30)[0]
    pick = np.sort(np.random.default_rng(configs.SEED_FD_4).choice(active, a.fd, replace=False))
    errs = {"fp64": [], "mixed": []}
    rows = []
    t0 = time.perf_counter()
    for e in pick:
        for pname in ("mu", "lam"):
            base = mu_m if pname == "mu" else lam_m
            h = a.fd_step * base[e]
            tops = []
            for sgn in (1.0, -1.0):
                p = base.copy()
                p[e] += sgn * h
                ctx.set_material_lame(p if pname == "mu" else mu_m,
                                      p if pname == "lam" else lam_m, nu)
                up, *_ = _solve_path(ctx, n, 1, L.FM_MIXED, 0.1, rtol=1e-30, u0=u,
                                     steps=[1], max_newton=a.fd_newton,
                                     allow_not_converged=True)
                tops.append(up[sel])
            dl = 0.5 * float(torch.sum((tops[0] - tops[1]) * (tops[0] + tops[1] - 2 * target)))
            fd = dl / (2 * h)
            k = 0 if pname == "mu" else 1
            for name in ("fp64", "mixed"):
                ge = float(grads[name][k][e])
                errs[name].append(abs(ge - fd) / max(abs(fd), 1e-300))
            rows.append((int(e), pname, fd, float(grads["fp64"][k][e])))
    ctx.set_material_lame(mu_m, lam_m, nu)
    res["fd_s"] = round(time.perf_counter() - t0, 1)
    res["fd_elements"] = int(a.fd)
    res["fd_step_rel"] = a.fd_step
    res["fd_rel_err"] = {name: {"max": float(np.max(v)), "median": float(np.median(v)),
                                "n_above_1e-6": int(np.sum(np.asarray(v) > 1e-6))}
                         for name, v in errs.items()}
    res["fd_sample"] = [{"e": r[0], "p": r[1], "fd": r[2], "adj": r[3]} for r in rows[:4]]
    return res


def case_incompressible(a):
    """Near-incompressible block (48^3 x 6 tets, jitter 0.1 h, nu = 0.49,
    u_z = -0.4 in 20 load steps), the whole load path in mixed precision and
    in FP64 with the same inexact-Newton settings (inner PCG to a.inner_tol,
    mixed from the projected previous correction, ILU(0) every a.ilu_every
    solves, the engine's line search), Newton and PCG
    counts per load step, the mixed-vs-FP64 difference at the end, and the
    adjoint dL/dmu (FP64 and mixed) for L = 1/2 |u_top - u*|^2 with u* from
    the log-normal mu field (sigma 0.2).  The reference's tangent clamps its
    volumetric term at max(1 - 2 nu, 0.1) = 0.1 against the exact 0.02, so
    Newton contracts by about 0.99 per iteration here: thousands of
    iterations per load step, each cheap."""
    P = configs.near_incompressible_block(a.N)
    nu = P.nu
    ctx = problem_context(P)
    n = ctx.n_dofs
    out = {"case": "incompressible", "N": a.N, "tets": ctx.n_elems, "nu": nu,
           "load_steps": min(a.steps, P.n_steps), "of": P.n_steps, "inner_tol": a.inner_tol,
           "ilu_every": a.ilu_every}
    base = dict(newton_rtol=1e-10, inner_tol=a.inner_tol, predictor_tol=1e-6,
                max_newton=a.max_newton, max_pcg=20000, line_search=10, ls_c=1e-4,
                ilu_every=a.ilu_every)

    def path(prec, label):
        cfg = dict(base, prec=prec, initial_guess=1 if prec == L.FM_MIXED else 0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u = torch.zeros(n, dtype=torch.float64, device="cuda")
        per = []
        for s in range(1, min(a.steps, P.n_steps) + 1):
            r = ctx.newton_step_cfg(u, s / P.n_steps, **cfg)
            per.append((r["newton_iters"], r["pcg_iters"]))
            print(f"[{label}] step {s}: newton {per[-1][0]} pcg {per[-1][1]} "
                  f"t {time.perf_counter() - t0:.1f}s", file=sys.stderr, flush=True)
        torch.cuda.synchronize()
        return u, {"s": round(time.perf_counter() - t0, 2),
                   "newton": sum(k for k, _ in per), "pcg": sum(p for _, p in per),
                   "newton_by_step": [k for k, _ in per],
                   "pcg_per_newton_by_step": [round(p / max(k, 1), 2) for k, p in per]}

    u_m, out["mixed"] = path(L.FM_MIXED, "mixed")
    u_d, out["fp64"] = path(L.FM_FP64, "fp64")
    out["mixed_vs_fp64_rel"] = float(torch.linalg.norm(u_m - u_d) / torch.linalg.norm(u_d))
    # u* from the 'true' field, then the adjoint of the top-face loss
    sel = torch.as_tensor(configs.top_face_xy_dofs(P.xyz), device="cuda")
    ctx.set_material(P.E, nu, P.meta["E_true"])
    u_t, out["forward_true_mixed"] = path(L.FM_MIXED, "true")
    ctx.set_material(P.E, nu, P.E_elem)
    g = torch.zeros_like(u_d)
    g[sel] = u_d[sel] - u_t[sel]
    t0 = time.perf_counter()
    gm64, _, _, s64, p64 = ctx.adjoint(u_d, g, tol=1e-10, inner_tol=1e-6, max_sweeps=a.sweeps,
                                       prec=L.FM_FP64)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    gm32, _, _, s32, p32 = ctx.adjoint(u_d, g, tol=1e-10, inner_tol=0.1, max_sweeps=a.sweeps,
                                       prec=L.FM_MIXED)
    t32 = time.perf_counter() - t0
    out["adjoint"] = {"fp64_sweeps": s64, "fp64_pcg": p64, "fp64_s": round(t64, 2),
                      "mixed_sweeps": s32, "mixed_pcg": p32, "mixed_s": round(t32, 2),
                      "loss": float(0.5 * torch.sum(g[sel] ** 2)),
                      "dLdmu_norm": float(torch.linalg.norm(gm64)),
                      "mixed_vs_fp64_rel": float(torch.linalg.norm(gm32 - gm64) /
                                                 torch.linalg.norm(gm64))}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m flexmesh_b200.cases")
    ap.add_argument("case", choices=["trsv", "ilu", "assemble", "newton", "adjoint",
                                     "incompressible"])
    ap.add_argument("--N", type=int, default=None)
    ap.add_argument("--prec", choices=list(PREC), default="fp64")
    ap.add_argument("--applies", type=int, default=4)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--fd", type=int, default=64)
    ap.add_argument("--inner-tol", type=float, default=0.1)
    ap.add_argument("--line-search", type=int, default=0)
    ap.add_argument("--fd-newton", type=int, default=80)
    ap.add_argument("--fd-step", type=float, default=1e-6)
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--max-newton", type=int, default=3000)
    ap.add_argument("--levels", type=int, default=1)
    ap.add_argument("--predictor-tol", type=float, default=1e-6)
    ap.add_argument("--ilu-every", type=int, default=1)
    ap.add_argument("--initial-guess", type=int, default=0)
    ap.add_argument("--save-u", default=None)
    ap.add_argument("--sweeps", type=int, default=500)
    ap.add_argument("--steps", type=int, default=1000, help="load steps to run (all by default)")
    a = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("cases need a CUDA device")
    default_N = {"trsv": 64, "ilu": 64, "assemble": 128, "newton": 64, "adjoint": 32,
                 "incompressible": 48}
    if a.N is None:
        a.N = default_N[a.case]
    fn = {"trsv": case_trsv, "ilu": case_ilu, "assemble": case_assemble, "newton": case_newton,
          "adjoint": case_adjoint, "incompressible": case_incompressible}[a.case]
    print(json.dumps(fn(a)), flush=True)


if __name__ == "__main__":
    main()
