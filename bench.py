#!/usr/bin/env python
"""Benchmark of the FlexMesh hot path on B200: Newton load steps of the
1.57M-tet block (64^3 hexes x 6 tets, jittered, log-normal mu, top face
u_z = -0.2 in 10 load steps), mixed precision (FP32 tangent/ILU(0)/PCG with
FP64 det F, ln J, residual and Newton update).

A step is one load step of that load path: the Dirichlet predictor plus
Newton iterations to ||R|| < 1e-10 ||R_0||.  Steps walk the load levels
1, 2, ..., 10, 1, ...; W warm-up steps run first, then K timed steps.
value = tets/s through Newton iterations = n_tets * (Newton iterations in
the timed steps) / timed seconds (CUDA events on the library's stream).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: replicas only (the path does not shard; each rank solves its own
copy of the block, no collectives); value sums the ranks' work over the
max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "atlas-flexmesh_b200"))

METRIC = "Newton solve s & tets/s, 1.57M-tet block: mixed vs FP64 GPU at rel err ≤1e-8"
WORKLOAD = "scale-up block 64^3x6 tets (1,572,864 tets, 823,875 DOF), jitter 0.15h, " \
           "log-normal mu sigma 0.3, top u_z=-0.2 in 10 load steps"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flexmesh", choices=["flexmesh", "reference"])
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--inner-tol", type=float, default=0.2)
    ap.add_argument("--fp64-steps", type=int, default=1,
                    help="timed FP64 load steps for the mixed/FP64 comparison (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl" if args.impl == "flexmesh" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region"""

    def __init__(self, gpu):
        self.gpu = gpu
        self.p = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_gpu{gpu}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
            sm = sorted(float(r[0]) for r in rows)
            mx = max(float(r[1]) for r in rows)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4)
                              if r[3 + i].strip() == "Active"})
            return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": reasons,
                    "samples": len(rows)}
        except Exception as e:  # nvidia-smi unavailable
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(e)[:80]}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(key):
    """DRAM bytes per call of one kernel class, measured by ncu on this
    workload and recorded in the committed summaries under profiles/ as
    'machine-readable: traffic_bytes_per_call <key> <bytes>' (None if absent)"""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                parts = line.split()
                if (len(parts) == 4 and parts[0] == "machine-readable:" and
                        parts[1] == "traffic_bytes_per_call" and parts[2] == key):
                    return int(parts[3])
    return None


def trsv_bytes(nnz, n, w, wv):
    """algorithmic bytes of one preconditioner apply (forward + backward)"""
    return (w + 4) * (nnz - n) + w * n + 8 * (n + 1) + 4 * wv * n


def asm_bytes(n_elems, n_nodes, nnz, w, per_elem_mat=8):
    return (16 + per_elem_mat) * n_elems + 48 * n_nodes + w * nnz + 8 * 3 * n_nodes


# ---------------------------------------------------------------------------
def run_flexmesh(args, rank, world, local, dist):
    import numpy as np
    import torch

    import flexmesh_b200 as F
    from flexmesh_b200 import configs

    torch.cuda.set_device(local)
    P = configs.scaleup_block(args.N)
    ctx = F.Context(local)
    ctx.set_mesh(P.xyz, P.conn, P.elem_volume)
    ctx.set_material(P.E, P.nu, P.E_elem)
    ctx.set_bc(P.mask, P.bc_value)
    E, n = P.n_elems, P.xyz.size
    u = torch.zeros(n, dtype=torch.float64, device=f"cuda:{local}")
    S = P.n_steps

    def load_step(uu, i, prec, tol):
        lvl = i % S + 1
        if lvl == 1:
            uu.zero_()
        return ctx.newton_step(uu, lvl / S, rtol=1e-10, inner_tol=tol, max_newton=400,
                               max_pcg=20000, prec=prec)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    for i in range(args.warmup):
        load_step(u, i, F.FM_MIXED, args.inner_tol)
    u_start = u.clone()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    newton = pcg = 0
    with Clocks(local) as clk:
        ev0.record()
        for i in range(args.warmup, args.warmup + args.steps):
            r = load_step(u, i, F.FM_MIXED, args.inner_tol)
            newton += r["newton_iters"]
            pcg += r["pcg_iters"]
        ev1.record()
        barrier()
    t = ev0.elapsed_time(ev1) / 1e3
    if dist:
        tt = torch.tensor([t], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    u_mixed = u.clone()

    # kernel breakdown and launch count: the same load steps replayed from the
    # same state with the library's event profiler on (kept out of the timed
    # run: its event records add host work to every kernel group)
    up = u_start.clone()
    ctx.profile_enable(True)
    for i in range(args.warmup, args.warmup + args.steps):
        load_step(up, i, F.FM_MIXED, args.inner_tol)
    prof = ctx.profile_read()
    ctx.profile_enable(False)
    barrier()
    replay_same = bool(torch.equal(up, u_mixed))

    # e2e: the same load steps through the host-buffer C-ABI call (copies inside)
    uh = u_start.cpu().numpy().copy()
    barrier()
    t0 = time.perf_counter()
    e_newton = 0
    for i in range(args.warmup, args.warmup + args.steps):
        lvl = i % S + 1
        if lvl == 1:
            uh[:] = 0.0
        r = ctx.newton_step_host(uh, lvl / S, rtol=1e-10, inner_tol=args.inner_tol,
                                 max_newton=400, max_pcg=20000, prec=F.FM_MIXED)
        e_newton += r["newton_iters"]
    te = time.perf_counter() - t0

    # FP64 comparison over the first timed load step(s), same starting state
    fp64 = None
    if args.fp64_steps > 0:
        u64 = u_start.clone()
        um = u_start.clone()
        k = min(args.fp64_steps, args.steps)
        barrier()
        ev0.record()
        n64 = p64 = 0
        for i in range(args.warmup, args.warmup + k):
            r = load_step(u64, i, F.FM_FP64, 1e-12)
            n64 += r["newton_iters"]
            p64 += r["pcg_iters"]
        ev1.record()
        barrier()
        t64 = ev0.elapsed_time(ev1) / 1e3
        ev0.record()
        nm = 0
        for i in range(args.warmup, args.warmup + k):
            nm += load_step(um, i, F.FM_MIXED, args.inner_tol)["newton_iters"]
        ev1.record()
        barrier()
        tm = ev0.elapsed_time(ev1) / 1e3
        err = (torch.linalg.norm(um - u64) / torch.linalg.norm(u64)).item()
        fp64 = {"load_steps": k, "fp64_s": t64, "fp64_newton": n64, "fp64_pcg": p64,
                "mixed_s": tm, "mixed_newton": nm, "speedup_mixed_vs_fp64": t64 / tm,
                "rel_err_mixed_vs_fp64": err}

    hbm, peak_kind = peaks()
    nnz = ctx.nnz
    # dominant kernel class by device time
    dom = max(prof, key=lambda k: prof[k]["ms"])
    launches = sum(v["kernels"] for v in prof.values())
    w = 4  # FP32 values in the mixed inner solve
    per = {"trsv": trsv_bytes(nnz, n, w, 4), "spmv": (w + 4) * nnz + 4 * (n + 1) + 2 * 4 * n,
           "ilu0": (2 * w + 4) * nnz + 4 * (n + 1),
           "assemble": asm_bytes(E, P.n_nodes, nnz, w)}
    roof = None
    if dom in per and prof[dom]["calls"]:
        avg_s = prof[dom]["ms"] / 1e3 / prof[dom]["calls"]
        ach = per[dom] / avg_s / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(ach / hbm, 4),
                "traffic": profiled_traffic(f"{dom}_mixed_n{args.N}"),
                "peak_kind": peak_kind, "bytes_per_launch": per[dom],
                "avg_launch_ms": round(avg_s * 1e3, 4)}
    value = E * newton * world / t
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "tets/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3 / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic (seeded jitter and log-normal mu, numpy PCG64)",
        "config": {"workload": WORKLOAD, "precision": "mixed", "inner_tol": args.inner_tol,
                   "newton_rtol": 1e-10, "load_levels": [i % S + 1 for i in
                                                          range(args.warmup,
                                                                args.warmup + args.steps)],
                   "l2": "inputs (K 182 MB fp32, LU 182 MB) exceed the 126 MB L2",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "newton_iters": newton, "pcg_iters": pcg,
        "newton_solve_s_est": round(t / args.steps * S, 3),
        "e2e": {"value": round(E * e_newton * world / te, 1), "unit": "tets/s",
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": int(launches), "profile": prof,
        "profile_note": "kernel classes and launch count from a replay of the timed load "
                        "steps with the event profiler on; replay bit-identical: "
                        + str(replay_same),
        "roofline": roof,
        "fp64_compare": fp64,
    }
    return line, ctx, P


def cpu_baseline_sample(P, nnz_expected, pcg_per_newton, threads):
    """The reference's own assembly (oracle/_ref, all threads) plus the
    bit-identical O(nnz) ILU(0) and PCG port of the oracle on a bounded
    sample, extrapolated to one Newton iteration."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nn, E = P.n_nodes, P.n_elems
    rp, ci = O.pattern(nn, P.conn, "solve")
    u = np.zeros(P.xyz.size)
    R = O.ref()
    kind = "reference" if R is not None else "port"
    t0 = time.perf_counter()
    if R is not None:
        # assemble_global_threadlocal takes one E per problem; the per-element
        # field does not change its cost, so the scalar E times the same work
        K = np.zeros(ci.size)
        f = np.zeros(P.xyz.size)
        R.ref_assemble(nn, P.xyz, E, P.conn, P.elem_volume, P.E, P.nu, u, rp, ci, K, f, threads)
    else:
        mu, lam = P.lame()
        slot = O.slot_map(nn, P.conn, rp, ci)
        t0 = time.perf_counter()
        K, f = O.assemble(P.xyz, P.conn, mu, lam, P.nu, u, slot, ci.size,
                          (P.elem_volume >= 1e-30).astype(np.uint8))
    t_asm = time.perf_counter() - t0
    Rv = -f
    O.apply_bc(rp, ci, K, Rv, P.mask)
    Rv = np.random.default_rng(0).standard_normal(Rv.size)
    Rv[P.mask == 1] = 0
    t0 = time.perf_counter()
    LU, d, _ = O.ilu0(rp, ci, K)
    t_ilu = time.perf_counter() - t0
    t0 = time.perf_counter()
    k = 3
    O.pcg_ilu0(rp, ci, K, Rv, tol=1e-300, max_iter=k)
    t_pcg = (time.perf_counter() - t0) / k
    t_newton = t_asm + t_ilu + pcg_per_newton * t_pcg
    return {"value": round(E / t_newton, 1), "unit": "tets/s", "cores": threads, "kind": kind,
            "sample": f"one Newton iteration at N={P.N} extrapolated: reference assembly "
                      f"({t_asm:.2f}s, {threads} threads), ILU(0) port ({t_ilu:.2f}s, 1 thread), "
                      f"{pcg_per_newton:.0f} PCG-ILU(0) iterations at {t_pcg:.3f}s "
                      f"(port, 1 thread; FP64 count of the GPU run)"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation on the host cores."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from flexmesh_b200 import configs

    P = configs.scaleup_block(args.N)
    threads = os.cpu_count() or 1
    pcg_per_newton = 300.0  # FP64 PCG-ILU(0) iterations per Newton iteration at N=64, 1e-12
    vals = []
    for i in range(args.warmup + args.steps):
        s = cpu_baseline_sample(P, None, pcg_per_newton, threads)
        if i >= args.warmup:
            vals.append(s)
    v = sum(x["value"] for x in vals) / len(vals)
    t_step = P.n_elems / v
    return {"metric": METRIC, "value": round(v, 1), "unit": "tets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_step * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "precision": "fp64 (the reference has no mixed path)"},
            "cpu_baseline": {"value": round(v, 1), "unit": "tets/s", "cores": threads,
                             "kind": vals[-1]["kind"], "sample": vals[-1]["sample"]},
            "e2e": {"value": round(v, 1), "unit": "tets/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank, world, local, dist = dist_init(args)
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    line, ctx, P = run_flexmesh(args, rank, world, local, dist)
    if rank == 0:
        line["clocks"] = Clocks(local).summary()
        if not args.no_cpu_baseline:
            fp = line.get("fp64_compare") or {}
            per = (fp.get("fp64_pcg", 0) / max(fp.get("fp64_newton", 1), 1)) or 300.0
            try:
                line["cpu_baseline"] = cpu_baseline_sample(P, ctx.nnz, per, os.cpu_count() or 1)
            except Exception as e:  # the checker must not break the GPU line
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
