#!/usr/bin/env python
"""Benchmark of the FlexMesh hot path on B200: the Newton solve of the
1.57M-tet block (64^3 hexes x 6 tets, interior nodes jittered by 0.15 h,
log-normal mu with sigma 0.3, top face u_z = -0.2 in 10 load steps) in mixed
precision (FP32 tangent/ILU(0)/PCG with FP64 det F, ln J, residual and
Newton update), beside the plain FP64 GPU path.

A step is one load step: the Dirichlet predictor plus Newton iterations to
||R|| < 1e-10 ||R_0||.  W warm-up steps walk load levels 1, 2, ...; the K
timed steps then start the load path again from u = 0 and walk levels
1..10, 1..10, ... so every 10 timed steps are one complete Newton solve.

    value        = n_tets * (Newton iterations in the timed steps) / timed s
                   (tets/s through Newton iterations; CUDA events on the
                   library's stream)
    newton_solve = measured seconds of each complete 10-level load path
    fp64_compare = the same load path in plain FP64 (PCG to 1e-12): its
                   seconds, the mixed/FP64 speed-up and ||u - u_FP64|| / ||u||
                   at the last load level
    e2e          = one complete load path through the host-buffer C-ABI call
                   (u copied host -> device and back inside every step)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: replicas only (the path does not shard; each rank solves its own
copy of the block, no collectives); value sums the ranks' work over the
max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "atlas-flexmesh_b200"))

METRIC = "Newton solve s & tets/s, 1.57M-tet block: mixed vs FP64 GPU at rel err ≤1e-8"
WORKLOAD = "scale-up block 64^3x6 tets (1,572,864 tets, 823,875 DOF), jitter 0.15h, " \
           "log-normal mu sigma 0.3, top u_z=-0.2 in 10 load steps"

# Newton settings of the mixed path (fm_newton_config fields).  Both paths
# run the engine's Armijo line search on every iteration (10 trials,
# c = 1e-4, FEM/adaptive_fem_engine.hpp:2581): without it the reference's
# tangent stops contracting at load levels 8-10 of this block.  Mixed: inner
# PCG to 0.8 from the projected previous correction, ILU(0) refactored every
# third solve (the fastest of the measured settings; at most 145 Newton
# iterations in a load step against the cap of 400, where 0.9 needs more
# than 400 at load level 6; every Newton stop test is on the FP64 residual,
# so all converge to the same u).
MIXED = dict(newton_rtol=1e-10, inner_tol=0.8, predictor_tol=1e-6, max_newton=400,
             max_pcg=20000, line_search=10, ls_c=1e-4, initial_guess=1, ilu_every=3)
# the plain FP64 path: PCG to 1e-12
FP64 = dict(newton_rtol=1e-10, inner_tol=1e-12, max_newton=400, max_pcg=20000, line_search=10,
            ls_c=1e-4)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flexmesh", choices=["flexmesh", "reference"])
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--inner-tol", type=float, default=MIXED["inner_tol"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 load path")
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
                                timeout=datetime.timedelta(seconds=900))
        pg = dist
    return rank, world, local, pg


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region (samples
    kept in memory)"""

    def __init__(self, gpu):
        self.gpu = gpu
        self.p = None
        self.rows = []

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out, _ = self.p.communicate()
            self.rows = [r.split(",") for r in (out or "").strip().splitlines() if r.strip()]

    def summary(self):
        try:
            rows = self.rows
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
    import torch

    import flexmesh_b200 as F
    from flexmesh_b200 import configs

    torch.cuda.set_device(local)
    P = configs.scaleup_block(args.N)
    ctx = F.Context(local)
    ctx.set_mesh(P.xyz, P.conn, P.elem_volume)
    ctx.set_material(P.E, P.nu, P.E_elem)
    ctx.set_bc(P.mask, P.bc_value)
    E, n, S = P.n_elems, P.xyz.size, P.n_steps
    dev = f"cuda:{local}"
    mixed = dict(MIXED, inner_tol=args.inner_tol, prec=F.FM_MIXED)
    fp64 = dict(FP64, prec=F.FM_FP64)

    def load_step(uu, lvl, cfg):
        if lvl == 1:
            uu.zero_()
        return ctx.newton_step_cfg(uu, lvl / S, **cfg)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    u = torch.zeros(n, dtype=torch.float64, device=dev)
    for i in range(args.warmup):
        load_step(u, i % S + 1, mixed)
    barrier()
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    newton = pcg = 0
    per_step = []
    ctx.profile_enable(False)  # zero the launch counters
    with Clocks(local) as clk:
        ev[0].record(stream)
        for j in range(args.steps):
            r = load_step(u, j % S + 1, mixed)
            ev[j + 1].record(stream)
            newton += r["newton_iters"]
            pcg += r["pcg_iters"]
            per_step.append((j % S + 1, r["newton_iters"], r["pcg_iters"], r["backtracks"]))
        barrier()
    launches = sum(v["kernels"] for v in ctx.profile_read().values())
    t = ev[0].elapsed_time(ev[-1]) / 1e3
    step_s = [ev[j].elapsed_time(ev[j + 1]) / 1e3 for j in range(args.steps)]
    if dist:
        tt = torch.tensor([t], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    u_mixed = u.clone()
    paths = [sum(step_s[p * S:(p + 1) * S]) for p in range(args.steps // S)]
    u_path_end = u_mixed if args.steps % S == 0 else None

    # kernel breakdown: one complete load path replayed with the library's
    # event profiler on (kept out of the timed run: its event records add
    # host work to every kernel group); the replay must reproduce the timed
    # path's displacements bit for bit
    up = torch.zeros_like(u)
    ctx.profile_enable(True)
    for lvl in range(1, S + 1):
        load_step(up, lvl, mixed)
    prof = ctx.profile_read()
    ctx.profile_enable(False)
    barrier()
    replay_same = bool(torch.equal(up, u_path_end)) if u_path_end is not None else None

    # e2e: one complete load path through the host-buffer call (copies inside)
    uh = torch.zeros(n, dtype=torch.float64).numpy()
    barrier()
    t0 = time.perf_counter()
    e_newton = 0
    for lvl in range(1, S + 1):
        if lvl == 1:
            uh[:] = 0.0
        r = ctx.newton_step_cfg(uh, lvl / S, **mixed)
        e_newton += r["newton_iters"]
    te = time.perf_counter() - t0
    if dist:
        tt = torch.tensor([te], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    e2e_same = bool((torch.from_numpy(uh).to(dev) == up).all().item())

    # the plain FP64 path over the same complete load path (rank 0: the
    # replicas would repeat it; no collective inside)
    fp = None
    if not args.no_fp64 and rank == 0:
        u64 = torch.zeros_like(u)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n64 = p64 = 0
        lv64 = []
        for lvl in range(1, S + 1):
            r = load_step(u64, lvl, fp64)
            n64 += r["newton_iters"]
            p64 += r["pcg_iters"]
            lv64.append((lvl, r["newton_iters"], r["pcg_iters"]))
        e1.record(stream)
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1) / 1e3
        err = (torch.linalg.norm(up - u64) / torch.linalg.norm(u64)).item()
        t_mixed_path = sum(paths) / len(paths) if paths else None
        fp = {"newton_solve_s": round(t64, 3), "newton": n64, "pcg": p64,
              "per_level": lv64, "mixed_newton_solve_s": t_mixed_path,
              "speedup_mixed_vs_fp64": round(t64 / t_mixed_path, 3) if t_mixed_path else None,
              "rel_err_mixed_vs_fp64": err, "rel_err_at": f"load level {S}"}

    hbm, peak_kind = peaks()
    nnz = ctx.nnz
    dom = max(prof, key=lambda k: prof[k]["ms"])
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
    tets_eval = int((P.elem_volume >= 1e-30).sum())
    line = {
        "metric": METRIC, "value": round(E * newton * world / t, 1), "unit": "tets/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3 / args.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic (seeded jitter and log-normal mu, numpy PCG64)",
        "config": {"workload": WORKLOAD, "precision": "mixed", "newton": mixed | {"prec": "mixed"},
                   "load_levels": [s[0] for s in per_step],
                   "l2": "inputs (K 182 MB fp32, LU 182 MB) exceed the 126 MB L2",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "newton_solve_s": [round(x, 3) for x in paths],
        "newton_iters": newton, "pcg_iters": pcg,
        "per_step": [{"level": a, "newton": b, "pcg": c, "backtracks": d, "s": round(s, 3)}
                     for (a, b, c, d), s in zip(per_step, step_s)],
        "tets": E, "tets_evaluated": tets_eval,
        "tets_note": "value counts all 6 tets per hex; the split's zero-volume sliver of each "
                     "hex (stored volume 0, skipped as the reference skips it) is in the count",
        "e2e": {"value": round(E * e_newton * world / te, 1), "unit": "tets/s",
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                "newton_solve_s": round(te, 3), "same_result": e2e_same},
        "gpu_launches": int(launches), "profile": prof,
        "profile_note": "kernel classes from one complete load path replayed with the event "
                        "profiler on; replay bit-identical to the timed path: " + str(replay_same),
        "roofline": roof,
        "fp64_compare": fp,
        "clocks": clk.summary(),
    }
    return line, ctx, P


def ref_mesher():
    """the unit cube of the reference's own generate_unit_cube_mesh
    (oracle/_ref), else the oracle's restatement of it"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O

    R = O.ref()
    if R is None:
        return O.unit_cube, "oracle port"

    def mesh(N):
        import ctypes as C
        h = R.ref_mesh_new(N)
        nn, ne, nl = C.c_uint32(), C.c_uint32(), C.c_uint32()
        R.ref_mesh_sizes(h, C.byref(nn), C.byref(ne), C.byref(nl))
        xyz = np.zeros(3 * nn.value)
        conn = np.zeros(4 * ne.value, np.uint32)
        vol = np.zeros(ne.value)
        p = np.zeros(nn.value + 1, np.uint32)
        l = np.zeros(max(nl.value, 1), np.uint32)
        R.ref_mesh_get(h, xyz, conn, vol, p, l)
        R.ref_mesh_free(h)
        return xyz, conn

    return mesh, "reference generate_unit_cube_mesh"


_PATTERN = {}


def cpu_sample(P, pcg_per_newton, threads, pcg_sample=3):
    """One bounded sample of the reference CPU path on the scale-up block:
    the reference's own assemble_global_threadlocal (oracle/_ref, all
    threads; its per-call hash map included), the bit-identical O(nnz)
    ILU(0) port and pcg_sample PCG-ILU(0) iterations of the port.  Returns
    (timed seconds, extrapolated seconds of one Newton iteration = t_asm +
    t_ilu + pcg_per_newton * t_pcg_iteration, kind, text)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nn = P.n_nodes
    key = (P.N, nn)
    if key not in _PATTERN:
        _PATTERN[key] = O.pattern(nn, P.conn, "solve")
    rp, ci = _PATTERN[key]
    u = np.zeros(P.xyz.size)
    R = O.ref()
    t0 = time.perf_counter()
    if R is not None:
        # the reference's assembly takes one (E, nu) per problem; the
        # element kernel's cost does not depend on E, so the median E of the
        # block stands in for the per-element field
        K = np.zeros(ci.size)
        f = np.zeros(P.xyz.size)
        R.ref_assemble(nn, P.xyz, P.n_elems, P.conn, P.elem_volume, P.E, P.nu, u, rp, ci, K, f,
                       threads)
        kind = "reference"
    else:
        mu, lam = P.lame()
        slot = O.slot_map(nn, P.conn, rp, ci)
        t0 = time.perf_counter()
        K, f = O.assemble(P.xyz, P.conn, mu, lam, P.nu, u, slot, ci.size,
                          (P.elem_volume >= 1e-30).astype(np.uint8))
        kind = "port"
    t_asm = time.perf_counter() - t0
    Rv = -f
    O.apply_bc(rp, ci, K, Rv, P.mask)
    Rv = np.random.default_rng(0).standard_normal(Rv.size)
    Rv[P.mask == 1] = 0
    t0 = time.perf_counter()
    O.ilu0(rp, ci, K)
    t_ilu = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.pcg_ilu0(rp, ci, K, Rv, tol=1e-300, max_iter=pcg_sample)
    t_pcg = (time.perf_counter() - t0) / pcg_sample
    t_newton = t_asm + t_ilu + pcg_per_newton * t_pcg
    timed = t_asm + t_ilu + pcg_sample * t_pcg
    text = (f"N={P.N}: assembly {t_asm:.2f}s ({kind} assemble_global_threadlocal, {threads} "
            f"threads), ILU(0) {t_ilu:.2f}s (O(nnz) port bit-identical to the reference's, 1 "
            f"thread), PCG-ILU(0) {t_pcg:.3f}s per iteration (port, 1 thread); one Newton "
            f"iteration = assembly + ILU(0) + {pcg_per_newton:.1f} PCG iterations")
    return timed, t_newton, kind, text


def measured_pcg_per_newton():
    """FP64 PCG iterations per Newton iteration of this load path, measured
    on the GPU (same stop test, iteration counts equal to the reference's)
    and committed with the bench summary under profiles/"""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                p = line.split()
                if len(p) == 3 and p[0] == "machine-readable:" and p[1] == "fp64_pcg_per_newton":
                    return float(p[2]), os.path.basename(path)
    return 300.0, "default estimate"


def run_reference(args, rank, world):
    """The reference's own CPU implementation on the host cores; rank 0 only."""
    if rank != 0:
        return None
    from flexmesh_b200 import configs

    mesher, mesh_kind = ref_mesher()
    P = configs.scaleup_block(args.N, mesher=mesher)
    threads = os.cpu_count() or 1
    k, k_src = measured_pcg_per_newton()
    timed, vals = [], []
    for i in range(args.warmup + args.steps):
        ts, tn, kind, text = cpu_sample(P, k, threads)
        if i >= args.warmup:
            timed.append(ts)
            vals.append(tn)
    t_newton = sum(vals) / len(vals)
    v = P.n_elems / t_newton
    return {"metric": METRIC, "value": round(v, 1), "unit": "tets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * sum(timed) / len(timed), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "precision": "fp64 (the reference has no mixed path)",
                       "mesh": mesh_kind},
            "step": "one bounded sample per step: assembly + ILU(0) + 3 PCG-ILU(0) iterations "
                    "(ms_per_step is its measured time)",
            "value_formula": f"n_tets / (t_asm + t_ilu + {k:.1f} t_pcg_iteration): one Newton "
                             f"iteration, PCG count per Newton iteration from {k_src}",
            "newton_iteration_s": round(t_newton, 3),
            "cpu_baseline": {"value": round(v, 1), "unit": "tets/s", "cores": threads,
                             "kind": kind, "sample": text},
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
        if not args.no_cpu_baseline:
            fp = line.get("fp64_compare") or {}
            k = fp["pcg"] / max(fp["newton"], 1) if fp else measured_pcg_per_newton()[0]
            try:
                ts, tn, kind, text = cpu_sample(P, k, os.cpu_count() or 1)
                line["cpu_baseline"] = {"value": round(P.n_elems / tn, 1), "unit": "tets/s",
                                        "cores": os.cpu_count() or 1, "kind": kind,
                                        "sample": text + f" ({k:.1f}: this run's FP64 count)"}
            except Exception as e:  # the checker must not break the GPU line
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
