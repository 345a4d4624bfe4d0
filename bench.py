#!/usr/bin/env python
"""Benchmark of the recursive-block SpTRSV on B200.

Metric: solves/s at <= 1e-12 relative error (plus GB/s, p50/p99 latency).
Workload of the headline line: plain FP64 forward solve, 1 right-hand side,
lv = -1 (the reference's automatic rule), on the lower factor of the 2D
5-point Laplacian on a 1024 x 1024 grid (n = 1,048,576, nnz = 3,143,680,
2,047 levels).  Inputs are seeded synthetic stand-ins for the SuiteSparse
matrices the reference evaluates on (values U(-1,1), diagonal 1 + sum of
|off-diagonals|, x_true U(-1,1), b = L x_true).  L2 is flushed (a 256 MB
write) before every timed solve: the factor (58.7 MB) fits in the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs N independent replicas (the solve has no data-path collective:
a triangular solve is one dependency chain), one process per GPU launched by
torch.distributed.run; value = all ranks' solves / max-over-ranks time.
The reference arm (--impl reference) times the CPU implementation of the
path on the host: the reference ships no CPU triangular solve, so this is the
serial FP64 substitution port (oracle/), single-threaded.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "recblock-sptrsv_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "solves/s (plain FP64, 1 RHS, <=1e-12 rel err)"
WORKLOAD = "2D 5-pt Laplacian lower factor 1024x1024 (n=1048576, nnz=3143680, 2047 levels), forward, FP64, k=1, lv=-1"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-sweep", action="store_true", help="skip the structure/variant side measurements")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, side measurements and the CPU baseline "
                                                               "(short runs for profilers)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- inputs ----
def make_system(kind, sub, seed_x=1):
    """Seeded L (or U = L^T), its CSC input, b and x_true (numpy/scipy only)."""
    import scipy.sparse as sp

    import rbs

    specs = {
        "c1a": dict(kind=rbs.GEN_LAPLACE2D, grid=1024, seed=101),
        "c1b": dict(kind=rbs.GEN_ZIPF, n=2000000, zipf_alpha=2.1, zipf_max=1000, seed=102),
        "c1c": dict(kind=rbs.GEN_CHAIN, n=1000000, chain_bw=3, seed=103),
        "c0": dict(kind=rbs.GEN_BAND_POISSON, n=16384, lam=6, band=512, seed=100),
    }
    rp, ci, va = rbs.gen_lower_csr(**specs[kind])
    n = len(rp) - 1
    L = sp.csr_matrix((va, ci, rp), shape=(n, n))
    A = L if sub == rbs.FORWARD else L.T.tocsr()
    csc = A.tocsc()
    csc.sort_indices()
    x_true = rbs.gen_uniform(specs[kind]["seed"] + seed_x, n)
    b = A @ x_true
    return dict(n=n, nnz=A.nnz, cp=csc.indptr.astype(np.int32), ri=csc.indices.astype(np.int32),
                cv=csc.data.astype(np.float64), b=b, x_true=x_true, A=A)


# ---------------------------------------------------------------- clocks ----
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- reference ----
def cpu_serial(system, budget_s, max_reps):
    """Time the oracle's serial FP64 substitution (the CPU arm)."""
    from oracle import oracle

    A = system["A"]
    rp, ci, va = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    import rbs
    sub = rbs.FORWARD
    x = oracle.sptrsv_csr(rp, ci, va, sub, system["b"])  # warm-up + reference solution
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_reps and time.perf_counter() < t_end:
        t0 = time.perf_counter()
        oracle.sptrsv_csr(rp, ci, va, sub, system["b"])
        times.append(time.perf_counter() - t0)
    return x, times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sysm = make_system("c1a", 0)
    from oracle import oracle

    A = sysm["A"]
    rp, ci, va = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    for _ in range(args.warmup):
        oracle.sptrsv_csr(rp, ci, va, 0, sysm["b"])
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        x = oracle.sptrsv_csr(rp, ci, va, 0, sysm["b"])
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps / total
    err = float(np.linalg.norm(x - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))
    import platform
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "arm": "serial FP64 substitution on the host (the reference has no CPU "
                                               "solve; oracle/oracle.c), 1 thread"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": 1, "kind": "port",
                         "sample": f"{args.steps} full c1a forward solves", "cpu": platform.processor() or "x86_64",
                         "nproc": os.cpu_count()},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "rel_err_vs_x_true": err,
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ ours ----
def timed_solves(plan, db, dx, steps, flush, k=1, prec=0):
    import torch

    ms = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        st = plan.solve(db, dx, k=k, prec=prec)
        ms.append(st.ms)
    return ms, st


def launches_per_solve(plan):
    import rbs
    kern = plan.export("kernel")
    lr = plan.export("longrow")
    return 2 + int((kern != rbs.K_EMPTY).sum()) + int((lr > 0).sum())


def run_ours(args):
    import torch
    import torch.distributed as dist

    import rbs

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    def barrier():
        if world > 1:
            t = torch.zeros(1, device=dev)
            dist.all_reduce(t)
        torch.cuda.synchronize()

    def allmax(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    sysm = make_system("c1a", rbs.FORWARD)
    plan = rbs.analyse(sysm["cp"], sysm["ri"], sysm["cv"], substitution=rbs.FORWARD, lv=-1,
                       opts=rbs.options(max_rhs=32))
    info = plan.info()
    db = torch.tensor(sysm["b"], dtype=torch.float64, device=dev)
    dx = torch.empty_like(db)
    timed_solves(plan, db, dx, args.warmup, flush)
    plan.profile(True)
    clocks = Clocks(dev.index)
    clocks.start()
    barrier()
    ms, st = timed_solves(plan, db, dx, args.steps, flush)
    barrier()
    clk = clocks.stop()
    x = dx.cpu().numpy()
    rel = float(np.linalg.norm(x - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))
    total_ms = allmax(float(sum(ms)))
    value = world * args.steps * 1000.0 / total_ms
    ms_per_step = total_ms / args.steps
    useful = st.useful_bytes
    # per-block device time -> dominant kernel kind and its roofline
    bms, bbytes, solves = plan.block_times()
    kern = plan.export("kernel")
    by_kind = {}
    for b in range(len(kern)):
        d = by_kind.setdefault(int(kern[b]), [0.0, 0.0, 0])
        d[0] += bms[b]
        d[1] += bbytes[b]
        d[2] += 1
    dom = max(by_kind, key=lambda kk: by_kind[kk][0])
    dom_ms_per_solve = by_kind[dom][0] / max(solves, 1)
    dom_launch_ms = dom_ms_per_solve / by_kind[dom][2]
    dom_bytes_per_launch = by_kind[dom][1] / by_kind[dom][2]
    peak, peak_kind = peaks()
    achieved = dom_bytes_per_launch / (dom_launch_ms / 1000) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(rbs.KERNEL_NAMES[dom])
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind, "kernel": rbs.KERNEL_NAMES[dom],
                "kernel_share": by_kind[dom][0] / max(sum(v[0] for v in by_kind.values()), 1e-30),
                "bytes_per_launch": dom_bytes_per_launch, "launch_ms": dom_launch_ms,
                "solve_frac": useful / (ms_per_step / 1000) / 1e9 / peak}
    plan.profile(False)

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "solves/s", "ms_per_step": ms_per_step,
                              "roofline": roofline, "note": "--no-extras run (profiling)"}))
        if world > 1:
            dist.destroy_process_group()
        return

    # end to end through the host-array API (pinned buffers, H2D + solve + D2H per step)
    hb = torch.empty(sysm["n"], dtype=torch.float64, pin_memory=True)
    hx = torch.empty(sysm["n"], dtype=torch.float64, pin_memory=True)
    hb.copy_(torch.from_numpy(sysm["b"]))
    hbn, hxn = hb.numpy(), hx.numpy()
    for _ in range(2):
        plan.solve_host(hbn, x=hxn)
    e2e = []
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plan.solve_host(hbn, x=hxn)
        e2e.append(time.perf_counter() - t0)
    barrier()
    e2e_total = allmax(float(sum(e2e)))
    e2e_rel = float(np.linalg.norm(hxn - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded stand-in for SuiteSparse inputs)",
        "config": {"workload": WORKLOAD, "global_batch": world, "parallelism": f"replicas{world}",
                   "l2": "flushed before every timed solve (256 MB write)", "lv": info.lv,
                   "kernels": {rbs.KERNEL_NAMES[i]: info.kernels[i] for i in range(7) if info.kernels[i]}},
        "gb_per_s": useful / (ms_per_step / 1000) / 1e9,
        "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
        "rel_err_vs_x_true": rel,
        "roofline": roofline,
        "e2e": {"value": world * args.steps / e2e_total, "unit": "solves/s", "h2d_bytes_per_step": 8 * sysm["n"],
                "d2h_bytes_per_step": 8 * sysm["n"], "rel_err_vs_x_true": e2e_rel,
                "path": "rbs_solve_host (C ABI, pinned host arrays)"},
        "gpu_launches": launches_per_solve(plan) * args.steps,
        "clocks": clk,
        "analyse_ms": info.analyse_ms,
    }

    if not args.no_sweep:
        side = {}
        # precision / batching variants on the same factor
        for name, k, prec in (("mixed_k1", 1, rbs.PREC_MIXED), ("fp64_k8", 8, rbs.PREC_FP64),
                              ("mixed_k8", 8, rbs.PREC_MIXED), ("fp64_k32", 32, rbs.PREC_FP64),
                              ("mixed_k32", 32, rbs.PREC_MIXED)):
            B = np.stack([sysm["b"]] * k)
            dB = torch.tensor(B, dtype=torch.float64, device=dev).reshape(-1)
            dX = torch.empty_like(dB)
            timed_solves(plan, dB, dX, 2, flush, k=k, prec=prec)
            vms, vst = timed_solves(plan, dB, dX, max(3, args.steps // 10), flush, k=k, prec=prec)
            X = dX.cpu().numpy().reshape(k, -1)
            verr = max(float(np.linalg.norm(X[c] - sysm["x_true"]) / np.linalg.norm(sysm["x_true"])) for c in range(k))
            side[name] = {"solves_per_s": k * 1000.0 / float(np.mean(vms)), "ms": float(np.mean(vms)),
                          "iterations": vst.iterations, "rel_err_vs_x_true": verr,
                          "moved_gb": vst.moved_bytes / 1e9}
        line["variants_c1a"] = side
        del plan
        # the other config-1 structures and directions
        sweep = {}
        for kind, sub in (("c1a", rbs.BACKWARD), ("c1b", rbs.FORWARD), ("c1b", rbs.BACKWARD), ("c1c", rbs.FORWARD),
                          ("c1c", rbs.BACKWARD)):
            s2 = make_system(kind, sub)
            p2 = rbs.analyse(s2["cp"], s2["ri"], s2["cv"], substitution=sub, lv=-1)
            d_b = torch.tensor(s2["b"], dtype=torch.float64, device=dev)
            d_x = torch.empty_like(d_b)
            timed_solves(p2, d_b, d_x, 2, flush)
            sms, sst = timed_solves(p2, d_b, d_x, max(3, args.steps // 10), flush)
            xs = d_x.cpu().numpy()
            inf2 = p2.info()
            sweep[f"{kind}_{'fwd' if sub == 0 else 'bwd'}"] = {
                "solves_per_s": 1000.0 / float(np.mean(sms)), "ms": float(np.mean(sms)),
                "gb_per_s": sst.useful_bytes / (float(np.mean(sms)) / 1000) / 1e9,
                "rel_err_vs_x_true": float(np.linalg.norm(xs - s2["x_true"]) / np.linalg.norm(s2["x_true"])),
                "n": s2["n"], "nnz": s2["nnz"], "nlevel": inf2.nlevel, "lv": inf2.lv,
                "kernels": {rbs.KERNEL_NAMES[i]: inf2.kernels[i] for i in range(7) if inf2.kernels[i]}}
            del p2
        line["sweep_config1"] = sweep

    if rank == 0 and world == 1:
        xo, times = cpu_serial(sysm, budget_s=8.0, max_reps=200)
        import platform
        line["cpu_baseline"] = {"value": len(times) / sum(times), "unit": "solves/s", "cores": 1, "kind": "port",
                                "sample": f"{len(times)} full c1a forward solves, serial FP64 substitution",
                                "cpu": platform.processor() or "x86_64", "nproc": os.cpu_count()}
        line["rel_err_vs_oracle"] = float(np.linalg.norm(x - xo) / np.linalg.norm(xo))
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
