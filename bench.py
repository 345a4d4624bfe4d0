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
  python bench.py --side analysis|batched|blocks|ic0|ilu0|mtx|serve [--case c1b]

The headline value is timed on the block walk replayed from its CUDA graph;
the roofline's per-kernel times come from a second pass of the same steps
with CUDA events around every block.  Side measurements (multi-RHS, other
structures, mixed precision, analysis, factors, Matrix Market input,
batched systems, serving) follow on one GPU; --side runs one alone.

N > 1 runs N independent replicas (the solve has no data-path collective:
a triangular solve is one dependency chain), one process per GPU launched by
torch.distributed.run; value = all ranks' solves / max-over-ranks time.
The reference arm (--impl reference) times the CPU implementation of the
path on the host: the reference ships no CPU triangular solve, so this is the
fastest of the oracle's serial FP64 substitution and its level-scheduled
substitution over the level-ordered matrix on 1..all host threads (oracle/),
chosen untimed.
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
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-sweep", action="store_true", help="skip the structure/variant side measurements")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-system batched measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving measurement")
    ap.add_argument("--case", default="c1a", choices=["c1a", "c1b", "c1c", "c2r", "c0"],
                    help="structure of the timed solve (profiling runs; the benchmark line is c1a)")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, side measurements and the CPU baseline "
                                                               "(short runs for profilers)")
    ap.add_argument("--side", default=None, choices=sorted(SIDE_FUNCS),
                    help="run one side measurement alone on cuda:0 and print its JSON (no benchmark line)")
    ap.add_argument("--ks", default="1,8,32,64,128", help="right-hand-side counts of the multi_rhs side measurement")
    ap.add_argument("--precs", default="fp64,mixed", help="precisions of the multi_rhs side measurement")
    ap.add_argument("--sides", default=None,
                    help="comma-separated side measurements to run after the benchmark line's own "
                         f"(default: {','.join(SIDE_DEFAULT)}; each in a child process)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- inputs ----
FORWARD, BACKWARD = 0, 1
SPECS = {
    "c1a": dict(kind=1, grid=1024, seed=101),
    "c1b": dict(kind=2, n=2000000, zipf_alpha=2.1, zipf_max=1000, seed=102),
    "c1c": dict(kind=3, n=1000000, chain_bw=3, seed=103),
    "c0": dict(kind=0, n=16384, lam=6, band=512, seed=100),
    "c2r": dict(kind=0, n=4000000, lam=10, band=4096, seed=104),
}


def make_system(kind, sub, seed_x=1, gen=None):
    """Seeded L (or U = L^T), its CSC input, b and x_true.  `gen` supplies
    gen_lower_csr / gen_uniform: the library's generator for this
    library's arm, the oracle's bit-identical restatement (oracle/gen.c,
    tests/test_oracle_gen.py) for the CPU arm, which must not load the
    library under test."""
    import scipy.sparse as sp

    if gen is None:
        import rbs as gen
    rp, ci, va = gen.gen_lower_csr(**SPECS[kind])
    n = len(rp) - 1
    L = sp.csr_matrix((va, ci, rp), shape=(n, n))
    A = L if sub == FORWARD else L.T.tocsr()
    csc = A.tocsc()
    csc.sort_indices()
    x_true = gen.gen_uniform(SPECS[kind]["seed"] + seed_x, n)
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
def cpu_candidates():
    """Thread counts tried for the CPU arm: 1, 2, 4, ... up to the host
    threads this process may use, and that count itself."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    ts, t = [], 1
    while t < n:
        ts.append(t)
        t *= 2
    return ts + [n]


def cpu_best(system, reps=3):
    """The fastest CPU configuration for the system's forward solve, chosen
    untimed: the oracle's serial FP64 substitution (1 thread, over a copy of
    the rows with the diagonal apart) or its level-scheduled substitution
    over the level-ordered matrix on T host threads (T from
    cpu_candidates()).  Returns (name, threads, solve
    function b -> x, reference solution).  Both give the same x bit for bit;
    the level order's analysis is done once, outside any timing, as the
    reference's preprocessing is."""
    from oracle import oracle

    A = system["A"]
    rp, ci, va = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    b = system["b"]
    x_serial = oracle.sptrsv_csr(rp, ci, va, FORWARD, b)
    lvl = oracle.LevelSolver(rp, ci, va, FORWARD)
    cands = [("serial substitution", 1, lambda bb: lvl.solve(bb, threads=0))]
    for t in cpu_candidates():
        cands.append(("level-scheduled substitution", t, lambda bb, t=t: lvl.solve(bb, threads=t)))
    best = None
    for name, t, fn in cands:
        x = fn(b)
        if not np.array_equal(x, x_serial):
            continue
        dt = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn(b)
            dt.append(time.perf_counter() - t0)
        if best is None or min(dt) < best[0]:
            best = (min(dt), name, t, fn)
    return best[1], best[2], best[3], x_serial


def cpu_timed(fn, b, budget_s, max_reps):
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_reps and time.perf_counter() < t_end:
        t0 = time.perf_counter()
        fn(b)
        times.append(time.perf_counter() - t0)
    return times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    sysm = make_system("c1a", FORWARD, gen=oracle)
    name, threads, fn, _ = cpu_best(sysm)
    for _ in range(args.warmup):
        fn(sysm["b"])
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        x = fn(sysm["b"])
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps / total
    err = float(np.linalg.norm(x - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))
    import platform
    arm = (f"{name} in FP64 on the host, {threads} thread(s): the fastest of the oracle's serial substitution and "
           f"its level-scheduled substitution on 1..{cpu_candidates()[-1]} threads (the reference has no CPU solve; "
           "oracle/oracle.c)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "arm": arm},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full c1a forward solves, {name}; inputs from the oracle's "
                                   "generator (bit-identical to the library's)",
                         "cpu": platform.processor() or "x86_64", "nproc": os.cpu_count()},
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


def replica_throughput(rank_total_ms, steps, world, allmax):
    """Whole-job solves/s of `world` independent replicas that each timed
    `steps` solves: all ranks' solves over the slowest rank's time (max over
    ranks, `allmax`), and that time per step."""
    total = allmax(rank_total_ms)
    return world * steps * 1000.0 / total, total / steps


def rel(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


def measure(plan, dB, dX, flush, reps, k=1, prec=0):
    """Mean device ms of `reps` solves after two warm-up solves."""
    timed_solves(plan, dB, dX, 2, flush, k=k, prec=prec)
    ms, st = timed_solves(plan, dB, dX, reps, flush, k=k, prec=prec)
    return float(np.mean(ms)), st


def side_multi_rhs(dev, args):
    """Multi-RHS column blocks on the 2D-Laplacian factor: k in {1, 8, 32,
    128}, FP64 and FP32 sweeps + FP64 refinement.  Columns of X_true are
    U(-1,1); B = L X_true."""
    import torch

    import rbs

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    sysm = make_system("c1a", FORWARD)
    plan = rbs.analyse(sysm["cp"], sysm["ri"], sysm["cv"], substitution=FORWARD, lv=-1)
    out = {}
    reps = max(3, args.steps // 10)
    A = sysm["A"]
    precs = [(nm, p) for nm, p in (("fp64", rbs.PREC_FP64), ("mixed", rbs.PREC_MIXED)) if nm in args.precs.split(",")]
    for k in [int(v) for v in args.ks.split(",")]:
        Xt = np.stack([sysm["x_true"]] + [rbs.gen_uniform(1000 + c, sysm["n"]) for c in range(1, k)])
        B = np.ascontiguousarray((A @ Xt.T).T)
        dB = torch.tensor(B, dtype=torch.float64, device=dev).reshape(-1)
        dX = torch.empty_like(dB)
        for pname, prec in precs:
            ms, st = measure(plan, dB, dX, flush, reps, k=k, prec=prec)
            X = dX.cpu().numpy().reshape(k, -1)
            out[f"{pname}_k{k}"] = {"solves_per_s": k * 1000.0 / ms, "ms": ms, "iterations": st.iterations,
                                    "rel_err_vs_x_true": max(rel(X[c], Xt[c]) for c in range(k)),
                                    "useful_gb": st.useful_bytes / 1e9, "moved_gb": st.moved_bytes / 1e9,
                                    "gb_per_s": st.useful_bytes / (ms / 1000) / 1e9}
        del dB, dX
    if "fp64_k1" in out:
        base = out["fp64_k1"]["solves_per_s"]
        for v in out.values():
            v["x_plain_fp64_k1"] = v["solves_per_s"] / base
    return out


def side_structures(dev, args):
    """Config-1 structures and directions other than the headline."""
    import torch

    import rbs

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    sweep = {}
    for kind, sub in (("c1a", rbs.BACKWARD), ("c1b", rbs.FORWARD), ("c1b", rbs.BACKWARD), ("c1c", rbs.FORWARD),
                      ("c1c", rbs.BACKWARD)):
        s2 = make_system(kind, sub)
        p2 = rbs.analyse(s2["cp"], s2["ri"], s2["cv"], substitution=sub, lv=-1)
        d_b = torch.tensor(s2["b"], dtype=torch.float64, device=dev)
        d_x = torch.empty_like(d_b)
        ms, st = measure(p2, d_b, d_x, flush, max(3, args.steps // 10))
        xs = d_x.cpu().numpy()
        inf2 = p2.info()
        sweep[f"{kind}_{'fwd' if sub == 0 else 'bwd'}"] = {
            "solves_per_s": 1000.0 / ms, "ms": ms, "gb_per_s": st.useful_bytes / (ms / 1000) / 1e9,
            "rel_err_vs_x_true": rel(xs, s2["x_true"]), "n": s2["n"], "nnz": s2["nnz"], "nlevel": inf2.nlevel,
            "lv": inf2.lv, "analyse_ms": inf2.analyse_ms,
            "kernels": {rbs.KERNEL_NAMES[i]: inf2.kernels[i] for i in range(7) if inf2.kernels[i]}}
        del p2
    return sweep


def side_analysis(dev, args):
    """Analysis time: host (rbs_analyse on host arrays) against device
    (rbs_analyse_device on device arrays: level sets, reordering and the
    processing-order CSR on the GPU, the execution layout on the host); the
    integer outputs are identical (tests/test_device_analysis_gpu.py)."""
    import torch

    import rbs

    out = {}
    # one warm-up device analysis: the first call loads the kernels
    w = make_system("c0", rbs.FORWARD)
    wd = [torch.tensor(w[k], device=dev) for k in ("cp", "ri", "cv")]
    rbs.analyse_device(wd[0], wd[1], wd[2], w["n"], w["nnz"], substitution=rbs.FORWARD, lv=-1,
                       opts=rbs.options(host_only=1))
    for kind in ("c1a", "c1b", "c1c", "c2r"):
        s2 = make_system(kind, rbs.FORWARD)
        t0 = time.perf_counter()
        ph = rbs.analyse(s2["cp"], s2["ri"], s2["cv"], substitution=rbs.FORWARD, lv=-1, opts=rbs.options(host_only=1))
        host_s = time.perf_counter() - t0
        d = [torch.tensor(s2[k], device=dev) for k in ("cp", "ri", "cv")]
        times = []
        for _ in range(3):  # the first call of a size also loads the kernels it needs
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            pd = rbs.analyse_device(d[0], d[1], d[2], s2["n"], s2["nnz"], substitution=rbs.FORWARD, lv=-1,
                                    opts=rbs.options(host_only=1))
            times.append(time.perf_counter() - t0)
        dev_s = min(times[1:])
        same = bool((ph.export("levelItem") == pd.export("levelItem")).all() and
                    (ph.export("recblock_Index") == pd.export("recblock_Index")).all())
        out[kind] = {"n": s2["n"], "nnz": s2["nnz"], "nlevel": ph.info().nlevel,
                     "host_ms": 1000 * host_s, "device_path_ms": 1000 * dev_s, "device_path_first_call_ms": 1000 * times[0],
                     "device_part_ms": float(pd.export("analyse_ms")[1]),
                     "level_search_on_device": bool(pd.export("analyse_ms")[2]), "identical": same}
        del ph, pd, d
    return out


def side_ilu0(dev, args):
    """ILU(0) of the full 2D 5-point Laplacian pattern on a 1024 x 1024 grid
    (both triangles, U(-1,1) values, dominant diagonal) on the device, and
    one preconditioner apply z = U^-1 L^-1 b through this library's plans."""
    import scipy.sparse as sp
    import torch

    import rbs

    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=1024, seed=401)
    n = len(rp) - 1
    S = sp.tril(sp.csr_matrix((va, ci, rp), shape=(n, n)), k=-1).tocsr()
    T = S.T.tocsr()
    T.data = np.random.default_rng(402).uniform(-1, 1, T.nnz)
    off = (S + T).tocsr()
    A = (off + sp.diags(1.0 + np.asarray(abs(off).sum(axis=1)).ravel())).tocsr()
    A.sort_indices()
    d = [torch.tensor(a, device=dev) for a in (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data)]
    dlu = torch.empty_like(d[2])
    rbs.ilu0_device(d[0], d[1], d[2], dlu)  # first call loads the kernels
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rbs.ilu0_device(d[0], d[1], d[2], dlu)
        times.append(time.perf_counter() - t0)
    lu = dlu.cpu().numpy()
    # split into L (unit diagonal written out) and U, plans for both
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    low = A.indices < rows
    Lm = (sp.csr_matrix((lu[low], A.indices[low], np.r_[0, np.cumsum(np.bincount(rows[low], minlength=n))]),
                        shape=(n, n)) + sp.identity(n, format="csr")).tocsr()
    Um = sp.csr_matrix((lu[~low], A.indices[~low], np.r_[0, np.cumsum(np.bincount(rows[~low], minlength=n))]),
                       shape=(n, n))
    Lm.sort_indices()
    Um.sort_indices()
    Lp = rbs.analyse(Lm.indptr.astype(np.int32), Lm.indices.astype(np.int32), Lm.data, substitution=rbs.FORWARD,
                     lv=-1, fmt=rbs.FMT_CSR)
    Up = rbs.analyse(Um.indptr.astype(np.int32), Um.indices.astype(np.int32), Um.data, substitution=rbs.BACKWARD,
                     lv=-1, fmt=rbs.FMT_CSR)
    db = torch.tensor(rbs.gen_uniform(403, n), device=dev)
    y, z = torch.empty_like(db), torch.empty_like(db)
    apply_ms = []
    for _ in range(5):
        a = Lp.solve(db, y).ms
        apply_ms.append(a + Up.solve(y, z).ms)
    return {"n": n, "nnz": int(A.nnz), "factor_ms": 1000 * float(np.median(times)),
            "apply_ms": float(np.median(apply_ms[1:])),
            "apply_kernels": {"L": rbs.KERNEL_NAMES[int(np.bincount(Lp.export("kernel")).argmax())],
                              "U": rbs.KERNEL_NAMES[int(np.bincount(Up.export("kernel")).argmax())]}}


def side_mtx(dev, args):
    """Matrix Market input (main.cu:120-236's steps): the 2D 5-point
    Laplacian pattern on a 1024 x 1024 grid in symmetric storage with
    U(-1,1) values written %.17g, read and expanded to CSR on the device
    (rbs_mtx_read), then cut into the forward triangle's CSC
    (rbs_mtx_triangle).  CPU side: the reference's own mmio_info +
    mmio_data (oracle/_ref/mtx_dump when built, else the oracle's reader),
    then the oracle's triangle extraction and transposition.  The file is
    in the page cache for both sides."""
    import tempfile

    import torch

    import rbs
    from oracle import oracle

    rp, ci, _ = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=1024, seed=77)
    va = rbs.gen_uniform(78, len(ci))
    n = len(rp) - 1
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "laplace2d_1024.mtx")
        rbs.mtx_write(path, rp, ci, va, symmetric=True)
        size = os.path.getsize(path)
        M = rbs.mtx_read(path)  # first call: page cache, kernels, pinned staging
        M.triangle(rbs.FORWARD, rbs.FMT_CSC)
        reads, parses, tris, totals = [], [], [], []
        for _ in range(5):
            del M
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            M = rbs.mtx_read(path)
            t1 = time.perf_counter()
            p, x, v = M.triangle(rbs.FORWARD, rbs.FMT_CSC)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            reads.append(M.info.read_ms)
            parses.append(M.info.parse_ms)
            tris.append(1000 * (t2 - t1))
            totals.append(1000 * (t2 - t0))
        ref_ms = oracle.reference_mtx_ms(path)
        t0 = time.perf_counter()
        o = oracle.mtx_read(path)
        t1 = time.perf_counter()
        tp, ti, tv = oracle.tri_extract(o["rowptr"], o["colidx"], o["val"], rbs.FORWARD)
        cp, cr, cv = oracle.transpose(tp, ti, tv)
        t2 = time.perf_counter()
        drp, dci, dva = M.csr()
        same = bool(np.array_equal(drp.cpu().numpy(), o["rowptr"]) and np.array_equal(dci.cpu().numpy(), o["colidx"])
                    and np.array_equal(dva.cpu().numpy().view(np.uint64), o["val"].view(np.uint64))
                    and np.array_equal(p.cpu().numpy(), cp) and np.array_equal(x.cpu().numpy(), cr)
                    and np.array_equal(v.cpu().numpy().view(np.uint64), cv.view(np.uint64)))
        read_cpu_ms = ref_ms if ref_ms is not None else 1000 * (t1 - t0)
        cpu_total = read_cpu_ms + 1000 * (t2 - t1)
        gpu_total = float(np.median(totals))
        return {"file_mb": size / 1e6, "entries_file": int(M.info.nnz_file), "entries_csr": int(M.info.nnz), "n": n,
                "device_ms": {"read_to_hbm": float(np.median(reads)), "parse_to_csr": float(np.median(parses)),
                              "triangle_csc": float(np.median(tris)), "total": gpu_total},
                "file_gb_per_s": size / (gpu_total * 1e6), "host_values": int(M.info.host_values),
                "cpu_ms": {"read": read_cpu_ms,
                           "read_by": "reference mmio_info + mmio_data" if ref_ms is not None else "oracle port",
                           "extract_transpose": 1000 * (t2 - t1), "total": cpu_total},
                "speedup_vs_cpu": cpu_total / gpu_total, "identical": same}


def side_ic0(dev, args):
    """IC(0) of the 2D 5-point Laplacian on a 1024 x 1024 grid given as its
    lower triangle (U(-1,1) off-diagonal values, dominant diagonal) on the
    device, and one preconditioner apply z = L^-T L^-1 b: L through a CSR
    forward plan, L^T through the same arrays read as CSC (backward)."""
    import scipy.sparse as sp
    import torch

    import rbs

    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=1024, seed=411)
    n = len(rp) - 1
    S = sp.tril(sp.csr_matrix((va, ci, rp), shape=(n, n)), k=-1).tocsr()
    S = sp.csr_matrix((np.random.default_rng(412).uniform(-1, 1, S.nnz), S.indices, S.indptr), shape=(n, n))
    Lo = (S + sp.diags(1.0 + np.asarray(abs(S + S.T).sum(axis=1)).ravel())).tocsr()
    Lo.sort_indices()
    h = (Lo.indptr.astype(np.int32), Lo.indices.astype(np.int32), Lo.data)
    d = [torch.tensor(a, device=dev) for a in h]
    dl = torch.empty_like(d[2])
    rbs.ic0_device(d[0], d[1], d[2], dl)  # first call loads the kernels
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rbs.ic0_device(d[0], d[1], d[2], dl)
        times.append(time.perf_counter() - t0)
    l = dl.cpu().numpy()
    Lp = rbs.analyse(h[0], h[1], l, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
    Ltp = rbs.analyse(h[0], h[1], l, substitution=rbs.BACKWARD, lv=-1, fmt=rbs.FMT_CSC)
    db = torch.tensor(rbs.gen_uniform(413, n), device=dev)
    y, z = torch.empty_like(db), torch.empty_like(db)
    apply_ms = []
    for _ in range(5):
        a = Lp.solve(db, y).ms
        apply_ms.append(a + Ltp.solve(y, z).ms)
    return {"n": n, "nnz_lower": int(Lo.nnz), "factor_ms": 1000 * float(np.median(times)),
            "apply_ms": float(np.median(apply_ms[1:]))}


def side_mixed(dev, args):
    """FP32 sweeps + FP64 refinement against the plain FP64 solve on the
    2D-Laplacian factor, the power-law factor and the n = 4M Poisson(10)
    band-4096 factor; errors against the serial FP64 oracle."""
    import torch

    import rbs
    from oracle import oracle

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {}
    for kind in ("c1a", "c1b", "c2r"):
        s2 = make_system(kind, rbs.FORWARD)
        A = s2["A"]
        xo = oracle.sptrsv_csr(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, rbs.FORWARD, s2["b"])
        p2 = rbs.analyse(s2["cp"], s2["ri"], s2["cv"], substitution=rbs.FORWARD, lv=-1)
        d_b = torch.tensor(s2["b"], dtype=torch.float64, device=dev)
        d_x = torch.empty_like(d_b)
        reps = max(3, args.steps // 10)
        ms64, st64 = measure(p2, d_b, d_x, flush, reps)
        e64 = rel(d_x.cpu().numpy(), xo)
        msmx, stmx = measure(p2, d_b, d_x, flush, reps, prec=rbs.PREC_MIXED)
        emx = rel(d_x.cpu().numpy(), xo)
        out[kind] = {"n": s2["n"], "nnz": s2["nnz"], "nlevel": p2.info().nlevel,
                     "fp64": {"ms": ms64, "solves_per_s": 1000.0 / ms64, "rel_err_vs_oracle": e64,
                              "gb_per_s": st64.useful_bytes / (ms64 / 1000) / 1e9},
                     "mixed": {"ms": msmx, "solves_per_s": 1000.0 / msmx, "rel_err_vs_oracle": emx,
                               "iterations": stmx.iterations, "useful_gb": stmx.useful_bytes / 1e9,
                               "moved_gb": stmx.moved_bytes / 1e9,
                               "gb_per_s_useful": stmx.useful_bytes / (msmx / 1000) / 1e9}}
        del p2, d_b, d_x
    return out


def side_batched(dev, args):
    """512 independent lower-triangular systems (n log-uniform in [1k, 200k],
    Poisson(8) off-diagonals in a band of 256, one RHS each) solved as one
    block-diagonal plan (one graph-captured walk, measured kernel choice),
    against the plain FP64 path: each system alone through its own plan."""
    import torch

    import rbs

    rng = np.random.default_rng(303)
    ns = np.exp(rng.uniform(np.log(1000), np.log(200000), 512)).astype(int)
    systems, bs, xts = [], [], []
    for i, n in enumerate(ns):
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=int(n), lam=8, band=256, seed=5000 + i)
        xt = rbs.gen_uniform(9000 + i, int(n))
        import scipy.sparse as sp
        b = sp.csr_matrix((va, ci, rp), shape=(int(n), int(n))) @ xt
        systems.append((rp, ci, va))
        bs.append(b)
        xts.append(xt)
    t0 = time.perf_counter()
    plan, offs = rbs.batch_analyse(systems, substitution=rbs.FORWARD, fmt=rbs.FMT_CSR,
                                   opts=rbs.options(select=rbs.SELECT_TUNE))
    t_an = time.perf_counter() - t0
    B = np.concatenate(bs)
    Xt = np.concatenate(xts)
    dB = torch.tensor(B, dtype=torch.float64, device=dev)
    dX = torch.empty_like(dB)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    res = {"systems": 512, "rows": int(ns.sum()), "nnz": int(sum(len(s[1]) for s in systems)),
           "analyse_s": t_an, "nlevel": plan.info().nlevel, "lv": plan.info().lv}
    for pname, prec in (("fp64", rbs.PREC_FP64), ("mixed", rbs.PREC_MIXED)):
        ms, st = measure(plan, dB, dX, flush, 5, prec=prec)
        X = dX.cpu().numpy()
        err = max(rel(X[offs[i]:offs[i + 1]], xts[i]) for i in range(512))
        res[f"batched_{pname}"] = {"ms": ms, "solves_per_s": 512 * 1000.0 / ms, "iterations": st.iterations,
                                   "max_rel_err_vs_x_true": err, "gb_per_s": st.useful_bytes / (ms / 1000) / 1e9}
    del plan, dB, dX
    # plain FP64, one plan and one solve per system (warm L2: conservative for the ratio)
    plain_ms = 0.0
    perr = 0.0
    for i, (rp, ci, va) in enumerate(systems):
        p1 = rbs.analyse(rp, ci, va, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
        d_b = torch.tensor(bs[i], dtype=torch.float64, device=dev)
        d_x = torch.empty_like(d_b)
        for _ in range(2):
            p1.solve(d_b, d_x)
        ms = [p1.solve(d_b, d_x).ms for _ in range(3)]
        plain_ms += float(np.mean(ms))
        perr = max(perr, rel(d_x.cpu().numpy(), xts[i]))
        del p1
    res["plain_fp64_per_system"] = {"ms_total": plain_ms, "solves_per_s": 512 * 1000.0 / plain_ms,
                                    "max_rel_err_vs_x_true": perr}
    for pname in ("fp64", "mixed"):
        res[f"batched_{pname}"]["x_plain_fp64"] = res[f"batched_{pname}"]["solves_per_s"] / \
            res["plain_fp64_per_system"]["solves_per_s"]
    return res


def serving_factors(count=64, seed=404):
    """64 factors, n log-uniform in [10k, 2M], structures cycling through
    the 2D Laplacian, power-law rows and the banded chain."""
    import rbs

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        kind = i % 3
        if kind == 0:
            L = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=max(2, int(round(np.sqrt(n)))), seed=7000 + i)
        elif kind == 1:
            L = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=n, zipf_alpha=2.1, zipf_max=1000, seed=7000 + i)
        else:
            L = rbs.gen_lower_csr(rbs.GEN_CHAIN, n=n, chain_bw=3, seed=7000 + i)
        out.append(L)
    return out


def side_serving(dev, args, n_requests=1000, loads=(500, 1000, 2000, 10000, 50000), batch_rhs=32):
    """Poisson request arrivals over 64 device-resident factors; each
    request carries 1-16 right-hand sides in device arrays; the server
    batches within factors (one multi-RHS solve per batch, columns read in
    place) and across them (batches of all factors overlap on the device),
    once with FP32 sweeps + FP64 refinement and once in FP64 (the solves are
    latency-bound, so the FP64 sweep, one walk instead of two or three, is
    the faster choice here), and once more in FP64 with the small factors
    served in groups (one block-diagonal plan per group: requests of
    different factors share a launch).  Baselines, on the same arrivals and
    device arrays: one plain FP64 rbs_solve of each request's k columns in
    arrival order on the caller's thread, and the plain FP64 single-RHS path
    (one rbs_solve per right-hand side, back to back)."""
    import threading

    import torch

    import rbs

    facs = serving_factors()
    ns = [len(L[0]) - 1 for L in facs]
    t0 = time.perf_counter()
    plans = [rbs.analyse(*L, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR) for L in facs]
    t_an = time.perf_counter() - t0
    rng = np.random.default_rng(505)
    # per factor: 16 right-hand-side columns and a 16-column output area on
    # the device (a request of k columns uses the first k)
    dB = [torch.tensor(rbs.gen_uniform(11000 + i, 16 * n), device=dev) for i, n in enumerate(ns)]
    dX = [torch.empty_like(b) for b in dB]
    res = {"factors": 64, "rows": int(sum(ns)), "nnz": int(sum(len(L[1]) for L in facs)), "analyse_s": t_an,
           "requests_per_load": n_requests, "rhs_per_request": "uniform 1..16", "max_batch_rhs": batch_rhs,
           "hbm_budget_gb": 150, "requests": "device arrays (rbs_server_submit_device)", "loads": {}}

    def schedule(rate):
        gaps = rng.exponential(1.0 / rate, n_requests)
        return np.cumsum(gaps), rng.integers(0, 64, n_requests), rng.integers(1, 17, n_requests)

    scheds = {rate: schedule(rate) for rate in loads}
    for p in plans:  # the plain arms run at the widest request too: work vectors and graphs exist before timing
        p.reserve(16)
    for f in range(64):
        for k in (1, 16):
            for _ in range(2):
                plans[f].solve(dB[f], dX[f], k=k)
    # plain: one FP64 solve per request, in arrival order, on the caller's thread
    plain = {}
    for rate in loads:
        arr, fid, ks = scheds[rate]
        lat = []
        torch.cuda.synchronize()
        t_start = time.perf_counter()
        for a, f, k in zip(arr, fid, ks):
            while time.perf_counter() - t_start < a:
                pass
            plans[f].solve(dB[f], dX[f], k=int(k))
            lat.append(time.perf_counter() - t_start - a)
        span = time.perf_counter() - t_start
        plain[rate] = {"p50_ms": 1000 * float(np.percentile(lat, 50)), "p99_ms": 1000 * float(np.percentile(lat, 99)),
                       "solves_per_s": float(ks.sum()) / span, "requests_per_s": n_requests / span}
    # plain FP64 single-RHS path: one solve per right-hand side, back to back,
    # on the first 200 requests of the 1000 req/s schedule
    arr, fid, ks = scheds[loads[1] if len(loads) > 1 else loads[0]]
    torch.cuda.synchronize()
    t_start = time.perf_counter()
    nsol = 0
    for f, k in zip(fid[:200], ks[:200]):
        n = ns[f]
        for c in range(int(k)):
            plans[f].solve(dB[f][c * n:(c + 1) * n], dX[f][c * n:(c + 1) * n], k=1)
            nsol += 1
    single = nsol / (time.perf_counter() - t_start)
    res["plain_fp64_single_rhs"] = {"solves_per_s": single, "sample": "first 200 requests, one solve per RHS"}
    srv = rbs.Server(150 << 30, max_batch_rhs=batch_rhs)
    old_si = sys.getswitchinterval()
    sys.setswitchinterval(1e-4)  # the submit loop and the waiter share the interpreter
    fids = [srv.add_factor(p) for p in plans]
    plans = None
    # warm-up: every factor once at one and at 16 columns, in both served
    # precisions (captures the block walks)
    for f in range(64):
        for k in (1, 16):
            for prec in (rbs.PREC_MIXED, rbs.PREC_FP64):
                srv.wait(srv.submit_device(fids[f], dB[f], dX[f], k=k, prec=prec))

    def serve(rate, prec, srv, fids):
        arr, fid, ks = scheds[rate]
        srv.reset_stats()
        tickets = []
        lats = []
        failure = []

        def waiter():
            try:
                for i in range(n_requests):
                    while i >= len(tickets):
                        time.sleep(0)
                    lats.append(srv.wait(tickets[i])[0])
            except Exception as e:  # handed to the main thread below
                failure.append(e)

        th = threading.Thread(target=waiter)
        th.start()
        lag = []
        t_start = time.perf_counter()
        try:
            for a, f, k in zip(arr, fid, ks):
                while time.perf_counter() - t_start < a:
                    pass
                lag.append(1000 * (time.perf_counter() - t_start - a))
                tickets.append(srv.submit_device(fids[f], dB[f], dX[f], k=int(k), prec=prec))
        finally:
            th.join()
        if failure:
            raise failure[0]
        span = time.perf_counter() - t_start
        lats = np.array(lats) + np.array(lag)  # latency from the scheduled arrival, as for the plain arm
        st = srv.stats()
        return {"p50_ms": float(np.percentile(lats, 50)), "p99_ms": float(np.percentile(lats, 99)),
                "solves_per_s": float(ks.sum()) / span, "requests_per_s": n_requests / span,
                "mean_batch_rhs": st.mean_batch_rhs, "batches": st.batches}

    try:
        for rate in loads:
            row = {"served_mixed": serve(rate, rbs.PREC_MIXED, srv, fids),
                   "served_fp64": serve(rate, rbs.PREC_FP64, srv, fids), "plain_fp64": plain[rate]}
            for arm in ("served_mixed", "served_fp64"):
                row[f"{arm}_x_plain_fp64"] = row[arm]["solves_per_s"] / plain[rate]["solves_per_s"]
                row[f"{arm}_x_plain_fp64_single_rhs"] = row[arm]["solves_per_s"] / single
            res["loads"][str(rate)] = row
        # accuracy: every factor once, b = L x_true, served mixed vs x_true
        import scipy.sparse as sp
        worst = 0.0
        for i, (rp, ci, va) in enumerate(facs):
            xt = rbs.gen_uniform(13000 + i, ns[i])
            b = torch.tensor(sp.csr_matrix((va, ci, rp), shape=(ns[i], ns[i])) @ xt, device=dev)
            x = torch.empty_like(b)
            srv.wait(srv.submit_device(fids[i], b, x, k=1, prec=rbs.PREC_MIXED))
            worst = max(worst, rel(x.cpu().numpy(), xt))
        res["max_rel_err_vs_x_true"] = worst
        srv.close()
        srv = None
        # Grouped: the small Laplacian and power-law factors (<= 100k rows)
        # in groups of up to 16, each group one block-diagonal plan whose
        # batches solve requests of all its members in one launch; chains
        # stay alone (a group walks as deep as its deepest member).  FP64.
        srv = rbs.Server(150 << 30, max_batch_rhs=batch_rhs)
        small = [i for i in range(64) if ns[i] <= 100000 and i % 3 != 2]
        gids = [None] * 64
        for g0 in range(0, len(small), 16):
            mem = small[g0:g0 + 16]
            gplan, offs = rbs.batch_analyse([tuple(facs[i]) for i in mem], substitution=rbs.FORWARD, fmt=rbs.FMT_CSR)
            for i, fid_i in zip(mem, srv.add_group(gplan, offs)):
                gids[i] = fid_i
        for i in range(64):
            if gids[i] is None:
                gids[i] = srv.add_factor(rbs.analyse(*facs[i], substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR))
        for f in range(64):
            for k in (1, 16):
                srv.wait(srv.submit_device(gids[f], dB[f], dX[f], k=k, prec=rbs.PREC_FP64))
        res["grouped"] = {"groups": (len(small) + 15) // 16, "members": len(small),
                          "rule": "Laplacian and power-law factors of <= 100k rows, up to 16 per group"}
        for rate in loads:
            row = res["loads"][str(rate)]
            row["served_fp64_grouped"] = serve(rate, rbs.PREC_FP64, srv, gids)
            row["served_fp64_grouped_x_plain_fp64_single_rhs"] = row["served_fp64_grouped"]["solves_per_s"] / single
        worst = 0.0
        for i in small:
            rp, ci, va = facs[i]
            xt = rbs.gen_uniform(13000 + i, ns[i])
            b = torch.tensor(sp.csr_matrix((va, ci, rp), shape=(ns[i], ns[i])) @ xt, device=dev)
            x = torch.empty_like(b)
            srv.wait(srv.submit_device(gids[i], b, x, k=1, prec=rbs.PREC_FP64))
            worst = max(worst, rel(x.cpu().numpy(), xt))
        res["grouped"]["max_rel_err_vs_x_true"] = worst
    finally:
        sys.setswitchinterval(old_si)
        if srv is not None:
            srv.close()
    return res


def profiled_traffic(kind):
    """DRAM bytes (read + write) per launch of the dominant kernel from the
    committed ncu summary of the same workload (profiles/), or None."""
    path = {"level": os.path.join(ROOT, "profiles", "k_tri_level_ca_c1a.md")}.get(kind)
    if not path or not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def launches_per_solve(plan):
    import rbs
    kern = plan.export("kernel")
    lr = plan.export("longrow")
    mr = plan.export("medrow")
    return 2 + int((kern != rbs.K_EMPTY).sum()) + int((lr > 0).sum()) + int((mr > 0).sum())


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
    sysm = make_system(args.case, rbs.FORWARD)
    plan = rbs.analyse(sysm["cp"], sysm["ri"], sysm["cv"], substitution=rbs.FORWARD, lv=-1,
                       opts=rbs.options(max_rhs=32))
    info = plan.info()
    db = torch.tensor(sysm["b"], dtype=torch.float64, device=dev)
    dx = torch.empty_like(db)
    timed_solves(plan, db, dx, args.warmup, flush)  # the second solve captures the block walk's graph
    clocks = Clocks(dev.index)
    clocks.start()
    barrier()
    ms, st = timed_solves(plan, db, dx, args.steps, flush)
    barrier()
    clk = clocks.stop()
    x = dx.cpu().numpy()
    rel = float(np.linalg.norm(x - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))
    value, ms_per_step = replica_throughput(float(sum(ms)), args.steps, world, allmax)
    useful = st.useful_bytes
    # per-block device time -> dominant kernel kind and its roofline: the
    # same steps once more with CUDA events around every block (events force
    # eager launches instead of the graph replay, so this pass is slower and
    # is not the value above)
    plan.profile(True)
    barrier()
    pms, _ = timed_solves(plan, db, dx, args.steps, flush)
    barrier()
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
    traffic = profiled_traffic(rbs.KERNEL_NAMES[dom])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind, "kernel": rbs.KERNEL_NAMES[dom],
                "kernel_share": by_kind[dom][0] / max(sum(v[0] for v in by_kind.values()), 1e-30),
                "bytes_per_launch": dom_bytes_per_launch, "launch_ms": dom_launch_ms,
                "solve_frac": useful / (ms_per_step / 1000) / 1e9 / peak,
                "timing": "per-block CUDA events on the plan's stream, second pass of the same steps "
                          f"(eager launches: {float(np.mean(pms)):.3f} ms per solve against "
                          f"{ms_per_step:.3f} ms replayed from the graph)"}
    plan.profile(False)

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "solves/s", "ms_per_step": ms_per_step,
                              "case": args.case, "roofline": roofline, "note": "--no-extras run (profiling)"}))
        if world > 1:
            dist.destroy_process_group()
        return

    # end to end through the host-array API: pinned b and x, and every step
    # uploads its b and downloads its x.  Main figure: the asynchronous call
    # (rbs_solve_host_async) issued step after step, so a step's copies
    # overlap its neighbours' solves; the L2 flush runs on the plan's stream
    # between the solves, as for the device-timed value.  Also reported: one
    # synchronous call per step (rbs_solve_host), the copies in series.
    hb = torch.empty(sysm["n"], dtype=torch.float64, pin_memory=True)
    hx = torch.empty(sysm["n"], dtype=torch.float64, pin_memory=True)
    hb.copy_(torch.from_numpy(sysm["b"]))
    hbn, hxn = hb.numpy(), hx.numpy()
    plan.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    for _ in range(3):
        flush.zero_()
        plan.solve_host_async(hbn, hxn)
    plan.sync()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        plan.solve_host_async(hbn, hxn)
    plan.sync()
    e2e_async_total = allmax(time.perf_counter() - t0)
    e2e_rel = float(np.linalg.norm(hxn - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))
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
    e2e_sync_rel = float(np.linalg.norm(hxn - sysm["x_true"]) / np.linalg.norm(sysm["x_true"]))

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded stand-in for SuiteSparse inputs)",
        "config": {"workload": WORKLOAD if args.case == "c1a" else args.case, "global_batch": world,
                   "parallelism": f"replicas{world}",
                   "l2": "flushed before every timed solve (256 MB write)", "lv": info.lv,
                   "kernels": {rbs.KERNEL_NAMES[i]: info.kernels[i] for i in range(7) if info.kernels[i]}},
        "gb_per_s": useful / (ms_per_step / 1000) / 1e9,
        "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
        "rel_err_vs_x_true": rel,
        "roofline": roofline,
        # the single right-hand side is bounded by its dependency chain: every
        # one of the global levels needs the previous level's results
        "latency_floor": {"levels": info.nlevel, "us_per_level": 1000.0 * ms_per_step / max(info.nlevel, 1),
                          "hbm_time_us": useful / (peak * 1e9) * 1e6,
                          "note": "time per solve / global levels, against the HBM time of the useful bytes"},
        "e2e": {"value": world * args.steps / e2e_async_total, "unit": "solves/s",
                "h2d_bytes_per_step": 8 * sysm["n"], "d2h_bytes_per_step": 8 * sysm["n"], "rel_err_vs_x_true": e2e_rel,
                "path": "rbs_solve_host_async (C ABI, pinned host arrays, one upload and one download per step, "
                        "steps issued back to back, L2 flushed between solves on the plan's stream), wall clock "
                        "around all steps and the final rbs_plan_sync",
                "sync_call": {"value": world * args.steps / e2e_total, "unit": "solves/s",
                              "rel_err_vs_x_true": e2e_sync_rel,
                              "path": "rbs_solve_host per step (copies, solve and status check in series), "
                                      "wall clock per call"}},
        "gpu_launches": launches_per_solve(plan) * args.steps,
        "clocks": clk,
        "analyse_ms": info.analyse_ms,
    }

    del plan
    torch.cuda.empty_cache()
    if rank == 0 and world == 1:
        cname, cthreads, cfn, xo = cpu_best(sysm)
        times = cpu_timed(cfn, sysm["b"], budget_s=8.0, max_reps=200)
        import platform
        line["cpu_baseline"] = {"value": len(times) / sum(times), "unit": "solves/s", "cores": cthreads,
                                "kind": "port",
                                "sample": f"{len(times)} full c1a forward solves, {cname} in FP64, {cthreads} "
                                          "thread(s), the fastest CPU configuration",
                                "cpu": platform.processor() or "x86_64", "nproc": os.cpu_count()}
        line["rel_err_vs_oracle"] = float(np.linalg.norm(x - xo) / np.linalg.norm(xo))
    # side measurements (other configurations) on a single GPU only (with N
    # replicas they would repeat the same numbers N times), each in a process
    # of its own: a failing section is recorded, it cannot void this line
    if world == 1:
        for name in side_list(args):
            line[SIDE_KEYS[name]] = run_side(name, args)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


SIDE_KEYS = {"multi_rhs": "config3_multi_rhs_c1a", "structures": "sweep_config1", "mixed": "config2_mixed",
             "analysis": "analysis_host_vs_device", "ilu0": "ilu0_laplace2d_1024", "ic0": "ic0_laplace2d_1024",
             "mtx": "mtx_ingest_laplace2d_1024", "batched": "config3_batched_512", "serve": "config4_serving",
             "blocks": "blocks"}
SIDE_FUNCS = {"multi_rhs": "side_multi_rhs", "structures": "side_structures", "mixed": "side_mixed",
              "analysis": "side_analysis", "ilu0": "side_ilu0", "ic0": "side_ic0", "mtx": "side_mtx",
              "batched": "side_batched", "serve": "side_serving", "blocks": "side_blocks"}
SIDE_DEFAULT = ["multi_rhs", "structures", "mixed", "batched", "serve", "analysis", "ilu0", "ic0", "mtx"]


def side_list(args):
    if args.no_extras:
        return []
    if args.sides is not None:
        return [x for x in args.sides.split(",") if x]
    out = list(SIDE_DEFAULT)
    if args.no_sweep:
        out = [x for x in out if x not in ("multi_rhs", "structures", "mixed", "analysis", "ilu0", "ic0", "mtx")]
    if args.no_batch:
        out.remove("batched")
    if args.no_serve:
        out.remove("serve")
    return out


def run_side(name, args, timeout=900):
    """One side measurement in a child process (bench.py --side NAME): its
    JSON, or {"error": ...} with the end of its output."""
    cmd = [sys.executable, os.path.abspath(__file__), "--side", name, "--steps", str(args.steps), "--warmup",
           str(args.warmup), "--case", args.case]
    t0 = time.perf_counter()
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout} s"}
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        return {"error": f"exit {p.returncode}", "tail": (p.stderr or p.stdout)[-1500:], "wall_s": wall}
    for ln in reversed(p.stdout.strip().splitlines()):
        try:
            d = json.loads(ln)
        except ValueError:
            continue
        if isinstance(d, dict) and name in d:
            out = d[name]
            if isinstance(out, dict):
                out["wall_s"] = wall
            return out
    return {"error": "no JSON line", "tail": p.stdout[-1500:], "wall_s": wall}


def side_blocks(dev, args):
    """Per-block device time of the --case structure, forward and backward:
    CUDA events around every block (eager launches), the ten slowest blocks
    with their kernel, rows and entries, and the graph-replayed solve time."""
    import torch

    import rbs

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {}
    for sub, tag in ((rbs.FORWARD, "fwd"), (rbs.BACKWARD, "bwd")):
        s = make_system(args.case, sub)
        db = torch.tensor(s["b"], device=dev)
        dx = torch.empty_like(db)
        p = rbs.analyse(s["cp"], s["ri"], s["cv"], substitution=sub, lv=-1)
        ms, _ = measure(p, db, dx, flush, 20)
        p.profile(True)
        timed_solves(p, db, dx, 10, flush)
        bms, _, n = p.block_times()
        p.profile(False)
        kern, bm, bnnz = p.export("kernel"), p.export("blk_m"), p.export("blk_nnz")
        top = np.argsort(-np.asarray(bms))[:10]
        out[tag] = {"graph_ms": ms, "profiled_ms": float(sum(bms)) / max(n, 1),
                    "blocks": [{"block": int(b), "kernel": rbs.KERNEL_NAMES[int(kern[b])], "rows": int(bm[b]),
                                "entries": int(bnnz[b]), "ms": float(bms[b]) / max(n, 1)} for b in top]}
        del p
    return out


def main():
    args = parse()
    if args.side:
        import torch
        print(json.dumps({args.side: globals()[SIDE_FUNCS[args.side]](torch.device("cuda:0"), args)}))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
