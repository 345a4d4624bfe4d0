"""The request server at the serving workload's shape (smaller n): 64
factors cycling through the 2D Laplacian, power-law (Zipf 2.1, rows up to
1000 entries) and banded-chain structures, plans analysed for one
right-hand side (the server reserves its batch width at admission), a
batch width of 32, FP32 sweeps + FP64 refinement, requests of 1..16
right-hand sides in device arrays and in host arrays, submitted in bursts
so that batches fill.  Every column is checked against the serial FP64
oracle and against the same column solved alone (relative 2-norm error
<= 1e-12 for both)."""
import numpy as np
import pytest

import rbs
from _util import rel_err
from oracle import oracle

TOL = 1e-12
pytestmark = pytest.mark.gpu


def factors(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(40000))))
        kind = i % 3
        if kind == 0:
            L = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=max(2, int(round(np.sqrt(n)))), seed=9000 + i)
        elif kind == 1:
            L = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=n, zipf_alpha=2.1, zipf_max=1000, seed=9000 + i)
        else:
            L = rbs.gen_lower_csr(rbs.GEN_CHAIN, n=n, chain_bw=3, seed=9000 + i)
        out.append(L)
    return out


def test_server_at_serving_shape(cuda):
    import torch
    facs = factors(64, 31)
    srv = rbs.Server(hbm_budget_bytes=40 << 30, max_batch_rhs=32)
    fids, alone = [], []
    for L in facs:
        fids.append(srv.add_factor(rbs.analyse(*L, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)))
        alone.append(rbs.analyse(*L, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR))
    rng = np.random.default_rng(77)
    reqs = []
    for q in range(300):
        f = int(rng.integers(0, 64))
        k = int(rng.integers(1, 17))
        rp, ci, va = facs[f]
        n = len(rp) - 1
        X = np.stack([rbs.gen_uniform(50000 + 20 * q + c, n) for c in range(k)])
        B = np.ascontiguousarray(np.stack([oracle.spmv_csr(rp, ci, va, X[c]) for c in range(k)]))
        on_device = q % 2 == 0
        r = dict(f=f, k=k, B=B, device=on_device)
        if on_device:
            r["dB"] = torch.tensor(B.reshape(-1), device=cuda)
            r["dX"] = torch.full_like(r["dB"], float("nan"))
        else:
            r["X"] = np.full_like(B, np.nan)
        reqs.append(r)
    # bursts of 60 requests, waited on in submission order
    for lo in range(0, len(reqs), 60):
        tickets = []
        for r in reqs[lo:lo + 60]:
            if r["device"]:
                tickets.append(srv.submit_device(fids[r["f"]], r["dB"], r["dX"], k=r["k"], prec=rbs.PREC_MIXED))
            else:
                tickets.append(srv.submit(fids[r["f"]], r["B"], r["X"], k=r["k"], prec=rbs.PREC_MIXED))
        for t, r in zip(tickets, reqs[lo:lo + 60]):
            lat, bk = srv.wait(t)
            assert lat > 0 and r["k"] <= bk <= 32
    st = srv.stats()
    assert st.completed == len(reqs) and st.mean_batch_rhs > 1
    for r in reqs:
        rp, ci, va = facs[r["f"]]
        n = len(rp) - 1
        X = r["dX"].cpu().numpy().reshape(r["k"], n) if r["device"] else r["X"]
        dB = torch.tensor(r["B"].reshape(-1), device=cuda)
        dXa = torch.empty_like(dB)
        alone[r["f"]].solve(dB, dXa, k=r["k"], prec=rbs.PREC_MIXED)
        Xa = dXa.cpu().numpy().reshape(r["k"], n)
        for c in range(r["k"]):
            xo = oracle.sptrsv_csr(rp, ci, va, rbs.FORWARD, r["B"][c])
            assert rel_err(X[c], xo) <= TOL, (r["f"], c)
            assert rel_err(X[c], Xa[c]) <= TOL, (r["f"], c)
    srv.close()


def test_reserve_then_solve_wider_and_narrower(cuda):
    # work vectors reserved for 32 columns: solves of 1..32 columns, FP64 and
    # mixed, in any order, all against the oracle
    import torch
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=20000, zipf_alpha=2.1, zipf_max=1000, seed=5)
    n = len(rp) - 1
    plan = rbs.analyse(rp, ci, va, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
    plan.reserve(32)
    for k in (32, 1, 17, 3, 32, 8):
        X = np.stack([rbs.gen_uniform(300 + c, n) for c in range(k)])
        B = np.stack([oracle.spmv_csr(rp, ci, va, X[c]) for c in range(k)])
        dB = torch.tensor(B.reshape(-1), device=cuda)
        for prec in (rbs.PREC_FP64, rbs.PREC_MIXED):
            dX = torch.empty_like(dB)
            plan.solve(dB, dX, k=k, prec=prec)
            got = dX.cpu().numpy().reshape(k, n)
            for c in range(k):
                assert rel_err(got[c], oracle.sptrsv_csr(rp, ci, va, rbs.FORWARD, B[c])) <= TOL, (k, prec, c)


def test_server_group_serves_members_in_one_launch(cuda):
    # twelve small factors as one group (a block-diagonal plan), next to two
    # single factors: requests of all members share launches (the server's
    # batch count stays far below the request count), host and device
    # arrays, FP64 and mixed; every column against the oracle and against the
    # same factor solved alone
    import torch
    facs = factors(14, 53)
    facs = [f for f in facs if len(f[0]) - 1 <= 12000][:12] + facs[:2]
    members, singles = facs[:-2], facs[-2:]
    srv = rbs.Server(hbm_budget_bytes=40 << 30, max_batch_rhs=16)
    gplan, offs = rbs.batch_analyse([tuple(L) for L in members], substitution=rbs.FORWARD, fmt=rbs.FMT_CSR)
    fids = srv.add_group(gplan, offs)
    fids += [srv.add_factor(rbs.analyse(*L, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)) for L in singles]
    alone = [rbs.analyse(*L, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR) for L in facs]
    rng = np.random.default_rng(91)
    reqs = []
    for q in range(160):
        f = int(rng.integers(0, len(facs)))
        k = int(rng.integers(1, 5))
        rp, ci, va = facs[f]
        n = len(rp) - 1
        X = np.stack([rbs.gen_uniform(80000 + 20 * q + c, n) for c in range(k)])
        B = np.ascontiguousarray(np.stack([oracle.spmv_csr(rp, ci, va, X[c]) for c in range(k)]))
        prec = rbs.PREC_MIXED if q % 2 else rbs.PREC_FP64
        r = dict(f=f, k=k, B=B, prec=prec, device=q % 3 != 0)
        if r["device"]:
            r["dB"] = torch.tensor(B.reshape(-1), device=cuda)
            r["dX"] = torch.full_like(r["dB"], float("nan"))
        else:
            r["X"] = np.full_like(B, np.nan)
        reqs.append(r)
    tickets = []
    for r in reqs:
        if r["device"]:
            tickets.append(srv.submit_device(fids[r["f"]], r["dB"], r["dX"], k=r["k"], prec=r["prec"]))
        else:
            tickets.append(srv.submit(fids[r["f"]], r["B"], r["X"], k=r["k"], prec=r["prec"]))
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    assert st.completed == len(reqs)
    assert st.batches < len(reqs) / 2, st.batches  # members and requests shared launches
    for r in reqs:
        rp, ci, va = facs[r["f"]]
        n = len(rp) - 1
        X = r["dX"].cpu().numpy().reshape(r["k"], n) if r["device"] else r["X"]
        dB = torch.tensor(r["B"].reshape(-1), device=cuda)
        dXa = torch.empty_like(dB)
        alone[r["f"]].solve(dB, dXa, k=r["k"], prec=r["prec"])
        Xa = dXa.cpu().numpy().reshape(r["k"], n)
        for c in range(r["k"]):
            xo = oracle.sptrsv_csr(rp, ci, va, rbs.FORWARD, r["B"][c])
            assert rel_err(X[c], xo) <= TOL, (r["f"], c, r["prec"])
            assert rel_err(X[c], Xa[c]) <= TOL, (r["f"], c, r["prec"])
    srv.close()
