"""Parity of the CUDA solve with the serial FP64 oracle (tolerance: relative
2-norm error <= 1e-12, the bound of the solve metric), through the
C ABI, on every golden case, both directions, every selection mode,
multi-RHS and mixed precision."""
import numpy as np
import pytest

import rbs
from _util import FIXTURES, load_fixture, rel_err
from oracle import oracle

TOL = 1e-12
pytestmark = pytest.mark.gpu


def system(cp, ri, va, sub, k=1, seed=5):
    """CSR of A (original numbering), right-hand sides and oracle solutions."""
    arp, aci, ava = oracle.transpose(cp, ri, va)  # CSC(A) -> CSR(A)
    n = len(cp) - 1
    X = np.stack([rbs.gen_uniform(seed + c, n) for c in range(k)])
    B = np.stack([oracle.spmv_csr(arp, aci, ava, X[c]) for c in range(k)])
    Xref = oracle.sptrsv_csr(arp, aci, ava, sub, B)
    return B, Xref


def solve(plan, B, dev, k=1, prec=rbs.PREC_FP64):
    import torch
    db = torch.tensor(np.ascontiguousarray(B), dtype=torch.float64, device=dev).reshape(-1)
    dx = torch.full_like(db, float("nan"))
    st = plan.solve(db, dx, k=k, prec=prec)
    return dx.cpu().numpy().reshape(B.shape), st


@pytest.mark.parametrize("select", [rbs.SELECT_AUTO, rbs.SELECT_REFERENCE])
@pytest.mark.parametrize("name", FIXTURES)
def test_golden_parity(cuda, name, select):
    g, cp, ri, va, sub, lv = load_fixture(name)
    B, Xref = system(cp, ri, va, sub)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(select=select))
    X, _ = solve(plan, B, cuda)
    assert rel_err(X, Xref) <= TOL
    # a second solve reuses the plan and its work vectors
    X2, _ = solve(plan, B, cuda)
    assert rel_err(X2, Xref) <= TOL


@pytest.mark.parametrize("k", [2, 3, 8, 32, 128, 130])
@pytest.mark.parametrize("name", ["band_lv3_fwd", "zipf_lv2_bwd", "longrows_lv2_fwd"])
def test_multi_rhs(cuda, name, k):
    g, cp, ri, va, sub, lv = load_fixture(name)
    B, Xref = system(cp, ri, va, sub, k=k)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(max_rhs=k))
    X, _ = solve(plan, B, cuda, k=k)
    for c in range(k):
        assert rel_err(X[c], Xref[c]) <= TOL, c


@pytest.mark.parametrize("name", ["band_auto_fwd", "laplace40_lv2_bwd", "zipf_lv3_fwd", "dense_lv2_fwd",
                                  "chain_method1_fwd", "longrows_lv2_bwd"])
@pytest.mark.parametrize("k", [1, 8])
def test_mixed_precision(cuda, name, k):
    g, cp, ri, va, sub, lv = load_fixture(name)
    B, Xref = system(cp, ri, va, sub, k=k)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(max_rhs=k))
    X, st = solve(plan, B, cuda, k=k, prec=rbs.PREC_MIXED)
    assert st.iterations >= 1
    for c in range(k):
        assert rel_err(X[c], Xref[c]) <= TOL, (c, st.iterations)


def test_fp32_sweep_is_single_precision_accurate(cuda):
    g, cp, ri, va, sub, lv = load_fixture("band_lv3_fwd")
    B, Xref = system(cp, ri, va, sub)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv)
    X, _ = solve(plan, B, cuda, prec=rbs.PREC_FP32)
    assert 1e-12 < rel_err(X, Xref) <= 1e-5


def test_host_api_and_reference_shim(cuda):
    import torch
    g, cp, ri, va, sub, lv = load_fixture("band_auto_fwd")
    B, Xref = system(cp, ri, va, sub)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv)
    X, st = plan.solve_host(B[0])
    assert rel_err(X, Xref[0]) <= TOL and st.ms > 0
    n = len(cp) - 1
    d_cp = torch.tensor(cp, dtype=torch.int32, device=cuda)
    d_ri = torch.tensor(ri, dtype=torch.int32, device=cuda)
    d_va = torch.tensor(va, dtype=torch.float64, device=cuda)
    d_b = torch.tensor(B[0], dtype=torch.float64, device=cuda)
    d_x = torch.zeros(n, dtype=torch.float64, device=cuda)
    import os
    os.environ["RBS_BENCH_REPEAT"] = "3"
    cal, pre = rbs.recblocking_solver_cuda(d_cp, d_ri, d_va, n, n, len(ri), d_x, d_b, sub, lv)
    assert cal > 0 and pre > 0
    assert rel_err(d_x.cpu().numpy(), Xref[0]) <= TOL
    np.testing.assert_array_equal(d_b.cpu().numpy(), B[0])  # b is left untouched


def test_async_and_external_stream(cuda):
    import torch
    g, cp, ri, va, sub, lv = load_fixture("zipf_lv2_fwd")
    B, Xref = system(cp, ri, va, sub)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv)
    s = torch.cuda.Stream()
    plan.set_stream(s.cuda_stream)
    db = torch.tensor(B[0], dtype=torch.float64, device=cuda)
    dx = torch.empty_like(db)
    torch.cuda.synchronize()
    plan.solve_async(db, dx)
    plan.sync()
    assert rel_err(dx.cpu().numpy(), Xref[0]) <= TOL
    plan.set_stream(None)


def test_device_analysis_entry(cuda):
    import torch
    g, cp, ri, va, sub, lv = load_fixture("laplace40_lv2_fwd")
    n = len(cp) - 1
    plan = rbs.analyse_device(torch.tensor(cp, dtype=torch.int32, device=cuda),
                              torch.tensor(ri, dtype=torch.int32, device=cuda),
                              torch.tensor(va, dtype=torch.float64, device=cuda), n, len(ri), substitution=sub, lv=lv)
    np.testing.assert_array_equal(plan.export("levelItem"), g["ref_levelItem"])
    B, Xref = system(cp, ri, va, sub)
    X, _ = solve(plan, B, cuda)
    assert rel_err(X, Xref) <= TOL


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
@pytest.mark.parametrize("grid", [64, 300])
def test_multi_rhs_staged_level_triangles(cuda, grid, sub):
    # 2D-Laplacian factors: their triangles run the staged level kernel with
    # one CTA per group of two right-hand-side columns; widths 8 and up also
    # take the transposing gather and scatter (odd widths leave padding
    # columns in the last group).  Every column against the oracle, FP64 and mixed
    # at 1e-12, FP32 at single precision.
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=grid, seed=grid + sub)
    cp, ri, cv = oracle.transpose(rp, ci, va) if sub == rbs.FORWARD else (rp, ci, va)
    plan = rbs.analyse(cp, ri, cv, substitution=sub, lv=-1, opts=rbs.options(max_rhs=128))
    kern = plan.export("kernel")
    assert (kern[0::2] == rbs.K_LEVEL).sum() >= 1
    for k in (2, 5, 8, 32, 64, 100, 128):
        B, Xref = system(cp, ri, cv, sub, k=k, seed=7 * k)
        for prec, tol in ((rbs.PREC_FP64, TOL), (rbs.PREC_MIXED, TOL), (rbs.PREC_FP32, 1e-5)):
            X, _ = solve(plan, B, cuda, k=k, prec=prec)
            for c in range(k):
                assert rel_err(X[c], Xref[c]) <= tol, (k, prec, c)


@pytest.mark.parametrize("select", [rbs.SELECT_AUTO, rbs.SELECT_TUNE])
def test_overlapped_walk_alternating_widths(cuda, select):
    # grouped multi-column solves move the columns inside the block walk
    # (triangle by triangle, on a second stream) and leave the x work vector
    # without its sentinel; a single-column walk afterwards (under TUNE it may
    # poll for the sentinel) refills it first.  Widths, precisions and a
    # leading dimension larger than n alternate, twice (eager, then graph
    # replays); every column against the oracle.
    import torch
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=200, seed=41)
    cp, ri, cv = oracle.transpose(rp, ci, va)
    n = len(cp) - 1
    plan = rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=-1, opts=rbs.options(select=select))
    seq = [(8, rbs.PREC_FP64, n), (1, rbs.PREC_FP64, n), (8, rbs.PREC_FP32, n), (8, rbs.PREC_MIXED, n),
           (1, rbs.PREC_FP64, n), (3, rbs.PREC_FP64, n + 7), (1, rbs.PREC_FP32, n), (16, rbs.PREC_FP64, n)]
    for rep in range(2):
        for q, (k, prec, ld) in enumerate(seq):
            B, Xref = system(cp, ri, cv, rbs.FORWARD, k=k, seed=1000 * rep + 50 * q)
            hb = np.zeros((k, ld))
            hb[:, :n] = B
            db = torch.tensor(hb, dtype=torch.float64, device=cuda).reshape(-1)
            dx = torch.full_like(db, float("nan"))
            plan.solve(db, dx, k=k, ld=ld, prec=prec)
            X = dx.cpu().numpy().reshape(k, ld)
            assert np.isnan(X[:, n:]).all(), (rep, q)  # padding rows of the caller's columns untouched
            tol = 1e-5 if prec == rbs.PREC_FP32 else TOL
            for c in range(k):
                assert rel_err(X[c, :n], Xref[c]) <= tol, (rep, q, k, prec, c)


def test_host_async_pipelined(cuda):
    # several asynchronous host-array solves in flight on two staging slots,
    # pinned buffers, widths 1 and 3 (a wider call drains and regrows the
    # slots), FP64 and FP32; mixed runs synchronously; all against the oracle
    import torch
    g, cp, ri, va, sub, lv = load_fixture("laplace40_lv2_fwd")
    n = len(cp) - 1
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv)
    jobs = []
    for q, (k, prec) in enumerate([(1, rbs.PREC_FP64)] * 4 + [(3, rbs.PREC_FP64), (1, rbs.PREC_FP32),
                                                              (3, rbs.PREC_MIXED), (1, rbs.PREC_FP64)]):
        B, Xref = system(cp, ri, va, sub, k=k, seed=100 + 10 * q)
        hb = torch.empty(k * n, dtype=torch.float64, pin_memory=True)
        hx = torch.full((k * n,), float("nan"), dtype=torch.float64, pin_memory=True)
        hb.copy_(torch.from_numpy(np.ascontiguousarray(B).reshape(-1)))
        plan.solve_host_async(hb.numpy(), hx.numpy(), k=k, prec=prec)
        jobs.append((k, prec, Xref, hb, hx))
    plan.sync()
    for k, prec, Xref, hb, hx in jobs:
        X = hx.numpy().reshape(k, n)
        tol = 1e-5 if prec == rbs.PREC_FP32 else TOL
        for c in range(k):
            assert rel_err(X[c], Xref[c]) <= tol, (k, prec, c)
