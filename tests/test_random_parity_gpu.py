"""Randomised parity sweep: seeded structures of every generator kind at
several sizes, every recursion depth choice, both directions, the three
kernel-selection modes, FP64 / mixed / FP32 and several right-hand sides;
every solve against the serial FP64 oracle, and the device analysis against
the host analysis."""
import numpy as np
import pytest

import rbs
from _util import rel_err
from oracle import oracle

pytestmark = pytest.mark.gpu

SELECTS = [rbs.SELECT_REFERENCE, rbs.SELECT_AUTO, rbs.SELECT_TUNE]


def random_system(seed):
    rng = np.random.default_rng(seed)
    kind = seed % 5
    n = int(rng.integers(800, 20000))
    if kind == 0:
        return rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=float(rng.uniform(1, 14)),
                                 band=int(rng.integers(2, 2000)), seed=seed)
    if kind == 1:
        return rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=int(rng.integers(20, 140)), seed=seed)
    if kind == 2:
        return rbs.gen_lower_csr(rbs.GEN_ZIPF, n=n, zipf_alpha=float(rng.uniform(1.6, 2.6)),
                                 zipf_max=int(rng.integers(10, 3000)), seed=seed)
    if kind == 3:
        return rbs.gen_lower_csr(rbs.GEN_CHAIN, n=n, chain_bw=int(rng.integers(1, 6)), seed=seed)
    return rbs.gen_lower_csr(rbs.GEN_DIAG, n=n, seed=seed)


@pytest.mark.parametrize("seed", range(30))
def test_random_parity(cuda, seed):
    import torch
    rng = np.random.default_rng(1000 + seed)
    rp, ci, va = random_system(seed)
    n = len(rp) - 1
    sub = int(rng.integers(0, 2))
    lv = int(rng.choice([-1, 0, 1, 2, 3]))
    while lv > 0 and (1 << lv) > n:
        lv -= 1
    select = SELECTS[seed % 3]
    if sub == rbs.FORWARD:
        A, (arp, aci, ava) = oracle.transpose(rp, ci, va), (rp, ci, va)  # CSC of L; CSR of L
    else:
        A, (arp, aci, ava) = (rp, ci, va), oracle.transpose(rp, ci, va)  # CSC of U = L^T; CSR of U
    host = rbs.analyse(*A, substitution=sub, lv=lv, opts=rbs.options(select=select, max_rhs=8))
    d = [torch.tensor(np.asarray(a), device=cuda) for a in A]
    dev = rbs.analyse_device(d[0], d[1], d[2], n, len(A[1]), substitution=sub, lv=lv,
                             opts=rbs.options(select=select, host_only=1))
    for key in ("levelItem", "levelPtr", "recblock_Ptr", "recblock_Index", "method", "blk_nnz"):
        np.testing.assert_array_equal(dev.export(key), host.export(key), err_msg=key)
    k = int(rng.choice([1, 3, 8]))
    X = np.stack([rbs.gen_uniform(seed * 10 + c, n) for c in range(k)])
    B = np.stack([oracle.spmv_csr(arp, aci, ava, X[c]) for c in range(k)])
    Xo = np.stack([oracle.sptrsv_csr(arp, aci, ava, sub, B[c]) for c in range(k)])
    dB = torch.tensor(B, device=cuda).reshape(-1)
    for prec, tol in ((rbs.PREC_FP64, 1e-12), (rbs.PREC_MIXED, 1e-12), (rbs.PREC_FP32, 1e-4)):
        dX = torch.empty_like(dB)
        host.solve(dB, dX, k=k, prec=prec)
        got = dX.cpu().numpy().reshape(k, n)
        for c in range(k):
            assert rel_err(got[c], Xo[c]) <= tol, (prec, c)


@pytest.mark.parametrize("seed", range(10))
def test_random_batch_parity(cuda, seed):
    # many systems in one plan (one CTA per system in the level-chunk kernel,
    # or whatever the selection picks for the block-diagonal triangle)
    import torch
    rng = np.random.default_rng(5000 + seed)
    count = int(rng.integers(2, 12))
    systems = [random_system(100 * seed + i) for i in range(count)]
    sub = int(rng.integers(0, 2))
    select = SELECTS[seed % 3]
    inputs, csrs = [], []
    for rp, ci, va in systems:
        if sub == rbs.FORWARD:
            inputs.append(oracle.transpose(rp, ci, va))
            csrs.append((rp, ci, va))
        else:
            inputs.append((rp, ci, va))
            csrs.append(oracle.transpose(rp, ci, va))
    plan, offs = rbs.batch_analyse(inputs, substitution=sub, opts=rbs.options(select=select))
    bs, xs = [], []
    for i, (arp, aci, ava) in enumerate(csrs):
        n = len(arp) - 1
        b = oracle.spmv_csr(arp, aci, ava, rbs.gen_uniform(700 + i, n))
        bs.append(b)
        xs.append(oracle.sptrsv_csr(arp, aci, ava, sub, b))
    dB = torch.tensor(np.concatenate(bs), device=cuda)
    for prec, tol in ((rbs.PREC_FP64, 1e-12), (rbs.PREC_MIXED, 1e-12), (rbs.PREC_FP32, 1e-4)):
        dX = torch.empty_like(dB)
        plan.solve(dB, dX, prec=prec)
        X = dX.cpu().numpy()
        for i in range(count):
            assert rel_err(X[offs[i]:offs[i + 1]], xs[i]) <= tol, (prec, i)
