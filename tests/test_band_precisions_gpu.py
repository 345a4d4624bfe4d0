"""Band-scan triangles in every precision: chosen by the cost model on a
long chain, and by the tuner on a short one (the tuner picks kernels after
the device state exists, so the band-scan scratch must already fit)."""
import numpy as np
import pytest

import rbs
from _util import rel_err
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,select", [(200000, rbs.SELECT_AUTO), (1489, rbs.SELECT_TUNE), (20000, rbs.SELECT_TUNE)])
@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_band_scan_precisions(cuda, n, select, sub):
    import torch
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_CHAIN, n=n, chain_bw=4, seed=n + 3)
    if sub == rbs.FORWARD:
        A, (arp, aci, ava) = oracle.transpose(rp, ci, va), (rp, ci, va)
    else:
        A, (arp, aci, ava) = (rp, ci, va), oracle.transpose(rp, ci, va)
    plan = rbs.analyse(*A, substitution=sub, lv=-1 if n > 10000 else 0, opts=rbs.options(select=select, max_rhs=4))
    assert (plan.export("kernel") == rbs.K_BANDSCAN).any()
    k = 4
    X = np.stack([rbs.gen_uniform(20 + c, n) for c in range(k)])
    B = np.stack([oracle.spmv_csr(arp, aci, ava, X[c]) for c in range(k)])
    Xo = np.stack([oracle.sptrsv_csr(arp, aci, ava, sub, B[c]) for c in range(k)])
    for kk in (1, k):
        dB = torch.tensor(B[:kk], device=cuda).reshape(-1)
        for prec, tol in ((rbs.PREC_FP64, 1e-12), (rbs.PREC_FP32, 1e-4), (rbs.PREC_MIXED, 1e-12)):
            dX = torch.empty_like(dB)
            plan.solve(dB, dX, k=kk, prec=prec)
            got = dX.cpu().numpy().reshape(kk, n)
            for c in range(kk):
                assert rel_err(got[c], Xo[c]) <= tol, (kk, prec, c)


@pytest.mark.parametrize("bw", [1, 2, 7])
def test_band_scan_widths_many_ctas(cuda, bw):
    # one deep triangle (lv = 0) of 300,000 rows: band widths W = 1, 2 and 8
    # (chunks of 4 or 8 rows, so the maps pass spans more than a hundred CTAs
    # and the scan pass composes their totals), one and three columns, FP64
    # and mixed against the oracle
    import torch
    n = 300000
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_CHAIN, n=n, chain_bw=bw, seed=700 + bw)
    cp, ri, cv = oracle.transpose(rp, ci, va)
    plan = rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=0, opts=rbs.options(max_rhs=4))
    assert (plan.export("kernel") == rbs.K_BANDSCAN).all()
    k = 3
    X = np.stack([rbs.gen_uniform(50 + c, n) for c in range(k)])
    B = np.stack([oracle.spmv_csr(rp, ci, va, X[c]) for c in range(k)])
    Xo = np.stack([oracle.sptrsv_csr(rp, ci, va, rbs.FORWARD, B[c]) for c in range(k)])
    for kk in (1, k):
        dB = torch.tensor(B[:kk], device=cuda).reshape(-1)
        for prec in (rbs.PREC_FP64, rbs.PREC_MIXED):
            dX = torch.empty_like(dB)
            plan.solve(dB, dX, k=kk, prec=prec)
            got = dX.cpu().numpy().reshape(kk, n)
            for c in range(kk):
                assert rel_err(got[c], Xo[c]) <= 1e-12, (bw, kk, prec, c)
