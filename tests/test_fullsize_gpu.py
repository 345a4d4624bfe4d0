"""Parity at the benchmark configurations' full sizes (config 0, the three
config-1 structures forward and backward, the config-2 4M-row factor), FP64
and mixed precision, against the serial FP64 oracle."""
import numpy as np
import pytest

import rbs
from _util import rel_err
from oracle import oracle

TOL = 1e-12
pytestmark = pytest.mark.gpu

CONFIGS = {
    "c0_band": dict(kind=rbs.GEN_BAND_POISSON, n=16384, lam=6, band=512, seed=100),
    "c1a_laplace": dict(kind=rbs.GEN_LAPLACE2D, grid=1024, seed=101),
    "c1b_zipf": dict(kind=rbs.GEN_ZIPF, n=2000000, zipf_alpha=2.1, zipf_max=1000, seed=102),
    "c1c_chain": dict(kind=rbs.GEN_CHAIN, n=1000000, chain_bw=3, seed=103),
    "c2_band4m": dict(kind=rbs.GEN_BAND_POISSON, n=4000000, lam=10, band=4096, seed=104),
}


def build(cfg, sub):
    rp, ci, va = rbs.gen_lower_csr(**cfg)
    if sub == rbs.FORWARD:
        cp, ri, cv = oracle.transpose(rp, ci, va)
        arp, aci, ava = rp, ci, va
    else:
        cp, ri, cv = rp, ci, va
        arp, aci, ava = oracle.transpose(rp, ci, va)
    n = len(rp) - 1
    x = rbs.gen_uniform(cfg["seed"] + 7, n)
    b = oracle.spmv_csr(arp, aci, ava, x)
    xref = oracle.sptrsv_csr(arp, aci, ava, sub, b)
    return cp, ri, cv, b, xref


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
@pytest.mark.parametrize("name", ["c0_band", "c1a_laplace", "c1b_zipf", "c1c_chain"])
def test_fullsize_fp64(cuda, name, sub):
    import torch
    cp, ri, cv, b, xref = build(CONFIGS[name], sub)
    plan = rbs.analyse(cp, ri, cv, substitution=sub, lv=-1)
    db = torch.tensor(b, device=cuda)
    dx = torch.empty_like(db)
    plan.solve(db, dx)
    assert rel_err(dx.cpu().numpy(), xref) <= TOL
    dx2 = torch.empty_like(db)
    plan.solve(db, dx2, prec=rbs.PREC_MIXED)
    assert rel_err(dx2.cpu().numpy(), xref) <= TOL


def test_fullsize_config2(cuda):
    import torch
    cp, ri, cv, b, xref = build(CONFIGS["c2_band4m"], rbs.FORWARD)
    plan = rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=-1)
    db = torch.tensor(b, device=cuda)
    dx = torch.empty_like(db)
    st = plan.solve(db, dx, prec=rbs.PREC_MIXED)
    assert rel_err(dx.cpu().numpy(), xref) <= TOL, st.iterations
