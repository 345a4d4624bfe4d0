"""Which execution layouts a plan carries (host analysis, no GPU): outside
tuning the CTA sync-free kernel's ELL chunks exist only for level triangles
that have neither a staged level-ELL nor a level-chunk layout (the kernel
choice falls back to them only then); a tuning plan carries them for every
candidate, with the same chunks where both have them."""
import numpy as np
import pytest

import rbs
from oracle import oracle


def systems():
    yield "laplace", rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=120, seed=1)
    yield "band", rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=20000, lam=10, band=400, seed=2)
    yield "zipf", rbs.gen_lower_csr(rbs.GEN_ZIPF, n=20000, zipf_alpha=2.0, zipf_max=200, seed=3)


@pytest.mark.parametrize("name,csr", list(systems()), ids=lambda v: v if isinstance(v, str) else "")
def test_ell_only_where_it_can_run(name, csr):
    rp, ci, va = csr
    cp, ri, cv = oracle.transpose(rp, ci, va)
    plans = {sel: rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=-1,
                              opts=rbs.options(host_only=1, select=sel))
             for sel in (rbs.SELECT_AUTO, rbs.SELECT_TUNE)}
    auto = plans[rbs.SELECT_AUTO]
    eb = auto.export("ell_block").reshape(-1, 2)
    cb = auto.export("ca_block").reshape(-1, 4)
    lb = auto.export("lc_block").reshape(-1, 3)
    for b in range(len(eb)):
        if eb[b, 0] >= 0:
            assert cb[b, 0] < 0 and lb[b, 0] < 0, b
    tune = plans[rbs.SELECT_TUNE]
    te = tune.export("ell_block").reshape(-1, 2)
    assert (te[:, 0] >= 0).sum() >= (eb[:, 0] >= 0).sum()
    # where both plans carry a block's ELL chunks, they carry the same chunks
    ta, tc = tune.export("ell_chunks").reshape(-1, 4), auto.export("ell_chunks").reshape(-1, 4)
    for b in range(len(eb)):
        if eb[b, 0] >= 0 and te[b, 0] >= 0:
            assert eb[b, 1] == te[b, 1]
            np.testing.assert_array_equal(tc[eb[b, 0]:eb[b, 0] + eb[b, 1], :3], ta[te[b, 0]:te[b, 0] + te[b, 1], :3])
