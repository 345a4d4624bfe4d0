"""The value oracle's own rounding error is far below the 1e-12 parity
tolerance: plain serial substitution against the same substitution with
Neumaier-compensated row sums (oracle.c) on the structures the GPU parity
tests use, both directions, agree to 1e-14 relative (2-norm), and both
recover a known solution (b = L x_true) to 1e-12.  The level-scheduled
threaded substitution (the benchmark's CPU baseline) equals the serial one
bit for bit."""
import numpy as np
import pytest

import rbs
from oracle import oracle


def structures():
    yield "laplace", rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=200, seed=3)
    yield "band", rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=60000, lam=8, band=512, seed=4)
    yield "zipf", rbs.gen_lower_csr(rbs.GEN_ZIPF, n=60000, zipf_alpha=2.1, zipf_max=1000, seed=5)
    yield "chain", rbs.gen_lower_csr(rbs.GEN_CHAIN, n=60000, chain_bw=3, seed=6)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name,csr", list(structures()), ids=lambda v: v if isinstance(v, str) else "")
@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_oracle_error_is_below_the_parity_tolerance(name, csr, sub):
    rp, ci, va = csr
    if sub == rbs.BACKWARD:  # U = L^T: L's CSC is U's CSR
        rp, ci, va = oracle.transpose(rp, ci, va)
    n = len(rp) - 1
    x_true = rbs.gen_uniform(17, n)
    b = oracle.spmv_csr(rp, ci, va, x_true)
    x = oracle.sptrsv_csr(rp, ci, va, sub, b)
    xc = oracle.sptrsv_csr(rp, ci, va, sub, b, compensated=True)
    assert rel(x, xc) <= 1e-14
    assert rel(x, x_true) <= 1e-12 and rel(xc, x_true) <= 1e-12


@pytest.mark.parametrize("name,csr", list(structures()), ids=lambda v: v if isinstance(v, str) else "")
@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_level_scheduled_cpu_solve_equals_serial(name, csr, sub):
    # the benchmark's threaded CPU baseline (oracle.LevelSolver) gives the
    # serial substitution's x bit for bit at any thread count
    rp, ci, va = csr
    if sub == rbs.BACKWARD:
        rp, ci, va = oracle.transpose(rp, ci, va)
    b = rbs.gen_uniform(23, len(rp) - 1)
    x = oracle.sptrsv_csr(rp, ci, va, sub, b)
    lvl = oracle.LevelSolver(rp, ci, va, sub)
    for threads in (0, 1, 3, 8):  # 0: serial over the rows' own order
        assert np.array_equal(lvl.solve(b, threads=threads).view(np.uint64), x.view(np.uint64)), threads
