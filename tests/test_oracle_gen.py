"""The oracle's restatement of the seeded generators (oracle/gen.c) gives
the same arrays as the library's (include/rbs_gen.h) bit for bit, so the
CPU side of the benchmark can build its inputs without loading the library
under test.  Covers every kind, the benchmark's own specifications and
edge shapes (one row, Floyd sampling with k above and below 64, k equal to
the range)."""
import numpy as np
import pytest

import rbs
from oracle import oracle

SPECS = [
    dict(kind=rbs.GEN_BAND_POISSON, n=16384, lam=6, band=512, seed=100),        # the n = 16,384 case
    dict(kind=rbs.GEN_BAND_POISSON, n=3000, lam=90, band=120, seed=3),           # Floyd with k > 64
    dict(kind=rbs.GEN_BAND_POISSON, n=500, lam=30, band=8, seed=4),              # k capped at the range
    dict(kind=rbs.GEN_BAND_POISSON, n=2000, lam=4, band=0, seed=5),              # unbounded band
    dict(kind=rbs.GEN_LAPLACE2D, grid=1024, seed=101),                           # the 2D Laplacian 1024^2
    dict(kind=rbs.GEN_LAPLACE2D, grid=1, seed=9),
    dict(kind=rbs.GEN_ZIPF, n=200000, zipf_alpha=2.1, zipf_max=1000, seed=102),  # power-law rows
    dict(kind=rbs.GEN_ZIPF, n=5000, zipf_alpha=1.2, zipf_max=3000, seed=6),
    dict(kind=rbs.GEN_CHAIN, n=100000, chain_bw=3, seed=103),
    dict(kind=rbs.GEN_CHAIN, n=7, chain_bw=9, seed=7),
    dict(kind=rbs.GEN_DIAG, n=1000, seed=8),
    dict(kind=rbs.GEN_BAND_POISSON, n=1, lam=3, band=4, seed=10),
]


@pytest.mark.parametrize("spec", SPECS, ids=[f"{s['kind']}-{s.get('n', s.get('grid'))}-{s['seed']}" for s in SPECS])
def test_generator_bit_identical(spec):
    a = rbs.gen_lower_csr(**spec)
    b = oracle.gen_lower_csr(**spec)
    for x, y, name in zip(a, b, ("rowptr", "colidx", "val")):
        assert x.dtype == y.dtype and x.shape == y.shape, name
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), name


@pytest.mark.parametrize("seed,n,lo,hi", [(0, 1, -1.0, 1.0), (102, 100000, -1.0, 1.0), (7, 5000, 2.0, 3.5)])
def test_uniform_bit_identical(seed, n, lo, hi):
    a = rbs.gen_uniform(seed, n, lo, hi)
    b = oracle.gen_uniform(seed, n, lo, hi)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_mt19937_64_known_answer():
    # the C++ standard fixes the 10000th output of a default-seeded (5489)
    # std::mt19937_64 at 9981545732273789042; a uniform draw exposes its top
    # 53 bits: (word >> 11) * 2^-53 on [0, 1)
    u = oracle.gen_uniform(5489, 10000, 0.0, 1.0)[-1]
    assert u == (9981545732273789042 >> 11) * 2.0 ** -53
