"""IC(0) (rbs_ic0_device) -- incomplete Cholesky of an SPD matrix given as
its lower triangle -- against the oracle's serial row algorithm bit for bit,
and the preconditioner apply L^-T L^-1 b with L^T solved from L's own
arrays read as CSC (no transpose formed).  The oracle itself is checked on
the CPU: L L^T equals A on the pattern."""
import numpy as np
import pytest
import scipy.sparse as sp

import rbs
from _util import rel_err
from oracle import oracle


def spd_lower(kind, seed, n):
    """Lower triangle (diagonal last, columns ascending) of an SPD matrix:
    a generator's strict pattern, U(-1,1) values, diagonal 1 + the row's
    absolute off-diagonal sum in the full symmetric matrix."""
    rng = np.random.default_rng(seed)
    if kind == "laplace":
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=int(round(np.sqrt(n))), seed=seed)
    elif kind == "band":
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=6, band=400, seed=seed)
    else:
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=n, zipf_alpha=2.1, zipf_max=200, seed=seed)
    m = len(rp) - 1
    S = sp.tril(sp.csr_matrix((va, ci, rp), shape=(m, m)), k=-1).tocsr()
    S = sp.csr_matrix((rng.uniform(-1, 1, S.nnz), S.indices, S.indptr), shape=(m, m))
    d = 1.0 + np.asarray(abs(S + S.T).sum(axis=1)).ravel()
    L = (S + sp.diags(d)).tocsr()
    L.sort_indices()
    return L.indptr.astype(np.int32), L.indices.astype(np.int32), L.data.astype(np.float64)


@pytest.mark.parametrize("kind", ["laplace", "band", "zipf"])
def test_oracle_ic0_reproduces_a_on_its_pattern(kind):
    rp, ci, va = spd_lower(kind, 3, 3000)
    n = len(rp) - 1
    l = oracle.ic0_csr(rp, ci, va)
    Lm = sp.csr_matrix((l, ci, rp), shape=(n, n))
    Al = sp.csr_matrix((va, ci, rp), shape=(n, n))
    A = Al + sp.tril(Al, -1).T
    pattern = sp.csr_matrix((np.ones(len(ci)), ci, rp), shape=(n, n))
    R = (Lm @ Lm.T - A).multiply(pattern)
    assert abs(R).max() <= 1e-12 * abs(A).max()


def factor(cuda, rp, ci, va):
    import torch
    d = [torch.tensor(a, device=cuda) for a in (rp, ci, va)]
    dl = torch.empty_like(d[2])
    rbs.ic0_device(d[0], d[1], d[2], dl)
    return dl.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n", [("laplace", 6000), ("band", 6000), ("zipf", 6000), ("laplace", 1024 * 1024)])
def test_ic0_matches_oracle_bit_for_bit(cuda, kind, n):
    rp, ci, va = spd_lower(kind, 51, n)
    got = factor(cuda, rp, ci, va)
    assert np.array_equal(got.view(np.uint64), oracle.ic0_csr(rp, ci, va).view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["laplace", "zipf"])
def test_ic0_preconditioner_apply_with_transposed_solve(cuda, kind):
    import torch
    rp, ci, va = spd_lower(kind, 52, 20000)
    n = len(rp) - 1
    l = factor(cuda, rp, ci, va)
    Lp = rbs.analyse(rp, ci, l, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
    # L's CSR arrays are L^T's CSC: the backward plan solves L^T z = y
    Ltp = rbs.analyse(rp, ci, l, substitution=rbs.BACKWARD, lv=-1, fmt=rbs.FMT_CSC)
    b = rbs.gen_uniform(53, n)
    tp, ti, tv = oracle.transpose(rp, ci, l)
    z_ref = oracle.sptrsv_csr(tp, ti, tv, rbs.BACKWARD, oracle.sptrsv_csr(rp, ci, l, rbs.FORWARD, b))
    db = torch.tensor(b, device=cuda)
    y, z = torch.empty_like(db), torch.empty_like(db)
    Lp.solve(db, y)
    Ltp.solve(y, z)
    assert rel_err(z.cpu().numpy(), z_ref) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("defect", ["upper_entry", "diagonal_not_last", "not_positive"])
def test_ic0_rejects(cuda, defect):
    import torch
    rp, ci, va = spd_lower("band", 54, 2000)
    ci, va = ci.copy(), va.copy()
    i = 500
    if defect == "upper_entry":
        ci[rp[i + 1] - 1] = i + 1  # the diagonal's slot now holds a column above it
    elif defect == "diagonal_not_last":
        ci[rp[i]:rp[i + 1]] = np.roll(ci[rp[i]:rp[i + 1]], 1)
    else:
        va[rp[i + 1] - 1] = -1.0
    d = [torch.tensor(a, device=cuda) for a in (rp, ci, va)]
    with pytest.raises(rbs.RbsError) as e:
        rbs.ic0_device(d[0], d[1], d[2], torch.empty_like(d[2]))
    assert e.value.code == rbs.ERR_STRUCTURE, str(e.value)
