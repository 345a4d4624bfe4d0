"""ILU(0) on the device (rbs_ilu0_device) -- the factor producer for this
solver in preconditioned Krylov methods -- against the oracle's serial IKJ
ILU(0) bit for bit, and the preconditioner apply U^-1 L^-1 b through this
library's own triangle plans against the oracle's serial substitutions."""
import numpy as np
import pytest
import scipy.sparse as sp

import rbs
from _util import rel_err
from oracle import oracle

pytestmark = pytest.mark.gpu


def strict_lower(kind, seed, n):
    if kind == "laplace":
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=int(round(np.sqrt(n))), seed=seed)
    elif kind == "band":
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=6, band=400, seed=seed)
    else:
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=n, zipf_alpha=2.1, zipf_max=200, seed=seed)
    m = len(rp) - 1
    L = sp.csr_matrix((va, ci, rp), shape=(m, m))
    return sp.tril(L, k=-1).tocsr()


def general_matrix(kind, seed, n, symmetric_pattern=True):
    """Square CSR with a dominant diagonal: strict lower part from a
    generator, strict upper part from its transpose (or from another
    generator), fresh U(-1,1) values."""
    rng = np.random.default_rng(seed)
    S = strict_lower(kind, seed, n)
    m = S.shape[0]
    T = S.T.tocsr() if symmetric_pattern else strict_lower("band", seed + 1, m).T.tocsr()
    T = sp.csr_matrix((rng.uniform(-1, 1, T.nnz), T.indices, T.indptr), shape=(m, m))
    off = (S + T).tocsr()
    d = 1.0 + np.asarray(abs(off).sum(axis=1)).ravel()
    A = (off + sp.diags(d)).tocsr()
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)


def split(rp, ci, lu):
    """L (strict lower of lu + unit diagonal) and U (upper of lu) as CSR."""
    n = len(rp) - 1
    lr, lc, lv, ur, uc, uv = [0], [], [], [0], [], []
    for i in range(n):
        for p in range(rp[i], rp[i + 1]):
            if ci[p] < i:
                lc.append(ci[p]); lv.append(lu[p])
            else:
                uc.append(ci[p]); uv.append(lu[p])
        lc.append(i); lv.append(1.0)
        lr.append(len(lc)); ur.append(len(uc))
    f = lambda r, c, v: (np.array(r, np.int32), np.array(c, np.int32), np.array(v))
    return f(lr, lc, lv), f(ur, uc, uv)


def factor(cuda, rp, ci, va):
    import torch
    d = [torch.tensor(a, device=cuda) for a in (rp, ci, va)]
    dlu = torch.empty_like(d[2])
    rbs.ilu0_device(d[0], d[1], d[2], dlu)
    return dlu.cpu().numpy()


@pytest.mark.parametrize("kind,symmetric", [("laplace", True), ("band", True), ("zipf", True), ("band", False),
                                            ("zipf", False)])
def test_ilu0_matches_oracle_bit_for_bit(cuda, kind, symmetric):
    rp, ci, va = general_matrix(kind, 41, 6000, symmetric)
    lu = factor(cuda, rp, ci, va)
    ref = oracle.ilu0_csr(rp, ci, va)
    assert np.array_equal(lu, ref)


def test_ilu0_at_size(cuda):
    rp, ci, va = general_matrix("laplace", 42, 1024 * 1024)
    lu = factor(cuda, rp, ci, va)
    assert np.array_equal(lu, oracle.ilu0_csr(rp, ci, va))


@pytest.mark.parametrize("kind", ["laplace", "zipf"])
def test_ilu0_preconditioner_apply(cuda, kind):
    import torch
    rp, ci, va = general_matrix(kind, 43, 20000)
    lu = factor(cuda, rp, ci, va)
    (lr, lc, lv), (ur, uc, uv) = split(rp, ci, lu)
    n = len(rp) - 1
    Lp = rbs.analyse(lr, lc, lv, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
    Up = rbs.analyse(ur, uc, uv, substitution=rbs.BACKWARD, lv=-1, fmt=rbs.FMT_CSR)
    b = rbs.gen_uniform(44, n)
    z_ref = oracle.sptrsv_csr(ur, uc, uv, rbs.BACKWARD, oracle.sptrsv_csr(lr, lc, lv, rbs.FORWARD, b))
    db = torch.tensor(b, device=cuda)
    y, z = torch.empty_like(db), torch.empty_like(db)
    Lp.solve(db, y)
    Up.solve(y, z)
    assert rel_err(z.cpu().numpy(), z_ref) <= 1e-12


@pytest.mark.parametrize("defect", ["no_diagonal", "unsorted"])
def test_ilu0_rejects_bad_structure(cuda, defect):
    import torch
    rp, ci, va = general_matrix("band", 45, 2000)
    ci = ci.copy()
    n = len(rp) - 1
    if defect == "no_diagonal":
        # a row whose diagonal can become column i+1 with the row still sorted
        for i in range(100, n - 1):
            p = next(q for q in range(rp[i], rp[i + 1]) if ci[q] == i)
            if p + 1 == rp[i + 1] or ci[p + 1] > i + 1:
                ci[p] = i + 1
                break
    else:
        i = 100
        ci[rp[i]:rp[i + 1]] = ci[rp[i]:rp[i + 1]][::-1].copy()
    d = [torch.tensor(a, device=cuda) for a in (rp, ci, va)]
    with pytest.raises(rbs.RbsError) as e:
        rbs.ilu0_device(d[0], d[1], d[2], torch.empty_like(d[2]))
    assert e.value.code == rbs.ERR_STRUCTURE
