"""The pieces around the solve chained the way a preconditioned-solver user
chains them: a Matrix Market file read on the device (rbs_mtx_read), its
lower triangle factored by IC(0) on the device (rbs_ic0_device), and the
preconditioner applied with two plans over the factor's one set of arrays
(L forward as CSR, L^T backward as the same arrays read as CSC) -- checked
step by step against the oracle's reader, IC(0) and substitutions; the same
file through ILU(0) with L and U plans."""
import numpy as np
import pytest
import scipy.sparse as sp

import rbs
from _util import rel_err
from oracle import oracle

pytestmark = pytest.mark.gpu


def spd_file(path, grid, seed):
    """Lower triangle of a 2D 5-point pattern with U(-1,1) off-diagonals and
    a dominant diagonal, written in symmetric storage."""
    rp, ci, _ = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=grid, seed=seed)
    n = len(rp) - 1
    S = sp.tril(sp.csr_matrix((np.ones(len(ci)), ci, rp), shape=(n, n)), k=-1).tocsr()
    S.data = np.random.default_rng(seed).uniform(-1, 1, S.nnz)
    d = 1.0 + np.asarray(abs(S + S.T).sum(axis=1)).ravel()
    Lo = (S + sp.diags(d)).tocsr()
    Lo.sort_indices()
    rbs.mtx_write(path, Lo.indptr.astype(np.int32), Lo.indices.astype(np.int32), Lo.data, symmetric=True)
    return n


def test_mtx_to_ic0_to_preconditioner(cuda, tmp_path):
    import torch
    path = str(tmp_path / "spd.mtx")
    n = spd_file(path, 300, 71)
    M = rbs.mtx_read(path)
    o = oracle.mtx_read(path)
    drp, dci, dva = M.csr()
    np.testing.assert_array_equal(dci.cpu().numpy(), o["colidx"])
    # the lower triangle with the diagonal last (rows of the expanded CSR
    # hold their own entries first, in file order: ascending columns)
    A = sp.csr_matrix((o["val"], o["colidx"], o["rowptr"]), shape=(n, n))
    Lo = sp.tril(A).tocsr()
    Lo.sort_indices()
    rp, ci, va = Lo.indptr.astype(np.int32), Lo.indices.astype(np.int32), Lo.data
    d = [torch.tensor(a, device=cuda) for a in (rp, ci, va)]
    dl = torch.empty_like(d[2])
    rbs.ic0_device(d[0], d[1], d[2], dl)
    l = dl.cpu().numpy()
    assert np.array_equal(l.view(np.uint64), oracle.ic0_csr(rp, ci, va).view(np.uint64))
    Lp = rbs.analyse(rp, ci, l, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
    Ltp = rbs.analyse(rp, ci, l, substitution=rbs.BACKWARD, lv=-1, fmt=rbs.FMT_CSC)
    tp, ti, tv = oracle.transpose(rp, ci, l)
    for seed in (72, 73):  # two applications in a row on the same plans
        b = rbs.gen_uniform(seed, n)
        z_ref = oracle.sptrsv_csr(tp, ti, tv, rbs.BACKWARD, oracle.sptrsv_csr(rp, ci, l, rbs.FORWARD, b))
        db = torch.tensor(b, device=cuda)
        y, z = torch.empty_like(db), torch.empty_like(db)
        Lp.solve(db, y)
        Ltp.solve(y, z)
        assert rel_err(z.cpu().numpy(), z_ref) <= 1e-12


def test_mtx_to_ilu0_to_preconditioner(cuda, tmp_path):
    import torch
    path = str(tmp_path / "spd.mtx")
    n = spd_file(path, 200, 81)
    M = rbs.mtx_read(path)
    drp, dci, dva = (t.cpu().numpy() for t in M.csr())
    A = sp.csr_matrix((dva, dci, drp), shape=(n, n))
    A.sort_indices()  # ILU(0) wants ascending columns; the reader keeps file order
    rp, ci, va = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    d = [torch.tensor(a, device=cuda) for a in (rp, ci, va)]
    dlu = torch.empty_like(d[2])
    rbs.ilu0_device(d[0], d[1], d[2], dlu)
    lu = dlu.cpu().numpy()
    assert np.array_equal(lu.view(np.uint64), oracle.ilu0_csr(rp, ci, va).view(np.uint64))
    rows = np.repeat(np.arange(n), np.diff(rp))
    low = ci < rows
    L = (sp.csr_matrix((lu[low], ci[low], np.r_[0, np.cumsum(np.bincount(rows[low], minlength=n))]), shape=(n, n))
         + sp.identity(n, format="csr")).tocsr()
    U = sp.csr_matrix((lu[~low], ci[~low], np.r_[0, np.cumsum(np.bincount(rows[~low], minlength=n))]), shape=(n, n))
    L.sort_indices()
    U.sort_indices()
    Lt = (L.indptr.astype(np.int32), L.indices.astype(np.int32), L.data)
    Ut = (U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data)
    Lp = rbs.analyse(*Lt, substitution=rbs.FORWARD, lv=-1, fmt=rbs.FMT_CSR)
    Up = rbs.analyse(*Ut, substitution=rbs.BACKWARD, lv=-1, fmt=rbs.FMT_CSR)
    b = rbs.gen_uniform(82, n)
    z_ref = oracle.sptrsv_csr(*Ut, rbs.BACKWARD, oracle.sptrsv_csr(*Lt, rbs.FORWARD, b))
    db = torch.tensor(b, device=cuda)
    y, z = torch.empty_like(db), torch.empty_like(db)
    Lp.solve(db, y)
    Up.solve(y, z)
    assert rel_err(z.cpu().numpy(), z_ref) <= 1e-12
