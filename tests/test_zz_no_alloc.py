"""rbs_sptrsv_csr_noalloc: the solve for callers that cannot allocate device
memory (their framework's caching allocator holds the free memory, or their
loop forbids cudaMalloc/cudaFree after start-up).  Its scratch is a static
device array inside the library.  Checked through the C ABI against the
planned solve (rbs_analyse + rbs_solve) and against the serial FP64 oracle,
on two calls in a row, with the same tolerance as the other parity tests;
then its edge cases: rows of 40..200 entries (the widest lane groups), a
system of exactly the scratch limit's row count, and malformed rows (a
missing diagonal, an entry above the diagonal), which must come back as
RBS_ERR_STRUCTURE without a fault or a wait.  Collected last on purpose."""
import numpy as np
import pytest

import rbs
from oracle import oracle

TOL = 1e-12
pytestmark = pytest.mark.gpu


def _system(sub, seed, n=50000, lam=6, band=512):
    import scipy.sparse as sp
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=lam, band=band, seed=seed)
    n = len(rp) - 1
    L = sp.csr_matrix((va, ci, rp), shape=(n, n))
    A = L if sub == rbs.FORWARD else L.T.tocsr()
    A.sort_indices()
    return A


def _device_csr(A, cuda):
    import torch
    return (torch.tensor(A.indptr, dtype=torch.int32, device=cuda),
            torch.tensor(A.indices, dtype=torch.int32, device=cuda),
            torch.tensor(A.data, dtype=torch.float64, device=cuda))


def _rel(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


def _oracle(A, sub, b):
    return oracle.sptrsv_csr(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, sub, b)


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_noalloc_matches_planned_solve_and_oracle_twice(cuda, sub):
    import torch
    A = _system(sub, seed=300 + sub)
    n = A.shape[0]
    csc = A.tocsc()
    csc.sort_indices()
    plan = rbs.analyse(csc.indptr, csc.indices, csc.data, substitution=sub, lv=-1)
    d_rp, d_ci, d_va = _device_csr(A, cuda)
    for call in range(2):
        b = A @ rbs.gen_uniform(400 + call, n)
        d_b = torch.tensor(b, dtype=torch.float64, device=cuda)
        x_plan = torch.empty_like(d_b)
        plan.solve(d_b, x_plan)
        x_na = torch.full_like(d_b, float("nan"))
        rbs.sptrsv_csr_noalloc(d_rp, d_ci, d_va, n, sub, d_b, x_na)
        got = x_na.cpu().numpy()
        assert _rel(got, x_plan.cpu().numpy()) <= TOL, call
        assert _rel(got, _oracle(A, sub, b)) <= TOL, call


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_noalloc_dense_rows(cuda, sub):
    # 60 entries per row on average, up to about 200: lane groups of 16 and 32
    import torch
    A = _system(sub, seed=310 + sub, n=6000, lam=60, band=200)
    n = A.shape[0]
    assert A.nnz / n >= 40
    d_rp, d_ci, d_va = _device_csr(A, cuda)
    b = A @ rbs.gen_uniform(311, n)
    d_b = torch.tensor(b, device=cuda)
    x = torch.full_like(d_b, float("nan"))
    rbs.sptrsv_csr_noalloc(d_rp, d_ci, d_va, n, sub, d_b, x)
    assert _rel(x.cpu().numpy(), _oracle(A, sub, b)) <= TOL


def test_noalloc_at_the_row_limit(cuda):
    import torch
    A = _system(rbs.FORWARD, seed=320, n=rbs.NOALLOC_MAX_ROWS, lam=3, band=64)
    n = A.shape[0]
    assert n == rbs.NOALLOC_MAX_ROWS
    d_rp, d_ci, d_va = _device_csr(A, cuda)
    b = A @ rbs.gen_uniform(321, n)
    d_b = torch.tensor(b, device=cuda)
    x = torch.full_like(d_b, float("nan"))
    rbs.sptrsv_csr_noalloc(d_rp, d_ci, d_va, n, rbs.FORWARD, d_b, x)
    assert _rel(x.cpu().numpy(), _oracle(A, rbs.FORWARD, b)) <= TOL


def _malformed(kind):
    # built on the host: a lower CSR of 5000 rows, then one row broken
    import scipy.sparse as sp
    A = _system(rbs.FORWARD, seed=330, n=5000, lam=4, band=64).tolil()
    r = 2500
    if kind == "missing_diagonal":
        A[r, r] = 0.0
    else:  # an entry above the diagonal, whose x a forward walk never produces first
        A[r, r + 7] = 0.5
    A = sp.csr_matrix(A)
    A.eliminate_zeros()
    A.sort_indices()
    return A


@pytest.mark.parametrize("kind", ["missing_diagonal", "above_diagonal"])
def test_noalloc_reports_malformed_rows(cuda, kind):
    import torch
    A = _malformed(kind)
    n = A.shape[0]
    d_rp, d_ci, d_va = _device_csr(A, cuda)
    d_b = torch.ones(n, dtype=torch.float64, device=cuda)
    x = torch.zeros_like(d_b)
    with pytest.raises(rbs.RbsError) as e:
        rbs.sptrsv_csr_noalloc(d_rp, d_ci, d_va, n, rbs.FORWARD, d_b, x)
    assert e.value.code == rbs.ERR_STRUCTURE
    # the device is still usable: a well-formed system solves afterwards
    A2 = _system(rbs.FORWARD, seed=331, n=3000)
    d2 = _device_csr(A2, cuda)
    b2 = A2 @ rbs.gen_uniform(332, A2.shape[0])
    x2 = torch.full((A2.shape[0],), float("nan"), dtype=torch.float64, device=cuda)
    rbs.sptrsv_csr_noalloc(*d2, A2.shape[0], rbs.FORWARD, torch.tensor(b2, device=cuda), x2)
    assert _rel(x2.cpu().numpy(), _oracle(A2, rbs.FORWARD, b2)) <= TOL


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    dummy_i = torch.zeros(4, dtype=torch.int32, device=cuda)
    dummy_d = torch.zeros(4, dtype=torch.float64, device=cuda)
    with pytest.raises(rbs.RbsError) as e:
        rbs.sptrsv_csr_noalloc(dummy_i, dummy_i, dummy_d, rbs.NOALLOC_MAX_ROWS + 1, rbs.FORWARD, dummy_d, dummy_d)
    assert e.value.code == rbs.ERR_ARG and "scratch limit" in str(e.value)
