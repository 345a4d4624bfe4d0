"""rbs_sptrsv_csr_noalloc: the solve for callers that cannot allocate device
memory (their framework's caching allocator holds the free memory, or their
loop forbids cudaMalloc/cudaFree after start-up).  Its scratch is a static
device array inside the library.  Checked through the C ABI against the
planned solve (rbs_analyse + rbs_solve) on two calls in a row, with the
same tolerance as the other parity tests.  Collected last on purpose."""
import numpy as np
import pytest

import rbs

TOL = 1e-12
pytestmark = pytest.mark.gpu


def _system(sub, seed):
    import scipy.sparse as sp
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=50000, lam=6, band=512, seed=seed)
    n = len(rp) - 1
    L = sp.csr_matrix((va, ci, rp), shape=(n, n))
    A = L if sub == rbs.FORWARD else L.T.tocsr()
    A.sort_indices()
    return A


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_noalloc_matches_planned_solve_twice(cuda, sub):
    import torch
    A = _system(sub, seed=300 + sub)
    n = A.shape[0]
    csc = A.tocsc()
    csc.sort_indices()
    plan = rbs.analyse(csc.indptr, csc.indices, csc.data, substitution=sub, lv=-1)
    d_rp = torch.tensor(A.indptr, dtype=torch.int32, device=cuda)
    d_ci = torch.tensor(A.indices, dtype=torch.int32, device=cuda)
    d_va = torch.tensor(A.data, dtype=torch.float64, device=cuda)
    for call in range(2):
        b = A @ rbs.gen_uniform(400 + call, n)
        d_b = torch.tensor(b, dtype=torch.float64, device=cuda)
        x_plan = torch.empty_like(d_b)
        plan.solve(d_b, x_plan)
        x_na = torch.full_like(d_b, float("nan"))
        rbs.sptrsv_csr_noalloc(d_rp, d_ci, d_va, n, sub, d_b, x_na)
        ref = x_plan.cpu().numpy()
        got = x_na.cpu().numpy()
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= TOL, (call, err)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    dummy_i = torch.zeros(4, dtype=torch.int32, device=cuda)
    dummy_d = torch.zeros(4, dtype=torch.float64, device=cuda)
    with pytest.raises(rbs.RbsError) as e:
        rbs.sptrsv_csr_noalloc(dummy_i, dummy_i, dummy_d, rbs.NOALLOC_MAX_ROWS + 1, rbs.FORWARD, dummy_d, dummy_d)
    assert e.value.code == rbs.ERR_ARG and "scratch limit" in str(e.value)
