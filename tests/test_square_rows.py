"""Host analysis of squares with a heavy tail of long rows: for the single-RHS
solve, every square whose lane group is narrower than a warp lists its rows
of 9..2048 entries for the warp-per-row pass (export "medrow"), and no other
block lists any.  A chain keeps the level order equal to the natural order,
so the square of lv = 1 is exactly rows [n/2, n) x columns [0, n/2)."""
import numpy as np
import pytest

import rbs
from oracle import oracle


def chain_with_long_rows(n, long_rows, long_len, seed):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        cols = set()
        if i > 0:
            cols.add(i - 1)  # the chain: level(i) = i
        if i >= n // 2:
            k = long_len if i in long_rows else 2
            cols.update(rng.choice(n // 2, size=k, replace=False).tolist())
        cols.discard(i)
        rows.append(sorted(c for c in cols if c < i))
    rp = np.zeros(n + 1, np.int32)
    ci, va = [], []
    for i, cs in enumerate(rows):
        ci.extend(cs + [i])
        va.extend([0.1] * len(cs) + [1.0])
        rp[i + 1] = len(ci)
    return rp, np.array(ci, np.int32), np.array(va)


@pytest.mark.parametrize("long_len,expect_rows", [(40, 5), (9, 5), (2048, 5), (2049, 0), (8, 0)])
def test_square_medium_rows_listed(long_len, expect_rows):
    n = 6000
    long_rows = {n // 2 + 7, n // 2 + 100, n // 2 + 1500, n - 20, n - 1}
    rp, ci, va = chain_with_long_rows(n, long_rows, long_len, 5)
    cp, ri, cv = oracle.transpose(rp, ci, va)  # the CSC the analysis takes
    plan = rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=1, opts=rbs.options(host_only=1))
    kern = plan.export("kernel")
    med = plan.export("medrow")
    assert len(med) == 3 and kern[1] == rbs.K_SPMV
    assert med[0] == 0 and med[2] == 0
    # the square's rows: 2 (or long_len) entries; rows of more than 2048
    # entries go to the long-row kernel instead
    assert med[1] == expect_rows


@pytest.mark.gpu
@pytest.mark.parametrize("long_len", [40, 700, 2048, 3000])
def test_square_with_long_rows_solves(cuda, long_len):
    # the warp-per-row pass (and, past 2048 entries, the long-row kernel)
    # against the serial oracle; the warp-per-row sum has a fixed order, so
    # two solves agree bit for bit when no row is longer than 2048
    import torch
    from _util import rel_err
    n = 8000
    long_rows = {n // 2 + 3, n // 2 + 999, n - 2}
    rp, ci, va = chain_with_long_rows(n, long_rows, long_len, 9)
    cp, ri, cv = oracle.transpose(rp, ci, va)
    plan = rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=1)
    assert plan.export("medrow")[1] == (3 if long_len <= 2048 else 0)
    b = rbs.gen_uniform(10, n)
    x_ref = oracle.sptrsv_csr(rp, ci, va, rbs.FORWARD, b)
    db = torch.tensor(b, device=cuda)
    x1, x2 = torch.empty_like(db), torch.empty_like(db)
    plan.solve(db, x1)
    plan.solve(db, x2)
    assert rel_err(x1.cpu().numpy(), x_ref) <= 1e-12
    if long_len <= 2048:
        assert torch.equal(x1, x2)
