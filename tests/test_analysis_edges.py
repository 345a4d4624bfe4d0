"""Host analysis on edge-shaped inputs against the oracle's restatement of
the reference analysis (itself pinned by the reference-built golden
vectors): one row, 2^lv == n (one-row triangles), n not a multiple of
2^lv, diagonal-only systems (empty squares), a dense lower triangle, a row
longer than the long-row threshold (2048), both directions."""
import numpy as np
import pytest

import rbs
from _util import INT_KEYS
from oracle import oracle


def _lower(rows, seed):
    rng = np.random.default_rng(seed)
    rp, ci, va = [0], [], []
    for i, cols in enumerate(rows):
        v = rng.uniform(-1, 1, len(cols))
        ci.extend(cols)
        va.extend(v)
        ci.append(i)
        va.append(1.0 + np.abs(v).sum())
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(va)


def _band(n, w, seed):
    rng = np.random.default_rng(seed)
    return _lower([sorted(rng.choice(np.arange(max(0, i - w), i), size=min(i, 3), replace=False).tolist())
                   for i in range(n)], seed)


CASES = {
    "one_row_lv0": (lambda: _lower([[]], 1), 0),
    "two_rows_lv1": (lambda: _lower([[], [0]], 2), 1),
    "eight_rows_lv3": (lambda: _band(8, 3, 3), 3),
    "diag_only_lv3": (lambda: _lower([[] for _ in range(100)], 4), 3),
    "dense_lv2": (lambda: _lower([list(range(i)) for i in range(64)], 5), 2),
    "ragged_n1001_lv3": (lambda: _band(1001, 40, 6), 3),
    "long_row_lv2": (lambda: _lower([[] if i < 4999 else list(range(4999)) for i in range(5000)], 7), 2),
}


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
@pytest.mark.parametrize("name", sorted(CASES))
def test_edge_analysis_matches_oracle(name, sub):
    make, lv = CASES[name]
    rp, ci, va = make()
    # forward input: CSC(L); backward input: CSC(L^T) = L's CSR arrays
    cp, ri, cv = oracle.transpose(rp, ci, va) if sub == rbs.FORWARD else (rp, ci, va)
    ref = oracle.analyse(cp, ri, cv, sub, lv)
    for select in (rbs.SELECT_AUTO, rbs.SELECT_TUNE):
        plan = rbs.analyse(cp, ri, cv, substitution=sub, lv=lv, opts=rbs.options(host_only=1, select=select))
        for k in INT_KEYS:
            want, got = ref[k], plan.export(k)
            if k.startswith("subtri") or k.startswith("subrec"):
                mask = want != -1
                want, got = want[mask], got[mask]
            np.testing.assert_array_equal(got, want, err_msg=f"{name}: {k}")
        np.testing.assert_array_equal(plan.export("recblock_Val"), ref["recblock_Val"])
