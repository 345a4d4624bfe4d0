"""The library's analysis (rbs_analyse, host side) reproduces the
reference's integer outputs bit for bit: level order, block bounds, nnz per
block, method codes, local level sets and the packed recblock_* arrays."""
import numpy as np
import pytest

import rbs
from _util import FIXTURES, INT_KEYS, load_fixture, val_digest


def host_plan(cp, ri, va, sub, lv, select=rbs.SELECT_AUTO, fmt=rbs.FMT_CSC):
    return rbs.analyse(cp, ri, va, substitution=sub, lv=lv, fmt=fmt, opts=rbs.options(host_only=1, select=select))


@pytest.mark.parametrize("name", FIXTURES)
def test_analysis_matches_reference(name):
    g, cp, ri, va, sub, lv = load_fixture(name)
    plan = host_plan(cp, ri, va, sub, lv)
    assert plan.info().lv == lv
    for k in INT_KEYS:
        ref = g["ref_" + k]
        got = plan.export(k)
        if k.startswith("subtri") or k.startswith("subrec"):
            mask = ref != -1
            ref, got = ref[mask], got[mask]
        np.testing.assert_array_equal(got, ref, err_msg=f"{name}: {k}")
    assert val_digest(plan.export("recblock_Val")) == g["ref_recblock_Val_sha256"].tobytes()
    sq = np.arange(1, len(g["ref_method"]), 2)
    ok = g["ref_method"][sq] >= 0
    np.testing.assert_array_equal(plan.export("longrow")[sq][ok], g["ref_longrow"][sq][ok])


@pytest.mark.parametrize("name", ["band_lv3_fwd", "zipf_lv2_bwd"])
def test_csr_input_gives_same_analysis(name):
    # RBS_FMT_CSR is transposed to the reference's CSC layout first
    from oracle import oracle
    g, cp, ri, va, sub, lv = load_fixture(name)
    rp, ci, v2 = oracle.transpose(cp, ri, va)  # CSC -> CSR
    plan = host_plan(rp, ci, v2, sub, lv, fmt=rbs.FMT_CSR)
    np.testing.assert_array_equal(plan.export("levelItem"), g["ref_levelItem"])
    np.testing.assert_array_equal(plan.export("recblock_Index"), g["ref_recblock_Index"])


def test_reference_select_maps_methods_to_kernels():
    g, cp, ri, va, sub, lv = load_fixture("band_lv3_fwd")
    plan = host_plan(cp, ri, va, sub, lv, select=rbs.SELECT_REFERENCE)
    meth, kern = plan.export("method"), plan.export("kernel")
    tri_map = {0: rbs.K_DIAG, 2: rbs.K_LEVEL, 3: rbs.K_SYNCFREE}
    for b in range(0, len(meth), 2):
        assert kern[b] == tri_map[meth[b]]
    for b in range(1, len(meth), 2):
        assert kern[b] == rbs.K_SPMV


def test_permutation_is_the_bfs_order():
    g, cp, ri, va, sub, lv = load_fixture("laplace40_lv2_fwd")
    plan = host_plan(cp, ri, va, sub, lv)
    perm = plan.export("perm")
    np.testing.assert_array_equal(np.sort(perm), np.arange(len(cp) - 1))
    np.testing.assert_array_equal(perm, g["ref_levelItem"])
