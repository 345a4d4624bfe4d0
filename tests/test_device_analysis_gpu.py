"""Analysis on the device (rbs_analyse_device: validation, findlevel, level
reordering and the processing-order CSR run as CUDA kernels) reproduces the
reference's integer outputs bit for bit: checked against the reference's
golden vectors, against the host analysis on the benchmark structures, and
its reordered CSC against the oracle's restatement of
levelset_reordering_colrow_csc."""
import numpy as np
import pytest

import rbs
from _util import FIXTURES, INT_KEYS, load_fixture, rel_err, val_digest
from oracle import oracle

pytestmark = pytest.mark.gpu


def dev_plan(cuda, ptr, idx, val, sub, lv, fmt=rbs.FMT_CSC, select=rbs.SELECT_AUTO, host_only=1):
    import torch
    d = [torch.tensor(np.asarray(a), device=cuda) for a in (ptr, idx)]
    dv = torch.tensor(np.asarray(val, np.float64), device=cuda)
    return rbs.analyse_device(d[0], d[1], dv, len(ptr) - 1, len(idx), substitution=sub, lv=lv, fmt=fmt,
                              opts=rbs.options(host_only=host_only, select=select))


@pytest.mark.parametrize("name", FIXTURES)
def test_device_analysis_matches_reference(cuda, name):
    g, cp, ri, va, sub, lv = load_fixture(name)
    plan = dev_plan(cuda, cp.astype(np.int32), ri.astype(np.int32), va, sub, lv)
    assert plan.export("analyse_ms")[1] > 0  # the level sets came from the device
    for k in INT_KEYS:
        ref = g["ref_" + k]
        got = plan.export(k)
        if k.startswith("subtri") or k.startswith("subrec"):
            mask = ref != -1
            ref, got = ref[mask], got[mask]
        np.testing.assert_array_equal(got, ref, err_msg=f"{name}: {k}")
    assert val_digest(plan.export("recblock_Val")) == g["ref_recblock_Val_sha256"].tobytes()
    ncp, nri, _, _ = oracle.reorder_colrow(cp, ri, va, sub)
    np.testing.assert_array_equal(plan.export("reordered_colptr"), ncp)
    np.testing.assert_array_equal(plan.export("reordered_rowidx"), nri)


SYSTEMS = {
    "laplace2d_1024": dict(kind=rbs.GEN_LAPLACE2D, grid=1024, seed=101),       # 2047 narrow levels
    "powerlaw_2M": dict(kind=rbs.GEN_ZIPF, n=2000000, zipf_alpha=2.1, zipf_max=1000, seed=102),  # wide levels
    "chain_200k": dict(kind=rbs.GEN_CHAIN, n=200000, chain_bw=3, seed=103),    # one row per level
    "band_poisson": dict(kind=rbs.GEN_BAND_POISSON, n=16384, lam=6, band=512, seed=100),
}


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_device_analysis_matches_host_at_size(cuda, name, sub):
    import torch
    rp, ci, va = rbs.gen_lower_csr(**SYSTEMS[name])
    A = oracle.transpose(rp, ci, va) if sub == rbs.FORWARD else (rp, ci, va)  # CSC of L, or of U = L^T
    host = rbs.analyse(*A, substitution=sub, lv=-1, opts=rbs.options(host_only=1))
    dev = dev_plan(cuda, *A, sub, -1, host_only=0)
    for k in ("levelItem", "levelPtr", "perm", "blk_nnz", "method", "nlv", "kernel", "reordered_colptr",
              "reordered_rowidx", "recblock_Ptr", "recblock_Index"):
        np.testing.assert_array_equal(dev.export(k), host.export(k), err_msg=f"{name}: {k}")
    # the level search ran on the device, except for the chain (one row per
    # level), which it hands to the host after a few thousand levels
    assert dev.export("analyse_ms")[2] == (0 if name.startswith("chain") else 1)
    # and the plan built from the device analysis solves
    n = len(A[0]) - 1
    arp, aci, ava = (rp, ci, va) if sub == rbs.FORWARD else oracle.transpose(*A)
    b = oracle.spmv_csr(arp, aci, ava, rbs.gen_uniform(7, n))
    x = oracle.sptrsv_csr(arp, aci, ava, sub, b)
    db = torch.tensor(b, device=cuda)
    dx = torch.empty_like(db)
    dev.solve(db, dx)
    assert rel_err(dx.cpu().numpy(), x) <= 1e-12


def test_device_analysis_csr_input(cuda):
    g, cp, ri, va, sub, lv = load_fixture("zipf_lv3_fwd")
    rp, ci, v2 = oracle.transpose(cp, ri, va)  # CSC -> CSR (rows ascending in each column afterwards)
    plan = dev_plan(cuda, rp, ci, v2, sub, lv, fmt=rbs.FMT_CSR)
    np.testing.assert_array_equal(plan.export("levelItem"), g["ref_levelItem"])
    np.testing.assert_array_equal(plan.export("recblock_Index"), g["ref_recblock_Index"])


@pytest.mark.parametrize("defect", ["no_diagonal", "zero_diagonal", "outside", "bad_index"])
def test_device_analysis_rejects_bad_structure(cuda, defect):
    g, cp, ri, va, sub, lv = load_fixture("band_lv0_fwd")
    cp, ri, va = cp.astype(np.int32).copy(), ri.astype(np.int32).copy(), va.copy()
    c = 5
    if defect == "no_diagonal":
        ri[cp[c]] = ri[cp[c] + 1] if cp[c + 1] - cp[c] > 1 else c + 1
    elif defect == "zero_diagonal":
        va[cp[c]] = 0.0
    elif defect == "outside":
        ri[cp[c + 1] - 1] = 0  # row 0 < column c in a lower triangle
    else:
        ri[cp[c + 1] - 1] = len(cp) + 10
    with pytest.raises(rbs.RbsError) as e:
        dev_plan(cuda, cp, ri, va, sub, lv)
    assert e.value.code == rbs.ERR_STRUCTURE
