"""Saved plans (rbs_plan_save / rbs_plan_load) restore the analysis exactly:
every reference-format array and the execution layouts, without a new level
search; bad files (wrong magic, truncated, damaged: a file digest covers
every byte) are rejected."""
import os

import numpy as np
import pytest

import rbs
from _util import FIXTURES, INT_KEYS, load_fixture, rel_err

EXTRA = ["kernel", "perm", "levelPtr", "reordered_colptr", "reordered_rowidx", "lc_tab", "lc_segs", "ca_tab",
         "ell_chunks", "block_rows"]


@pytest.mark.parametrize("name", ["band_lv3_fwd", "zipf_lv2_bwd", "chain_method1_fwd", "laplace40_lv2_bwd"])
def test_save_load_roundtrip(tmp_path, name):
    g, cp, ri, va, sub, lv = load_fixture(name)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(host_only=1, select=rbs.SELECT_TUNE))
    path = tmp_path / "plan.rbs"
    plan.save(path)
    back = rbs.load_plan(path, rbs.options(host_only=1))
    for k in INT_KEYS + EXTRA:
        np.testing.assert_array_equal(back.export(k), plan.export(k), err_msg=k)
    np.testing.assert_array_equal(back.export("recblock_Val"), plan.export("recblock_Val"))
    assert back.info().nlevel == plan.info().nlevel and back.info().lv == plan.info().lv


def test_load_rejects_bad_files(tmp_path):
    g, cp, ri, va, sub, lv = load_fixture("band_lv0_fwd")
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(host_only=1))
    good = tmp_path / "p.rbs"
    plan.save(good)
    raw = good.read_bytes()
    bad = tmp_path / "bad.rbs"
    bad.write_bytes(b"NOTAPLAN" + raw[8:])
    with pytest.raises(rbs.RbsError):
        rbs.load_plan(bad, rbs.options(host_only=1))
    cut = tmp_path / "cut.rbs"
    cut.write_bytes(raw[: len(raw) // 2])
    with pytest.raises(rbs.RbsError):
        rbs.load_plan(cut, rbs.options(host_only=1))
    with pytest.raises(rbs.RbsError):
        rbs.load_plan(tmp_path / "missing.rbs", rbs.options(host_only=1))
    # one flipped bit anywhere in the body (here inside the pools), or bytes
    # appended, fail the file digest before anything reaches the device
    for at in (len(raw) // 3, len(raw) - 9):
        flip = bytearray(raw)
        flip[at] ^= 0x10
        (tmp_path / "flip.rbs").write_bytes(bytes(flip))
        with pytest.raises(rbs.RbsError) as e:
            rbs.load_plan(tmp_path / "flip.rbs", rbs.options(host_only=1))
        assert "damaged" in str(e.value)
    (tmp_path / "long.rbs").write_bytes(raw + b"\0")
    with pytest.raises(rbs.RbsError):
        rbs.load_plan(tmp_path / "long.rbs", rbs.options(host_only=1))
    # a file of a build with other layout constants (row-length classes of
    # the squares, level-chunk layout): the 8-byte signature after the magic
    # differs, and the file is refused as not of this build before its
    # contents are read
    other = bytearray(raw)
    other[8] ^= 0x01
    (tmp_path / "other.rbs").write_bytes(bytes(other))
    with pytest.raises(rbs.RbsError) as e:
        rbs.load_plan(tmp_path / "other.rbs", rbs.options(host_only=1))
    assert "not a plan file of this build" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["band_auto_fwd", "zipf_lv3_bwd"])
def test_loaded_plan_solves(cuda, tmp_path, name):
    import torch

    from oracle import oracle
    g, cp, ri, va, sub, lv = load_fixture(name)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv)
    path = tmp_path / "plan.rbs"
    plan.save(path)
    back = rbs.load_plan(path)
    rp, ci, v2 = oracle.transpose(cp, ri, va)
    n = len(cp) - 1
    b = oracle.spmv_csr(rp, ci, v2, rbs.gen_uniform(11, n))
    xo = oracle.sptrsv_csr(rp, ci, v2, sub, b)
    db = torch.tensor(b, device=cuda)
    x1, x2 = torch.empty_like(db), torch.empty_like(db)
    plan.solve(db, x1)
    back.solve(db, x2)
    assert torch.equal(x1, x2)  # same layouts, same kernels: same bits
    assert rel_err(x2.cpu().numpy(), xo) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["band", "zipf"])
def test_transposed_solve_without_materialising(cuda, kind):
    # L^T x = b from L's own CSR arrays: a lower factor's CSR is its
    # transpose's CSC, so the arrays go in as an upper triangle (backward)
    import torch

    from oracle import oracle
    if kind == "band":
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=20000, lam=6, band=300, seed=31)
    else:
        rp, ci, va = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=20000, zipf_alpha=2.1, zipf_max=200, seed=32)
    n = len(rp) - 1
    plan = rbs.analyse(rp, ci, va, substitution=rbs.BACKWARD, lv=-1, fmt=rbs.FMT_CSC)
    up, ui, uv = oracle.transpose(rp, ci, va)  # explicit L^T (CSR), for the oracle only
    b = oracle.spmv_csr(up, ui, uv, rbs.gen_uniform(12, n))
    xo = oracle.sptrsv_csr(up, ui, uv, rbs.BACKWARD, b)
    db = torch.tensor(b, device=cuda)
    dx = torch.empty_like(db)
    plan.solve(db, dx)
    assert rel_err(dx.cpu().numpy(), xo) <= 1e-12
