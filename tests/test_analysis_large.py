"""Integer analysis at the benchmark's full sizes is the REFERENCE's, bit for
bit.  tests/golden/large_digests.json holds what recblock-sptrsv's own
analysis (get_recblock_size + L_/U_preprocessing, run by
tests/golden/make_golden_large.py through oracle/_ref/ref_dump) gives on
the benchmark systems -- the n = 16,384 band, the 2D Laplacian 1024^2, the
2M-row power-law factor, the 1M-row chain and the 4M-row band-4096 factor,
forward and backward, lv by the reference's automatic rule: every
per-block array in full and a SHA-256 of every large array.  The host
analysis (rbs_analyse) is checked here on the CPU, the device analysis
(rbs_analyse_device) on the GPU."""
import hashlib
import json
import os

import numpy as np
import pytest

import rbs
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "large_digests.json")
with open(GOLDEN) as _f:
    LARGE = json.load(_f)


def _inputs(case):
    rp, ci, va = rbs.gen_lower_csr(**case["spec"])
    cp, ri, cv = oracle.transpose(rp, ci, va) if case["substitution"] == 0 else (rp, ci, va)
    got = hashlib.sha256(cp.astype(np.int32).tobytes() + ri.astype(np.int32).tobytes() +
                         cv.astype(np.float64).tobytes()).hexdigest()
    assert got == case["input_sha256"], "regenerated input differs from the one the reference analysed"
    return cp.astype(np.int32), ri.astype(np.int32), cv.astype(np.float64)


def _check(plan, case, name):
    assert plan.info().lv == case["lv"], name
    for k, want in case["digests"].items():
        got = plan.export(k)
        got = np.ascontiguousarray(got, np.float64 if k == "recblock_Val" else np.int32)
        assert hashlib.sha256(got.tobytes()).hexdigest() == want, f"{name}: {k}"
    full = {k: np.asarray(v, np.int64) for k, v in case["full"].items()}
    for k, ref in full.items():
        got = np.asarray(plan.export(k), np.int64)
        if k.startswith("subtri") or k.startswith("subrec"):  # the reference leaves -1 where undefined
            mask = ref != -1
            ref, got = ref[mask], got[mask]
        elif k == "longrow":  # defined for squares the reference analyses (method >= 0)
            sq = np.arange(1, len(ref), 2)
            ok = full["method"][sq] >= 0
            ref, got = ref[sq][ok], got[sq][ok]
        np.testing.assert_array_equal(got, ref, err_msg=f"{name}: {k}")


@pytest.mark.parametrize("name", sorted(LARGE))
def test_host_analysis_is_the_references_at_full_size(name):
    case = LARGE[name]
    cp, ri, va = _inputs(case)
    plan = rbs.analyse(cp, ri, va, substitution=case["substitution"], lv=-1, opts=rbs.options(host_only=1))
    _check(plan, case, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(LARGE))
def test_device_analysis_is_the_references_at_full_size(cuda, name):
    import torch
    case = LARGE[name]
    cp, ri, va = _inputs(case)
    d = [torch.tensor(a, device=cuda) for a in (cp, ri, va)]
    plan = rbs.analyse_device(d[0], d[1], d[2], len(cp) - 1, len(ri), substitution=case["substitution"], lv=-1,
                              opts=rbs.options(host_only=1))
    _check(plan, case, name)
