"""Pin the integer analysis at the benchmark's full sizes to the REFERENCE.

Runs oracle/_ref/ref_dump (recblock-sptrsv's own get_recblock_size +
L_/U_preprocessing, recblocking_preprocess.h:298-385 and :387-1474, built
from the reference sources by oracle/Makefile) on the benchmark systems at
their full sizes, both directions, lv by the reference's automatic rule
(main.cu:245-254), and writes tests/golden/large_digests.json: per case the
sizes and lv, the per-block method and local level counts in full, and a
SHA-256 of every other output array (levelItem, block bounds, recblock_*,
local level sets).  The arrays themselves are tens of MB, so only their
digests are committed.  Inputs come from the oracle's generator
(oracle/gen.c, bit-identical to the library's); forward input = CSC of L,
backward input = CSC of U = L^T = the CSR arrays of L.

Needs the reference sources; run here, not on a GPU box:
    make -C oracle ref REF=<reference recblock-sptrsv dir> && python tests/golden/make_golden_large.py
"""
import hashlib
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle  # noqa: E402

# the benchmark's seeded systems at full size (bench.py SPECS)
LARGE = {
    "c0_band16k": dict(kind=0, n=16384, lam=6, band=512, seed=100),
    "c1a_laplace1024": dict(kind=1, grid=1024, seed=101),
    "c1b_zipf2m": dict(kind=2, n=2000000, zipf_alpha=2.1, zipf_max=1000, seed=102),
    "c1c_chain1m": dict(kind=3, n=1000000, chain_bw=3, seed=103),
    "c2r_band4m": dict(kind=0, n=4000000, lam=10, band=4096, seed=104),
}
FULL_MAX = 4096  # per-block arrays (at most 2^(lv+1) entries) are kept whole


def inputs(spec, sub):
    rp, ci, va = oracle.gen_lower_csr(**spec)
    if sub == 0:
        return oracle.transpose(rp, ci, va)
    return rp, ci, va


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    if not os.path.exists(oracle.REF_DUMP):
        sys.exit("oracle/_ref/ref_dump missing: run make -C oracle ref REF=<reference recblock-sptrsv dir>")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, spec in LARGE.items():
            for sub, tag in ((0, "fwd"), (1, "bwd")):
                cp, ri, va = inputs(spec, sub)
                n = len(cp) - 1
                lv = oracle.auto_lv(n, 0)
                t0 = time.time()
                ref = oracle.run_reference_dump(cp, ri, va, sub, lv, tmp)
                case = {"spec": spec, "substitution": sub, "n": n, "nnz": int(len(ri)), "lv": lv,
                        "input_sha256": hashlib.sha256(cp.tobytes() + ri.tobytes() + va.tobytes()).hexdigest(),
                        "digests": {}, "full": {}}
                for k, v in sorted(ref.items()):
                    if len(v) <= FULL_MAX and v.dtype == np.int32:
                        case["full"][k] = v.astype(int).tolist()
                    else:
                        case["digests"][k] = digest(v)
                out[f"{name}_{tag}"] = case
                print(f"{name}_{tag}: n={n} nnz={len(ri)} lv={lv} methods={ref['method'].tolist()} "
                      f"({time.time() - t0:.1f} s)", flush=True)
    with open(os.path.join(HERE, "large_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
