"""Generate golden vectors from the REFERENCE's own analysis.

Runs oracle/_ref/ref_dump (recblock-sptrsv's get_recblock_size +
L_/U_preprocessing compiled from the reference sources by oracle/Makefile)
on every case in cases.py, both directions, and writes
tests/golden/<case>_<fwd|bwd>.npz with the inputs (unless regenerated from
the seed) and every output.  Needs the reference sources; run here, not on
a GPU box:  make -C oracle ref REF=<reference recblock-sptrsv dir> && python tests/golden/make_golden.py
"""
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    if not os.path.exists(oracle.REF_DUMP):
        sys.exit("oracle/_ref/ref_dump missing: run make -C oracle ref REF=<reference recblock-sptrsv dir>")
    with tempfile.TemporaryDirectory() as tmp:
        for name, spec in cases.CASES.items():
            for sub, tag in ((0, "fwd"), (1, "bwd")):
                cp, ri, va = cases.inputs(spec, sub)
                lv = spec["lv"] if spec["lv"] >= 0 else oracle.auto_lv(len(cp) - 1, 0)
                ref = oracle.run_reference_dump(cp, ri, va, sub, lv, tmp)
                out = {f"ref_{k}": v for k, v in ref.items()}
                out["lv"] = np.array([lv], np.int32)
                out["substitution"] = np.array([sub], np.int32)
                # the packed values are the input values rearranged: keep a digest
                val = out.pop("ref_recblock_Val")
                out["ref_recblock_Val_sha256"] = np.frombuffer(hashlib.sha256(val.tobytes()).digest(), np.uint8)
                out["input_sha256"] = np.frombuffer(
                    hashlib.sha256(cp.tobytes() + ri.tobytes() + va.tobytes()).digest(), np.uint8)
                if name not in cases.SPEC_ONLY:
                    out["colptr"], out["rowidx"], out["val"] = cp, ri, va
                path = os.path.join(HERE, f"{name}_{tag}.npz")
                np.savez_compressed(path, **out)
                meth = ref["method"]
                print(f"{name}_{tag}: n={len(cp)-1} nnz={len(ri)} lv={lv} methods={meth.tolist()} "
                      f"-> {os.path.getsize(path)//1024} KB")


if __name__ == "__main__":
    main()
