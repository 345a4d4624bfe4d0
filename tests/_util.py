"""Shared helpers for the tests (golden fixture loading, relative errors)."""
import hashlib
import os

import numpy as np

import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Integer arrays compared bit-for-bit with the reference's own analysis.
INT_KEYS = ["levelItem", "loc_off", "tmp_off", "blk_m", "blk_n", "blk_nnz", "subtri_up", "subtri_down", "subrec_up",
            "subrec_down", "subrec_right", "subrec_left", "sizes", "ptr_offset", "index_offset", "dcsrindex_offset",
            "recblock_Ptr", "recblock_Index", "recblock_dcsr_rowidx", "method", "nlv", "lvl_ptr", "lvl_item", "m_lv",
            "offset_lv", "nnz_lv"]

FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_fixture(name):
    """Return (golden dict, colptr, rowidx, val, substitution, lv)."""
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    case = name.rsplit("_", 1)[0]
    sub = int(g["substitution"][0])
    if "colptr" in g:
        cp, ri, va = g["colptr"], g["rowidx"], g["val"]
    else:
        cp, ri, va = cases.inputs(cases.CASES[case], sub)
    digest = hashlib.sha256(np.ascontiguousarray(cp, np.int32).tobytes() + np.ascontiguousarray(ri, np.int32).tobytes()
                            + np.ascontiguousarray(va, np.float64).tobytes()).digest()
    assert digest == g["input_sha256"].tobytes(), f"{name}: regenerated input differs from the fixture's input"
    return g, cp, ri, va, sub, int(g["lv"][0])


def val_digest(v):
    return hashlib.sha256(np.ascontiguousarray(v, np.float64).tobytes()).digest()


def rel_err(x, ref):
    x = np.asarray(x, np.float64).ravel()
    ref = np.asarray(ref, np.float64).ravel()
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))
