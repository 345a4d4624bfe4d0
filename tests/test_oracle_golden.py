"""Pin the oracle: its restated analysis must equal the reference's own
outputs (golden vectors from oracle/_ref/ref_dump) bit for bit."""
import numpy as np
import pytest

from _util import FIXTURES, INT_KEYS, load_fixture, val_digest
from oracle import oracle


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_reference(name):
    g, cp, ri, va, sub, lv = load_fixture(name)
    o = oracle.analyse(cp, ri, va, sub, lv)
    for k in INT_KEYS:
        ref = g["ref_" + k]
        got = o[k]
        if k.startswith("subtri") or k.startswith("subrec"):
            mask = ref != -1  # entries the reference leaves unset
            ref, got = ref[mask], got[mask]
        np.testing.assert_array_equal(got, ref, err_msg=f"{name}: {k}")
    assert val_digest(o["recblock_Val"]) == g["ref_recblock_Val_sha256"].tobytes()
    # long rows of square blocks
    sq = np.arange(1, len(o["method"]), 2)
    np.testing.assert_array_equal(o["longrow"][sq][o["method"][sq] >= 0], g["ref_longrow"][sq][g["ref_method"][sq] >= 0])


def test_golden_covers_every_method():
    tri, sq, longrows = set(), set(), 0
    for name in FIXTURES:
        g = np.load(__import__("os").path.join(__import__("_util").GOLDEN, name + ".npz"))
        m = g["ref_method"]
        tri |= set(m[0::2].tolist())
        sq |= set(m[1::2].tolist())
        longrows += int(g["ref_longrow"].sum())
    assert tri == {0, 1, 2, 3}
    assert sq >= {0, 1, 2, 3}
    assert longrows > 0


def test_auto_lv_rule():
    # main.cu:245-254
    assert oracle.auto_lv(16384, 0) == 1
    assert oracle.auto_lv(1048576, 0) == 3
    assert oracle.auto_lv(2000000, 0) == 4
    assert oracle.auto_lv(4000000, 0) == 5
    assert oracle.auto_lv(1048576, 1) == 4
