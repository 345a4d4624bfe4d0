"""The C-ABI library loads, exports every function include/*.h declares, and
rejects malformed input with a status (no GPU needed: host-only analysis)."""
import ctypes
import os
import re

import numpy as np
import pytest

import rbs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, re.M):
            if m.group(1) not in ("if", "for", "while", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert "rbs_analyse" in names and "recblocking_solver_cuda" in names
    lib = ctypes.CDLL(rbs._LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(rbs.EXPORTS) <= set(names)


def test_options_default():
    o = rbs.options()
    assert o.select == rbs.SELECT_AUTO and o.device == -1 and o.max_rhs == 1 and o.ir_tol == 1e-13


def test_auto_lv_matches_reference_rule():
    from oracle import oracle
    for m in (2, 1000, 16384, 200000, 1048576, 2000000, 4000000, 30000000):
        for d in (0, 1):
            assert rbs.auto_lv(m, d) == oracle.auto_lv(m, d)


def _lower_csc(n=64, seed=0):
    from oracle import oracle
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=3, band=16, seed=seed)
    return oracle.transpose(rp, ci, va)


def _expect(code, *args, **kw):
    with pytest.raises(rbs.RbsError) as e:
        rbs.analyse(*args, opts=rbs.options(host_only=1), **kw)
    assert e.value.code == code, str(e.value)


def test_missing_diagonal_is_a_structure_error():
    cp, ri, va = _lower_csc()
    # drop the diagonal of column 5 (it is the first entry in forward layout)
    k = cp[5]
    keep = np.ones(len(ri), bool)
    keep[k] = False
    cp2 = cp.copy()
    cp2[6:] -= 1
    _expect(rbs.ERR_STRUCTURE, cp2, ri[keep], va[keep], substitution=rbs.FORWARD, lv=1)


def test_wrong_triangle_is_a_structure_error():
    cp, ri, va = _lower_csc()
    _expect(rbs.ERR_STRUCTURE, cp, ri, va, substitution=rbs.BACKWARD, lv=1)


def test_zero_diagonal_and_bad_index():
    cp, ri, va = _lower_csc()
    v2 = va.copy()
    v2[cp[3]] = 0.0
    _expect(rbs.ERR_STRUCTURE, cp, ri, v2, substitution=rbs.FORWARD, lv=1)
    r2 = ri.copy()
    r2[-1] = 10**6
    _expect(rbs.ERR_STRUCTURE, cp, r2, va, substitution=rbs.FORWARD, lv=1)


def test_bad_arguments():
    cp, ri, va = _lower_csc()
    _expect(rbs.ERR_ARG, cp, ri, va, substitution=7, lv=1)
    _expect(rbs.ERR_ARG, cp, ri, va, substitution=rbs.FORWARD, lv=10)  # 2^10 > n


def test_host_only_plan_refuses_to_solve():
    cp, ri, va = _lower_csc()
    plan = rbs.analyse(cp, ri, va, lv=1, opts=rbs.options(host_only=1))
    b = np.ones(len(cp) - 1)
    with pytest.raises(rbs.RbsError) as e:
        plan.solve_host(b)
    assert e.value.code == rbs.ERR_ARG


def test_empty_square_block_is_handled():
    # a diagonal matrix: every square block is empty (the reference divides
    # by zero there, recblocking_preprocess.h:825); here they become no-ops
    n = 256
    cp = np.arange(n + 1, dtype=np.int32)
    ri = np.arange(n, dtype=np.int32)
    va = np.linspace(1, 2, n)
    plan = rbs.analyse(cp, ri, va, lv=3, opts=rbs.options(host_only=1))
    meth = plan.export("method")
    kern = plan.export("kernel")
    assert (meth[1::2] == -1).all() and (kern[1::2] == rbs.K_EMPTY).all()
    assert (kern[0::2] == rbs.K_DIAG).all()


def _big_upper_csc(n=700000):
    # a lower CSR read as the CSC of its transpose: an upper triangle whose
    # columns hold the diagonal last (backward substitution)
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=2, band=8, seed=4)
    return rp, ci, va.copy()


def _message(*args, **kw):
    with pytest.raises(rbs.RbsError) as e:
        rbs.analyse(*args, opts=rbs.options(host_only=1), **kw)
    assert e.value.code == rbs.ERR_STRUCTURE, str(e.value)
    return str(e.value)


def test_large_input_reports_the_first_fault():
    # the checks run over chunks of columns and entries on host threads; the
    # error still names the first bad column or entry, as a serial scan does
    cp, ri, va = _big_upper_csc()
    for a, b in ((5, 650000), (300001, 600000), (699999, 699999)):
        v2 = va.copy()
        v2[cp[b + 1] - 1] = 0.0
        v2[cp[a + 1] - 1] = 0.0
        assert f"zero diagonal in column {a}" in _message(cp, ri, v2, substitution=rbs.BACKWARD, lv=2)
    r2 = ri.copy()
    k1, k2 = 123457, len(ri) - 3
    r2[k2] = -1
    r2[k1] = 10**7
    assert f"index out of range at entry {k1}" in _message(cp, r2, va, substitution=rbs.BACKWARD, lv=2)
    c2 = cp.copy()
    c2[650001] = c2[650000] - 1
    c2[400001] = c2[400000] - 1
    assert "pointer array decreases at 400000" in _message(c2, ri, va, substitution=rbs.BACKWARD, lv=2)
    # a column below the diagonal in an upper system: the wrong-triangle rule
    r3 = ri.copy()
    col = 500000 + int(np.argmax(np.diff(cp[500000:500100]) > 1))  # a column with an off-diagonal entry
    r3[cp[col]] = col + 1
    assert f"entry ({col + 1},{col}) outside the upper triangle" in _message(cp, r3, va, substitution=rbs.BACKWARD, lv=2)


def test_batch_reports_the_first_bad_system():
    systems = [rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=3000, lam=3, band=20, seed=s) for s in range(6)]
    bad = [list(s) for s in systems]
    for i in (4, 2):
        p = bad[i][0].copy()
        p[-1] += 1
        bad[i][0] = p
    with pytest.raises(rbs.RbsError) as e:
        rbs.batch_analyse([tuple(s) for s in bad], substitution=rbs.FORWARD, fmt=rbs.FMT_CSR,
                          opts=rbs.options(host_only=1))
    assert e.value.code == rbs.ERR_STRUCTURE and "system 2 " in str(e.value)
