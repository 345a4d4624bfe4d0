"""Seeded parity cases shared by make_golden.py and the tests.

Each case is a lower-triangular CSR L (columns ascending, diagonal last) plus
a direction and a recursion depth.  The forward input of the solver is
CSC(L); the backward input is CSC(L^T), which is L's CSR arrays.
"""
from __future__ import annotations

import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(_ROOT, "recblock-sptrsv_b200"))
sys.path.insert(0, _ROOT)


def _csr_from_rows(rows, seed):
    """rows: list of sorted off-diagonal column lists; values U(-1,1), diag 1+sum|off|."""
    rng = np.random.default_rng(seed)
    rp = [0]
    ci, va = [], []
    for i, cols in enumerate(rows):
        v = rng.uniform(-1, 1, len(cols))
        ci.extend(cols)
        va.extend(v)
        ci.append(i)
        va.append(1.0 + np.abs(v).sum())
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(va, np.float64)


def build(spec):
    """Return (rowptr, colidx, val) of L for a case spec."""
    import rbs

    kind = spec["kind"]
    if kind == "band":
        return rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=spec["n"], lam=spec["lam"], band=spec["band"], seed=spec["seed"])
    if kind == "laplace":
        return rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=spec["grid"], seed=spec["seed"])
    if kind == "zipf":
        return rbs.gen_lower_csr(rbs.GEN_ZIPF, n=spec["n"], zipf_alpha=spec["alpha"], zipf_max=spec["zmax"],
                                 seed=spec["seed"])
    if kind == "chain":
        return rbs.gen_lower_csr(rbs.GEN_CHAIN, n=spec["n"], chain_bw=spec["bw"], seed=spec["seed"])
    rng = np.random.default_rng(spec["seed"])
    n = spec["n"]
    if kind == "bipartite":
        # triangles diagonal-only, all coupling in the squares
        s = n // (1 << spec["lv"])
        rows = []
        for i in range(n):
            t = min(i // s, (1 << spec["lv"]) - 1)
            lo = 0
            hi = t * s
            k = min(int(rng.poisson(3)), hi - lo)
            rows.append(sorted(rng.choice(hi - lo, size=k, replace=False) + lo) if k else [])
        return _csr_from_rows(rows, spec["seed"] + 1)
    if kind == "longrows":
        # banded base plus a few dense rows (> 2048 entries inside one square)
        rows = []
        for i in range(n):
            if i >= n - spec["ndense"]:
                rows.append(list(range(0, spec["dense_to"])))
            else:
                lo = max(0, i - spec["band"])
                k = min(int(rng.poisson(spec["lam"])), i - lo)
                rows.append(sorted(rng.choice(i - lo, size=k, replace=False) + lo) if k else [])
        return _csr_from_rows(rows, spec["seed"] + 1)
    if kind == "dense":
        rows = []
        for i in range(n):
            k = min(int(rng.poisson(spec["lam"])), i)
            rows.append(sorted(rng.choice(i, size=k, replace=False)) if k else [])
        return _csr_from_rows(rows, spec["seed"] + 1)
    raise ValueError(kind)


def inputs(spec, substitution):
    """(colptr, rowidx, val) of the solver input in the reference's CSC layout."""
    from oracle import oracle

    rp, ci, va = build(spec)
    if substitution == 0:
        return oracle.transpose(rp, ci, va)
    return rp, ci, va


CASES = {
    "band_auto": dict(kind="band", n=3000, lam=6, band=256, seed=11, lv=-1),
    "band_lv3": dict(kind="band", n=3000, lam=6, band=256, seed=12, lv=3),
    "laplace40_lv2": dict(kind="laplace", grid=40, seed=13, lv=2),
    "zipf_lv2": dict(kind="zipf", n=4000, alpha=2.1, zmax=200, seed=14, lv=2),
    "zipf_lv3": dict(kind="zipf", n=4000, alpha=2.1, zmax=200, seed=15, lv=3),
    "chain_method1": dict(kind="chain", n=44000, bw=3, seed=16, lv=1),
    "bipartite_lv1": dict(kind="bipartite", n=2000, seed=17, lv=1),
    "longrows_lv2": dict(kind="longrows", n=4400, lam=3, band=48, ndense=3, dense_to=4300, seed=18, lv=2),
    "dense_lv2": dict(kind="dense", n=1200, lam=30, seed=19, lv=2),
    "band_lv0": dict(kind="band", n=800, lam=5, band=100, seed=20, lv=0),
}
# fixtures that store only outputs: inputs come from the seeded C generator
# (include/rbs_gen.h) and are checked against the stored input digest
SPEC_ONLY = {"band_auto", "band_lv3", "laplace40_lv2", "zipf_lv2", "zipf_lv3", "chain_method1", "band_lv0"}
