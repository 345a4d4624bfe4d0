"""Level-chunk layout (csrc/level_lc.cuh) checked on the CPU.

The layout is exported from a host-only analysis and replayed by a Python
model of the kernel's schedule: chunk records are "copied" into a ring at
the iteration the host scheduled, gathered LC_D chunks ahead, solved in
order with a window of the last LC_XW rows.  The model asserts every rule
the kernel relies on (no live ring bytes overwritten, mbarrier slots free,
old dependencies final when gathered, recent dependencies present in the
window) and its solution is compared with the serial FP64 oracle.
"""
import numpy as np
import pytest

import rbs
from _util import rel_err
from oracle import oracle


def _pad4(n):
    return (n + 3) & ~3


def _padv(n, es):
    return ((n * es + 15) // 16) * 16 // es


def _static(nr, no, nrec, ncols, hdr):
    ints = hdr + 2 * _pad4(nr) + _pad4(nr + 1) + _pad4(ncols + 1) + _pad4(nrec) + _pad4(no)
    return 4 * ints + 8 * (_padv(nr, 8) + _padv(nrec, 8) + _padv(no, 8))


def _foot(nr, no, nrec, ncols, hdr):
    # gathered x of the old entries, then the right-hand-side area with
    # 32 bytes of slack for a 16-byte-aligned bulk copy
    return _static(nr, no, nrec, ncols, hdr) + 8 * (_padv(no, 8) + _padv(nr + 4, 8))


def _parse(words, src16, hdr):
    """Sections of one FP64 record (mirrors LcView)."""
    w = words[src16 * 4:]
    nr, no, nrec, vbase, rnext, ncols, maxlen, blo = (int(v) for v in w[:8])
    o = hdr

    def ints(cnt):
        nonlocal o
        v = w[o:o + cnt]
        o += _pad4(cnt)
        return v

    def dbl(cnt):
        nonlocal o
        v = w[o:o + 2 * cnt].copy().view(np.float64)
        o += 2 * _padv(cnt, 8)
        return v

    dest = ints(nr)
    rlen = ints(nr)
    rpo = ints(nr + 1)
    cs = ints(ncols + 1)
    inv = dbl(nr)
    colr = ints(nrec)
    valr = dbl(nrec)
    colo = ints(no)
    valo = dbl(no)
    return dict(nr=nr, no=no, nrec=nrec, vbase=vbase, rnext=rnext, ncols=ncols, maxlen=maxlen, blo=blo, dest=dest,
                rlen=rlen, rpo=rpo,
                cs=cs, inv=inv, colr=colr, valr=valr, colo=colo, valo=valo)


def emulate(plan, b_proc):
    XW, NB, D, RMAX, T, RING, FMAX, HDR = (int(v) for v in plan.export("lc_consts"))
    tab = plan.export("lc_tab").reshape(-1, 10)
    segs = plan.export("lc_segs").reshape(-1, 3)
    words = plan.export("lc_rec64")
    blk = plan.export("lc_block").reshape(-1, 3)
    br = plan.export("block_rows").reshape(-1, 2)
    x = np.full(len(b_proc), np.nan)
    nblocks = 0
    for b in range(0, len(br), 2):
        if blk[b, 0] < 0:
            continue
        nblocks += 1
        r0, m = int(br[b, 0]), int(br[b, 1])
        xb = x[r0:r0 + m]
        bb = b_proc[r0:r0 + m]
        for s in range(blk[b, 0], blk[b, 0] + blk[b, 1]):
            c0, nch, ring0 = (int(v) for v in segs[s])
            recs = [_parse(words, int(tab[c0 + j, 0]), HDR) for j in range(nch)]
            assert nch == 0 or int(tab[c0, 4]) == ring0
            live, issued, gathered = {}, [0], {}
            chunk_of = {}

            def issue_upto(it):
                while issued[0] < nch and tab[c0 + issued[0], 5] <= it:
                    j = issued[0]
                    r = recs[j]
                    lo = int(tab[c0 + j, 4]) * 16
                    f = _foot(r["nr"], r["no"], r["nrec"], r["ncols"], HDR)
                    assert f <= FMAX and lo + f <= RING
                    assert int(tab[c0 + j, 1]) * 16 == _static(r["nr"], r["no"], r["nrec"], r["ncols"], HDR)
                    blo, bn = int(tab[c0 + j, 6]), int(tab[c0 + j, 7])
                    assert blo == r["blo"]
                    if blo >= 0:  # contiguous rows: bulk right-hand side
                        assert bn == r["nr"] and sorted(r["dest"]) == list(range(blo, blo + bn))
                    assert int(tab[c0 + j, 8]) * 16 == _static(r["nr"], r["no"], r["nrec"], r["ncols"], HDR) + \
                        8 * _padv(r["no"], 8)
                    for k, (a, e) in live.items():
                        assert not (a < lo + f and lo < e), f"chunk {j} overwrites live chunk {k}"
                    if j >= NB:  # slot reuse: the previous user was gathered before a barrier that precedes `it`
                        g = j - NB - D  # its gather iteration (-1: the prologue, before iteration 0's barrier)
                        assert it >= max(g, -1) + 1 and it >= 1, "mbarrier slot still in use"
                    live[j] = (lo, lo + f)
                    issued[0] += 1

            def gather(j):
                assert j < issued[0], f"chunk {j} gathered before its copy was issued"
                r = recs[j]
                vals = xb[r["colo"]]
                assert not np.isnan(vals).any(), "old dependency not final when gathered"
                gathered[j] = (vals, bb[r["dest"]])

            issue_upto(0)
            for j in range(min(D, nch)):
                gather(j)
            win = np.full(XW, np.nan)
            for c in range(nch):
                issue_upto(c)
                if c + D < nch:
                    gather(c + D)
                r = recs[c]
                assert r["nr"] <= RMAX
                if c + 1 < nch:
                    assert r["rnext"] == int(tab[c0 + c + 1, 4])
                gx, bs = gathered.pop(c)
                rl = r["rlen"]
                assert (np.diff(rl) <= 0).all() and (len(rl) == 0 or rl[0] <= r["ncols"])
                for t in range(r["nr"]):
                    o0, o1 = r["rpo"][t], r["rpo"][t + 1]
                    es = r["cs"][:rl[t]] + t
                    assert (es < r["cs"][1:rl[t] + 1]).all(), "jagged column overrun"
                    wv = win[r["colr"][es]]
                    assert not np.isnan(wv).any(), "recent dependency missing from the window"
                    ssum = np.dot(r["valr"][es], wv) + np.dot(r["valo"][o0:o1], gx[o0:o1])
                    xv = (bs[t] - ssum) * r["inv"][t]
                    win[(r["vbase"] + t) & (XW - 1)] = xv
                    assert np.isnan(xb[r["dest"][t]])
                    xb[r["dest"][t]] = xv
                    chunk_of[int(r["dest"][t])] = c
                del live[c]
    return x, nblocks


def _system(kind, **kw):
    return rbs.gen_lower_csr(kind, **kw)


CASES = {
    "band_poisson": (rbs.GEN_BAND_POISSON, dict(n=16384, lam=6, band=512, seed=11)),
    "band_dense": (rbs.GEN_BAND_POISSON, dict(n=30000, lam=30, band=4096, seed=12)),
    "laplace_wide": (rbs.GEN_LAPLACE2D, dict(grid=1100, seed=13)),
    "zipf": (rbs.GEN_ZIPF, dict(n=20000, zipf_alpha=2.1, zipf_max=300, seed=14)),
    "chain": (rbs.GEN_CHAIN, dict(n=3000, chain_bw=3, seed=15)),
}


@pytest.mark.parametrize("lv", [0, -1])
@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
@pytest.mark.parametrize("case", sorted(CASES))
def test_lc_schedule_matches_oracle(case, sub, lv):
    if case == "laplace_wide" and (sub, lv) != (rbs.FORWARD, 0):
        pytest.skip("one wide-level case is enough")
    kind, kw = CASES[case]
    rp, ci, va = _system(kind, **kw)
    n = len(rp) - 1
    if sub == rbs.FORWARD:
        arp, aci, ava = rp, ci, va
    else:
        arp, aci, ava = oracle.transpose(rp, ci, va)
    plan = rbs.analyse(arp, aci, ava, substitution=sub, lv=lv, fmt=rbs.FMT_CSR,
                       opts=rbs.options(select=rbs.SELECT_TUNE, host_only=1))
    b = oracle.spmv_csr(arp, aci, ava, rbs.gen_uniform(kw["seed"] + 7, n))
    perm = plan.export("perm")
    x_proc, nblocks = emulate(plan, b[perm])
    assert nblocks > 0
    if lv == 0:
        # one triangle: the replay is the whole solve (with squares the
        # triangles' right-hand sides would need the square updates first,
        # so lv = -1 checks the schedule rules only)
        xo = oracle.sptrsv_csr(arp, aci, ava, sub, b)
        assert rel_err(x_proc, xo[perm]) <= 1e-12


def test_lc_batch_segments():
    systems = []
    rng = np.random.default_rng(5)
    for i in range(9):
        n = int(rng.integers(500, 4000))
        kind = i % 3
        if kind == 0:
            systems.append(_system(rbs.GEN_BAND_POISSON, n=n, lam=8, band=256, seed=100 + i))
        elif kind == 1:
            systems.append(_system(rbs.GEN_LAPLACE2D, grid=int(np.sqrt(n)), seed=100 + i))
        else:
            systems.append(_system(rbs.GEN_CHAIN, n=n, chain_bw=3, seed=100 + i))
    plan, offs = rbs.batch_analyse(systems, fmt=rbs.FMT_CSR, opts=rbs.options(select=rbs.SELECT_TUNE, host_only=1))
    bs, xs = [], []
    for i, (rp, ci, va) in enumerate(systems):
        b = oracle.spmv_csr(rp, ci, va, rbs.gen_uniform(300 + i, len(rp) - 1))
        bs.append(b)
        xs.append(oracle.sptrsv_csr(rp, ci, va, rbs.FORWARD, b))
    B = np.concatenate(bs)
    perm = plan.export("perm")
    x_proc, nblocks = emulate(plan, B[perm])
    assert nblocks == 1
    segs = plan.export("lc_segs").reshape(-1, 3)
    assert len(segs) == len(systems)
    x = np.empty_like(x_proc)
    x[perm] = x_proc
    for i in range(len(systems)):
        assert rel_err(x[offs[i]:offs[i + 1]], xs[i]) <= 1e-12
