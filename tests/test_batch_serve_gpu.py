"""Batched many-system plans, measured kernel selection and the request
server: every result checked against the serial FP64 oracle and against the
same system solved alone (relative 2-norm error <= 1e-12)."""
import threading

import numpy as np
import pytest

import rbs
from _util import load_fixture, rel_err
from oracle import oracle

TOL = 1e-12
pytestmark = pytest.mark.gpu


def small_systems(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = i % 4
        n = int(rng.integers(300, 3000))
        if kind == 0:
            L = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=n, lam=8, band=256, seed=seed * 100 + i)
        elif kind == 1:
            L = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=int(np.sqrt(n)) + 1, seed=seed * 100 + i)
        elif kind == 2:
            L = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=n, zipf_alpha=2.1, zipf_max=100, seed=seed * 100 + i)
        else:
            L = rbs.gen_lower_csr(rbs.GEN_CHAIN, n=n, chain_bw=3, seed=seed * 100 + i)
        out.append(L)
    return out


def as_input(L, sub):
    rp, ci, va = L
    if sub == rbs.FORWARD:
        return oracle.transpose(rp, ci, va), (rp, ci, va)
    return (rp, ci, va), oracle.transpose(rp, ci, va)


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
def test_batch_matches_oracle_and_alone(cuda, sub):
    import torch
    systems = small_systems(12, 7 + sub)
    inputs, Bs, Xrefs, alone = [], [], [], []
    for i, L in enumerate(systems):
        (cp, ri, cv), (arp, aci, ava) = as_input(L, sub)
        inputs.append((cp, ri, cv))
        b = oracle.spmv_csr(arp, aci, ava, rbs.gen_uniform(50 + i, len(cp) - 1))
        Bs.append(b)
        Xrefs.append(oracle.sptrsv_csr(arp, aci, ava, sub, b))
        plan = rbs.analyse(cp, ri, cv, substitution=sub, lv=-1)
        alone.append(plan.solve_host(b)[0])
    plan, offs = rbs.batch_analyse(inputs, substitution=sub)
    B = np.concatenate(Bs)
    db = torch.tensor(B, device=cuda)
    dx = torch.empty_like(db)
    plan.solve(db, dx)
    X = dx.cpu().numpy()
    for i in range(len(systems)):
        xi = X[offs[i]:offs[i + 1]]
        assert rel_err(xi, Xrefs[i]) <= TOL, i
        assert rel_err(xi, alone[i]) <= TOL, i
    # mixed precision on the batch as well
    plan.solve(db, dx, prec=rbs.PREC_MIXED)
    X2 = dx.cpu().numpy()
    for i in range(len(systems)):
        assert rel_err(X2[offs[i]:offs[i + 1]], Xrefs[i]) <= TOL, i


@pytest.mark.parametrize("name", ["band_lv3_fwd", "laplace40_lv2_bwd", "zipf_lv2_fwd", "chain_method1_bwd"])
def test_tuned_selection_parity(cuda, name):
    g, cp, ri, va, sub, lv = load_fixture(name)
    arp, aci, ava = oracle.transpose(cp, ri, va)
    b = oracle.spmv_csr(arp, aci, ava, rbs.gen_uniform(3, len(cp) - 1))
    xref = oracle.sptrsv_csr(arp, aci, ava, sub, b)
    plan = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(select=rbs.SELECT_TUNE))
    kern = plan.export("kernel")
    assert set(kern[0::2].tolist()) <= {rbs.K_DIAG, rbs.K_SYNCFREE, rbs.K_LEVEL, rbs.K_BANDSCAN}
    x, _ = plan.solve_host(b)
    assert rel_err(x, xref) <= TOL


def test_server_alone_vs_mixed(cuda):
    systems = small_systems(4, 11)
    srv = rbs.Server(hbm_budget_bytes=8 << 30, max_batch_rhs=16)
    fids, alone_plans, mats = [], [], []
    for L in systems:
        (cp, ri, cv), (arp, aci, ava) = as_input(L, rbs.FORWARD)
        fids.append(srv.add_factor(rbs.analyse(cp, ri, cv, lv=-1, opts=rbs.options(max_rhs=16))))
        alone_plans.append(rbs.analyse(cp, ri, cv, lv=-1, opts=rbs.options(max_rhs=16)))
        mats.append((arp, aci, ava))
    rng = np.random.default_rng(5)
    reqs = []
    for q in range(90):
        f = int(rng.integers(0, len(systems)))
        k = int(rng.integers(1, 5))
        n = len(mats[f][0]) - 1
        X = np.stack([rbs.gen_uniform(1000 + 10 * q + c, n) for c in range(k)])
        B = np.ascontiguousarray(np.stack([oracle.spmv_csr(*mats[f], X[c]) for c in range(k)]))
        prec = rbs.PREC_MIXED if q % 3 == 0 else rbs.PREC_FP64
        reqs.append(dict(f=f, k=k, B=B, X=np.zeros_like(B), prec=prec))
    tickets = [None] * len(reqs)

    def submitter(lo, hi):
        for i in range(lo, hi):
            r = reqs[i]
            tickets[i] = srv.submit(fids[r["f"]], r["B"], r["X"], r["k"], r["prec"])

    ths = [threading.Thread(target=submitter, args=(i * 30, i * 30 + 30)) for i in range(3)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    grew = False
    for i, r in enumerate(reqs):
        lat, bk = srv.wait(tickets[i])
        assert lat > 0 and bk >= r["k"]
        grew = grew or bk > r["k"]
    st = srv.stats()
    assert st.completed == len(reqs) and st.p99_ms >= st.p50_ms > 0
    for r in reqs:
        arp, aci, ava = mats[r["f"]]
        plan = alone_plans[r["f"]]
        for c in range(r["k"]):
            xa, _ = plan.solve_host(r["B"][c])
            xo = oracle.sptrsv_csr(arp, aci, ava, rbs.FORWARD, r["B"][c])
            assert rel_err(r["X"][c], xa) <= TOL
            assert rel_err(r["X"][c], xo) <= TOL
    assert grew, "no request was batched with another"
    srv.close()


def test_server_budget_admission(cuda):
    (cp, ri, cv), _ = as_input(small_systems(1, 3)[0], rbs.FORWARD)
    srv = rbs.Server(hbm_budget_bytes=1 << 12, max_batch_rhs=4)
    plan = rbs.analyse(cp, ri, cv, lv=-1)
    with pytest.raises(rbs.RbsError) as e:
        srv.add_factor(plan)
    assert e.value.code == rbs.ERR_BUDGET
    srv.close()
    assert plan.handle  # still the caller's


def test_bounded_wait_reports_timeout_and_plan_recovers(cuda):
    # a poll budget of one makes the sync-free kernel's dependency waits give
    # up: the solve must end with RBS_ERR_TIMEOUT, not hang, and the plan must
    # solve correctly afterwards with the default budget
    g, cp, ri, va, sub, lv = load_fixture("band_auto_fwd")
    arp, aci, ava = oracle.transpose(cp, ri, va)
    b = oracle.spmv_csr(arp, aci, ava, rbs.gen_uniform(9, len(cp) - 1))
    xref = oracle.sptrsv_csr(arp, aci, ava, sub, b)
    bad = rbs.analyse(cp, ri, va, substitution=sub, lv=lv,
                      opts=rbs.options(select=rbs.SELECT_REFERENCE, spin_limit=1))
    assert set(bad.export("kernel")[0::2].tolist()) == {rbs.K_SYNCFREE}
    with pytest.raises(rbs.RbsError) as e:
        bad.solve_host(b)
    assert e.value.code == rbs.ERR_TIMEOUT
    good = rbs.analyse(cp, ri, va, substitution=sub, lv=lv, opts=rbs.options(select=rbs.SELECT_REFERENCE))
    x, _ = good.solve_host(b)
    assert rel_err(x, xref) <= TOL


def test_cli_drop_in(cuda, tmp_path):
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "recblock-sptrsv_b200", "bin", "sptrsv")
    # a symmetric pattern (2D 5-point grid), as SuiteSparse files often are
    g = 30
    entries = []
    for r in range(g):
        for c in range(g):
            i = r * g + c + 1
            entries.append((i, i))
            if c + 1 < g:
                entries.append((i + 1, i))
            if r + 1 < g:
                entries.append((i + g, i))
    path = tmp_path / "grid.mtx"
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
        f.write(f"{g*g} {g*g} {len(entries)}\n")
        for i, j in entries:
            f.write(f"{i} {j}\n")
    for flag in ("-forward", "-backward"):
        out = subprocess.run([exe, "-d", "0", "-rhs", "1", "-lv", "-1", flag, "-mtx", str(path)], capture_output=True,
                             text=True, env={**os.environ, "RBS_SEED": "7", "RBS_BENCH_REPEAT": "3"}, timeout=120)
        assert out.returncode == 0, out.stderr
        assert "x check passed" in out.stdout, out.stdout
    bad = subprocess.run([exe, "-rhs", "1"], capture_output=True, text=True)
    assert bad.returncode == 2
