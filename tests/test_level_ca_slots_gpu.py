"""The staged level kernel's column forms: level-ELL widths 1, 2 and 4, with
every dependency inside the shared-memory window, so that the columns are
window slots (16-bit for widths 2 and 4, 32-bit for width 1).  Grid-like
factors built here: one dependency a grid row back (width 1), the 5-point
Laplacian (width 2) and a 9-point stencil's lower half (width 4).  Both
directions, FP64 and mixed precision, one and eight right-hand sides (the
multi-column launch stages the same slots), every column against the
serial FP64 oracle at 1e-12."""
import numpy as np
import pytest
import scipy.sparse as sp

import rbs
from _util import rel_err
from oracle import oracle

TOL = 1e-12
GRID = 128
pytestmark = pytest.mark.gpu


def stencil_lower(offsets, grid=GRID, seed=0):
    """Lower-triangular CSR on a grid x grid mesh in natural order: row
    (i, j) depends on (i + di, j + dj) for each offset that stays on the
    mesh and precedes it; off-diagonals uniform in [-0.25, 0.25], the
    diagonal 1 + the row's absolute off-diagonal sum."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(grid):
        for j in range(grid):
            r = i * grid + j
            for di, dj in offsets:
                ii, jj = i + di, j + dj
                if 0 <= ii < grid and 0 <= jj < grid and ii * grid + jj < r:
                    rows.append(r)
                    cols.append(ii * grid + jj)
    n = grid * grid
    off = rng.uniform(-0.25, 0.25, len(rows))
    L = sp.csr_matrix((off, (rows, cols)), shape=(n, n))
    d = 1.0 + np.asarray(abs(L).sum(axis=1)).ravel()
    L = (L + sp.diags(d)).tocsr()
    L.sort_indices()
    return L.indptr.astype(np.int32), L.indices.astype(np.int32), L.data.astype(np.float64)


SYSTEMS = {
    # width 1: (i-1, j)
    "one_back": (1, lambda: stencil_lower([(-1, 0)], seed=1)),
    # width 2: the 5-point Laplacian's lower factor
    "laplace5": (2, lambda: rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=GRID, seed=2)),
    # width 4: (i, j-1), (i-1, j-1), (i-1, j), (i-1, j+1)
    "nine_point": (4, lambda: stencil_lower([(0, -1), (-1, -1), (-1, 0), (-1, 1)], seed=3)),
}


def system(cp, ri, va, sub, k, seed):
    arp, aci, ava = oracle.transpose(cp, ri, va)
    n = len(cp) - 1
    X = np.stack([rbs.gen_uniform(seed + c, n) for c in range(k)])
    B = np.stack([oracle.spmv_csr(arp, aci, ava, X[c]) for c in range(k)])
    return B, oracle.sptrsv_csr(arp, aci, ava, sub, B)


@pytest.mark.parametrize("sub", [rbs.FORWARD, rbs.BACKWARD])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_window_slot_columns(cuda, name, sub):
    import torch
    width, make = SYSTEMS[name]
    rp, ci, va = make()
    # forward: L's CSC; backward: L's CSR read as the CSC of U = L^T
    cp, ri, cv = oracle.transpose(rp, ci, va) if sub == rbs.FORWARD else (rp, ci, va)
    plan = rbs.analyse(cp, ri, cv, substitution=sub, lv=-1, opts=rbs.options(max_rhs=8))
    kern = plan.export("kernel")
    cb = plan.export("ca_block").reshape(-1, 4)
    var = plan.export("lc_block").reshape(-1, 3)[:, 2]
    staged = [b for b in range(len(kern)) if kern[b] == rbs.K_LEVEL and var[b] == 1 and cb[b, 0] >= 0]
    # the path under test runs: staged level triangles of this width with window-slot columns
    assert staged, "no staged level triangle"
    assert all(cb[b, 2] == width and cb[b, 3] == 1 for b in staged), cb[staged]
    for k in (1, 8):
        B, Xref = system(cp, ri, cv, sub, k, seed=100 * k + sub)
        db = torch.tensor(np.ascontiguousarray(B), dtype=torch.float64, device=cuda).reshape(-1)
        for prec in (rbs.PREC_FP64, rbs.PREC_MIXED):
            dx = torch.full_like(db, float("nan"))
            plan.solve(db, dx, k=k, prec=prec)
            X = dx.cpu().numpy().reshape(B.shape)
            for c in range(k):
                assert rel_err(X[c], Xref[c]) <= TOL, (k, prec, c)
