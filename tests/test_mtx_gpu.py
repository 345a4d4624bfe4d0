"""Matrix Market input parsed on the device (rbs_mtx_*), against the
reference's own mmio_data outputs (tests/golden/mtx) and the oracle's
fscanf reader: CSR row pointers and columns identical, values identical bit
for bit; the triangle of main.cu:157-198 and its CSC (tranpose.h) identical
to the oracle's; larger seeded files with every value spelling; malformed
files rejected with a status; a full-size 2D Laplacian read, cut into its
triangle and solved end to end."""
import glob
import os

import numpy as np
import pytest

import rbs
from _util import rel_err
from oracle import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "mtx", "*.mtx")))


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


def check_csr(M, rp, ci, va):
    drp, dci, dva = M.csr()
    np.testing.assert_array_equal(drp.cpu().numpy(), rp)
    np.testing.assert_array_equal(dci.cpu().numpy(), ci)
    np.testing.assert_array_equal(bits(dva.cpu().numpy()), bits(va))


def lower_upper(rp, ci):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    return int((ci < rows).sum()), int((ci > rows).sum())


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_device_reader_matches_reference(cuda, path):
    g = np.load(path[:-4] + ".npz")
    for M in (rbs.mtx_read(path), rbs.mtx_read_buffer(open(path, "rb").read())):
        i = M.info
        assert (i.m, i.n, i.nnz, i.symmetric) == (int(g["m"]), int(g["n"]), len(g["colidx"]), int(g["symmetric"]))
        assert (i.nnz_lower, i.nnz_upper) == lower_upper(g["rowptr"], g["colidx"])
        check_csr(M, g["rowptr"], g["colidx"], g["val"])
    if os.path.basename(path) == "general_values.mtx":
        assert M.info.host_values == 5  # 1e-300, the 21-digit and 36-digit tokens, -1.79e308, 4.9e-324


@pytest.mark.parametrize("path", [p for p in FIXTURES if "rectangular" not in p and "integer_general" not in p],
                         ids=lambda p: os.path.basename(p)[:-4])
def test_device_triangle_matches_oracle(cuda, path):
    import torch
    g = np.load(path[:-4] + ".npz")
    M = rbs.mtx_read(path)
    for sub in (rbs.FORWARD, rbs.BACKWARD):
        nstrict = M.info.nnz_lower if sub == rbs.FORWARD else M.info.nnz_upper
        strict = np.random.default_rng(7).integers(1, 11, max(nstrict, 1)).astype(np.float64)[:nstrict]
        for sv in (None, strict):
            tp, ti, tv = oracle.tri_extract(g["rowptr"], g["colidx"], g["val"], sub, sv)
            dsv = None if sv is None else torch.tensor(sv, device=cuda)
            p, x, v = M.triangle(sub, rbs.FMT_CSR, dsv)
            np.testing.assert_array_equal(p.cpu().numpy(), tp)
            np.testing.assert_array_equal(x.cpu().numpy(), ti)
            np.testing.assert_array_equal(bits(v.cpu().numpy()), bits(tv))
            cp, cr, cv = oracle.transpose(tp, ti, tv)
            p, x, v = M.triangle(sub, rbs.FMT_CSC, dsv)
            np.testing.assert_array_equal(p.cpu().numpy(), cp)
            np.testing.assert_array_equal(x.cpu().numpy(), cr)
            np.testing.assert_array_equal(bits(v.cpu().numpy()), bits(cv))


def write_random(path, seed, n, nz, field="real", sym=False, spelling="17g"):
    rng = np.random.default_rng(seed)
    rows = rng.integers(1, n + 1, nz)
    cols = rng.integers(1, n + 1, nz)
    if sym:
        rows, cols = np.maximum(rows, cols), np.minimum(rows, cols)
    mant = rng.standard_normal(nz)
    ex = rng.integers(-70, 70, nz)
    vals = mant * 10.0 ** ex.astype(np.float64)
    lines = [f"%%MatrixMarket matrix coordinate {field} {'symmetric' if sym else 'general'}", "% seeded", f"{n} {n} {nz}"]
    for r, c, v, e in zip(rows, cols, vals, ex):
        if field == "pattern":
            lines.append(f"{r} {c}")
        elif field == "integer":
            lines.append(f"{r}\t{c}\t{int(e) * 1000 + int(r)}")
        elif spelling == "17g":
            lines.append(f"{r} {c} {v:.17g}")
        elif spelling == "16e":
            lines.append(f"{r}  {c}  {v:.16e}")
        else:  # short decimals with explicit signs and point forms
            lines.append(f"{r} {c} {v:+.4f}" if abs(v) < 1e6 else f"{r} {c} {v:.3E}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


@pytest.mark.parametrize("case", [
    (11, 20000, 300000, "real", True, "17g"),
    (12, 50000, 300000, "real", False, "16e"),
    (13, 30000, 200000, "real", False, "short"),
    (14, 40000, 250000, "pattern", True, None),
    (15, 10000, 100000, "integer", False, None),
    (16, 5, 2000, "real", True, "17g"),        # many duplicates per row
])
def test_device_reader_random_files(cuda, tmp_path, case):
    seed, n, nz, field, sym, spelling = case
    path = str(tmp_path / "r.mtx")
    write_random(path, seed, n, nz, field, sym, spelling)
    o = oracle.mtx_read(path)
    M = rbs.mtx_read(path)
    assert (M.info.m, M.info.nnz, M.info.nnz_file) == (n, len(o["colidx"]), nz)
    check_csr(M, o["rowptr"], o["colidx"], o["val"])


@pytest.mark.parametrize("body,code", [
    ("3 3 2\n1 1 1.0\n", rbs.ERR_ARG),                       # truncated
    ("3 3 2\n1 1 1.0\n2 4 1.0\n", rbs.ERR_STRUCTURE),         # column out of range
    ("3 3 2\n1 1 1.0\n0 2 1.0\n", rbs.ERR_STRUCTURE),         # row 0
    ("3 3 2\n1 1 1.5x\n2 2 1.0\n", rbs.ERR_ARG),              # malformed value
    ("3 3 2\n1 1 1.0\n2 b 1.0\n", rbs.ERR_ARG),               # malformed index
    ("3 3 2\n1 1 1.0\n2 2 1e\n", rbs.ERR_ARG),                # exponent without digits
])
def test_device_reader_rejects_bad_entries(cuda, body, code):
    text = "%%MatrixMarket matrix coordinate real general\n" + body
    with pytest.raises(rbs.RbsError) as e:
        rbs.mtx_read_buffer(text.encode())
    assert e.value.code == code, str(e.value)


def test_long_and_out_of_window_tokens_go_through_the_host(cuda):
    # values whose decimal exponent lies outside the device's exact window,
    # one of them longer than a host slot (100 zeros after the point)
    tiny = "0." + "0" * 100 + "123"
    text = ("%%MatrixMarket matrix coordinate real general\n3 3 4\n"
            f"1 1 {tiny}\n2 2 1e-200\n3 3 -2.5e+300\n3 1 0.5\n")
    M = rbs.mtx_read_buffer(text.encode())
    assert M.info.host_values == 3
    _, _, va = M.csr()
    # rows ascending, file order inside row 3: (3,3) then (3,1)
    np.testing.assert_array_equal(bits(va.cpu().numpy()), bits(np.array([float(tiny), 1e-200, -2.5e300, 0.5])))


@pytest.mark.parametrize("sym", [False, True])
def test_write_read_round_trip_at_size(cuda, tmp_path, sym):
    # rbs_mtx_write's %.17g values read back bit for bit; a symmetric file
    # (lower triangle written) expands to L + L^T - diag(L)
    rp, ci, _ = rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=1024, seed=61)
    va = rbs.gen_uniform(62, len(ci)) * 10.0 ** np.random.default_rng(63).integers(-40, 40, len(ci))
    path = str(tmp_path / "w.mtx")
    rbs.mtx_write(path, rp, ci, va, symmetric=sym)
    M = rbs.mtx_read(path)
    if not sym:
        check_csr(M, rp, ci, va)
    else:
        o = oracle.mtx_read(path)
        check_csr(M, o["rowptr"], o["colidx"], o["val"])
        # the lower part of every row, in file order, is the written row
        drp, dci, dva = (t.cpu().numpy() for t in M.csr())
        rows = np.repeat(np.arange(len(drp) - 1), np.diff(drp))
        low = dci <= rows
        np.testing.assert_array_equal(dci[low], ci)
        np.testing.assert_array_equal(bits(dva[low]), bits(va))


def test_triangle_needs_square(cuda):
    M = rbs.mtx_read(os.path.join(ROOT, "tests", "golden", "mtx", "rectangular.mtx"))
    with pytest.raises(rbs.RbsError) as e:
        M.triangle(rbs.FORWARD)
    assert e.value.code == rbs.ERR_STRUCTURE


def laplacian_file(path, g):
    """The lower triangle of the 5-point Laplacian on a g x g grid in
    symmetric storage, column by column as collections store it."""
    n = g * g
    j = np.arange(n, dtype=np.int64)
    r = np.stack([j, np.where(j % g != g - 1, j + 1, -1), np.where(j + g < n, j + g, -1)], 1)  # per column
    c = np.repeat(j, 3).reshape(n, 3)
    keep = r >= 0
    r, c = r[keep] + 1, c[keep] + 1
    v = np.where(r == c, 4, -1)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{n} {n} {len(r)}\n")
        f.write(("%d %d %d\n" * len(r)) % tuple(np.stack([r, c, v], 1).ravel().tolist()))
    return n


def test_fullsize_laplacian_read_extract_solve(cuda, tmp_path):
    import torch
    path = str(tmp_path / "lap.mtx")
    n = laplacian_file(path, 1024)
    o = oracle.mtx_read(path)
    M = rbs.mtx_read(path)
    assert M.info.nnz == len(o["colidx"]) == 5 * n - 4 * 1024
    check_csr(M, o["rowptr"], o["colidx"], o["val"])
    for sub in (rbs.FORWARD, rbs.BACKWARD):
        nstrict = M.info.nnz_lower if sub == rbs.FORWARD else M.info.nnz_upper
        # small strict values against the unit diagonal keep T well conditioned
        sv = rbs.gen_uniform(3 + sub, nstrict, -0.2, 0.2)
        tp, ti, tv = oracle.tri_extract(o["rowptr"], o["colidx"], o["val"], sub, sv)
        cp, cr, cv = oracle.transpose(tp, ti, tv)
        p, x, v = M.triangle(sub, rbs.FMT_CSC, torch.tensor(sv, device=cuda))
        np.testing.assert_array_equal(p.cpu().numpy(), cp)
        np.testing.assert_array_equal(x.cpu().numpy(), cr)
        np.testing.assert_array_equal(bits(v.cpu().numpy()), bits(cv))
        # main.cu's flow from here: analyse the device CSC and solve T x = b
        plan = rbs.analyse_device(p, x, v, n, v.numel(), substitution=sub)
        xr = rbs.gen_uniform(9, n)
        b = oracle.spmv_csr(tp, ti, tv, xr)
        db = torch.tensor(b, device=cuda)
        dx = torch.empty_like(db)
        plan.solve(db, dx)
        assert rel_err(dx.cpu().numpy(), oracle.sptrsv_csr(tp, ti, tv, sub, b)) <= 1e-12
