"""Matrix Market input without a GPU: the oracle's reader pinned against the
reference's own mmio_data outputs (tests/golden/mtx/*.npz, made by
make_mtx_golden.py from oracle/_ref/mtx_dump), the oracle's triangle
extraction checked against main.cu:157-198's rules, the device reader's
token parser (csrc/mtx_parse.cuh) built for the host and checked against
strtod bit for bit, and the library's header checks, which fail before any
device work."""
import glob
import os
import subprocess

import numpy as np
import pytest

import rbs
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "mtx", "*.mtx")))


def golden(path):
    return np.load(path[:-4] + ".npz")


def test_fixture_set_is_complete():
    names = {os.path.basename(p)[:-4] for p in FIXTURES}
    assert {"general_values", "symmetric_lower", "pattern_symmetric", "integer_general", "complex_hermitian",
            "skew_symmetric", "whitespace", "rectangular", "no_entries", "random_sym_17g"} <= names
    for p in FIXTURES:
        assert os.path.exists(p[:-4] + ".npz"), p


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_reader_matches_reference(path):
    g = golden(path)
    o = oracle.mtx_read(path)
    assert (o["m"], o["n"], o["symmetric"]) == (int(g["m"]), int(g["n"]), int(g["symmetric"]))
    np.testing.assert_array_equal(o["rowptr"], g["rowptr"])
    np.testing.assert_array_equal(o["colidx"], g["colidx"])
    np.testing.assert_array_equal(o["val"].view(np.uint64), g["val"].view(np.uint64))


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


@pytest.mark.parametrize("text,code", [
    ("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1\n", -5),        # truncated
    ("%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1\n", -6),        # row out of range
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", -3),          # array storage
    ("%%MatrixMarket matrix coordinate quaternion general\n1 1 0\n", -3),         # unknown field
    ("%MatrixMarket matrix coordinate real general\n1 1 0\n", -2),                # bad banner
])
def test_oracle_reader_errors(tmp_path, text, code):
    with pytest.raises(RuntimeError) as e:
        oracle.mtx_read(_write(tmp_path, "bad.mtx", text))
    assert e.value.args[1] == code


@pytest.mark.parametrize("sub", [oracle.FORWARD, oracle.BACKWARD])
@pytest.mark.parametrize("name", ["general_values", "symmetric_lower", "random_sym_17g", "random_gen_16e"])
def test_oracle_triangle_rules(sub, name):
    g = golden(os.path.join(ROOT, "tests", "golden", "mtx", name + ".mtx"))
    rp, ci, va = g["rowptr"], g["colidx"], g["val"]
    m = len(rp) - 1
    strict = np.arange(1, 1 + len(ci), dtype=np.float64)
    for sv in (None, strict):
        tp, ti, tv = oracle.tri_extract(rp, ci, va, sub, sv)
        r = 0
        for i in range(m):
            row = [(ci[k], va[k]) for k in range(rp[i], rp[i + 1]) if (ci[k] < i if sub == oracle.FORWARD else ci[k] > i)]
            got = list(zip(ti[tp[i]:tp[i + 1]], tv[tp[i]:tp[i + 1]]))
            diag, rest = (got[-1], got[:-1]) if sub == oracle.FORWARD else (got[0], got[1:])
            assert diag == (i, 1.0)
            assert [c for c, _ in rest] == [c for c, _ in row]
            want = [v for _, v in row] if sv is None else list(sv[r:r + len(row)])
            assert [v for _, v in rest] == want
            r += len(row)


def test_parser_matches_strtod(tmp_path):
    exe = str(tmp_path / "mtx_parse_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "recblock-sptrsv_b200", "csrc"),
                    os.path.join(ROOT, "tests", "mtx_parse_check.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe, "1000000"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    ok, host = map(int, out.stdout.split()[1:3])
    assert ok > 800000 and host < ok


@pytest.mark.parametrize("text,code", [
    ("%MatrixMarket matrix coordinate real general\n1 1 0\n", rbs.ERR_ARG),
    ("%%MatrixMarket matrix array real general\n2 2\n", rbs.ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix coordinate quaternion general\n1 1 0\n", rbs.ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix coordinate real general\n% no size line\n", rbs.ERR_ARG),
    ("%%MatrixMarket matrix coordinate real general\nthree by three\n", rbs.ERR_ARG),
    ("", rbs.ERR_ARG),
])
def test_library_header_errors(tmp_path, text, code):
    # rejected while reading the header, before any device call
    with pytest.raises(rbs.RbsError) as e:
        rbs.mtx_read_buffer(text.encode())
    assert e.value.code == code, str(e.value)
    with pytest.raises(rbs.RbsError) as e:
        rbs.mtx_read(_write(tmp_path, "h.mtx", text))
    assert e.value.code == code, str(e.value)


def test_library_missing_file(tmp_path):
    with pytest.raises(rbs.RbsError) as e:
        rbs.mtx_read(str(tmp_path / "absent.mtx"))
    assert e.value.code == rbs.ERR_ARG


@pytest.mark.parametrize("kind", ["general", "symmetric", "pattern"])
def test_writer_round_trips_through_the_oracle_reader(tmp_path, kind):
    # rbs_mtx_write is host code: %.17g values read back bit for bit by the
    # reference-style reader; symmetric files hold the lower triangle
    rp, ci, va = rbs.gen_lower_csr(rbs.GEN_ZIPF, n=3000, zipf_alpha=2.1, zipf_max=50, seed=21)
    va = va * 10.0 ** np.random.default_rng(22).integers(-30, 30, len(va))
    path = str(tmp_path / "w.mtx")
    rbs.mtx_write(path, rp, ci, None if kind == "pattern" else va, symmetric=kind == "symmetric")
    o = oracle.mtx_read(path)
    n = len(rp) - 1
    if kind == "general":
        np.testing.assert_array_equal(o["rowptr"], rp)
        np.testing.assert_array_equal(o["colidx"], ci)
        np.testing.assert_array_equal(o["val"].view(np.uint64), va.view(np.uint64))
    elif kind == "pattern":
        assert o["field"] == 2
        np.testing.assert_array_equal(o["colidx"], ci)
        assert (o["val"] == 1.0).all()
    else:
        assert o["symmetric"] == 1
        rows = np.repeat(np.arange(n), np.diff(o["rowptr"]))
        low = o["colidx"] <= rows
        np.testing.assert_array_equal(o["colidx"][low], ci)
        np.testing.assert_array_equal(o["val"][low].view(np.uint64), va.view(np.uint64))
        assert int((~low).sum()) == int((ci < np.repeat(np.arange(n), np.diff(rp))).sum())
