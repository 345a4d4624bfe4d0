"""Matrix Market fixtures and the REFERENCE's own reading of them.

Writes small .mtx files to tests/golden/mtx/ (hand-written corner cases and
seeded random matrices: every field, symmetry, comment and whitespace form
the reader must take) and runs oracle/_ref/mtx_dump -- recblock-sptrsv's
mmio_info + mmio_data compiled from the reference sources by oracle/Makefile
-- on each, saving its CSR as tests/golden/mtx/<name>.npz.  Needs the
reference sources; run here, not on a GPU box:
    make -C oracle ref REF=<reference recblock-sptrsv dir> && python tests/golden/make_mtx_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "mtx")
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle  # noqa: E402

HAND = {
    # duplicates, unsorted rows, empty rows, every value spelling
    "general_values": """%%MatrixMarket matrix coordinate real general
% values in many spellings
6 6 12
3 1 1.5
1 1 -0
6 6 1e-300
2 2 12345678901234567890.5
3 1 2.5E+3
5 2 .125
1 3 -7.
4 4 0.1
4 4 3.14159265358979323846264338327950288
6 1 -1.7976931348623157e308
2 6 4.9406564584124654e-324
5 5 1.0000000000000002
""",
    "symmetric_lower": """%%MatrixMarket matrix coordinate real symmetric
5 5 9
1 1 4
2 1 -1
2 2 4
3 2 -1
3 3 4
4 1 0.5
4 4 4
5 3 -1.25e-2
5 5 4
""",
    "pattern_symmetric": """%%MatrixMarket matrix coordinate pattern symmetric
4 4 5
1 1
3 1
4 2
4 3
2 2
""",
    "integer_general": """%%MatrixMarket matrix coordinate integer general
3 4 5
1 4 -3
3 3 7
2 1 +12
1 1 0
3 2 2147483647
""",
    "complex_hermitian": """%%MatrixMarket matrix coordinate complex hermitian
3 3 4
1 1 2.0 0.0
2 1 1.5 -0.5
3 2 -2.25 1e-3
3 3 1 0
""",
    "skew_symmetric": """%%MatrixMarket matrix coordinate real skew-symmetric
3 3 2
2 1 5
3 1 -6
""",
    # upper-case banner words, comments and blank lines, CRLF, tabs,
    # an entry split across lines, trailing spaces, no final newline
    "whitespace": "%%MatrixMarket MATRIX Coordinate REAL General\r\n%c1\r\n%\r\n\r\n"
                  "4 4 6\r\n1\t1\t1.0\r\n  2   2    2.0   \r\n3 3\r\n 3.0\r\n4 4 4.0\r\n4\t1\t-1.0\r\n3 2 -2e0",
    "rectangular": """%%MatrixMarket matrix coordinate real general
2 5 4
1 5 1
2 3 2
1 1 3
2 1 4
""",
    "no_entries": """%%MatrixMarket matrix coordinate real general
3 3 0
""",
}


def random_file(path, rng, n, nz, field, sym, fmt):
    rows = rng.integers(1, n + 1, nz)
    cols = rng.integers(1, n + 1, nz)
    if sym:  # stored lower triangle, as symmetric files are
        rows, cols = np.maximum(rows, cols), np.minimum(rows, cols)
    vals = rng.standard_normal(nz) * 10.0 ** rng.integers(-8, 8, nz)
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {'symmetric' if sym else 'general'}\n")
        f.write(f"{n} {n} {nz}\n")
        for r, c, v in zip(rows, cols, vals):
            if field == "pattern":
                f.write(f"{r} {c}\n")
            elif field == "integer":
                f.write(f"{r} {c} {int(v * 1000) % 100000}\n")
            else:
                f.write(f"{r} {c} {fmt % v}\n")


RANDOM = {
    "random_sym_17g": (1, 3000, 8000, "real", True, "%.17g"),
    "random_gen_16e": (2, 2500, 8000, "real", False, "%.16e"),
    "random_gen_6g": (3, 2000, 6000, "real", False, "%.6g"),
    "random_sym_pattern": (4, 2000, 5000, "pattern", True, None),
    "random_gen_integer": (5, 1500, 4000, "integer", False, None),
}


def main():
    if not os.path.exists(oracle.MTX_REF_DUMP):
        sys.exit("oracle/_ref/mtx_dump missing: run make -C oracle ref REF=<reference recblock-sptrsv dir>")
    os.makedirs(OUT, exist_ok=True)
    for name, text in HAND.items():
        with open(os.path.join(OUT, name + ".mtx"), "w", newline="") as f:
            f.write(text)
    for name, (seed, n, nz, field, sym, fmt) in RANDOM.items():
        random_file(os.path.join(OUT, name + ".mtx"), np.random.default_rng(seed), n, nz, field, sym, fmt)
    for name in list(HAND) + list(RANDOM):
        path = os.path.join(OUT, name + ".mtx")
        ref = oracle.run_reference_mtx(path)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **{k: np.asarray(v) for k, v in ref.items()})
        print(f"{name}: {ref['m']}x{ref['n']} nnz={len(ref['colidx'])} sym={ref['symmetric']}")


if __name__ == "__main__":
    main()
