"""Host analysis results do not depend on the number of host threads
(RBS_HOST_THREADS): plans of a CSC system, a CSR system and two batches
built with 1 and with 5 threads are byte-identical apart from the field
holding the analysis time (and the file digest, which covers it).  Sizes
are above the thresholds where the transposition, the row builds, the pool
fill and the per-system layouts run on threads."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import os, struct, sys
root, out = sys.argv[1], sys.argv[2]
sys.path.insert(0, os.path.join(root, "recblock-sptrsv_b200"))
sys.path.insert(0, os.path.join(root, "tests", "golden"))
import rbs
from oracle import oracle

def save(p, name):
    path = os.path.join(out, name + ".rbs")
    p.save(path)
    data = bytearray(open(path, "rb").read())
    ms = struct.pack("<d", float(p.export("analyse_ms")[0]))
    at = data.find(ms, 0, 256)
    assert at >= 0
    data[at:at + 8] = bytes(8)
    open(path, "wb").write(bytes(data[:-8]))  # without the file digest, which covers the time

rp, ci, va = rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=300000, lam=6, band=300, seed=11)
cp, ri, cv = oracle.transpose(rp, ci, va)
for sel in (rbs.SELECT_AUTO, rbs.SELECT_TUNE):
    save(rbs.analyse(cp, ri, cv, substitution=rbs.FORWARD, lv=-1, opts=rbs.options(host_only=1, select=sel)), f"csc{sel}")
    save(rbs.analyse(rp, ci, va, substitution=rbs.FORWARD, lv=3, fmt=rbs.FMT_CSR,
                     opts=rbs.options(host_only=1, select=sel)), f"csr{sel}")
systems = [rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=4000 + 997 * i, lam=5, band=64, seed=40 + i) for i in range(48)]
for lv in (0, 2):
    p, _ = rbs.batch_analyse(systems, substitution=rbs.FORWARD, lv=lv, fmt=rbs.FMT_CSR,
                             opts=rbs.options(host_only=1, select=rbs.SELECT_TUNE))
    save(p, f"batch{lv}")
"""


def _plans(tmp, threads):
    out = os.path.join(tmp, f"t{threads}")
    os.makedirs(out)
    env = dict(os.environ, RBS_HOST_THREADS=str(threads))
    subprocess.run([sys.executable, "-c", SCRIPT, ROOT, out], env=env, check=True, timeout=600)
    return {f: open(os.path.join(out, f), "rb").read() for f in sorted(os.listdir(out))}


def test_plans_do_not_depend_on_host_threads(tmp_path):
    one = _plans(str(tmp_path), 1)
    five = _plans(str(tmp_path), 5)
    assert len(one) == 6 and one.keys() == five.keys()
    for name in one:
        assert one[name] == five[name], name
