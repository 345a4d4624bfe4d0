"""Distinct plans may be analysed from several host threads at once (the
boundary's convention: thread-safe for distinct plans; the error message is
per thread): four threads analyse four systems, one of them malformed, each
twice; every plan equals the one the same analysis gives alone, and only the
malformed one fails, with its own message."""
import struct
import threading

import rbs
from oracle import oracle


def _bytes(plan, path):
    plan.save(path)
    data = bytearray(open(path, "rb").read())
    at = data.find(struct.pack("<d", float(plan.export("analyse_ms")[0])), 0, 256)
    data[at:at + 8] = bytes(8)
    return bytes(data[:-8])  # the file digest covers the time


def test_concurrent_host_analyses(tmp_path):
    systems = [rbs.gen_lower_csr(rbs.GEN_BAND_POISSON, n=150000, lam=5, band=200, seed=31),
               rbs.gen_lower_csr(rbs.GEN_ZIPF, n=120000, zipf_alpha=2.0, zipf_max=300, seed=32),
               rbs.gen_lower_csr(rbs.GEN_LAPLACE2D, grid=300, seed=33)]
    inputs = [oracle.transpose(*s) for s in systems]
    bad = tuple(a.copy() for a in inputs[0])
    bad[2][bad[0][777]] = 0.0  # zero diagonal in column 777
    inputs.append(bad)
    opts = rbs.options(host_only=1, select=rbs.SELECT_TUNE)
    alone = [_bytes(rbs.analyse(*inp, substitution=rbs.FORWARD, lv=-1, opts=opts), str(tmp_path / f"a{i}.rbs"))
             for i, inp in enumerate(inputs[:3])]
    results = {}

    def work(i):
        out = []
        for rep in range(2):
            try:
                p = rbs.analyse(*inputs[i], substitution=rbs.FORWARD, lv=-1, opts=opts)
                out.append(_bytes(p, str(tmp_path / f"t{i}_{rep}.rbs")))
            except rbs.RbsError as e:
                out.append(str(e))
        results[i] = out

    threads = [threading.Thread(target=work, args=(i,)) for i in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i in range(3):
        assert results[i] == [alone[i], alone[i]], i
    assert all("zero diagonal in column 777" in m for m in results[3]), results[3]
