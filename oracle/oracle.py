"""TEST INFRASTRUCTURE ONLY: ctypes binding of liboracle.so (oracle.c).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the library under test never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
REF_DUMP = os.path.join(_HERE, "_ref", "ref_dump")

FORWARD, BACKWARD = 0, 1


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)


if not os.path.exists(_LIB):
    build()

lib = ctypes.CDLL(_LIB)
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


class Blocks(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int) for f in ("lv", "sum_block", "m", "nnz", "ptr_size", "idx_size", "dcsr_size")] + [
        (f, _ip) for f in ("method", "nlv", "m_new", "longrow", "lenmax", "loc_off", "tmp_off", "blk_m", "blk_n",
                           "blk_nnz", "subtri_up", "subtri_down", "subrec_up", "subrec_down", "subrec_right",
                           "subrec_left", "ptr_offset", "index_offset", "dcsrindex_offset", "recblock_Ptr",
                           "recblock_Index")
    ] + [("recblock_Val", _dp)] + [
        (f, _ip) for f in ("recblock_dcsr_rowidx", "levelItem", "loc_item_off", "loc_ptr_off", "lvl_item", "lvl_ptr",
                           "m_lv", "offset_lv", "nnz_lv")
    ]


lib.orc_analyse.argtypes = [_ip, _ip, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.POINTER(Blocks)]
lib.orc_blocks_free.argtypes = [ctypes.POINTER(Blocks)]
lib.orc_sptrsv_csr.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, _dp, _dp]
lib.orc_sptrsv_csr_compensated.argtypes = lib.orc_sptrsv_csr.argtypes
lib.orc_spmv_csr.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp, _dp]
lib.orc_ilu0_csr.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp]
lib.orc_ic0_csr.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp]
lib.orc_spmv_csr.restype = None
lib.orc_transpose.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _ip, _ip, _dp]
lib.orc_transpose.restype = None
lib.orc_auto_lv.argtypes = [ctypes.c_int, ctypes.c_int]
lib.orc_mtx_read.argtypes = [ctypes.c_char_p] + [_ip] * 5 + [ctypes.POINTER(_ip), ctypes.POINTER(_ip),
                                                          ctypes.POINTER(_dp)]
lib.orc_free.argtypes = [ctypes.c_void_p]
lib.orc_free.restype = None
lib.orc_tri_extract.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, _dp, _ip, _ip, _dp]
MTX_REF_DUMP = os.path.join(_HERE, "_ref", "mtx_dump")


class _Levels(ctypes.Structure):
    _fields_ = ([("n", ctypes.c_int), ("nlevel", ctypes.c_int), ("substitution", ctypes.c_int)]
                + [(f, _ip) for f in ("lp", "item", "prp", "pci")] + [(f, _dp) for f in ("pva", "pdiag", "px")]
                + [(f, _ip) for f in ("nrp", "nci")] + [(f, _dp) for f in ("nva", "ndiag")])


lib.orc_levels_prepare.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, ctypes.POINTER(_Levels)]
lib.orc_levels_solve.argtypes = [ctypes.POINTER(_Levels), _dp, _dp, ctypes.c_int]
lib.orc_levels_solve.restype = None
lib.orc_levels_free.argtypes = [ctypes.POINTER(_Levels)]
lib.orc_levels_free.restype = None


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def transpose(ptr, idx, val, ncols=None):
    """CSR(rows) -> CSC, stable (tranpose.h:7-54)."""
    ptr, idx, val = _i(ptr), _i(idx), _d(val)
    m = len(ptr) - 1
    n = m if ncols is None else ncols
    tp = np.zeros(n + 1, np.int32)
    ti = np.zeros(max(len(idx), 1), np.int32)
    tv = np.zeros(max(len(idx), 1), np.float64)
    lib.orc_transpose(m, n, len(idx), ptr.ctypes.data_as(_ip), idx.ctypes.data_as(_ip), val.ctypes.data_as(_dp),
                      tp.ctypes.data_as(_ip), ti.ctypes.data_as(_ip), tv.ctypes.data_as(_dp))
    return tp, ti[: len(idx)], tv[: len(idx)]


def auto_lv(m, device_id=0):
    return lib.orc_auto_lv(m, device_id)


def reorder_colrow(colptr, rowidx, val, substitution):
    """Restated levelset_reordering_colrow_csc: (colptr_new, rowidx_new,
    val_new, levelItem) of the level-permuted CSC."""
    cp, ri, va = _i(colptr), _i(rowidx), _d(val)
    m, nnz = len(cp) - 1, len(ri)
    ncp, nri, nva, item = np.zeros(m + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz), np.zeros(m, np.int32)
    rc = lib.orc_reorder_colrow(cp.ctypes.data_as(_ip), ri.ctypes.data_as(_ip), va.ctypes.data_as(_dp), m, nnz,
                                substitution, ncp.ctypes.data_as(_ip), nri.ctypes.data_as(_ip),
                                nva.ctypes.data_as(_dp), item.ctypes.data_as(_ip))
    if rc != 0:
        raise RuntimeError("oracle reorder: level search stuck")
    return ncp, nri, nva, item


def analyse(colptr, rowidx, val, substitution, lv):
    """Restated reference analysis; returns a dict of numpy arrays named like the reference's variables."""
    cp, ri, va = _i(colptr), _i(rowidx), _d(val)
    m = len(cp) - 1
    b = Blocks()
    rc = lib.orc_analyse(cp.ctypes.data_as(_ip), ri.ctypes.data_as(_ip), va.ctypes.data_as(_dp), m, len(ri),
                         substitution, lv, ctypes.byref(b))
    if rc != 0:
        raise RuntimeError("oracle analysis: level search stuck")
    s = b.sum_block

    def arr(p, n, dt=np.int32):
        return np.ctypeslib.as_array(p, shape=(max(n, 1),))[:n].astype(dt).copy()

    out = {}
    for f in ("method", "nlv", "m_new", "longrow", "lenmax", "loc_off", "tmp_off", "blk_m", "blk_n", "blk_nnz",
              "subtri_up", "subtri_down", "subrec_up", "subrec_down", "subrec_right", "subrec_left"):
        out[f] = arr(getattr(b, f), s)
    for f in ("ptr_offset", "index_offset", "dcsrindex_offset"):
        out[f] = arr(getattr(b, f), s + 1)
    out["sizes"] = np.array([b.ptr_size, b.idx_size, b.dcsr_size], np.int32)
    out["recblock_Ptr"] = arr(b.recblock_Ptr, int(out["ptr_offset"][s]))
    out["recblock_Index"] = arr(b.recblock_Index, int(out["index_offset"][s]))
    out["recblock_Val"] = arr(b.recblock_Val, int(out["index_offset"][s]), np.float64)
    out["recblock_dcsr_rowidx"] = arr(b.recblock_dcsr_rowidx, int(out["dcsrindex_offset"][s]))
    out["levelItem"] = arr(b.levelItem, m)
    # local level sets of the triangles, concatenated in block order
    lp, li, mlv, olv, nlvv = [], [], [], [], []
    lvl_ptr_all = np.ctypeslib.as_array(b.lvl_ptr, shape=(m + (1 << lv),))
    lvl_item_all = np.ctypeslib.as_array(b.lvl_item, shape=(m,))
    mlv_all = np.ctypeslib.as_array(b.m_lv, shape=(m + (1 << lv),))
    olv_all = np.ctypeslib.as_array(b.offset_lv, shape=(m + (1 << lv),))
    nnzlv_all = np.ctypeslib.as_array(b.nnz_lv, shape=(m + (1 << lv),))
    ptr_off = np.ctypeslib.as_array(b.loc_ptr_off, shape=(s,))
    item_off = np.ctypeslib.as_array(b.loc_item_off, shape=(s,))
    for blk in range(0, s, 2):
        nl = int(out["nlv"][blk])
        po, io, bm = int(ptr_off[blk]), int(item_off[blk]), int(out["blk_m"][blk])
        lp.append(lvl_ptr_all[po:po + nl + 1])
        li.append(lvl_item_all[io:io + bm])
        if out["method"][blk] == 2:
            mlv.append(mlv_all[po:po + nl])
            olv.append(olv_all[po:po + nl])
            nlvv.append(nnzlv_all[po:po + nl])
    cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
    out["lvl_ptr"], out["lvl_item"] = cat(lp), cat(li)
    out["m_lv"], out["offset_lv"], out["nnz_lv"] = cat(mlv), cat(olv), cat(nlvv)
    lib.orc_blocks_free(ctypes.byref(b))
    return out


def sptrsv_csr(rowptr, colidx, val, substitution, b, compensated=False):
    """Serial FP64 substitution; b may be (n,) or (k, n)."""
    rp, ci, va = _i(rowptr), _i(colidx), _d(val)
    b = _d(b)
    n = len(rp) - 1
    f = lib.orc_sptrsv_csr_compensated if compensated else lib.orc_sptrsv_csr
    bs = b.reshape(-1, n)
    xs = np.zeros_like(bs)
    for c in range(bs.shape[0]):
        bc = np.ascontiguousarray(bs[c])
        xc = np.zeros(n)
        if f(n, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), va.ctypes.data_as(_dp), substitution,
             bc.ctypes.data_as(_dp), xc.ctypes.data_as(_dp)) != 0:
            raise RuntimeError("oracle substitution: zero or missing diagonal")
        xs[c] = xc
    return xs.reshape(b.shape)


class LevelSolver:
    """Level-scheduled substitution on host threads over a level-ordered copy
    of a CSR triangle (threads >= 1), or serial substitution over a copy in
    the rows' own order (threads == 0) (orc_levels_*): the benchmark's CPU
    baseline.  Results equal sptrsv_csr's bit for bit."""

    def __init__(self, rowptr, colidx, val, substitution):
        self._keep = (_i(rowptr), _i(colidx), _d(val))
        rp, ci, va = self._keep
        self.n = len(rp) - 1
        self._L = _Levels()
        if lib.orc_levels_prepare(self.n, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), va.ctypes.data_as(_dp),
                                  substitution, ctypes.byref(self._L)) != 0:
            raise RuntimeError("oracle level solver: missing/zero diagonal or entry outside the triangle")
        self.nlevel = self._L.nlevel

    def solve(self, b, x=None, threads=1):
        b = _d(b)
        if x is None:
            x = np.empty(self.n)
        lib.orc_levels_solve(ctypes.byref(self._L), b.ctypes.data_as(_dp), x.ctypes.data_as(_dp), int(threads))
        return x

    def __del__(self):
        if getattr(self, "_L", None) is not None:
            lib.orc_levels_free(ctypes.byref(self._L))
            self._L = None


def ilu0_csr(rowptr, colidx, val):
    """ILU(0) values in the pattern of a CSR matrix (strict L below, U on and above the diagonal)."""
    rp, ci, va = _i(rowptr), _i(colidx), _d(val)
    lu = np.zeros(len(ci))
    rc = lib.orc_ilu0_csr(len(rp) - 1, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), va.ctypes.data_as(_dp),
                          lu.ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError("oracle ILU(0): missing diagonal" if rc == -1 else "oracle ILU(0): zero pivot")
    return lu


def ic0_csr(rowptr, colidx, val):
    """IC(0) of an SPD matrix given as its lower-triangle CSR (diagonal last): L in that pattern."""
    rp, ci, va = _i(rowptr), _i(colidx), _d(val)
    out = np.zeros(len(ci))
    rc = lib.orc_ic0_csr(len(rp) - 1, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), va.ctypes.data_as(_dp),
                         out.ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError("oracle IC(0): bad structure" if rc == -1 else "oracle IC(0): pivot <= 0", rc)
    return out


def spmv_csr(rowptr, colidx, val, x):
    rp, ci, va, x = _i(rowptr), _i(colidx), _d(val), _d(x)
    y = np.zeros(len(rp) - 1)
    lib.orc_spmv_csr(len(rp) - 1, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), va.ctypes.data_as(_dp),
                     x.ctypes.data_as(_dp), y.ctypes.data_as(_dp))
    return y


def run_reference_dump(colptr, rowidx, val, substitution, lv, workdir):
    """Run the reference's own analysis (oracle/_ref/ref_dump) and read its outputs."""
    cp, ri, va = _i(colptr), _i(rowidx), _d(val)
    m = len(cp) - 1
    inp = os.path.join(workdir, "ref_in.bin")
    outp = os.path.join(workdir, "ref_out.bin")
    with open(inp, "wb") as f:
        np.array([m, len(ri), substitution, lv], np.int32).tofile(f)
        cp.tofile(f)
        ri.tofile(f)
        va.tofile(f)
    subprocess.run([REF_DUMP, inp, outp], check=True, stdout=subprocess.DEVNULL)
    res = {}
    with open(outp, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        name = data[pos:pos + 32].split(b"\0")[0].decode()
        kind = int(np.frombuffer(data, np.int32, 1, pos + 32)[0])
        cnt = int(np.frombuffer(data, np.int64, 1, pos + 36)[0])
        pos += 44
        dt = np.int32 if kind == 0 else np.float64
        res[name] = np.frombuffer(data, dt, cnt, pos).copy()
        pos += cnt * np.dtype(dt).itemsize
    return res


MTX_ERRORS = {-1: "cannot open", -2: "bad banner", -3: "not coordinate or unknown field", -4: "bad size line",
              -5: "truncated or malformed entry", -6: "index out of range"}


def mtx_read(path):
    """Matrix Market file -> CSR the way mmio_data does (mmio_highlevel.h:137-296).

    Returns dict(m, n, field, symmetric, rowptr, colidx, val); raises
    RuntimeError with the oracle's error code."""
    m, n, nnz, fld, sym = (ctypes.c_int() for _ in range(5))
    rp, ci, va = _ip(), _ip(), _dp()
    rc = lib.orc_mtx_read(os.fsencode(path), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(fld),
                          ctypes.byref(sym), ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(va))
    if rc != 0:
        raise RuntimeError(f"oracle mtx_read: {MTX_ERRORS.get(rc, rc)}", rc)
    try:
        out = dict(m=m.value, n=n.value, field=fld.value, symmetric=sym.value,
                   rowptr=np.ctypeslib.as_array(rp, (m.value + 1,)).copy(),
                   colidx=np.ctypeslib.as_array(ci, (max(nnz.value, 1),))[: nnz.value].copy(),
                   val=np.ctypeslib.as_array(va, (max(nnz.value, 1),))[: nnz.value].copy())
    finally:
        for p in (rp, ci, va):
            lib.orc_free(ctypes.cast(p, ctypes.c_void_p))
    return out


def tri_extract(rowptr, colidx, val, substitution, strict_val=None):
    """main.cu:157-198: unit-diagonal strictly lower (forward) / upper (backward) triangle of a square CSR."""
    rp, ci, va = _i(rowptr), _i(colidx), _d(val)
    m = len(rp) - 1
    cap = m + len(ci)
    tp = np.zeros(m + 1, np.int32)
    ti = np.zeros(max(cap, 1), np.int32)
    tv = np.zeros(max(cap, 1), np.float64)
    sv = None if strict_val is None else _d(strict_val)
    cnt = lib.orc_tri_extract(m, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip), va.ctypes.data_as(_dp), substitution,
                              None if sv is None else sv.ctypes.data_as(_dp), tp.ctypes.data_as(_ip),
                              ti.ctypes.data_as(_ip), tv.ctypes.data_as(_dp))
    return tp, ti[:cnt].copy(), tv[:cnt].copy()


def run_reference_mtx(path):
    """The reference's own mmio_info + mmio_data (oracle/_ref/mtx_dump) on a file."""
    out = subprocess.run([MTX_REF_DUMP, path], check=True, capture_output=True).stdout
    m, n, nnz, sym = np.frombuffer(out, np.int32, 4, 0)
    pos = 16
    rp = np.frombuffer(out, np.int32, m + 1, pos).copy()
    pos += 4 * (m + 1)
    ci = np.frombuffer(out, np.int32, nnz, pos).copy()
    pos += 4 * nnz
    va = np.frombuffer(out, np.float64, nnz, pos).copy()
    return dict(m=int(m), n=int(n), symmetric=int(sym), rowptr=rp, colidx=ci, val=va)


def reference_mtx_ms(path):
    """Wall milliseconds of the reference's own mmio_info + mmio_data on a
    file (oracle/_ref/mtx_dump --time), or None when it was not built."""
    if not os.path.exists(MTX_REF_DUMP):
        return None
    out = subprocess.run([MTX_REF_DUMP, "--time", path], check=True, capture_output=True, text=True).stdout
    return float(out.strip())


lib.orc_gen_lower_csr.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                  _ip, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_ip), ctypes.POINTER(_ip),
                                  ctypes.POINTER(_dp)]
lib.orc_gen_uniform.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_double, ctypes.c_double, _dp]

GEN_BAND_POISSON, GEN_LAPLACE2D, GEN_ZIPF, GEN_CHAIN, GEN_DIAG = range(5)


def gen_lower_csr(kind, n=0, grid=0, lam=0.0, band=0, zipf_alpha=0.0, zipf_max=0, chain_bw=0, seed=0):
    """The seeded lower-triangular CSR of include/rbs_gen.h (columns ascending, diagonal last)."""
    nn = ctypes.c_int()
    nnz = ctypes.c_longlong()
    rp, ci, va = _ip(), _ip(), _dp()
    rc = lib.orc_gen_lower_csr(kind, n, grid, lam, band, zipf_alpha, zipf_max, chain_bw, seed, ctypes.byref(nn),
                               ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(va))
    if rc:
        raise RuntimeError(f"orc_gen_lower_csr failed ({rc})")
    try:
        n_, z = nn.value, nnz.value
        return (np.ctypeslib.as_array(rp, shape=(n_ + 1,)).copy(),
                np.ctypeslib.as_array(ci, shape=(max(z, 1),))[:z].copy(),
                np.ctypeslib.as_array(va, shape=(max(z, 1),))[:z].copy())
    finally:
        for p in (rp, ci, va):
            lib.orc_free(p)


def gen_uniform(seed, n, lo=-1.0, hi=1.0):
    out = np.empty(n, dtype=np.float64)
    if lib.orc_gen_uniform(seed, n, lo, hi, out.ctypes.data_as(_dp)):
        raise RuntimeError("orc_gen_uniform failed")
    return out
