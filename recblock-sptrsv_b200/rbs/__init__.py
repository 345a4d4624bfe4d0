"""Python mirror of the recblock-sptrsv solver interface over librbs.so.

The product is the C ABI in include/rbs.h; this module binds it with ctypes
for tests, the benchmark and notebooks.  Function names follow the
reference's entry points:

  recblocking_solver_cuda(...)   recblocking_solver_cuda.h:21-32 (device pointers)
  recblocking_solver(...)        recblocking_solver.h:16-28 (host arrays)
  analyse(...) -> Plan           preprocess (levelset_reordering_colrow_csc +
                                 mat_preprocessing + per-block loop)
  Plan.solve(...)                L_calculate / U_calculate

Device buffers are passed as torch CUDA tensors (only their data_ptr is
used); host buffers as numpy arrays.  The library must be built
(`make -C recblock-sptrsv_b200`); importing this module without it raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(os.path.dirname(_HERE), "librbs.so")

FORWARD, BACKWARD = 0, 1
FMT_CSC, FMT_CSR = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2
SELECT_REFERENCE, SELECT_AUTO, SELECT_TUNE = 0, 1, 2
(K_DIAG, K_SYNCFREE, K_LEVEL, K_SEQ, K_BANDSCAN, K_SPMV, K_EMPTY) = range(7)
KERNEL_NAMES = ["diag", "syncfree", "level", "seq", "bandscan", "spmv", "empty"]

OK = 0
ERR_ARG, ERR_STRUCTURE, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT, ERR_NOCONV, ERR_BUDGET, ERR_UNSUPPORTED = range(1, 9)


class Options(ctypes.Structure):
    _fields_ = [
        ("select", ctypes.c_int),
        ("device", ctypes.c_int),
        ("lv_device_id", ctypes.c_int),
        ("host_only", ctypes.c_int),
        ("max_rhs", ctypes.c_int),
        ("mixed", ctypes.c_int),
        ("ir_tol", ctypes.c_double),
        ("ir_max_iter", ctypes.c_int),
        ("spin_limit", ctypes.c_longlong),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("ms", ctypes.c_double),
        ("iterations", ctypes.c_int),
        ("correction", ctypes.c_double),
        ("useful_bytes", ctypes.c_double),
        ("moved_bytes", ctypes.c_double),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("nnz", ctypes.c_int),
        ("lv", ctypes.c_int),
        ("substitution", ctypes.c_int),
        ("nlevel", ctypes.c_int),
        ("sum_block", ctypes.c_int),
        ("kernels", ctypes.c_int * 8),
        ("device_bytes", ctypes.c_longlong),
        ("analyse_ms", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("completed", ctypes.c_longlong),
        ("solves", ctypes.c_longlong),
        ("batches", ctypes.c_longlong),
        ("mean_batch_rhs", ctypes.c_double),
        ("p50_ms", ctypes.c_double),
        ("p99_ms", ctypes.c_double),
        ("solves_per_s", ctypes.c_double),
        ("factors", ctypes.c_int),
        ("hbm_used", ctypes.c_longlong),
    ]


class GenSpec(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("n", ctypes.c_int),
        ("grid", ctypes.c_int),
        ("lam", ctypes.c_double),
        ("band", ctypes.c_int),
        ("zipf_alpha", ctypes.c_double),
        ("zipf_max", ctypes.c_int),
        ("chain_bw", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
    ]


# every symbol include/rbs.h and include/rbs_gen.h declare
EXPORTS = [
    "rbs_options_default", "rbs_analyse", "rbs_analyse_device", "rbs_solve", "rbs_solve_host",
    "rbs_solve_async", "rbs_plan_sync", "rbs_plan_set_stream", "rbs_plan_info_get", "rbs_plan_export",
    "rbs_plan_free", "rbs_last_error", "rbs_auto_lv", "recblocking_solver_cuda", "recblocking_solver",
    "rbs_gen_lower_csr", "rbs_gen_uniform", "rbs_gen_free", "rbs_plan_profile", "rbs_plan_block_times",
    "rbs_sptrsv_csr_noalloc", "rbs_batch_analyse", "rbs_server_create", "rbs_server_add_factor",
    "rbs_server_submit", "rbs_server_submit_device", "rbs_server_add_group", "rbs_server_wait", "rbs_server_stats_get", "rbs_server_reset_stats", "rbs_server_destroy",
    "rbs_plan_save", "rbs_plan_load", "rbs_ilu0_device", "rbs_mtx_read", "rbs_mtx_read_buffer", "rbs_mtx_info_get",
    "rbs_mtx_csr", "rbs_mtx_triangle", "rbs_mtx_free", "rbs_mtx_write", "rbs_ic0_device", "rbs_plan_reserve", "rbs_solve_host_async",
]

MTX_REAL, MTX_INTEGER, MTX_PATTERN, MTX_COMPLEX = range(4)


class MtxInfo(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("n", ctypes.c_int), ("nnz_file", ctypes.c_longlong),
                ("nnz", ctypes.c_longlong), ("nnz_lower", ctypes.c_longlong), ("nnz_upper", ctypes.c_longlong),
                ("field", ctypes.c_int), ("symmetric", ctypes.c_int), ("host_values", ctypes.c_longlong),
                ("read_ms", ctypes.c_double), ("parse_ms", ctypes.c_double)]


class RbsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rbs error {code}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} not built; run make -C {os.path.dirname(_HERE)}")
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.rbs_options_default.argtypes = [ctypes.POINTER(Options)]
    lib.rbs_analyse.argtypes = [ip, ip, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(Options), ctypes.POINTER(P)]
    lib.rbs_analyse_device.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(Options), ctypes.POINTER(P)]
    lib.rbs_solve.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Stats)]
    lib.rbs_solve_host.argtypes = [P, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Stats)]
    lib.rbs_solve_async.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.rbs_plan_sync.argtypes = [P]
    lib.rbs_plan_set_stream.argtypes = [P, P]
    lib.rbs_plan_info_get.argtypes = [P, ctypes.POINTER(PlanInfo)]
    lib.rbs_plan_export.argtypes = [P, ctypes.c_char_p, P, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    lib.rbs_plan_free.argtypes = [P]
    lib.rbs_plan_save.argtypes = [P, ctypes.c_char_p]
    lib.rbs_ilu0_device.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, P, ctypes.POINTER(Options)]
    lib.rbs_ic0_device.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, P, ctypes.POINTER(Options)]
    lib.rbs_plan_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(Options), ctypes.POINTER(P)]
    lib.rbs_mtx_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(Options), ctypes.POINTER(P)]
    lib.rbs_mtx_read_buffer.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.POINTER(Options), ctypes.POINTER(P)]
    lib.rbs_mtx_info_get.argtypes = [P, ctypes.POINTER(MtxInfo)]
    lib.rbs_mtx_csr.argtypes = [P, P, P, P]
    lib.rbs_mtx_triangle.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, P]
    lib.rbs_mtx_free.argtypes = [P]
    lib.rbs_mtx_write.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ip, ip, dp, ctypes.c_int]
    lib.rbs_last_error.restype = ctypes.c_char_p
    lib.rbs_auto_lv.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.recblocking_solver_cuda.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int,
                                            ctypes.c_int, dp, dp]
    lib.recblocking_solver_cuda.restype = None
    lib.recblocking_solver.argtypes = [ip, ip, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    lib.recblocking_solver.restype = None
    lib.rbs_gen_lower_csr.argtypes = [ctypes.POINTER(GenSpec), ip, ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(dp)]
    lib.rbs_gen_uniform.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_double, ctypes.c_double, dp]
    lib.rbs_gen_free.argtypes = [P]
    lib.rbs_plan_profile.argtypes = [P, ctypes.c_int]
    lib.rbs_plan_block_times.argtypes = [P, dp, dp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    lib.rbs_sptrsv_csr_noalloc.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, P, P, P]
    lib.rbs_server_create.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(P)]
    lib.rbs_server_add_factor.argtypes = [P, P, ip]
    lib.rbs_server_submit.argtypes = [P, ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_longlong)]
    lib.rbs_server_submit_device.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_longlong)]
    lib.rbs_server_add_group.argtypes = [P, P, ctypes.c_int, ip, ip]
    lib.rbs_plan_reserve.argtypes = [P, ctypes.c_int]
    lib.rbs_solve_host_async.argtypes = [P, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.rbs_server_wait.argtypes = [P, ctypes.c_longlong, dp, ip]
    lib.rbs_server_stats_get.argtypes = [P, ctypes.POINTER(ServerStats)]
    lib.rbs_server_reset_stats.argtypes = [P]
    lib.rbs_server_destroy.argtypes = [P]
    lib.rbs_batch_analyse.argtypes = [ctypes.c_int, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(dp), ip, ip,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Options),
                                      ctypes.POINTER(P), ip]
    return lib


lib = _load()


def last_error() -> str:
    return lib.rbs_last_error().decode()


def _check(rc: int):
    if rc != OK:
        raise RbsError(rc, last_error())


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def options(**kw) -> Options:
    o = Options()
    lib.rbs_options_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def auto_lv(m: int, device_id: int = 0) -> int:
    return lib.rbs_auto_lv(m, device_id)


class Plan:
    """A device-resident analysis (permutation, block bounds, kernel plan)."""

    def __init__(self, handle: ctypes.c_void_p, n: int):
        self._h = handle
        self.n = n

    def __del__(self):
        self.free()

    def free(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.rbs_plan_free(self._h)
        self._h = None

    @property
    def handle(self):
        return self._h

    def info(self) -> PlanInfo:
        inf = PlanInfo()
        _check(lib.rbs_plan_info_get(self._h, ctypes.byref(inf)))
        return inf

    def export(self, name: str) -> np.ndarray:
        cnt = ctypes.c_longlong()
        _check(lib.rbs_plan_export(self._h, name.encode(), None, 0, ctypes.byref(cnt)))
        dt = np.float64 if name in ("recblock_Val", "block_bytes", "ell_val", "inv_diag", "analyse_ms", "ca_val") else np.int32
        out = np.empty(max(cnt.value, 1), dtype=dt)
        _check(lib.rbs_plan_export(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p), cnt.value,
                                   ctypes.byref(cnt)))
        return out[: cnt.value]

    def solve(self, b, x, k: int = 1, ld: int | None = None, prec: int = PREC_FP64) -> Stats:
        """Device solve: b, x are torch CUDA tensors (column-major n x k)."""
        st = Stats()
        ld = self.n if ld is None else ld
        _check(lib.rbs_solve(self._h, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()), k, ld, prec,
                             ctypes.byref(st)))
        return st

    def solve_async(self, b, x, k: int = 1, ld: int | None = None, prec: int = PREC_FP64):
        ld = self.n if ld is None else ld
        _check(lib.rbs_solve_async(self._h, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()), k, ld,
                                   prec))

    def sync(self):
        _check(lib.rbs_plan_sync(self._h))

    def solve_host(self, b: np.ndarray, k: int = 1, prec: int = PREC_FP64, x: np.ndarray | None = None):
        """Host solve: b is a numpy array (n,) or (k, n) (one row per RHS); x
        (same shape, e.g. a pinned buffer) receives the solution."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if x is None:
            x = np.zeros_like(b)
        assert x.flags.c_contiguous and x.dtype == np.float64 and x.shape == b.shape
        st = Stats()
        _check(lib.rbs_solve_host(self._h, _dp(b), _dp(x), k, self.n, prec, ctypes.byref(st)))
        return x, st

    def solve_host_async(self, b: np.ndarray, x: np.ndarray, k: int = 1, prec: int = PREC_FP64):
        """Enqueue a host-array solve (b, x: float64, (n,) or (k, n), ideally pinned, e.g. a
        torch pin_memory tensor's .numpy()); b unchanged and x unread until sync()."""
        assert b.flags.c_contiguous and x.flags.c_contiguous and b.dtype == np.float64 and x.dtype == np.float64
        assert b.size >= k * self.n and x.size >= k * self.n
        _check(lib.rbs_solve_host_async(self._h, _dp(b), _dp(x), k, self.n, prec))

    def profile(self, enable: bool = True):
        """Per-block CUDA-event timing of FP64/FP32 solves (resets the totals)."""
        _check(lib.rbs_plan_profile(self._h, int(enable)))

    def block_times(self):
        """(ms per block accumulated, algorithmic bytes per block per pass, timed solves)."""
        nb = self.info().sum_block
        ms = np.zeros(nb)
        by = np.zeros(nb)
        solves = ctypes.c_longlong()
        _check(lib.rbs_plan_block_times(self._h, _dp(ms), _dp(by), ctypes.byref(solves), nb))
        return ms, by, solves.value

    def save(self, path: str):
        """rbs_plan_save: the analysis to a file."""
        _check(lib.rbs_plan_save(self._h, str(path).encode()))

    def reserve(self, k: int):
        """Work vectors for k right-hand sides now (no allocation in later solves up to k)."""
        _check(lib.rbs_plan_reserve(self._h, k))

    def set_stream(self, stream_ptr: int | None):
        _check(lib.rbs_plan_set_stream(self._h, ctypes.c_void_p(stream_ptr) if stream_ptr else None))


def analyse(ptr: np.ndarray, idx: np.ndarray, val: np.ndarray, substitution: int = FORWARD, lv: int = -1,
            fmt: int = FMT_CSC, opts: Options | None = None) -> Plan:
    ptr = np.ascontiguousarray(ptr, dtype=np.int32)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    n = len(ptr) - 1
    h = ctypes.c_void_p()
    _check(lib.rbs_analyse(_ip(ptr), _ip(idx), _dp(val), n, len(idx), fmt, substitution, lv,
                           ctypes.byref(opts) if opts is not None else None, ctypes.byref(h)))
    return Plan(h, n)


def batch_analyse(systems, substitution: int = FORWARD, lv: int = -1, fmt: int = FMT_CSC,
                  opts: Options | None = None):
    """rbs_batch_analyse: systems is a list of (ptr, idx, val); returns (Plan, row_offsets)."""
    cnt = len(systems)
    keep = [(np.ascontiguousarray(p, np.int32), np.ascontiguousarray(i, np.int32), np.ascontiguousarray(v, np.float64))
            for p, i, v in systems]
    P = (ctypes.POINTER(ctypes.c_int) * cnt)(*[_ip(k[0]) for k in keep])
    I = (ctypes.POINTER(ctypes.c_int) * cnt)(*[_ip(k[1]) for k in keep])
    V = (ctypes.POINTER(ctypes.c_double) * cnt)(*[_dp(k[2]) for k in keep])
    ns = np.array([len(k[0]) - 1 for k in keep], np.int32)
    zs = np.array([len(k[1]) for k in keep], np.int32)
    offs = np.zeros(cnt + 1, np.int32)
    h = ctypes.c_void_p()
    _check(lib.rbs_batch_analyse(cnt, P, I, V, _ip(ns), _ip(zs), fmt, substitution, lv,
                                 ctypes.byref(opts) if opts is not None else None, ctypes.byref(h), _ip(offs)))
    return Plan(h, int(offs[-1])), offs


class Server:
    """rbs_server: device-resident factors, continuous batching, latency stats."""

    def __init__(self, hbm_budget_bytes: int, max_batch_rhs: int = 16):
        self._h = ctypes.c_void_p()
        _check(lib.rbs_server_create(hbm_budget_bytes, max_batch_rhs, ctypes.byref(self._h)))
        self._keep = {}

    def add_factor(self, plan: Plan) -> int:
        fid = ctypes.c_int()
        _check(lib.rbs_server_add_factor(self._h, plan.handle, ctypes.byref(fid)))
        plan._h = None  # owned by the server now
        return fid.value

    def add_group(self, plan: Plan, row_offsets) -> list:
        """A block-diagonal plan (batch_analyse) served as one unit: one factor id per system."""
        offs = np.ascontiguousarray(row_offsets, dtype=np.int32)
        count = len(offs) - 1
        ids = np.zeros(count, dtype=np.int32)
        _check(lib.rbs_server_add_group(self._h, plan.handle, count, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        plan._h = None  # owned by the server now
        return [int(v) for v in ids]

    def submit_device(self, factor: int, b, x, k: int = 1, prec: int = PREC_FP64) -> int:
        """Device arrays (torch CUDA tensors, float64, n*k elements, column-major), read and
        written in place; kept alive here until the wait."""
        t = ctypes.c_longlong()
        _check(lib.rbs_server_submit_device(self._h, factor, ctypes.c_void_p(b.data_ptr()),
                                            ctypes.c_void_p(x.data_ptr()), k, prec, ctypes.byref(t)))
        self._keep[t.value] = (b, x)
        return t.value

    def submit(self, factor: int, b: np.ndarray, x: np.ndarray, k: int = 1, prec: int = PREC_FP64) -> int:
        assert b.dtype == np.float64 and x.dtype == np.float64 and b.flags.c_contiguous and x.flags.c_contiguous
        t = ctypes.c_longlong()
        _check(lib.rbs_server_submit(self._h, factor, _dp(b), _dp(x), k, prec, ctypes.byref(t)))
        self._keep[t.value] = (b, x)
        return t.value

    def wait(self, ticket: int):
        lat = ctypes.c_double()
        bk = ctypes.c_int()
        rc = lib.rbs_server_wait(self._h, ticket, ctypes.byref(lat), ctypes.byref(bk))
        self._keep.pop(ticket, None)
        _check(rc)
        return lat.value, bk.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        _check(lib.rbs_server_stats_get(self._h, ctypes.byref(st)))
        return st

    def reset_stats(self):
        _check(lib.rbs_server_reset_stats(self._h))

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.rbs_server_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()


def ilu0_device(d_rowptr, d_colidx, d_val, d_lu, opts: Options | None = None):
    """rbs_ilu0_device on torch CUDA tensors: d_lu receives ILU(0) of the CSR matrix in its pattern."""
    n = d_rowptr.numel() - 1
    _check(lib.rbs_ilu0_device(ctypes.c_void_p(d_rowptr.data_ptr()), ctypes.c_void_p(d_colidx.data_ptr()),
                               ctypes.c_void_p(d_val.data_ptr()), n, d_colidx.numel(),
                               ctypes.c_void_p(d_lu.data_ptr()), ctypes.byref(opts) if opts is not None else None))


class Mtx:
    """A Matrix Market file parsed on the device (rbs_mtx_*): A's CSR in HBM,
    exported to torch tensors, and the triangle main.cu builds from it."""

    def __init__(self, h):
        self._h = h
        self.info = MtxInfo()
        _check(lib.rbs_mtx_info_get(h, ctypes.byref(self.info)))

    def csr(self, device="cuda"):
        import torch
        i = self.info
        rp = torch.empty(i.m + 1, dtype=torch.int32, device=device)
        ci = torch.empty(max(i.nnz, 1), dtype=torch.int32, device=device)
        va = torch.empty(max(i.nnz, 1), dtype=torch.float64, device=device)
        _check(lib.rbs_mtx_csr(self._h, ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(ci.data_ptr()),
                               ctypes.c_void_p(va.data_ptr())))
        return rp, ci[: i.nnz], va[: i.nnz]

    def triangle(self, substitution: int = FORWARD, fmt: int = FMT_CSC, strict_val=None, device="cuda"):
        """Unit-diagonal strictly lower (FORWARD) / upper (BACKWARD) triangle
        as (ptr, idx, val) torch tensors in CSC or CSR; strict_val: optional
        device tensor of the strict entries' values in row-major order."""
        import torch
        i = self.info
        cnt = i.m + (i.nnz_lower if substitution == FORWARD else i.nnz_upper)
        ptr = torch.empty(i.m + 1, dtype=torch.int32, device=device)
        idx = torch.empty(max(cnt, 1), dtype=torch.int32, device=device)
        val = torch.empty(max(cnt, 1), dtype=torch.float64, device=device)
        sv = None if strict_val is None else ctypes.c_void_p(strict_val.data_ptr())
        _check(lib.rbs_mtx_triangle(self._h, substitution, fmt, sv, ctypes.c_void_p(ptr.data_ptr()),
                                    ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(val.data_ptr())))
        return ptr, idx[:cnt], val[:cnt]

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.rbs_mtx_free(self._h)
        self._h = None

    def __del__(self):
        self.close()


def mtx_read(path: str, opts: Options | None = None) -> Mtx:
    """rbs_mtx_read: parse a Matrix Market file on the device."""
    h = ctypes.c_void_p()
    _check(lib.rbs_mtx_read(os.fsencode(str(path)), ctypes.byref(opts) if opts is not None else None, ctypes.byref(h)))
    return Mtx(h)


def mtx_read_buffer(data: bytes, opts: Options | None = None) -> Mtx:
    """rbs_mtx_read_buffer: parse a Matrix Market file image held in host memory."""
    h = ctypes.c_void_p()
    _check(lib.rbs_mtx_read_buffer(data, len(data), ctypes.byref(opts) if opts is not None else None,
                                   ctypes.byref(h)))
    return Mtx(h)


def mtx_write(path: str, rowptr: np.ndarray, colidx: np.ndarray, val: np.ndarray | None, ncols: int | None = None,
              symmetric: bool = False):
    """rbs_mtx_write: a host CSR as a Matrix Market coordinate file (%.17g values)."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    m = len(rp) - 1
    va = None if val is None else np.ascontiguousarray(val, np.float64)
    _check(lib.rbs_mtx_write(os.fsencode(str(path)), m, m if ncols is None else ncols, _ip(rp), _ip(ci),
                             None if va is None else _dp(va), int(bool(symmetric))))


def ic0_device(d_rowptr, d_colidx, d_val, d_l, opts: Options | None = None):
    """rbs_ic0_device on torch CUDA tensors: d_l receives IC(0) of the SPD
    matrix given as its lower-triangle CSR (diagonal last in every row)."""
    n = d_rowptr.numel() - 1
    _check(lib.rbs_ic0_device(ctypes.c_void_p(d_rowptr.data_ptr()), ctypes.c_void_p(d_colidx.data_ptr()),
                              ctypes.c_void_p(d_val.data_ptr()), n, d_colidx.numel(),
                              ctypes.c_void_p(d_l.data_ptr()), ctypes.byref(opts) if opts is not None else None))


def load_plan(path: str, opts: Options | None = None) -> Plan:
    """rbs_plan_load: a saved analysis, device state rebuilt unless opts.host_only."""
    h = ctypes.c_void_p()
    _check(lib.rbs_plan_load(str(path).encode(), ctypes.byref(opts) if opts is not None else None, ctypes.byref(h)))
    n = PlanInfo()
    _check(lib.rbs_plan_info_get(h, ctypes.byref(n)))
    return Plan(h, n.n)


def analyse_device(ptr, idx, val, n: int, nnz: int, substitution: int = FORWARD, lv: int = -1,
                   fmt: int = FMT_CSC, opts: Options | None = None) -> Plan:
    h = ctypes.c_void_p()
    _check(lib.rbs_analyse_device(ctypes.c_void_p(ptr.data_ptr()), ctypes.c_void_p(idx.data_ptr()),
                                  ctypes.c_void_p(val.data_ptr()), n, nnz, fmt, substitution, lv,
                                  ctypes.byref(opts) if opts is not None else None, ctypes.byref(h)))
    return Plan(h, n)


def recblocking_solver_cuda(d_colptr, d_rowidx, d_val, m: int, n: int, nnz: int, d_x, d_b, substitution: int,
                            lv: int):
    """recblocking_solver_cuda.h:21-32 with torch CUDA tensors; returns (cal_time, preprocess_time) in ms."""
    cal = ctypes.c_double(0.0)
    pre = ctypes.c_double(0.0)
    lib.recblocking_solver_cuda(ctypes.c_void_p(d_colptr.data_ptr()), ctypes.c_void_p(d_rowidx.data_ptr()),
                                ctypes.c_void_p(d_val.data_ptr()), m, n, nnz, ctypes.c_void_p(d_x.data_ptr()),
                                ctypes.c_void_p(d_b.data_ptr()), substitution, lv, ctypes.byref(cal),
                                ctypes.byref(pre))
    err = last_error()
    if err:
        raise RbsError(-1, err)
    return cal.value, pre.value


NOALLOC_MAX_ROWS = 1 << 20  # RBS_NOALLOC_MAX_ROWS


def sptrsv_csr_noalloc(d_rowptr, d_colidx, d_val, n: int, substitution: int, d_b, d_x, stream_ptr: int | None = None):
    """rbs_sptrsv_csr_noalloc: solve from a device CSR (diagonal inside the
    rows) with no device allocation; scratch is the library's static array."""
    _check(lib.rbs_sptrsv_csr_noalloc(ctypes.c_void_p(d_rowptr.data_ptr()), ctypes.c_void_p(d_colidx.data_ptr()),
                                      ctypes.c_void_p(d_val.data_ptr()), n, substitution,
                                      ctypes.c_void_p(d_b.data_ptr()), ctypes.c_void_p(d_x.data_ptr()),
                                      ctypes.c_void_p(stream_ptr) if stream_ptr else None))


# ---- synthetic inputs (include/rbs_gen.h) -------------------------------
GEN_BAND_POISSON, GEN_LAPLACE2D, GEN_ZIPF, GEN_CHAIN, GEN_DIAG = range(5)


def gen_lower_csr(kind: int, n: int = 0, grid: int = 0, lam: float = 0.0, band: int = 0, zipf_alpha: float = 0.0,
                  zipf_max: int = 0, chain_bw: int = 0, seed: int = 0):
    """Seeded lower-triangular CSR (columns ascending, diagonal last)."""
    spec = GenSpec(kind, n, grid, lam, band, zipf_alpha, zipf_max, chain_bw, seed)
    nn = ctypes.c_int()
    nnz = ctypes.c_longlong()
    rp = ctypes.POINTER(ctypes.c_int)()
    ci = ctypes.POINTER(ctypes.c_int)()
    va = ctypes.POINTER(ctypes.c_double)()
    _check(lib.rbs_gen_lower_csr(ctypes.byref(spec), ctypes.byref(nn), ctypes.byref(nnz), ctypes.byref(rp),
                                 ctypes.byref(ci), ctypes.byref(va)))
    try:
        n_, z = nn.value, nnz.value
        rowptr = np.ctypeslib.as_array(rp, shape=(n_ + 1,)).copy()
        colidx = np.ctypeslib.as_array(ci, shape=(max(z, 1),))[:z].copy()
        val = np.ctypeslib.as_array(va, shape=(max(z, 1),))[:z].copy()
    finally:
        lib.rbs_gen_free(ctypes.cast(rp, ctypes.c_void_p))
        lib.rbs_gen_free(ctypes.cast(ci, ctypes.c_void_p))
        lib.rbs_gen_free(ctypes.cast(va, ctypes.c_void_p))
    return rowptr, colidx, val


def gen_uniform(seed: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    _check(lib.rbs_gen_uniform(seed, n, lo, hi, _dp(out)))
    return out
