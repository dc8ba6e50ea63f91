"""Python binding of the casgemm C ABI (include/casgemm.h, include/casgemm_data.h).

A thin ctypes layer over libcasgemm.so: no computation happens here.  The
product path is the CUDA library; if it is missing, :func:`load` raises.

Mirrors the reference's call surface (fukien/contention-aware-spgemm): one
call per accumulator — ``hash``, ``hsersc``, ``hybacc`` for
ams_hashspgemm / ams_hserscspgemm / ams_hybaccspgemm — returning C with the
phase times of the reference's runtime_t (src/mm/mm_utils.h:48-54).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcasgemm.so")

ACCUM = {"hash": 0, "hsersc": 1, "hybacc": 2}
VAL_F64, VAL_I32 = 0, 1
STATUS = {
    0: "CAS_OK", 1: "CAS_ERR_BAD_INPUT", 2: "CAS_ERR_OOM", 3: "CAS_ERR_CUDA",
    4: "CAS_ERR_DEVICE", 5: "CAS_ERR_TIMEOUT", 6: "CAS_ERR_ABORTED", 7: "CAS_ERR_REJECTED",
}
SYMB_BINS = ["zero", "tiny", "h1k", "h2k", "h4k", "h8k", "h16k", "h32k", "dense"]
NUMC_BINS = ["zero", "tiny", "esc1k", "esc2k", "esc3k", "esc4k", "esc5k", "esc6k", "esc8k", "hash256", "hash1k",
             "hash4k", "dense"]


class CasCsr(ctypes.Structure):
    _fields_ = [
        ("num_row", ctypes.c_int64), ("num_col", ctypes.c_int64), ("num_nnz", ctypes.c_int64),
        ("row_ptrs", ctypes.c_void_p), ("cols", ctypes.c_void_p), ("rats", ctypes.c_void_p),
        ("col_bytes", ctypes.c_int32), ("val_type", ctypes.c_int32),
        ("on_device", ctypes.c_int32), ("owned", ctypes.c_int32),
    ]


class CasRuntime(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("init_time", "symb_time", "mgmt_time", "numc_time", "total_time")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class CasStats(ctypes.Structure):
    _fields_ = [
        ("flop", ctypes.c_int64), ("max_row_flp", ctypes.c_int64), ("nnz_c", ctypes.c_int64),
        ("symb_bin_rows", ctypes.c_int64 * 9), ("numc_bin_rows", ctypes.c_int64 * 13),
        ("kernel_launches", ctypes.c_int64), ("h2d_bytes", ctypes.c_double), ("d2h_bytes", ctypes.c_double),
        ("symb_bin_ms", ctypes.c_double * 9), ("numc_bin_ms", ctypes.c_double * 13),
        ("numc_bin_bytes", ctypes.c_double * 13), ("numc_bin_flop", ctypes.c_int64 * 13),
        ("esc_overflow_rows", ctypes.c_int64), ("esc_overflow_ms", ctypes.c_double),
        ("fused_rows", ctypes.c_int64), ("fused_flop", ctypes.c_int64), ("fused_bytes", ctypes.c_double),
        ("fused_ms", ctypes.c_double), ("d2h_direct_bytes", ctypes.c_double), ("split_rows", ctypes.c_int64),
        ("out_blocks", ctypes.c_int64), ("numc_bin_nnz", ctypes.c_int64 * 13),
    ]


class CasJob(ctypes.Structure):
    _fields_ = [
        ("A", CasCsr), ("B", CasCsr), ("row_digests", ctypes.c_void_p),
        ("flop", ctypes.c_int64), ("nnz_c", ctypes.c_int64), ("digest", ctypes.c_uint64),
        ("status", ctypes.c_int32),
    ]


class CasBatchStats(ctypes.Structure):
    _fields_ = [
        ("seconds", ctypes.c_double), ("waves", ctypes.c_int64), ("jobs_ok", ctypes.c_int64),
        ("flop", ctypes.c_int64), ("nnz_c", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
        ("h2d_bytes", ctypes.c_double), ("max_wave_bound", ctypes.c_double),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


BATCH_MODES = {"waves": 0, "per_call": 1, "concurrent": 2}


class CasServerOpts(ctypes.Structure):
    _fields_ = [
        ("slots", ctypes.c_int32), ("accum", ctypes.c_int32), ("mem_budget", ctypes.c_double),
        ("keep_output", ctypes.c_int32), ("dry_run", ctypes.c_int32), ("dry_run_ns_per_byte", ctypes.c_double),
    ]


class CasResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("chunks", ctypes.c_int32), ("flop", ctypes.c_int64), ("nnz_c", ctypes.c_int64),
        ("digest", ctypes.c_uint64), ("bound", ctypes.c_double), ("t_submit", ctypes.c_double),
        ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double), ("C", CasCsr),
    ]


class CasServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
        ("chunked", ctypes.c_int64), ("max_inflight", ctypes.c_int32), ("max_inflight_bytes", ctypes.c_double),
    ]


class CasTuning(ctypes.Structure):
    _fields_ = [
        ("acc_thres", ctypes.c_double), ("fusion", ctypes.c_int32), ("fused_min_products", ctypes.c_int32),
        ("esc_max_products", ctypes.c_int32), ("hash_max_nnz", ctypes.c_int32), ("esc_form", ctypes.c_int32),
        ("heavy_split", ctypes.c_int32), ("bin_order", ctypes.c_int32), ("out_blocks", ctypes.c_int32),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class CasError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libcasgemm.so (raises FileNotFoundError when it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `make -C {HERE}` (or __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    P, I64, I32, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
    sig = {
        "cas_create": (I32, [ctypes.c_int, ctypes.POINTER(P)]),
        "cas_destroy": (None, [P]),
        "cas_set_stream": (I32, [P, P]),
        "cas_set_acc_thres": (I32, [P, D]),
        "cas_last_error": (ctypes.c_char_p, [P]),
        "cas_set_profiling": (I32, [P, ctypes.c_int]),
        "cas_set_fusion": (I32, [P, ctypes.c_int]),
        "cas_set_tuning": (I32, [P, ctypes.POINTER(CasTuning)]),
        "cas_get_tuning": (I32, [P, ctypes.POINTER(CasTuning)]),
        "cas_get_stats": (I32, [P, ctypes.POINTER(CasStats)]),
        "cas_spgemm": (I32, [P, I32, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr),
                             ctypes.POINTER(CasRuntime)]),
        "cas_csr_free": (I32, [P, ctypes.POINTER(CasCsr)]),
        "cas_csr_digest": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(ctypes.c_uint64), P]),
        "cas_csr_transpose": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr)]),
        "cas_batch_run": (I32, [P, I32, ctypes.POINTER(CasJob), I64, I32, D, ctypes.POINTER(CasBatchStats)]),
        "cas_serve_create": (I32, [ctypes.c_int, ctypes.POINTER(CasServerOpts), ctypes.POINTER(P)]),
        "cas_serve_submit": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), ctypes.POINTER(I64)]),
        "cas_serve_poll": (I32, [P, I64, ctypes.POINTER(CasResult)]),
        "cas_serve_wait": (I32, [P, I64, D, ctypes.POINTER(CasResult)]),
        "cas_serve_stats": (I32, [P, ctypes.POINTER(CasServerStats)]),
        "cas_serve_clock": (D, [P]),
        "cas_serve_destroy": (None, [P]),
        "cas_flp_populate": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), P]),
        "cas_scan": (I32, [P, P, P, I64]),
        "cas_hash_symb": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), P, P]),
        "cas_hash_numc": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), P, ctypes.POINTER(CasCsr)]),
        "cas_hsersc_numc": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), P, ctypes.POINTER(CasCsr)]),
        "cas_hybacc_numc": (I32, [P, ctypes.POINTER(CasCsr), ctypes.POINTER(CasCsr), P, ctypes.POINTER(CasCsr)]),
        "cas_gen_rmat": (I32, [ctypes.c_int, ctypes.c_int, D, D, D, ctypes.c_uint64, P, P]),
        "cas_zipf_row_degrees": (D, [I64, I64, D, I64, P]),
        "cas_gen_zipf": (I64, [I64, I64, I64, D, I64, D, D, ctypes.c_uint64, P, P]),
        "cas_gen_int_values": (None, [I64, I32, I32, ctypes.c_uint64, P]),
        "cas_csr_transpose_host": (I32, [I64, I64, P, P, P, ctypes.c_int, P, P, P]),
        "cas_intprod_host": (I64, [I64, P, P, P]),
        "cas_mtx_read": (I64, [ctypes.c_char_p, ctypes.POINTER(I64), ctypes.POINTER(I64), P, P, P]),
        "cas_mtx_write": (I32, [ctypes.c_char_p, I64, I64, P, P, ctypes.c_int]),
        "cas_csr_write_bin": (I32, [ctypes.c_char_p, I64, I64, P, P, P]),
        "cas_csr_read_bin": (I64, [ctypes.c_char_p, ctypes.POINTER(I64), ctypes.POINTER(I64), P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


# ------------------------------------------------------------------ matrices
@dataclass
class Csr:
    """Host CSR: int64 row pointers, int32 columns, float64 or int32 values."""
    num_row: int
    num_col: int
    row_ptrs: np.ndarray
    cols: np.ndarray
    vals: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.row_ptrs[-1]) if len(self.row_ptrs) else 0

    @property
    def val_type(self) -> int:
        return VAL_I32 if self.vals.dtype == np.int32 else VAL_F64

    def as_cas(self) -> CasCsr:
        rp = np.ascontiguousarray(self.row_ptrs, dtype=np.int64)
        cols = np.ascontiguousarray(self.cols)
        vals = np.ascontiguousarray(self.vals)
        self._keep = (rp, cols, vals)
        return CasCsr(self.num_row, self.num_col, self.nnz, rp.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                      cols.dtype.itemsize, self.val_type, 0, 0)

    def transpose(self) -> "Csr":
        return transpose(self)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.vals, self.cols, self.row_ptrs), shape=(self.num_row, self.num_col))


@dataclass
class Result:
    """C = A*B on the host, with the call's phase times and counters."""
    csr: Csr
    runtime: dict
    stats: dict = field(default_factory=dict)


class DeviceCsr:
    """A device CSR described by raw pointers (e.g. torch CUDA tensors' data_ptr)."""

    def __init__(self, num_row, num_col, nnz, row_ptrs_ptr, cols_ptr, vals_ptr, val_type=VAL_F64, keep=None):
        self.c = CasCsr(num_row, num_col, nnz, row_ptrs_ptr, cols_ptr, vals_ptr, 4, val_type, 1, 0)
        self._keep = keep

    @property
    def num_row(self) -> int:
        return self.c.num_row

    @staticmethod
    def upload(M: "Csr", device: int = 0) -> "DeviceCsr":
        """A device copy of host CSR M (torch CUDA tensors, kept alive by the object)."""
        import torch
        dev = torch.device("cuda", device)
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (M.row_ptrs, M.cols, M.vals)]
        return DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                         M.val_type, keep=t)


class Context:
    """A casgemm context on one device (cas_create / cas_destroy)."""

    def __init__(self, device: int = 0, acc_thres: float = 2.0):
        self.lib = load()
        h = ctypes.c_void_p()
        st = self.lib.cas_create(device, ctypes.byref(h))
        if st != 0:
            raise CasError(st, "cas_create failed")
        self.h = h
        self.set_acc_thres(acc_thres)

    def close(self):
        if getattr(self, "h", None):
            self.lib.cas_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            raise CasError(st, self.lib.cas_last_error(self.h).decode())

    def set_acc_thres(self, thres: float):
        self._check(self.lib.cas_set_acc_thres(self.h, float(thres)))

    def get_tuning(self) -> dict:
        t = CasTuning()
        self._check(self.lib.cas_get_tuning(self.h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Change the routing of rows to kernels (cas_set_tuning); unnamed knobs keep their values."""
        cur = self.get_tuning()
        unknown = set(kw) - set(cur)
        if unknown:
            raise ValueError(f"unknown tuning knobs {sorted(unknown)}")
        cur.update(kw)
        t = CasTuning(float(cur["acc_thres"]), int(cur["fusion"]), int(cur["fused_min_products"]),
                      int(cur["esc_max_products"]), int(cur["hash_max_nnz"]), int(cur["esc_form"]),
                      int(cur["heavy_split"]), int(cur["bin_order"]), int(cur["out_blocks"]))
        self._check(self.lib.cas_set_tuning(self.h, ctypes.byref(t)))

    def set_fusion(self, on: bool):
        self._check(self.lib.cas_set_fusion(self.h, int(bool(on))))

    def set_profiling(self, on: bool):
        self._check(self.lib.cas_set_profiling(self.h, int(bool(on))))

    def set_stream(self, stream_ptr: Optional[int]):
        self._check(self.lib.cas_set_stream(self.h, stream_ptr))

    def stats(self) -> dict:
        s = CasStats()
        self._check(self.lib.cas_get_stats(self.h, ctypes.byref(s)))
        return {
            "flop": s.flop, "max_row_flp": s.max_row_flp, "nnz_c": s.nnz_c,
            "symb_bins": dict(zip(SYMB_BINS, list(s.symb_bin_rows))),
            "numc_bins": dict(zip(NUMC_BINS, list(s.numc_bin_rows))),
            "kernel_launches": s.kernel_launches, "h2d_bytes": s.h2d_bytes, "d2h_bytes": s.d2h_bytes,
            "symb_bin_ms": dict(zip(SYMB_BINS, list(s.symb_bin_ms))),
            "numc_bin_ms": dict(zip(NUMC_BINS, list(s.numc_bin_ms))),
            "numc_bin_bytes": dict(zip(NUMC_BINS, list(s.numc_bin_bytes))),
            "numc_bin_flop": dict(zip(NUMC_BINS, list(s.numc_bin_flop))),
            "esc_overflow_rows": s.esc_overflow_rows, "esc_overflow_ms": s.esc_overflow_ms,
            "fused_rows": s.fused_rows, "fused_flop": s.fused_flop, "fused_bytes": s.fused_bytes,
            "fused_ms": s.fused_ms, "d2h_direct_bytes": s.d2h_direct_bytes, "split_rows": s.split_rows,
            "out_blocks": s.out_blocks, "numc_bin_nnz": dict(zip(NUMC_BINS, list(s.numc_bin_nnz))),
        }

    def spgemm(self, A, B, accum: str = "hybacc", col_bytes: int = 4) -> Result:
        """C = A*B for host CSR inputs (Csr or CasCsr), returned on the host."""
        ca = A.as_cas() if isinstance(A, Csr) else A
        cb = B.as_cas() if isinstance(B, Csr) else B
        cc = CasCsr()
        cc.on_device = 0
        cc.col_bytes = col_bytes
        rt = CasRuntime()
        self._check(self.lib.cas_spgemm(self.h, ACCUM[accum], ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(cc),
                                        ctypes.byref(rt)))
        try:
            m, nnz = cc.num_row, cc.num_nnz
            rp = np.ctypeslib.as_array(ctypes.cast(cc.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (m + 1,)).copy()
            ctype = ctypes.c_int32 if cc.col_bytes == 4 else ctypes.c_int64
            vtype = ctypes.c_double if cc.val_type == VAL_F64 else ctypes.c_int64
            if nnz > 0:
                cols = np.ctypeslib.as_array(ctypes.cast(cc.cols, ctypes.POINTER(ctype)), (nnz,)).copy()
                vals = np.ctypeslib.as_array(ctypes.cast(cc.rats, ctypes.POINTER(vtype)), (nnz,)).copy()
            else:
                cols = np.zeros(0, np.int32 if cc.col_bytes == 4 else np.int64)
                vals = np.zeros(0, np.float64 if cc.val_type == VAL_F64 else np.int64)
            C = Csr(cc.num_row, cc.num_col, rp, cols, vals)
        finally:
            self.lib.cas_csr_free(self.h, ctypes.byref(cc))
        return Result(C, rt.as_dict(), self.stats())

    def spgemm_device(self, A: DeviceCsr, B: DeviceCsr, accum: str = "hybacc"):
        """C = A*B for device inputs; returns (CasCsr owned by the library, runtime).

        Release the result with :meth:`free`."""
        cc = CasCsr()
        cc.on_device = 1
        rt = CasRuntime()
        self._check(self.lib.cas_spgemm(self.h, ACCUM[accum], ctypes.byref(A.c), ctypes.byref(B.c),
                                        ctypes.byref(cc), ctypes.byref(rt)))
        return cc, rt.as_dict()

    def transpose(self, A) -> Csr:
        """B = A^T computed on the device (cas_csr_transpose), returned on the host."""
        ca = A.as_cas() if isinstance(A, Csr) else A.c
        cb = CasCsr()
        cb.on_device = 0
        self._check(self.lib.cas_csr_transpose(self.h, ctypes.byref(ca), ctypes.byref(cb)))
        try:
            n, nnz = cb.num_row, cb.num_nnz
            rp = np.ctypeslib.as_array(ctypes.cast(cb.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (n + 1,)).copy()
            vt, vdt = (ctypes.c_double, np.float64) if cb.val_type == VAL_F64 else (ctypes.c_int32, np.int32)
            cols = (np.ctypeslib.as_array(ctypes.cast(cb.cols, ctypes.POINTER(ctypes.c_int32)), (nnz,)).copy()
                    if nnz else np.zeros(0, np.int32))
            vals = (np.ctypeslib.as_array(ctypes.cast(cb.rats, ctypes.POINTER(vt)), (nnz,)).copy()
                    if nnz else np.zeros(0, vdt))
        finally:
            self.lib.cas_csr_free(self.h, ctypes.byref(cb))
        return Csr(n, A.num_row, rp, cols, vals)

    def transpose_device(self, A) -> CasCsr:
        """B = A^T on the device, owned by the library (release with :meth:`free`)."""
        ca = A.as_cas() if isinstance(A, Csr) else A.c
        cb = CasCsr()
        cb.on_device = 1
        self._check(self.lib.cas_csr_transpose(self.h, ctypes.byref(ca), ctypes.byref(cb)))
        return cb

    def free(self, cc: CasCsr):
        self._check(self.lib.cas_csr_free(self.h, ctypes.byref(cc)))

    def digest(self, cc: CasCsr, rows: bool = False):
        """Digest of a device CSR (cas_csr_digest); with rows, also its row digests."""
        d = ctypes.c_uint64()
        rd = np.empty(cc.num_row, np.uint64) if rows else None
        self._check(self.lib.cas_csr_digest(self.h, ctypes.byref(cc), ctypes.byref(d), _ptr(rd)))
        return (int(d.value), rd) if rows else int(d.value)

    def batch_run(self, jobs, accum: str = "hybacc", mode: str = "waves", wave_budget: float = 0.0,
                  row_digests: bool = False):
        """Independent products C_j = A_j * B_j (cas_batch_run).

        jobs: list of (A, B), each a host Csr or a DeviceCsr.  Returns (per-job
        dicts with flop, nnz_c, digest, status and optionally row_digests,
        batch stats)."""
        arr = (CasJob * max(1, len(jobs)))()
        keep = []
        rds = []
        for j, (A, B) in enumerate(jobs):
            ca = A.as_cas() if isinstance(A, Csr) else A.c
            cb = B.as_cas() if isinstance(B, Csr) else B.c
            keep.append((A, B))
            arr[j].A, arr[j].B = ca, cb
            rd = np.zeros(ca.num_row, np.uint64) if row_digests else None
            rds.append(rd)
            arr[j].row_digests = _ptr(rd) if rd is not None and len(rd) else None
        st = CasBatchStats()
        rc = self.lib.cas_batch_run(self.h, ACCUM[accum], arr, len(jobs), BATCH_MODES[mode], float(wave_budget),
                                    ctypes.byref(st))
        out = []
        for j in range(len(jobs)):
            d = {"flop": arr[j].flop, "nnz_c": arr[j].nnz_c, "digest": int(arr[j].digest),
                 "status": arr[j].status}
            if row_digests:
                d["row_digests"] = rds[j]
            out.append(d)
        if rc != 0:
            raise CasError(rc, self.lib.cas_last_error(self.h).decode())
        return out, st.as_dict()


class Server:
    """A request loop with continuous batching (cas_serve_*): submit returns at
    once; requests are admitted in order as slots and device memory free up,
    and run concurrently."""

    def __init__(self, device: int = 0, slots: int = 4, mem_budget: float = 60e9, accum: str = "hybacc",
                 keep_output: bool = False, dry_run: bool = False, dry_run_ns_per_byte: float = 0.0):
        self.lib = load()
        opts = CasServerOpts(slots, ACCUM[accum], float(mem_budget), int(keep_output), int(dry_run),
                             float(dry_run_ns_per_byte))
        h = ctypes.c_void_p()
        st = self.lib.cas_serve_create(device, ctypes.byref(opts), ctypes.byref(h))
        if st != 0:
            raise CasError(st, "cas_serve_create failed")
        self.h = h
        self._inputs = {}

    def submit(self, A, B) -> int:
        """Queues C = A * B.  A and B are both host Csr, or both DeviceCsr
        resident on the server's device (uploaded once, served many times)."""
        ca = A.as_cas() if isinstance(A, Csr) else A.c
        cb = B.as_cas() if isinstance(B, Csr) else B.c
        rid = ctypes.c_int64()
        st = self.lib.cas_serve_submit(self.h, ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(rid))
        if st != 0:
            raise CasError(st, "cas_serve_submit rejected the request")
        self._inputs[rid.value] = (A, B, ca, cb)  # the server reads these arrays until the request completes
        return rid.value

    def _result(self, rid, r: CasResult) -> dict:
        self._inputs.pop(rid, None)
        out = {"status": r.status, "chunks": r.chunks, "flop": r.flop, "nnz_c": r.nnz_c, "digest": int(r.digest),
               "bound": r.bound, "t_submit": r.t_submit, "t_admit": r.t_admit, "t_done": r.t_done}
        if r.C.owned:
            c = r.C
            rp = np.ctypeslib.as_array(ctypes.cast(c.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (c.num_row + 1,)).copy()
            vt = ctypes.c_double if c.val_type == VAL_F64 else ctypes.c_int64
            cols = (np.ctypeslib.as_array(ctypes.cast(c.cols, ctypes.POINTER(ctypes.c_int32)), (c.num_nnz,)).copy()
                    if c.num_nnz else np.zeros(0, np.int32))
            vals = (np.ctypeslib.as_array(ctypes.cast(c.rats, ctypes.POINTER(vt)), (c.num_nnz,)).copy()
                    if c.num_nnz else np.zeros(0, np.float64 if c.val_type == VAL_F64 else np.int64))
            out["C"] = Csr(c.num_row, c.num_col, rp, cols, vals)
            self.lib.cas_csr_free(None, ctypes.byref(r.C))
        return out

    def poll(self, rid: int):
        r = CasResult()
        st = self.lib.cas_serve_poll(self.h, rid, ctypes.byref(r))
        if st == 5:
            return None
        if st != 0:
            raise CasError(st, f"unknown request {rid}")
        return self._result(rid, r)

    def wait(self, rid: int, timeout: float = -1.0):
        r = CasResult()
        st = self.lib.cas_serve_wait(self.h, rid, float(timeout), ctypes.byref(r))
        if st == 5:
            return None
        if st != 0:
            raise CasError(st, f"unknown request {rid}")
        return self._result(rid, r)

    def stats(self) -> dict:
        s = CasServerStats()
        self.lib.cas_serve_stats(self.h, ctypes.byref(s))
        return {n: getattr(s, n) for n, _ in s._fields_}

    def clock(self) -> float:
        return self.lib.cas_serve_clock(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.cas_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Autotuner:
    """Picks the routing of rows to kernels (cas_tuning) per class of input.

    The class is a key from the degree distribution of the product: log2 of
    the mean products per row (rounded), log2 of the largest row's products
    over the mean (the skew, rounded down), log2 of the column count, and the
    value type.  For a
    class not yet in the cache, `tune` times every candidate setting on the
    given device matrices (best of `trials` runs by the pipeline's own CUDA
    events) and keeps the fastest; the cache is a JSON file, so a class is
    tuned once.  Every candidate computes the same C; only the speed differs.
    """

    CANDIDATES = ([{"acc_thres": a, "fusion": 1, "fused_min_products": lo, "esc_max_products": e,
                    "hash_max_nnz": 4096, "esc_form": f, "heavy_split": 1, "bin_order": 1}
                   for a in (1.5, 2.0, 5.0) for lo in (1024, 2048, 3072) for e in (4096, 8192) for f in (2, 1, 0)]
                  + [{"acc_thres": 2.0, "fusion": 0, "fused_min_products": 2048, "esc_max_products": 8192,
                      "hash_max_nnz": 4096, "esc_form": 1, "heavy_split": 1, "bin_order": 1},
                     {"acc_thres": 2.0, "fusion": 1, "fused_min_products": 2048, "esc_max_products": 8192,
                      "hash_max_nnz": 4096, "esc_form": 2, "heavy_split": 1, "bin_order": 0}])

    def __init__(self, ctx: "Context", cache_path: Optional[str] = None):
        self.ctx = ctx
        self.path = cache_path
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            import json
            with open(cache_path) as fh:
                self.cache = json.load(fh)

    @staticmethod
    def key(A: Csr, B: Csr) -> str:
        import math
        rows = np.diff(row_products_prefix(A, B))
        mean = float(rows.mean()) if len(rows) else 0.0
        mx = float(rows.max()) if len(rows) else 0.0
        lg = lambda x: int(round(math.log2(x))) if x > 0 else 0  # noqa: E731
        skew = int(math.floor(math.log2(mx / mean))) if mean > 0 and mx > 0 else 0
        vt = "i32" if A.vals.dtype == np.int32 else "f64"
        return f"p{lg(mean)}_s{skew}_c{lg(B.num_col)}_{vt}"

    def tune(self, key: str, dA: "DeviceCsr", dB: "DeviceCsr", accum: str = "hybacc", trials: int = 2) -> dict:
        if key in self.cache:
            return self.cache[key]
        saved = self.ctx.get_tuning()
        timed = []
        try:
            for cand in self.CANDIDATES:
                self.ctx.set_tuning(**cand)
                best = float("inf")
                for _ in range(trials):
                    cc, rt = self.ctx.spgemm_device(dA, dB, accum)
                    self.ctx.free(cc)
                    best = min(best, rt["total_time"])
                timed.append((best, cand))
        finally:
            self.ctx.set_tuning(**saved)
        best_t, best = min(timed, key=lambda x: x[0])
        default_t = next((t for t, c in timed if all(saved[k] == v for k, v in c.items())), None)  # as the context had
        self.cache[key] = dict(best, seconds=best_t, default_seconds=default_t)
        if self.path:
            import json
            with open(self.path, "w") as fh:
                json.dump(self.cache, fh, indent=1, sort_keys=True)
        return self.cache[key]

    def apply(self, key: str) -> bool:
        """Sets the cached choice for `key` on the context; False if the class was never tuned."""
        cfg = self.cache.get(key)
        if not cfg:
            return False
        self.ctx.set_tuning(**{k: cfg[k] for k in ("acc_thres", "fusion", "fused_min_products",
                                                    "esc_max_products", "hash_max_nnz", "esc_form", "heavy_split",
                                                    "bin_order")
                               if k in cfg})
        return True


# ---------------------------------------------------------------- data layer
def gen_rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int) -> Csr:
    """Symmetrised loop-free duplicate-free R-MAT graph (values 1.0)."""
    lib = load()
    n = 1 << scale
    nnz = 2 * edge_factor * n
    rp = np.empty(n + 1, np.int64)
    cols = np.empty(nnz, np.int32)
    st = lib.cas_gen_rmat(scale, edge_factor, a, b, c, seed, _ptr(rp), _ptr(cols))
    if st != 0:
        raise ValueError(f"cas_gen_rmat failed for scale={scale} ef={edge_factor}")
    return Csr(n, n, rp, cols, np.ones(nnz, np.float64))


def gen_g500(scale: int, edge_factor: int, seed: int) -> Csr:
    return gen_rmat(scale, edge_factor, 0.57, 0.19, 0.19, seed)


def gen_er(scale: int, edge_factor: int, seed: int) -> Csr:
    return gen_rmat(scale, edge_factor, 0.25, 0.25, 0.25, seed)


def gen_zipf(num_row: int, num_col: int, amax: int, target_nnz: int, seed: int,
             row_s: float = 1.2, col_s: float = 1.4, col_q: float = 1000.0) -> Csr:
    lib = load()
    rp = np.empty(num_row + 1, np.int64)
    nnz = lib.cas_gen_zipf(num_row, num_col, amax, row_s, target_nnz, col_s, col_q, seed, _ptr(rp), None)
    if nnz < 0:
        raise ValueError("cas_gen_zipf failed")
    cols = np.empty(nnz, np.int32)
    nnz2 = lib.cas_gen_zipf(num_row, num_col, amax, row_s, target_nnz, col_s, col_q, seed, _ptr(rp), _ptr(cols))
    if nnz2 != nnz:
        raise ValueError("cas_gen_zipf failed")
    return Csr(num_row, num_col, rp, cols, np.ones(nnz, np.float64))


def int_values(nnz: int, seed: int, lo: int = 1, hi: int = 8) -> np.ndarray:
    v = np.empty(nnz, np.int32)
    load().cas_gen_int_values(nnz, lo, hi, seed, _ptr(v))
    return v


def transpose(A: Csr) -> Csr:
    lib = load()
    rp = np.empty(A.num_col + 1, np.int64)
    cols = np.empty(A.nnz, np.int32)
    vals = np.empty(A.nnz, A.vals.dtype)
    cols_in = np.ascontiguousarray(A.cols, dtype=np.int32)
    st = lib.cas_csr_transpose_host(A.num_row, A.num_col, _ptr(np.ascontiguousarray(A.row_ptrs, np.int64)),
                                    _ptr(cols_in), _ptr(np.ascontiguousarray(A.vals)), A.vals.dtype.itemsize,
                                    _ptr(rp), _ptr(cols), _ptr(vals))
    if st != 0:
        raise ValueError("transpose failed")
    return Csr(A.num_col, A.num_row, rp, cols, vals)


def intprod(A: Csr, B: Csr) -> int:
    """Intermediate products of A*B (the reference's flop_cnt)."""
    return int(load().cas_intprod_host(A.num_row, _ptr(np.ascontiguousarray(A.row_ptrs, np.int64)),
                                       _ptr(np.ascontiguousarray(A.cols, np.int32)),
                                       _ptr(np.ascontiguousarray(B.row_ptrs, np.int64))))


def mtx_read(path: str) -> Csr:
    """MatrixMarket -> CSR with the reference loader's semantics (values forced to 1.0)."""
    lib = load()
    nr, nc = ctypes.c_int64(), ctypes.c_int64()
    nnz = lib.cas_mtx_read(path.encode(), ctypes.byref(nr), ctypes.byref(nc), None, None, None)
    if nnz < 0:
        raise ValueError(f"cannot read {path}")
    rp = np.empty(nr.value + 1, np.int64)
    cols = np.empty(nnz, np.int32)
    vals = np.empty(nnz, np.float64)
    if lib.cas_mtx_read(path.encode(), ctypes.byref(nr), ctypes.byref(nc), _ptr(rp), _ptr(cols), _ptr(vals)) != nnz:
        raise ValueError(f"cannot read {path}")
    return Csr(nr.value, nc.value, rp, cols, vals)


def mtx_write(path: str, A: Csr, symmetric: bool):
    if load().cas_mtx_write(path.encode(), A.num_row, A.num_col, _ptr(np.ascontiguousarray(A.row_ptrs, np.int64)),
                            _ptr(np.ascontiguousarray(A.cols, np.int32)), int(symmetric)) != 0:
        raise ValueError(f"cannot write {path}")


def csr_write_bin(path: str, A: Csr):
    """Binary CSR cache of A (cas_csr_write_bin); fp64 values."""
    vals = np.ascontiguousarray(A.vals, dtype=np.float64)
    if load().cas_csr_write_bin(path.encode(), A.num_row, A.num_col, _ptr(np.ascontiguousarray(A.row_ptrs, np.int64)),
                                _ptr(np.ascontiguousarray(A.cols, np.int32)), _ptr(vals)) != 0:
        raise ValueError(f"cannot write {path}")


def csr_read_bin(path: str) -> Csr:
    lib = load()
    nr, nc = ctypes.c_int64(), ctypes.c_int64()
    nnz = lib.cas_csr_read_bin(path.encode(), ctypes.byref(nr), ctypes.byref(nc), None, None, None)
    if nnz < 0:
        raise ValueError(f"cannot read {path}")
    rp = np.empty(nr.value + 1, np.int64)
    cols = np.empty(nnz, np.int32)
    vals = np.empty(nnz, np.float64)
    if lib.cas_csr_read_bin(path.encode(), ctypes.byref(nr), ctypes.byref(nc), _ptr(rp), _ptr(cols), _ptr(vals)) != nnz:
        raise ValueError(f"cannot read {path}")
    return Csr(nr.value, nc.value, rp, cols, vals)


# ---------------------------------------------------------- row sharding
def row_products_prefix(A: Csr, B: Csr) -> np.ndarray:
    """Prefix of intermediate products over the rows of A (num_row + 1 entries)."""
    cnt = np.diff(B.row_ptrs)[np.asarray(A.cols, dtype=np.int64)].astype(np.int64)
    return np.concatenate([[0], np.cumsum(cnt)])[A.row_ptrs]


def row_shard(prefix: np.ndarray, rank: int, world: int, r_end: Optional[int] = None):
    """Contiguous rows [r0, r1) of [0, r_end) holding about 1/world of their products.

    Rows of C are independent (C[r0:r1] = A[r0:r1] * B), so shards need no
    exchange; splitting by the product prefix is the lower_bound-on-prefix
    split of the reference's morsel packing (src/ams/ams_utils.c:1459-1465)."""
    n = len(prefix) - 1
    r_end = n if r_end is None else r_end
    if world <= 1:
        return 0, r_end
    ps = prefix[: r_end + 1]
    total = int(ps[-1])
    r0 = 0 if rank == 0 else int(np.searchsorted(ps, total * rank // world, side="left"))
    r1 = r_end if rank + 1 == world else int(np.searchsorted(ps, total * (rank + 1) // world, side="left"))
    return r0, r1


class _DeviceView:
    """A device array as __cuda_array_interface__ (zero copy, for torch.as_tensor)."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def device_tensors(cc: CasCsr):
    """torch views (no copy) of a device CSR's row pointers, columns and
    values, e.g. a C the library allocated; valid until it is freed."""
    import torch

    def view(ptr, n, typestr, dtype):
        if n == 0:
            return torch.empty(0, dtype=dtype, device="cuda")
        return torch.as_tensor(_DeviceView(ptr, n, typestr), device="cuda")

    vt = ("<f8", torch.float64) if cc.val_type == VAL_F64 else ("<i8", torch.int64)
    return (view(cc.row_ptrs, cc.num_row + 1, "<i8", torch.int64), view(cc.cols, cc.num_nnz, "<i4", torch.int32),
            view(cc.rats, cc.num_nnz, *vt))


def gather_shards(rp, cols, vals, r0: int, r1: int, num_row: int, root: int = 0):
    """Assembles the row shards of C from every rank on `root`.

    Each rank passes its shard, rows [r0, r1) of C, as torch tensors: row
    pointers starting at 0 (r1 - r0 + 1 entries), columns and values.  The
    ranks all-gather (r0, r1, nnz) of every shard; the root then receives
    each other rank's columns, values and row pointers by point-to-point
    transfers (NCCL over NVLink for CUDA tensors, gloo for host tensors) into
    its slice of C, and shifts the row pointers by the nnz of the shards
    before it.  Shards must cover [0, num_row) in rank order.  Returns (rp,
    cols, vals) of the whole C on the root and None elsewhere."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(), dist.get_rank()
    dev = cols.device
    meta = torch.tensor([r0, r1, int(rp[-1]) if len(rp) else 0], dtype=torch.int64, device=dev)
    allm = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(allm, meta)
    allm = [tuple(int(x) for x in m.tolist()) for m in allm]
    if [m[0] for m in allm] != sorted(m[0] for m in allm) or allm[0][0] != 0 or allm[-1][1] != num_row or \
            any(allm[q][1] != allm[q + 1][0] for q in range(world - 1)):
        raise ValueError("row shards must cover [0, num_row) in rank order")
    offs = [0]
    for m in allm:
        offs.append(offs[-1] + m[2])
    if rank != root:
        reqs = [dist.isend(rp.contiguous(), root)]
        if allm[rank][2] > 0:
            reqs += [dist.isend(cols.contiguous(), root), dist.isend(vals.contiguous(), root)]
        for r in reqs:
            r.wait()
        return None
    C_rp = torch.empty(num_row + 1, dtype=torch.int64, device=dev)
    C_cols = torch.empty(offs[-1], dtype=cols.dtype, device=dev)
    C_vals = torch.empty(offs[-1], dtype=vals.dtype, device=dev)
    parts, reqs = [], []
    for q, (a0, a1, n) in enumerate(allm):
        if q == root:
            parts.append((q, rp))
            C_cols[offs[q]:offs[q] + n] = cols
            C_vals[offs[q]:offs[q] + n] = vals
            continue
        buf = torch.empty(a1 - a0 + 1, dtype=torch.int64, device=dev)
        reqs.append(dist.irecv(buf, q))
        parts.append((q, buf))
        if n > 0:
            reqs.append(dist.irecv(C_cols[offs[q]:offs[q] + n], q))
            reqs.append(dist.irecv(C_vals[offs[q]:offs[q] + n], q))
    for r in reqs:
        r.wait()
    for q, part in parts:
        a0, a1, _ = allm[q]
        C_rp[a0:a1 + 1] = part + offs[q]
    return C_rp, C_cols, C_vals


def slice_rows(A: Csr, r0: int, r1: int) -> Csr:
    """Rows [r0, r1) of A as a CSR of its own (views, no copy of columns/values)."""
    s, e = int(A.row_ptrs[r0]), int(A.row_ptrs[r1])
    return Csr(r1 - r0, A.num_col, A.row_ptrs[r0:r1 + 1] - s, A.cols[s:e], A.vals[s:e])


# ------------------------------------------------------------ batch workload
def _splitmix(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 31)


def batch_spec(n: int = 512, seed: int = 4, scales=(10, 17), edge_factors=(2, 4, 8, 16, 32)):
    """The uneven batch: job j is a G500 R-MAT with scale uniform in
    [scales[0], scales[1]] and edge factor uniform over edge_factors, drawn
    from (seed, j) by SplitMix64; returns [(scale, edge_factor, graph_seed)]."""
    out = []
    span = scales[1] - scales[0] + 1
    for j in range(n):
        base = _splitmix((seed << 32) ^ j)
        s = scales[0] + _splitmix(base ^ 1) % span
        ef = edge_factors[_splitmix(base ^ 2) % len(edge_factors)]
        out.append((int(s), int(ef), int(_splitmix(base ^ 3) & 0xFFFFFFFF)))
    return out


def batch_job(scale: int, edge_factor: int, graph_seed: int, int_vals: bool = True):
    """One job of the batch: (A, B = A^T) with int32 values uniform in 1..8
    (accumulated in int64), or values 1.0."""
    A = gen_g500(scale, edge_factor, graph_seed)
    if int_vals:
        A = Csr(A.num_row, A.num_col, A.row_ptrs, A.cols, int_values(A.nnz, graph_seed ^ 0x5DEECE66D))
    return A, transpose(A)
