"""TEST INFRASTRUCTURE — ctypes access to the two CPU oracles.

* :func:`oracle_spgemm` — the project's C restatement (oracle/cas_oracle.c,
  liboracle_cas.so) of the reference's algorithm.
* :func:`ref_spgemm` — the reference itself (fukien/contention-aware-spgemm),
  compiled from its unmodified sources into oracle/_ref/libref_<algo>.so with
  a direct-call harness (oracle/ref_harness.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only to check or time the GPU product against; the product never
imports it.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_cas.so")
REF_DIR = os.path.join(HERE, "_ref")
ALGOS = {"hash": 0, "hsersc": 1, "hybacc": 2}
# AMS_ACC_THRES of each reference build (scripts/ams_rmat_run.sh:25-36)
REF_ACC_THRES = {"hash": 5.0, "hsersc": 5.0, "hybacc": 2.0}


class OrcCsr(ctypes.Structure):
    """The reference's csr_t (src/inc/store.h:49-56): int64 indices, fp64 values."""
    _fields_ = [
        ("num_row", ctypes.c_int64), ("num_col", ctypes.c_int64), ("num_nnz", ctypes.c_int64),
        ("row_ptrs", ctypes.c_void_p), ("cols", ctypes.c_void_p), ("rats", ctypes.c_void_p),
    ]


class RefRuntime(ctypes.Structure):
    """runtime_t (src/mm/mm_utils.h:48-54)."""
    _fields_ = [(n, ctypes.c_double) for n in ("init_time", "symb_time", "mgmt_time", "numc_time", "total_time")]


_orc = None
_refs = {}


def _load_oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            raise FileNotFoundError(f"{ORACLE_LIB} missing: run `make -C {HERE}`")
        lib = ctypes.CDLL(ORACLE_LIB)
        P = ctypes.c_void_p
        lib.orc_spgemm.restype = ctypes.c_int64
        lib.orc_spgemm.argtypes = [ctypes.POINTER(OrcCsr), ctypes.POINTER(OrcCsr), ctypes.POINTER(OrcCsr),
                                   ctypes.c_int, ctypes.c_double, ctypes.c_int]
        lib.orc_free.argtypes = [ctypes.POINTER(OrcCsr)]
        lib.orc_sort_rows.argtypes = [ctypes.POINTER(OrcCsr)]
        lib.orc_flp_populate.argtypes = [ctypes.POINTER(OrcCsr), ctypes.POINTER(OrcCsr), P]
        lib.orc_hash_symb.argtypes = [ctypes.POINTER(OrcCsr), ctypes.POINTER(OrcCsr), P, P]
        lib.orc_scan.argtypes = [P, P, ctypes.c_int64]
        lib.orc_intprod.restype = ctypes.c_int64
        lib.orc_intprod.argtypes = [ctypes.POINTER(OrcCsr), ctypes.POINTER(OrcCsr)]
        lib.orc_next_pow2.restype = ctypes.c_int64
        lib.orc_next_pow2.argtypes = [ctypes.c_int64]
        lib.orc_radix_sort_kv.argtypes = [P, P, P, P, ctypes.c_int64]
        lib.orc_row_digests.restype = ctypes.c_uint64
        lib.orc_row_digests.argtypes = [ctypes.POINTER(OrcCsr), ctypes.c_int64, P]
        lib.orc_pack_morsels.restype = ctypes.c_int64
        lib.orc_pack_morsels.argtypes = [ctypes.c_int64, P, P, P, ctypes.c_int64, ctypes.c_double, P, P, P, P,
                                         ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        _orc = lib
    return _orc


def _load_ref(algo: str, small: bool):
    key = (algo, small)
    if key not in _refs:
        path = os.path.join(REF_DIR, f"libref_{algo}{'_small' if small else ''}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C {HERE} ref` where the reference sources exist")
        lib = ctypes.CDLL(path)
        lib.ref_spgemm.restype = ctypes.c_int
        lib.ref_spgemm.argtypes = [ctypes.POINTER(OrcCsr)] * 3 + [ctypes.POINTER(RefRuntime)]
        lib.ref_free_csr.argtypes = [ctypes.POINTER(OrcCsr)]
        lib.ref_intprod.restype = ctypes.c_long
        lib.ref_intprod.argtypes = [ctypes.POINTER(OrcCsr), ctypes.POINTER(OrcCsr)]
        lib.ref_morsel_size.restype = ctypes.c_long
        lib.ref_thread_num.restype = ctypes.c_int
        lib.ref_acc_thres.restype = ctypes.c_double
        _refs[key] = lib
    return _refs[key]


def ref_available(algo: str = "hybacc", small: bool = True) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{algo}{'_small' if small else ''}.so"))


def to_orc(rp, cols, vals, num_col) -> Tuple[OrcCsr, tuple]:
    """Build a csr_t view (int64 columns, fp64 values); returns (struct, keep-alive)."""
    rp = np.ascontiguousarray(rp, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    s = OrcCsr(len(rp) - 1, num_col, int(rp[-1]) if len(rp) else 0, rp.ctypes.data, cols.ctypes.data,
               vals.ctypes.data)
    return s, (rp, cols, vals)


def _from_orc(c: OrcCsr):
    m, nnz = c.num_row, c.num_nnz
    rp = np.ctypeslib.as_array(ctypes.cast(c.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (m + 1,)).copy()
    if nnz > 0:
        cols = np.ctypeslib.as_array(ctypes.cast(c.cols, ctypes.POINTER(ctypes.c_int64)), (nnz,)).copy()
        vals = np.ctypeslib.as_array(ctypes.cast(c.rats, ctypes.POINTER(ctypes.c_double)), (nnz,)).copy()
    else:
        cols, vals = np.zeros(0, np.int64), np.zeros(0, np.float64)
    return rp, cols, vals


def sort_rows(rp, cols, vals):
    """Canonical per-row column order (the hash accumulators emit slot order)."""
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp))
    order = np.lexsort((cols, rows))
    return rp, cols[order], vals[order]


def oracle_spgemm(A, B, algo: str = "hybacc", acc_thres: Optional[float] = None, sort: bool = True):
    """C = A*B by the C restatement.  A, B: objects with num_row/num_col/row_ptrs/cols/vals.

    Returns (row_ptrs, cols int64, vals f64, flop)."""
    lib = _load_oracle()
    a, ka = to_orc(A.row_ptrs, A.cols, A.vals, A.num_col)
    b, kb = to_orc(B.row_ptrs, B.cols, B.vals, B.num_col)
    c = OrcCsr()
    thres = REF_ACC_THRES[algo] if acc_thres is None else acc_thres
    flop = lib.orc_spgemm(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ALGOS[algo], thres, int(sort))
    try:
        rp, cols, vals = _from_orc(c)
    finally:
        lib.orc_free(ctypes.byref(c))
    del ka, kb
    return rp, cols, vals, int(flop)


def ref_spgemm(A, B, algo: str = "hybacc", small: bool = True):
    """C = A*B by the reference's own kernels; rows sorted for comparison.

    Returns (row_ptrs, cols, vals, runtime dict) or None when the input is
    below one morsel (the reference would exit(1))."""
    lib = _load_ref(algo, small)
    a, ka = to_orc(A.row_ptrs, A.cols, A.vals, A.num_col)
    b, kb = to_orc(B.row_ptrs, B.cols, B.vals, B.num_col)
    c = OrcCsr()
    rt = RefRuntime()
    st = lib.ref_spgemm(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(rt))
    if st != 0:
        return None
    try:
        _load_oracle().orc_sort_rows(ctypes.byref(c))  # csr_t and orc_csr share one layout
        rp, cols, vals = _from_orc(c)
    finally:
        lib.ref_free_csr(ctypes.byref(c))
    del ka, kb
    return rp, cols, vals, {n: getattr(rt, n) for n, _ in RefRuntime._fields_}


class RefTimer:
    """Times the reference's own driver sequence on fixed inputs, the way its
    drivers do: each run builds C and frees it again
    (src/ams_hybaccspgemm.c:316-343), and only the reference's runtime_t is
    kept.  The csr_t views of A and B are built once, so a run costs the
    reference's four phases plus its own free_csr, with no copy of C into
    Python and no per-row sort."""

    def __init__(self, A, B, algo: str = "hybacc", small: bool = False):
        self.lib = _load_ref(algo, small)
        self.a, self.ka = to_orc(A.row_ptrs, A.cols, A.vals, A.num_col)
        self.b, self.kb = to_orc(B.row_ptrs, B.cols, B.vals, B.num_col)

    def run(self) -> Optional[dict]:
        """One run; the runtime dict, or None when A is below one morsel."""
        c = OrcCsr()
        rt = RefRuntime()
        st = self.lib.ref_spgemm(ctypes.byref(self.a), ctypes.byref(self.b), ctypes.byref(c), ctypes.byref(rt))
        if st != 0:
            return None
        nnz = int(c.num_nnz)
        self.lib.ref_free_csr(ctypes.byref(c))
        out = {n: getattr(rt, n) for n, _ in RefRuntime._fields_}
        out["nnz_c"] = nnz
        return out


def ref_row_digests(A, B, algo: str = "hybacc", small: bool = False, row_offset: int = 0):
    """C = A*B by the reference's own kernels, reduced to the row digests of
    the casgemm ABI (cas_csr_digest) after sorting each row by column, in C
    with OpenMP, so that outputs of hundreds of millions of entries are
    checked without copying them into Python.

    Returns (row_ptrs, row digests uint64[m], digest, runtime dict) or None
    below one morsel; `digest` counts row r as r + row_offset."""
    lib = _load_ref(algo, small)
    orc = _load_oracle()
    a, ka = to_orc(A.row_ptrs, A.cols, A.vals, A.num_col)
    b, kb = to_orc(B.row_ptrs, B.cols, B.vals, B.num_col)
    c = OrcCsr()
    rt = RefRuntime()
    st = lib.ref_spgemm(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(rt))
    if st != 0:
        return None
    try:
        orc.orc_sort_rows(ctypes.byref(c))
        rp = np.ctypeslib.as_array(ctypes.cast(c.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (c.num_row + 1,)).copy()
        rows = np.zeros(c.num_row, np.uint64)
        total = int(orc.orc_row_digests(ctypes.byref(c), int(row_offset), rows.ctypes.data))
    finally:
        lib.ref_free_csr(ctypes.byref(c))
    del ka, kb
    return rp, rows, total, {n: getattr(rt, n) for n, _ in RefRuntime._fields_}


def ref_load_mtx(path: str):
    """The reference's own MatrixMarket loader: (num_row, num_col, row_ptrs, cols, vals)."""
    lib = _load_ref("hybacc", True)
    lib.ref_load_mtx.argtypes = [ctypes.c_char_p, ctypes.POINTER(OrcCsr)]
    m = OrcCsr()
    lib.ref_load_mtx(path.encode(), ctypes.byref(m))
    try:
        rp, cols, vals = _from_orc(m)
        return m.num_row, m.num_col, rp, cols, vals
    finally:
        lib.ref_free_csr(ctypes.byref(m))


def ref_info(algo: str = "hybacc", small: bool = False) -> dict:
    lib = _load_ref(algo, small)
    return {"threads": lib.ref_thread_num(), "morsel": lib.ref_morsel_size(), "acc_thres": lib.ref_acc_thres()}


def oracle_lib():
    return _load_oracle()


# ------------------------------------------------------------------ digests
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays (mod 2^64)."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def csr_digest(rp, cols, vals):
    """The product digest of the casgemm ABI (cas_csr_digest), restated in numpy.

    Entry k of row r with column c and value v hashes to
    mix64(c * 0x9E3779B97F4A7C15 + k) ^ mix64(bits(v) + 0x632BE59BD9B4E019);
    a row's digest is the sum of its entries' hashes, and the product's is the
    sum over rows of mix64(row digest + r), all mod 2^64.  Returns
    (digest, row digests)."""
    rp = np.asarray(rp, np.int64)
    m = len(rp) - 1
    cols = np.asarray(cols).astype(np.int64).view(np.uint64)
    v = np.asarray(vals)
    bits = v.view(np.uint64) if v.dtype == np.float64 else v.astype(np.int64).view(np.uint64)
    row = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    k = (np.arange(len(cols), dtype=np.int64) - rp[:-1][row]).view(np.uint64)
    with np.errstate(over="ignore"):
        h = _mix64(cols * np.uint64(0x9E3779B97F4A7C15) + k) ^ _mix64(bits + np.uint64(0x632BE59BD9B4E019))
        rows = np.zeros(m, np.uint64)
        np.add.at(rows, row, h)
        d = _mix64(rows + np.arange(m, dtype=np.uint64))
        total = np.uint64(0)
        for chunk in np.array_split(d, max(1, len(d) // 65536)):
            total = total + np.add.reduce(chunk, dtype=np.uint64)
    return int(total), rows
