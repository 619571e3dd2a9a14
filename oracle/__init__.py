"""ctypes access to the checkers -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package.  The product (``partc_b200``) never imports it.

* :func:`contract` runs the C restatement of the reference's contraction (``oracle.c``).
* :func:`ref_self_contract` runs the reference's own ``fksCuckooTC`` path, compiled from its
  sources into ``oracle/_ref`` (present only where the reference was available at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_tc.so")
REF_BIN = os.path.join(HERE, "_ref", "ref_tc")

FLOPS_ONLY, COUNTS, VALUES = 0, 1, 2


def reference_dir(ref: Optional[str] = None) -> str:
    """Where the reference's sources are: the argument, else the environment variable
    ``PARTC_REFERENCE``, else a checkout named ``reference`` beside this repository."""
    if ref:
        return ref
    return os.environ.get("PARTC_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def build(ref: Optional[str] = None) -> None:
    """Compile the restatement and, where the reference sources exist, ``oracle/_ref``."""
    subprocess.run(["make", "-s", "-C", HERE, f"REF={reference_dir(ref)}"], check=True)


class _Coo(C.Structure):
    _fields_ = [("order", C.c_uint32), ("nnz", C.c_uint64), ("idx", C.c_void_p),
                ("vals", C.c_void_p), ("dims", C.c_void_p)]


class _Result(C.Structure):
    _fields_ = [("out_order", C.c_uint32), ("out_nnz", C.c_uint64), ("out_idx", C.POINTER(C.c_uint32)),
                ("out_val", C.POINTER(C.c_double)), ("flops", C.c_uint64), ("nrows", C.c_uint64),
                ("nfibers", C.c_uint64), ("row_key", C.POINTER(C.c_uint64)),
                ("row_flops", C.POINTER(C.c_uint64)), ("row_nnz", C.POINTER(C.c_uint64)),
                ("row_len", C.POINTER(C.c_uint32)), ("err", C.c_char * 128)]


class _RefResult(C.Structure):
    _fields_ = [("out_order", C.c_uint32), ("out_nnz", C.c_uint64), ("out_idx", C.POINTER(C.c_uint32)),
                ("out_val", C.POINTER(C.c_double)), ("t_insert_b", C.c_double), ("t_insert_a", C.c_double),
                ("t_preprocess", C.c_double), ("t_contract", C.c_double), ("t_wall", C.c_double)]


_lib = None
_ref = None


def _oracle():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = C.CDLL(ORACLE_SO)
        _lib.oracle_contract.restype = C.c_int
        _lib.oracle_contract.argtypes = [C.POINTER(_Coo), C.POINTER(_Coo), C.c_uint32, C.c_void_p, C.c_void_p,
                                         C.c_int, C.POINTER(_Result)]
        _lib.oracle_free.argtypes = [C.POINTER(_Result)]
    return _lib


def _coo(t, keep):
    idx = np.ascontiguousarray(t.idx, dtype=np.uint32)
    vals = np.ascontiguousarray(t.vals, dtype=np.float64)
    dims = np.ascontiguousarray(t.dims, dtype=np.uint32)
    keep.extend([idx, vals, dims])
    return _Coo(idx.shape[1], idx.shape[0], idx.ctypes.data, vals.ctypes.data, dims.ctypes.data)


def _arr(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def contract(A, B, c: int, a_modes, b_modes=None, mode: int = VALUES) -> dict:
    """O = A x B (B defaults to A: the reference's self-contraction).  Returns a dict with the
    output ``idx`` ([nnz, order] uint32) and ``vals`` plus per-row statistics."""
    lib = _oracle()
    B = A if B is None else B
    b_modes = a_modes if b_modes is None else b_modes
    keep: list = []
    ca, cb = _coo(A, keep), _coo(B, keep)
    am = np.ascontiguousarray(a_modes, dtype=np.uint32)
    bm = np.ascontiguousarray(b_modes, dtype=np.uint32)
    r = _Result()
    rc = lib.oracle_contract(C.byref(ca), C.byref(cb), c, am.ctypes.data, bm.ctypes.data, mode, C.byref(r))
    if rc != 0:
        msg = r.err.decode()
        lib.oracle_free(C.byref(r))
        raise ValueError(f"oracle: {msg}")
    out = {
        "order": r.out_order, "nnz": r.out_nnz, "flops": r.flops, "nrows": r.nrows, "nfibers": r.nfibers,
        "row_key": _arr(r.row_key, r.nrows, np.uint64), "row_flops": _arr(r.row_flops, r.nrows, np.uint64),
        "row_nnz": _arr(r.row_nnz, r.nrows, np.uint64), "row_len": _arr(r.row_len, r.nrows, np.uint32),
    }
    if mode == VALUES:
        out["idx"] = _arr(r.out_idx, r.out_nnz * r.out_order, np.uint32).reshape(-1, r.out_order)
        out["vals"] = _arr(r.out_val, r.out_nnz, np.float64)
    lib.oracle_free(C.byref(r))
    return out


REF_IO_SO = os.path.join(HERE, "_ref", "libref_io.so")
_refio = None


def ref_read_tns(path: str) -> dict:
    """The reference's own .tns reader (readTensor with pigo), compiled from its sources:
    0-based labels [N, d], values, and mode sizes."""
    global _refio
    if _refio is None:
        _refio = C.CDLL(REF_IO_SO)
        _refio.ref_read_tns.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.POINTER(C.c_uint32)),
                                        C.POINTER(C.POINTER(C.c_double))]
        _refio.ref_io_free.argtypes = [C.c_void_p]
    d, n = C.c_uint32(), C.c_uint32()
    ip, dp = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    vp = C.POINTER(C.c_double)()
    _refio.ref_read_tns(path.encode(), C.byref(d), C.byref(n), C.byref(ip), C.byref(dp), C.byref(vp))
    out = {"idx": _arr(ip, n.value * d.value, np.uint32).reshape(-1, d.value),
           "vals": _arr(vp, n.value, np.float64), "dims": _arr(dp, d.value, np.uint32)}
    for p in (ip, dp, vp):
        _refio.ref_io_free(C.cast(p, C.c_void_p))
    return out


def ref_io_available() -> bool:
    return os.path.exists(REF_IO_SO)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _refl():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_SO)
        _ref.ref_self_contract.restype = C.c_int
        _ref.ref_self_contract.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_void_p, C.c_int, C.POINTER(_RefResult)]
        _ref.ref_free.argtypes = [C.POINTER(_RefResult)]
    return _ref


def ref_self_contract(t, c: int, modes, keep_mask: Optional[np.ndarray] = None) -> dict:
    """Run the reference's own path (main.cpp:59-118) in-process.  The reference exits the
    process on an empty contraction or on a tensor with at most one nonzero; do not call it so."""
    lib = _refl()
    idx = np.ascontiguousarray(t.idx, dtype=np.uint32)
    vals = np.ascontiguousarray(t.vals, dtype=np.float64)
    dims = np.ascontiguousarray(t.dims, dtype=np.uint32)
    md = np.ascontiguousarray(modes, dtype=np.uint32)
    km = None if keep_mask is None else np.ascontiguousarray(keep_mask, dtype=np.uint8)
    r = _RefResult()
    lib.ref_self_contract(idx.ctypes.data, vals.ctypes.data, idx.shape[1], idx.shape[0], dims.ctypes.data, c,
                          md.ctypes.data, None if km is None else km.ctypes.data, 1, C.byref(r))
    out = {
        "order": r.out_order, "nnz": r.out_nnz,
        "idx": _arr(r.out_idx, r.out_nnz * r.out_order, np.uint32).reshape(-1, r.out_order),
        "vals": _arr(r.out_val, r.out_nnz, np.float64),
        "t_insert_b": r.t_insert_b, "t_insert_a": r.t_insert_a, "t_preprocess": r.t_preprocess,
        "t_contract": r.t_contract, "t_wall": r.t_wall,
    }
    lib.ref_free(C.byref(r))
    return out


def write_ref_input(path: str, t, c: int, modes) -> None:
    """Binary input for the ``ref_tc`` command-line program."""
    d, n = t.idx.shape[1], t.idx.shape[0]
    with open(path, "wb") as f:
        np.array([d, n, c], dtype=np.uint32).tofile(f)
        np.ascontiguousarray(t.dims, dtype=np.uint32).tofile(f)
        np.ascontiguousarray(modes, dtype=np.uint32).tofile(f)
        np.ascontiguousarray(t.idx, dtype=np.uint32).tofile(f)
        np.ascontiguousarray(t.vals, dtype=np.float64).tofile(f)


def canonical(idx: np.ndarray, vals: np.ndarray):
    """Sort an output tensor lexicographically by its index tuple (outputs are compared as sets)."""
    if idx.shape[0] == 0:
        return idx, vals
    order = np.lexsort(idx.T[::-1])
    return idx[order], vals[order]
