"""ctypes binding of the engine's C ABI (``include/partc.h``).

The CUDA library ``libpartc_b200.so`` is the product; this module only loads it and converts
numpy arrays.  There is no CPU fallback: if the library is missing or no B200 is visible, calls
fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpartc_b200.so")

PTC_HOST, PTC_DEVICE = 0, 1
PATH_TWO_PHASE, PATH_LEARNED = 0, 1

STATUS = {
    0: "PTC_OK", 1: "PTC_ERR_INVALID_ARGUMENT", 2: "PTC_ERR_INDEX_RANGE", 3: "PTC_ERR_KEY_OVERFLOW",
    4: "PTC_ERR_EMPTY_CONTRACTION", 5: "PTC_ERR_TOO_FEW_NONZEROS", 6: "PTC_ERR_HASH_BUILD",
    7: "PTC_ERR_OUT_OF_MEMORY", 8: "PTC_ERR_CUDA", 9: "PTC_ERR_NO_DEVICE",
    11: "PTC_ERR_OVERFLOW", 12: "PTC_ERR_INTERNAL",
}

# every function include/partc.h declares (checked by the CPU tests)
EXPORTS = [
    "ptc_options_init", "ptc_last_error", "ptc_status_string", "ptc_contract", "ptc_self_contract",
    "ptc_tensor_free", "ptc_device_count", "ptc_train_options_init", "ptc_sizer_create", "ptc_sizer_load",
    "ptc_sizer_save", "ptc_sizer_free", "ptc_sizer_get_params", "ptc_sizer_set_params", "ptc_sizer_collect",
    "ptc_sizer_train", "ptc_sizer_predict", "ptc_sizer_gradients", "ptc_buffer_free",
    "ptc_sizer_predict_noalloc", "ptc_batch_contract", "ptc_autotune", "ptc_read_tns", "ptc_write_tns",
    "ptc_device_pool_in_use",
]
SIZER_FEATURES = 16
SIZER_PARAMS = 5313


class PtcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))


class Coo(C.Structure):
    _fields_ = [("order", C.c_uint32), ("location", C.c_uint32), ("nnz", C.c_uint64),
                ("idx", C.c_void_p), ("vals", C.c_void_p), ("dims", C.c_void_p)]


class Tensor(C.Structure):
    _fields_ = [("order", C.c_uint32), ("location", C.c_uint32), ("nnz", C.c_uint64),
                ("idx", C.POINTER(C.c_uint32)), ("vals", C.POINTER(C.c_double)), ("opaque", C.c_void_p)]


class Options(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("device", C.c_int32), ("stream", C.c_void_p),
                ("path", C.c_uint32), ("output_location", C.c_uint32), ("verbose", C.c_uint32),
                ("panel_width", C.c_uint32), ("hash_seed", C.c_uint64), ("sizer", C.c_void_p),
                ("sort_rows", C.c_uint32), ("small_max_products", C.c_uint32),
                ("sort_max_avg_products", C.c_uint32), ("hash_load_pct", C.c_uint32),
                ("batch_wave_mib", C.c_uint32), ("warp_task_max_len", C.c_uint32), ("cuckoo_max_chain", C.c_uint32),
                ("cuckoo_max_attempts", C.c_uint32), ("large_rows", C.c_uint32), ("bitmap_max_len", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


class Stats(C.Structure):
    _fields_ = [("mult_adds", C.c_uint64), ("out_nnz", C.c_uint64), ("nrows", C.c_uint64),
                ("ncols", C.c_uint64), ("nfibers", C.c_uint64), ("a_nnz", C.c_uint64), ("b_nnz", C.c_uint64),
                ("t_total_ms", C.c_double), ("t_h2d_ms", C.c_double), ("t_build_ms", C.c_double),
                ("t_symbolic_ms", C.c_double), ("t_numeric_ms", C.c_double), ("t_d2h_ms", C.c_double),
                ("hash_attempts", C.c_uint32), ("panel_width", C.c_uint32),
                ("rows_small", C.c_uint64), ("rows_hash", C.c_uint64), ("hash_parts", C.c_uint64),
                ("rows_long", C.c_uint64), ("rerun_rows", C.c_uint64), ("sizer_mean_abs_log2_err", C.c_double),
                ("kernel_launches", C.c_uint64), ("batch_waves", C.c_uint64), ("rerun_items", C.c_uint64),
                ("reserved", C.c_double * 2)]

    def as_dict(self) -> dict:
        return {name: (getattr(self, name) if not name == "reserved" else None)
                for name, _ in self._fields_ if name != "reserved"}


class BatchItem(C.Structure):
    _fields_ = [("A", Coo), ("B", Coo), ("c", C.c_uint32), ("a_modes", C.c_uint32 * 16),
                ("b_modes", C.c_uint32 * 16)]


SINK = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.POINTER(Tensor))


class TuneReport(C.Structure):
    _fields_ = [("trials", C.c_uint32), ("repeats", C.c_uint32), ("default_ms", C.c_double),
                ("best_ms", C.c_double), ("reserved", C.c_double * 4)]

TUNE_KNOBS = ("large_rows", "bitmap_max_len", "panel_width", "warp_task_max_len", "small_max_products", "sort_max_avg_products",
              "hash_load_pct")


class TrainOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float),
                ("seed", C.c_uint64), ("device", C.c_int32), ("reserved", C.c_uint32 * 5)]


class TrainStats(C.Structure):
    _fields_ = [("first_epoch_loss", C.c_float), ("final_epoch_loss", C.c_float), ("epochs", C.c_uint32),
                ("steps", C.c_uint64), ("ms", C.c_double)]


_lib = None


def lib():
    """Load the CUDA library (built by ``python -m partc_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m partc_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.ptc_options_init.argtypes = [C.POINTER(Options)]
        L.ptc_options_init.restype = None
        L.ptc_last_error.restype = C.c_char_p
        L.ptc_status_string.argtypes = [C.c_int]
        L.ptc_status_string.restype = C.c_char_p
        L.ptc_contract.argtypes = [C.POINTER(Coo), C.POINTER(Coo), C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.POINTER(Options), C.POINTER(Tensor), C.POINTER(Stats)]
        L.ptc_contract.restype = C.c_int
        L.ptc_self_contract.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32,
                                        C.c_void_p, C.POINTER(Options), C.POINTER(Tensor), C.POINTER(Stats)]
        L.ptc_self_contract.restype = C.c_int
        L.ptc_tensor_free.argtypes = [C.POINTER(Tensor)]
        L.ptc_tensor_free.restype = None
        L.ptc_device_count.restype = C.c_int
        L.ptc_device_pool_in_use.argtypes = [C.c_int32, C.POINTER(C.c_uint64)]
        L.ptc_device_pool_in_use.restype = C.c_int
        L.ptc_batch_contract.argtypes = [C.POINTER(BatchItem), C.c_uint32, C.POINTER(Options), C.POINTER(Tensor),
                                         SINK, C.c_void_p, C.POINTER(Stats)]
        L.ptc_batch_contract.restype = C.c_int
        L.ptc_autotune.argtypes = [C.POINTER(BatchItem), C.c_uint32, C.POINTER(Options), C.c_uint32,
                                   C.POINTER(Options), C.POINTER(TuneReport)]
        L.ptc_autotune.restype = C.c_int
        L.ptc_read_tns.argtypes = [C.c_char_p, C.POINTER(Options), C.POINTER(Tensor), C.c_void_p]
        L.ptc_read_tns.restype = C.c_int
        L.ptc_write_tns.argtypes = [C.c_char_p, C.POINTER(Tensor)]
        L.ptc_write_tns.restype = C.c_int
        P, F = C.POINTER, C.c_float
        L.ptc_train_options_init.argtypes = [P(TrainOptions)]
        L.ptc_train_options_init.restype = None
        L.ptc_sizer_create.argtypes = [C.c_uint64, P(C.c_void_p)]
        L.ptc_sizer_load.argtypes = [C.c_char_p, P(C.c_void_p)]
        L.ptc_sizer_save.argtypes = [C.c_void_p, C.c_char_p]
        L.ptc_sizer_free.argtypes = [C.c_void_p]
        L.ptc_sizer_free.restype = None
        L.ptc_sizer_get_params.argtypes = [C.c_void_p, C.c_void_p]
        L.ptc_sizer_set_params.argtypes = [C.c_void_p, C.c_void_p]
        L.ptc_sizer_collect.argtypes = [P(Coo), P(Coo), C.c_uint32, C.c_void_p, C.c_void_p, P(Options),
                                        P(P(F)), P(P(F)), P(C.c_uint64)]
        L.ptc_sizer_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, P(TrainOptions),
                                      P(TrainStats)]
        L.ptc_sizer_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p]
        L.ptc_sizer_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p,
                                          P(F)]
        L.ptc_sizer_predict_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p]
        L.ptc_buffer_free.argtypes = [C.c_void_p]
        L.ptc_buffer_free.restype = None
        for name in ("ptc_sizer_create", "ptc_sizer_load", "ptc_sizer_save", "ptc_sizer_get_params",
                     "ptc_sizer_set_params", "ptc_sizer_collect", "ptc_sizer_train", "ptc_sizer_predict",
                     "ptc_sizer_gradients", "ptc_sizer_predict_noalloc"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def options(**kw) -> Options:
    o = Options()
    lib().ptc_options_init(C.byref(o))
    for k, v in kw.items():
        if k == "path" and isinstance(v, str):
            v = {"two_phase": PATH_TWO_PHASE, "learned": PATH_LEARNED}[v]
        if k == "output_location" and isinstance(v, str):
            v = {"host": PTC_HOST, "device": PTC_DEVICE}[v]
        if k == "large_rows" and isinstance(v, str):
            v = {"auto": 0, "bitmap": 1, "panels": 2}[v]
        setattr(o, k, v)
    return o


def _check(rc: int):
    if rc != 0:
        raise PtcError(rc, lib().ptc_last_error().decode())


def _host_coo(t, keep: list) -> Coo:
    idx = np.ascontiguousarray(t.idx, dtype=np.uint32)
    vals = np.ascontiguousarray(t.vals, dtype=np.float64)
    dims = np.ascontiguousarray(t.dims, dtype=np.uint32)
    keep += [idx, vals, dims]
    order = idx.shape[1] if idx.ndim == 2 else len(dims)
    return Coo(order, PTC_HOST, idx.shape[0] if idx.ndim == 2 else 0, idx.ctypes.data, vals.ctypes.data,
               dims.ctypes.data)


def device_coo(idx_ptr: int, vals_ptr: int, nnz: int, dims, keep: list) -> Coo:
    """Describe a tensor whose idx/vals already live in device memory (e.g. torch CUDA tensors)."""
    d = np.ascontiguousarray(dims, dtype=np.uint32)
    keep.append(d)
    return Coo(len(d), PTC_DEVICE, nnz, idx_ptr, vals_ptr, d.ctypes.data)


def contract(A, B=None, c: int = 1, a_modes=None, b_modes=None, *, keep_device: bool = False, **opt):
    """O = A x B through ``ptc_contract`` with host inputs.  Returns ``(idx, vals, stats)``:
    ``idx`` is ``uint32[nnz, order]``.  With ``keep_device=True`` the output stays on the device
    and a raw ``Tensor`` struct is returned instead of arrays (free it with :func:`free`)."""
    L = lib()
    keep: list = []
    ca = _host_coo(A, keep)
    cb = None if B is None else _host_coo(B, keep)
    am = np.ascontiguousarray(a_modes, dtype=np.uint32)
    bm = am if b_modes is None else np.ascontiguousarray(b_modes, dtype=np.uint32)
    if keep_device:
        opt.setdefault("output_location", PTC_DEVICE)
    o = options(**opt)
    out = Tensor()
    st = Stats()
    rc = L.ptc_contract(C.byref(ca), None if cb is None else C.byref(cb), c, am.ctypes.data, bm.ctypes.data,
                        C.byref(o), C.byref(out), C.byref(st))
    _check(rc)
    if o.output_location == PTC_DEVICE:
        return out, None, st.as_dict()
    idx, vals = _host_arrays(out)
    return idx, vals, st.as_dict()


class _Owner:
    """Releases a host ptc_tensor when the last numpy view of it is gone."""

    def __init__(self, t: Tensor):
        self.t = t

    def __del__(self):
        if _lib is not None:
            _lib.ptc_tensor_free(C.byref(self.t))


def _host_arrays(out: Tensor):
    """Zero-copy numpy views of a host output tensor (the views own it)."""
    n, d = out.nnz, out.order
    if n == 0:
        lib().ptc_tensor_free(C.byref(out))
        return np.zeros((0, d), np.uint32), np.zeros(0, np.float64)
    owner = _Owner(out)
    ib = (C.c_uint32 * (n * d)).from_address(C.addressof(out.idx.contents))
    vb = (C.c_double * n).from_address(C.addressof(out.vals.contents))
    ib._owner = owner
    vb._owner = owner
    idx = np.frombuffer(ib, dtype=np.uint32).reshape(n, d)
    vals = np.frombuffer(vb, dtype=np.float64)
    return idx, vals


def contract_coo(ca: Coo, cb: Optional[Coo], c: int, a_modes, b_modes=None, **opt):
    """Lower-level call on prepared ``Coo`` descriptors (host or device).  Returns the raw output
    ``Tensor`` (free with :func:`free`) and the stats dict."""
    L = lib()
    am = np.ascontiguousarray(a_modes, dtype=np.uint32)
    bm = am if b_modes is None else np.ascontiguousarray(b_modes, dtype=np.uint32)
    o = options(**opt)
    out = Tensor()
    st = Stats()
    rc = L.ptc_contract(C.byref(ca), None if cb is None else C.byref(cb), c, am.ctypes.data, bm.ctypes.data,
                        C.byref(o), C.byref(out), C.byref(st))
    _check(rc)
    return out, st.as_dict()


def free(t: Tensor) -> None:
    lib().ptc_tensor_free(C.byref(t))


def batch_items(work, keep: list, B_list=None):
    """``BatchItem`` array for workloads with ``.tensor``, ``.c``, ``.modes`` (self-contractions),
    or, where ``B_list[i]`` is given, ``(B tensor, b_modes)`` as item i's second operand."""
    arr = (BatchItem * len(work))()
    for i, w in enumerate(work):
        it = arr[i]
        it.A = _host_coo(w.tensor, keep)
        it.c = w.c
        for j, m in enumerate(w.modes):
            it.a_modes[j] = m
        if B_list is not None and B_list[i] is not None:
            bt, bm = B_list[i]
            it.B = _host_coo(bt, keep)
            for j, m in enumerate(bm):
                it.b_modes[j] = m
    return arr


def read_tns(path: str, **opt):
    """``ptc_read_tns`` (GPU parser): returns a ``gen.CooTensor`` with host numpy arrays."""
    from partc_b200.gen import CooTensor
    o = options(**opt)
    out = Tensor()
    dims = np.zeros(16, dtype=np.uint32)
    _check(lib().ptc_read_tns(path.encode(), C.byref(o), C.byref(out), dims.ctypes.data))
    d = out.order
    idx, vals = _host_arrays(out)
    return CooTensor(idx=idx.reshape(-1, d), vals=vals, dims=dims[:d].copy())


def write_tns(path: str, t) -> None:
    """``ptc_write_tns`` of a host tensor (``idx`` [nnz, d] uint32, ``vals``)."""
    idx = np.ascontiguousarray(t.idx, dtype=np.uint32)
    vals = np.ascontiguousarray(t.vals, dtype=np.float64)
    tt = Tensor(idx.shape[1], PTC_HOST, idx.shape[0], idx.ctypes.data_as(C.POINTER(C.c_uint32)),
                vals.ctypes.data_as(C.POINTER(C.c_double)), None)
    _check(lib().ptc_write_tns(path.encode(), C.byref(tt)))


def autotune(items, repeats: int = 3, **opt):
    """``ptc_autotune``: returns ``(knobs dict, report dict)``; pass the knobs to contract /
    batch_contract as keyword options."""
    o = options(**opt)
    best = Options()
    rep = TuneReport()
    _check(lib().ptc_autotune(items, len(items), C.byref(o), repeats, C.byref(best), C.byref(rep)))
    knobs = {k: int(getattr(best, k)) for k in TUNE_KNOBS}
    return knobs, {"trials": rep.trials, "repeats": rep.repeats, "default_ms": rep.default_ms,
                   "best_ms": rep.best_ms}


def batch_contract(items, *, outputs: str = "arrays", sink=None, **opt):
    """Run ``ptc_batch_contract`` on a ``BatchItem`` array.

    outputs="arrays": returns ``(list of (idx, vals), stats)`` with host numpy arrays;
    outputs="device": returns ``(list of Tensor, stats)`` kept on the device (free each);
    outputs="sink":   calls ``sink(i, tensor)`` for every item (views valid during the call);
    outputs="none":   discards the outputs (timing).
    """
    L = lib()
    n = len(items)
    if outputs == "device":
        opt.setdefault("output_location", PTC_DEVICE)
    o = options(**opt)
    st = Stats()
    outs = (Tensor * n)() if outputs in ("arrays", "device") else None
    cb = SINK(0)
    if outputs == "sink":
        def _cb(user, i, t):
            sink(int(i), t.contents)
        cb = SINK(_cb)
    rc = L.ptc_batch_contract(items, n, C.byref(o), outs, cb, None, C.byref(st))
    _check(rc)
    if outputs == "arrays":
        return [_host_arrays(Tensor.from_buffer_copy(outs[i])) for i in range(n)], st.as_dict()
    if outputs == "device":
        return [outs[i] for i in range(n)], st.as_dict()
    return None, st.as_dict()


def device_pool_in_use(device: int = -1) -> int:
    """Bytes of the device's stream-ordered pool still allocated (ptc_device_pool_in_use)."""
    v = C.c_uint64()
    _check(lib().ptc_device_pool_in_use(device, C.byref(v)))
    return int(v.value)


def device_count() -> int:
    return int(lib().ptc_device_count())


# ---- learned sizer -------------------------------------------------------------------------

class Sizer:
    """Owning handle of a ptc_sizer (the learned output-size predictor)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def create(cls, seed: int = 0) -> "Sizer":
        h = C.c_void_p()
        _check(lib().ptc_sizer_create(seed, C.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path: str) -> "Sizer":
        h = C.c_void_p()
        _check(lib().ptc_sizer_load(path.encode(), C.byref(h)))
        return cls(h)

    def save(self, path: str) -> None:
        _check(lib().ptc_sizer_save(self.h, path.encode()))

    def params(self) -> np.ndarray:
        out = np.empty(SIZER_PARAMS, dtype=np.float32)
        _check(lib().ptc_sizer_get_params(self.h, out.ctypes.data))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib().ptc_sizer_set_params(self.h, p.ctypes.data))

    def train(self, x: np.ndarray, t: np.ndarray, epochs=20, batch=8192, lr=2e-3, seed=7, device=-1) -> dict:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        o = TrainOptions()
        lib().ptc_train_options_init(C.byref(o))
        o.epochs, o.batch, o.lr, o.seed, o.device = epochs, batch, lr, seed, device
        st = TrainStats()
        _check(lib().ptc_sizer_train(self.h, x.ctypes.data, t.ctypes.data, len(t), C.byref(o), C.byref(st)))
        return {"first_epoch_loss": st.first_epoch_loss, "final_epoch_loss": st.final_epoch_loss,
                "epochs": st.epochs, "steps": st.steps, "ms": st.ms}

    def predict(self, x: np.ndarray, device=-1) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty(x.shape[0], dtype=np.float32)
        _check(lib().ptc_sizer_predict(self.h, x.ctypes.data, x.shape[0], device, out.ctypes.data))
        return out

    def predict_noalloc(self, x: np.ndarray, device=-1) -> np.ndarray:
        """Same as predict, through the entry point that allocates no device memory."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty(x.shape[0], dtype=np.float32)
        _check(lib().ptc_sizer_predict_noalloc(self.h, x.ctypes.data, x.shape[0], device, out.ctypes.data))
        return out

    def gradients(self, x: np.ndarray, t: np.ndarray, device=-1):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(SIZER_PARAMS, dtype=np.float32)
        loss = C.c_float()
        _check(lib().ptc_sizer_gradients(self.h, x.ctypes.data, t.ctypes.data, len(t), device, g.ctypes.data,
                                         C.byref(loss)))
        return float(loss.value), g

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ptc_sizer_free(self.h)
            self.h = None


def sizer_collect(A, B, c, a_modes, b_modes=None, **opt):
    """Features and log2(1 + exact output nnz) of the rows the learned path sizes."""
    L = lib()
    keep: list = []
    ca = _host_coo(A, keep)
    cb = None if B is None else _host_coo(B, keep)
    am = np.ascontiguousarray(a_modes, dtype=np.uint32)
    bm = am if b_modes is None else np.ascontiguousarray(b_modes, dtype=np.uint32)
    o = options(**opt)
    fx = C.POINTER(C.c_float)()
    ft = C.POINTER(C.c_float)()
    n = C.c_uint64()
    _check(L.ptc_sizer_collect(C.byref(ca), None if cb is None else C.byref(cb), c, am.ctypes.data, bm.ctypes.data,
                               C.byref(o), C.byref(fx), C.byref(ft), C.byref(n)))
    try:
        nn = n.value
        x = np.ctypeslib.as_array(fx, shape=(max(nn, 1) * SIZER_FEATURES,))[: nn * SIZER_FEATURES].reshape(
            nn, SIZER_FEATURES).copy()
        t = np.ctypeslib.as_array(ft, shape=(max(nn, 1),))[:nn].copy()
    finally:
        L.ptc_buffer_free(C.cast(fx, C.c_void_p))
        L.ptc_buffer_free(C.cast(ft, C.c_void_p))
    return x, t
