"""The C ABI library loads and exports every function include/partc.h declares; argument
validation happens on the host and needs no GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from partc_b200 import _lib, gen
from partc_b200 import build as b

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    if not os.path.exists(_lib.LIB_PATH):
        b.build()
    return _lib


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(ptc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_exports_every_declared_symbol(L):
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 7
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(names)


def test_options_defaults(L):
    o = L.options()
    assert o.struct_size == C.sizeof(_lib.Options)
    assert o.device == -1 and o.path == _lib.PATH_TWO_PHASE and o.output_location == _lib.PTC_HOST


def test_status_strings(L):
    lib = L.lib()
    for code, name in _lib.STATUS.items():
        assert lib.ptc_status_string(code).decode() == name


@pytest.mark.parametrize("bad", ["c0", "repeat", "range", "nullout", "panel"])
def test_invalid_arguments_rejected_on_host(L, bad):
    t = gen.random_coo([10, 10, 10], 100, [None] * 3, 1, "uniform01")
    c, modes, kw = 2, [0, 1, 2], {}
    if bad == "c0":
        c = 0
    elif bad == "repeat":
        modes = [0, 0, 2]
    elif bad == "range":
        modes = [0, 1, 3]
    elif bad == "panel":
        kw = {"panel_width": 300}
    if bad == "nullout":
        keep = []
        ca = _lib._host_coo(t, keep)
        m = np.array(modes, np.uint32)
        o = L.options()
        rc = L.lib().ptc_contract(C.byref(ca), None, c, m.ctypes.data, m.ctypes.data, C.byref(o), None, None)
        assert rc == 1
        return
    with pytest.raises(_lib.PtcError) as e:
        L.contract(t, None, c, modes, **kw)
    assert e.value.name == "PTC_ERR_INVALID_ARGUMENT"


def test_self_contraction_of_one_nonzero_is_an_error(L):
    t = gen.random_coo([10, 10, 10], 1, [None] * 3, 1, "uniform01")
    with pytest.raises(_lib.PtcError) as e:
        L.contract(t, None, 2, [0, 1, 2])
    assert e.value.name == "PTC_ERR_TOO_FEW_NONZEROS"
