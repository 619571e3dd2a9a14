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


def test_binding_layouts_match_the_header(L, tmp_path):
    """Every struct the ctypes binding mirrors has the header's size and field offsets (compiled
    with the host C compiler against include/partc.h)."""
    import subprocess
    structs = {"ptc_coo": _lib.Coo, "ptc_tensor": _lib.Tensor, "ptc_options": _lib.Options,
               "ptc_stats": _lib.Stats, "ptc_batch_item": _lib.BatchItem, "ptc_tune_report": _lib.TuneReport,
               "ptc_train_options": _lib.TrainOptions, "ptc_train_stats": _lib.TrainStats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "partc.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
