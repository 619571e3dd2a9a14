""".tns input and output.  The GPU reader must give exactly what the reference's own reader
(readTensor with pigo, compiled from its sources into oracle/_ref) gives: labels, mode sizes and
values bit for bit, including pigo's own decimal arithmetic on long fractions and exponents
(it differs from correctly rounded parsing on about 7% of these values).  Lines end in '\n' only:
pigo counts a '\r' as one more label."""
import os

import numpy as np
import pytest

from partc_b200 import _lib, gen

VALUE_TEXTS = ["0.5", "1", "-2.25", "3.14159265358979323846", "1e-3", "2.5E+2", "-7.0e1", "0.1", "123456789.987654321",
               "1.0000000000000002", "4.9e-300", "6.02214076e23", "+0.75", "0.000012345", "9.999999999999999e-1",
               ".5", "42.", "0.30000000000000004",
               # exponents pigo raises 10 to with std::pow although they are not integers, or that
               # carry an exponent of their own (its read_fp reads the exponent recursively)
               "2e0.5", "-3.5e-1.25", "1e1e1", "7E+0.125", "1.5e2.5e-1"]


def _write_tricky(path, rng, n=4000):
    dims = [7, 11, 13]
    lines = ["# a comment line", "% another comment", ""]
    for i in range(n):
        lab = [int(rng.integers(1, d + 1)) for d in dims]
        if i % 3 == 0:
            v = VALUE_TEXTS[i % len(VALUE_TEXTS)]
        else:
            v = repr(float(rng.normal() * 10.0 ** int(rng.integers(-5, 6))))
        sep = "\t" if i % 7 == 0 else " "
        lines.append(sep.join(str(x) for x in lab) + sep + v)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def test_reference_reader_available(oracle_mod):
    assert oracle_mod.ref_io_available()


@pytest.mark.gpu
def test_gpu_reader_matches_the_reference_reader(engine, oracle_mod, tmp_path):
    path = str(tmp_path / "t.tns")
    _write_tricky(path, np.random.default_rng(5))
    ref = oracle_mod.ref_read_tns(path)
    got = engine.read_tns(path)
    assert np.array_equal(got.idx, ref["idx"])
    assert np.array_equal(got.vals.view(np.uint64), ref["vals"].view(np.uint64))
    assert np.array_equal(got.dims, ref["dims"])


@pytest.mark.gpu
def test_write_then_read_round_trip(engine, oracle_mod, tmp_path):
    """Written with 17 significant digits, read back: the labels exactly; the values as the
    reference's reader reads them (its decimal arithmetic is not correctly rounded, so they can
    differ from the originals in the last bits)."""
    t = gen.random_coo([50, 40, 30, 9], 20000, [1.1] * 4, 3, "normal")
    path = str(tmp_path / "rt.tns")
    engine.write_tns(path, t)
    back = engine.read_tns(path)
    ref = oracle_mod.ref_read_tns(path)
    assert np.array_equal(back.idx, t.idx)
    assert np.array_equal(back.vals.view(np.uint64), ref["vals"].view(np.uint64))
    np.testing.assert_allclose(back.vals, t.vals, rtol=1e-15, atol=0)
    assert list(back.dims) == [int(t.idx[:, m].max()) + 1 for m in range(4)]


@pytest.mark.gpu
def test_reader_rejects_bad_lines(engine, tmp_path):
    path = str(tmp_path / "bad.tns")
    with open(path, "w") as f:
        f.write("1 2 3 0.5\n4 5 1.0\n")
    with pytest.raises(_lib.PtcError):
        engine.read_tns(path)
    with open(path, "w") as f:
        f.write("1 0 3 0.5\n")
    with pytest.raises(_lib.PtcError) as e:
        engine.read_tns(path)
    assert e.value.name == "PTC_ERR_INDEX_RANGE"
