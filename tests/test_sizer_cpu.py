"""Host-side parts of the learned sizer: parameter layout, save/load, the CPU reference network."""
import numpy as np

from partc_b200 import _lib
from oracle import sizer_ref


def test_param_layout_matches_reference():
    assert sizer_ref.NPARAM == _lib.SIZER_PARAMS


def test_create_save_load_roundtrip(tmp_path):
    s = _lib.Sizer.create(seed=3)
    p = s.params()
    assert p.shape == (_lib.SIZER_PARAMS,) and np.isfinite(p).all()
    # He-normal first layer, zero-ish biases
    w = sizer_ref.unflatten(p)
    assert 0.2 < w["W1"].std() < 0.5
    path = str(tmp_path / "s.bin")
    s.save(path)
    r = _lib.Sizer.load(path)
    assert np.array_equal(r.params(), p)
    q = p.copy()
    q[5] = 1.25
    r.set_params(q)
    assert r.params()[5] == np.float32(1.25)


def test_load_rejects_other_files(tmp_path):
    path = str(tmp_path / "bad.bin")
    open(path, "wb").write(b"not a sizer")
    try:
        _lib.Sizer.load(path)
        raise AssertionError("expected an error")
    except _lib.PtcError as e:
        assert e.name == "PTC_ERR_INVALID_ARGUMENT"


def test_bf16_rounding_reference():
    x = np.array([1.0, 1.00390625, 1.0078125, -3.14159, 1e-3], dtype=np.float32)
    r = sizer_ref.bf16_round(x)
    # representable values stay, others move by less than half a BF16 ulp
    assert r[0] == 1.0 and r[2] == 1.0078125
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)


def test_reference_gradient_is_consistent():
    """Finite differences of the reference loss agree with its analytic gradient (FP64 check of
    the oracle itself, with unrounded weights)."""
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(sizer_ref.NPARAM) * 0.1).astype(np.float64)
    x = rng.random((64, 16))
    t = rng.random(64) * 4

    def loss(flat):
        prm = {k: v.astype(np.float64) for k, v in sizer_ref.unflatten(flat).items()}
        y, _ = sizer_ref.forward({k: v.astype(np.float32) for k, v in prm.items()}, x)
        return float(np.mean((y.astype(np.float64) - t) ** 2))

    _, g = sizer_ref.loss_and_grads({k: v.astype(np.float32) for k, v in sizer_ref.unflatten(p).items()}, x, t)
    for i in [0, 17, 1024, 1100, 5200, 5312]:
        e = np.zeros_like(p)
        e[i] = 1e-3
        fd = (loss(p + e) - loss(p - e)) / 2e-3
        assert abs(fd - g[i]) <= 5e-3 * max(1.0, abs(g[i])), (i, fd, g[i])
