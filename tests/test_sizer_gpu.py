"""The learned sizer's CUDA kernels against the CPU reference network (oracle/sizer_ref.py)."""
import numpy as np
import pytest

from oracle import sizer_ref
from partc_b200 import _lib, gen

pytestmark = pytest.mark.gpu


def device_params(s):
    """The parameters as the device uses them: weights rounded to BF16, biases FP32."""
    prm = sizer_ref.unflatten(s.params())
    return {k: (sizer_ref.bf16_round(v) if k.startswith("W") or k == "w3" else v.astype(np.float32))
            for k, v in prm.items()}


def test_forward_matches_reference(engine):
    rng = np.random.default_rng(1)
    s = _lib.Sizer.create(seed=11)
    x = rng.random((3000, 16)).astype(np.float32)
    y = s.predict(x)
    yr, _ = sizer_ref.forward(device_params(s), x)
    np.testing.assert_allclose(y, yr, rtol=1e-4, atol=1e-4)


def test_gradients_match_reference(engine):
    """Gradients of the mean squared error from the hand-written backward kernels equal the CPU
    reference's (FP32 accumulation in a different order: relative 1e-3 of the largest entry)."""
    rng = np.random.default_rng(2)
    s = _lib.Sizer.create(seed=12)
    x = rng.random((5000, 16)).astype(np.float32)
    t = (rng.random(5000) * 10).astype(np.float32)
    loss, g = s.gradients(x, t)
    lr, gr = sizer_ref.loss_and_grads(device_params(s), x, t)
    assert abs(loss - lr) <= 1e-4 * max(1.0, abs(lr))
    scale = np.abs(gr).max()
    assert np.abs(g - gr).max() <= 1e-3 * scale, np.abs(g - gr).max() / scale
    # per block of parameters too
    o = 0
    for name, shape in sizer_ref.SHAPES:
        n = int(np.prod(shape))
        a, b = g[o:o + n], gr[o:o + n]
        assert np.abs(a - b).max() <= 1e-3 * max(np.abs(b).max(), 1e-6) + 1e-7, name
        o += n


def test_collect_targets_are_exact_counts(engine, oracle_mod):
    t = gen.random_coo([120, 140, 900, 17], 150_000, [1.1] * 4, 41, "uniform01")
    x, y = _lib.sizer_collect(t, None, 2, [0, 1, 2, 3])
    assert x.shape[1] == 16 and x.shape[0] == y.shape[0] > 0
    assert np.isfinite(x).all()
    o = oracle_mod.contract(t, None, 2, [0, 1, 2, 3], mode=oracle_mod.COUNTS)
    # the collected rows are the large rows -- more than 128 products, and at least 64 products
    # per A nonzero (fewer go to the sort-based accumulator) -- and their exact counts match
    F = o["row_flops"].astype(np.int64)
    big = (F > 128) & (F >= 64 * o["row_len"].astype(np.int64))
    expect = np.sort(np.log2(1.0 + o["row_nnz"][big].astype(np.float64)).astype(np.float32))
    got = np.sort(y)
    assert got.shape == expect.shape
    np.testing.assert_allclose(got, expect, rtol=1e-6)


def test_training_reduces_loss(engine):
    xs, ts = [], []
    for seed in range(3):
        w = gen.sizer_member(seed, nnz_scale=0.05)
        x, y = _lib.sizer_collect(w.tensor, None, w.c, w.modes)
        xs.append(x)
        ts.append(y)
    x = np.concatenate(xs)
    y = np.concatenate(ts)
    assert len(y) > 100
    s = _lib.Sizer.create(seed=5)
    r = s.train(x, y, epochs=30, batch=1024, lr=3e-3)
    assert r["final_epoch_loss"] < 0.25 * r["first_epoch_loss"], r
    pred = s.predict(x)
    assert np.mean(np.abs(pred - y)) < 1.0
