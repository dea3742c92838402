"""The proposal MLP's tensor-core kernels (tcgen05, BF16 x BF16 -> FP32 in tensor memory)
against the FP32 NumPy reference (tests/mlp_ref.py), through the C ABI:

* forward logits of 1000 rows (the last 128-row tile partial) and of 38400 rows (more
  tiles than resident CTAs: the persistent loop) within 2e-2 of the reference, and the
  proposal bits equal to logit > threshold;
* the gradient of the weighted logistic loss: every parameter block within 3e-2 of the
  block's largest reference value, the loss within 1e-3 relative. The tolerances cover
  BF16 rounding boundaries: the kernels and the reference round the same FP32 values, but
  their FP32 sums differ in the last bits, so an activation or gradient now and then
  rounds to the neighbouring BF16 value (2^-8 relative);
* Adam on the device learns a separable labelling (loss falls below a tenth of its start).
"""
import numpy as np
import pytest

import mlp_ref
import mwdg2_b200

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.uniform(-2.0, 2.0, size=(n, mwdg2_b200.MLP_FEATURES)).astype(np.float32)
    X[:, 108:112] = rng.integers(0, 2, size=(n, 4))
    X[:, 112] = 1.0
    labels = rng.integers(0, 16, size=n).astype(np.uint8)
    return X, labels


@pytest.mark.parametrize("n", [1000, 38400])
def test_forward_matches_reference(n):
    p = mwdg2_b200.mlp_init(3)
    p[8192:8256] = 0.05   # non-zero biases
    X, _ = _data(n, 7)
    logits, prop = mwdg2_b200.mlp_forward(p, X, threshold=0.25)
    ref, _ = mlp_ref.forward(p, X)
    err = float(np.max(np.abs(logits - ref)))
    assert err <= 2e-2 * max(1.0, float(np.max(np.abs(ref)))), f"max |logit error| {err:.3e}"
    np.testing.assert_array_equal(prop, (logits > 0.25).astype(np.uint8))


def test_gradient_matches_reference():
    p = mwdg2_b200.mlp_init(5)
    X, labels = _data(777, 11)
    grad, loss = mwdg2_b200.mlp_grad(p, X, labels, pos_weight=3.0)
    ref_loss, ref = mlp_ref.loss_and_grad(p, X, labels, pos_weight=3.0)
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss), (loss, ref_loss)
    o = 0
    for fo, fi in mlp_ref.SHAPES:
        for name, size in (("W", fo * fi), ("b", fo)):
            g, r = grad[o:o + size], ref[o:o + size]
            scale = float(np.max(np.abs(r)))
            err = float(np.max(np.abs(g - r)))
            assert err <= 3e-2 * scale + 1e-7, f"{name}{fo}x{fi}: error {err:.3e} of scale {scale:.3e}"
            o += size


def test_trainer_learns_separable_labels():
    rng = np.random.Generator(np.random.PCG64(13))
    X = rng.uniform(-1.0, 1.0, size=(4096, mwdg2_b200.MLP_FEATURES)).astype(np.float32)
    X[:, 112] = 1.0
    labels = ((X[:, 0] > 0) * 1 + (X[:, 1] > 0) * 2 + (X[:, 2] + X[:, 3] > 0) * 4 + (X[:, 4] < -0.5) * 8).astype(np.uint8)
    tr = mwdg2_b200.Trainer(mwdg2_b200.mlp_init(1), lr=3e-3)
    first = tr.step(X, labels)
    for _ in range(300):
        last = tr.step(X, labels)
    p = tr.params()
    tr.close()
    assert last < 0.1 * first, (first, last)
    _, prop = mwdg2_b200.mlp_forward(p, X)
    want = (labels[:, None] >> np.arange(4)) & 1
    assert float(np.mean(prop == want)) > 0.97
