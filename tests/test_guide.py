"""The path-guiding network (cr_guide): tensor-core inference and the training gradients against
the float64 CPU statement in oracle/guide_oracle.py, and online training on a known target.
"""
import numpy as np
import pytest

import guide_oracle as go


def random_params(rng, scale=0.3):
    p = rng.normal(0, scale, go.PARAMS).astype(np.float32)
    p[go.W4 + go.OUT * go.IN:go.WCOUNT] = 0  # padded output rows
    p[go.B4 + go.OUT:] = 0
    return p


def random_samples(rng, n):
    f = np.zeros((n, 13), np.float32)
    f[:, 0:3] = rng.uniform(0, 1, (n, 3))
    for a, b in ((3, 6), (6, 9), (9, 12)):
        v = rng.normal(size=(n, 3))
        f[:, a:b] = v / np.linalg.norm(v, axis=1, keepdims=True)
    f[:, 12] = rng.uniform(0.1, 2.0, n)
    return f


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = random_params(rng).astype(np.float64)
    s = random_samples(rng, 7)
    # perturb parameters that are exactly representable in FP16 steps, so rounding is stable
    p = go.fp16_round(p)
    loss, g = go.loss_and_gradient(p, s)
    for i in [go.W1 + 3, go.W2 + 100, go.W3 + 777, go.W4 + 5, go.B4 + 1, go.B4 + 7]:
        h = 2.0 ** -6
        up, dn = p.copy(), p.copy()
        up[i] += h
        dn[i] -= h
        num = (go.loss_and_gradient(up, s)[0] - go.loss_and_gradient(dn, s)[0]) / (2 * h)
        assert num == pytest.approx(g[i], rel=2e-2, abs=1e-4), i


@pytest.mark.gpu
def test_inference_matches_oracle(crgpu, gpu):
    rng = np.random.default_rng(11)
    gd = crgpu.Guide(seed=3)
    p = random_params(rng)
    gd.set_parameters(p)
    feats = random_samples(rng, 1000)[:, :9]
    got = gd.evaluate(feats)
    want = go.forward(p, feats)
    err = np.abs(got - want)
    # activations are rounded to FP16 between layers (~5e-4 relative each), so the error scales
    # with the outputs
    assert np.max(err / (1 + np.abs(want))) < 2e-2, float(np.max(err))
    assert np.mean(err) < 2e-3 * (1 + np.mean(np.abs(want))), (float(np.mean(err)), float(np.mean(np.abs(want))))
    gd.close()


@pytest.mark.gpu
def test_training_gradients_match_oracle(crgpu, gpu):
    rng = np.random.default_rng(12)
    gd = crgpu.Guide(seed=4)
    p = random_params(rng, scale=0.15)
    gd.set_parameters(p)
    s = random_samples(rng, 1000)  # not a multiple of the 128-sample blocks
    g, loss = gd.gradients(s)
    want_loss, want = go.loss_and_gradient(p, s)
    assert loss == pytest.approx(want_loss, rel=1e-4)
    scale = np.max(np.abs(want))
    # FP32 on the device against FP64 here: pre-activations near zero can fall on either side of
    # a ReLU, so compare to the gradient's scale
    assert np.max(np.abs(g - want)) < 3e-3 * scale, (float(np.max(np.abs(g - want))), float(scale))
    assert np.linalg.norm(g - want) < 1e-3 * np.linalg.norm(want)
    gd.close()


@pytest.mark.gpu
def test_training_learns_a_direction_field(crgpu, gpu):
    """Directions drawn around a position-dependent axis: Adam (lr 1e-3) lowers the loss and
    the learned mixture puts its density near the axis."""
    rng = np.random.default_rng(13)
    n = 20000
    s = random_samples(rng, n)
    axis = s[:, 0:3] - 0.5
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    jitter = rng.normal(0, 0.1, (n, 3))
    d = axis + jitter
    s[:, 9:12] = d / np.linalg.norm(d, axis=1, keepdims=True)
    s[:, 12] = 1.0
    gd = crgpu.Guide(seed=5)
    before = gd.gradients(s)[1] / n
    gd.train(s, steps=400, batch=4096)
    after = gd.gradients(s)[1] / n
    assert after < before - 1.5, (before, after)
    out = gd.evaluate(s[:512, :9])
    q_axis = go.mixture_pdf(out, axis[:512])
    q_away = go.mixture_pdf(out, -axis[:512])
    assert np.median(q_axis) > 20 * np.median(q_away)
    gd.close()
