"""Float64 CPU statement of the path-guiding network (cpu-renderer_b200/csrc/cr_guide.cuh,
cr_guide.cu) — TEST INFRASTRUCTURE ONLY: the checker for tests/test_guide.py; the product never
imports it.

The network has no counterpart in the reference; this module restates its definition
independently: the input encoding, the four dense layers with the FP16-rounded weights that
inference uses, the mixture of 8 von Mises-Fisher lobes, and the weighted negative
log-likelihood the training kernels minimise. Gradients come from torch's autograd in float64
on the CPU.
"""
import math

import numpy as np
import torch

IN, WIDTH, LOBES, OUT, OUT_PAD, FEATURES = 64, 64, 8, 40, 48, 9
W1, W2, W3 = 0, WIDTH * IN, 2 * WIDTH * IN
W4 = 3 * WIDTH * IN
WCOUNT = W4 + OUT_PAD * WIDTH
B1, B2, B3, B4 = WCOUNT, WCOUNT + WIDTH, WCOUNT + 2 * WIDTH, WCOUNT + 3 * WIDTH
PARAMS = B4 + OUT_PAD
LOG_KAPPA_MIN, LOG_KAPPA_MAX = -3.0, 9.0


def fp16_round(p):
    return np.asarray(p, np.float32).astype(np.float16).astype(np.float64)


OCTAVES = 8


def encode(features):
    """features (n, 9) -> inputs (n, 64): the features, then sin and cos of 2^k pi position,
    k = 0..7 (57 inputs, the rest zero)."""
    f = np.asarray(features, np.float64)
    x = np.zeros((len(f), IN))
    x[:, :FEATURES] = f
    o = FEATURES
    for k in range(OCTAVES):
        s = float(1 << k) * math.pi
        for d in range(3):
            x[:, o] = np.sin(s * f[:, d])
            x[:, o + 1] = np.cos(s * f[:, d])
            o += 2
    return x


def _layers(p):
    w = lambda off, rows: p[off:off + rows * IN].reshape(rows, IN)
    return [(w(W1, WIDTH), p[B1:B1 + WIDTH]), (w(W2, WIDTH), p[B2:B2 + WIDTH]),
            (w(W3, WIDTH), p[B3:B3 + WIDTH]), (w(W4, OUT_PAD), p[B4:B4 + OUT_PAD])]


def forward(params, features):
    """Network outputs (n, 40) with the FP16-rounded parameters."""
    p = torch.tensor(fp16_round(params))
    h = torch.tensor(encode(features))
    layers = _layers(p)
    for i, (w, b) in enumerate(layers):
        h = h @ w.T + b
        if i < 3:
            h = torch.relu(h)
    return h[:, :OUT].numpy()


def _nll(out, dirs):
    o = out[:, :OUT].reshape(-1, LOBES, 5)
    logpi = torch.log_softmax(o[:, :, 0], dim=1)
    kappa = torch.exp(torch.clamp(o[:, :, 1], LOG_KAPPA_MIN, LOG_KAPPA_MAX))
    m = o[:, :, 2:5]
    mu = m / torch.linalg.norm(m, dim=2, keepdim=True)
    c = (mu * dirs[:, None, :]).sum(dim=2)
    logvmf = torch.log(kappa) - math.log(2 * math.pi) - torch.log(-torch.expm1(-2 * kappa)) + kappa * (c - 1)
    return -torch.logsumexp(logpi + logvmf, dim=1)


def loss_and_gradient(params, samples):
    """samples (n, 13): features, direction, weight. Returns (sum_i w_i * -log q_i, d/dparams)."""
    s = np.asarray(samples, np.float64)
    p = torch.tensor(fp16_round(params), requires_grad=True)
    h = torch.tensor(encode(s[:, :9]))
    layers = _layers(p)
    for i, (w, b) in enumerate(layers):
        h = h @ w.T + b
        if i < 3:
            h = torch.relu(h)
    loss = (torch.tensor(s[:, 12]) * _nll(h, torch.tensor(s[:, 9:12]))).sum()
    loss.backward()
    return float(loss.detach()), p.grad.numpy()


def mixture_pdf(outputs, dirs):
    """q(dir) of each row's mixture."""
    out = torch.tensor(np.asarray(outputs, np.float64))
    return torch.exp(-_nll(out, torch.tensor(np.asarray(dirs, np.float64)))).numpy()
