"""CPU (numpy) reference of the learned-radius network -- TEST INFRASTRUCTURE ONLY.

The same definition the CUDA kernels implement (stl2sdf.jl_b200/csrc/radius.cu): Fourier features
of normalised coordinates, three hidden layers of 64 with FP16-rounded weights and FP16-rounded
inputs to the first two mma layers, FP32 accumulation, softplus output, and the loss
mean((log(dhat + eps) - log(t + eps))^2).  Used to check the GPU forward, the GPU gradients and the
tensor-core inference kernel.  The reference project has no such network; this checks the GPU code
against its own specification.
"""

from __future__ import annotations

import numpy as np

FREQ = 4
FEAT = 3 + 6 * FREQ
IN = 32
HID = 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID * HID
OFF_W4 = OFF_B3 + HID
OFF_B4 = OFF_W4 + HID
PARAMS = OFF_B4 + 1
EPS = 1e-3


def h16(x):
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float32)


def unpack(P):
    P = np.asarray(P, np.float32)
    W1 = h16(P[OFF_W1:OFF_B1]).reshape(HID, IN)
    b1 = P[OFF_B1:OFF_W2]
    W2 = h16(P[OFF_W2:OFF_B2]).reshape(HID, HID)
    b2 = P[OFF_B2:OFF_W3]
    W3 = h16(P[OFF_W3:OFF_B3]).reshape(HID, HID)
    b3 = P[OFF_B3:OFF_W4]
    w4 = h16(P[OFF_W4:OFF_B4])
    b4 = P[OFF_B4]
    return W1, b1, W2, b2, W3, b3, w4, b4


def features(x):
    x = np.asarray(x, np.float32).reshape(-1, 3)
    f = np.zeros((x.shape[0], IN), np.float32)
    f[:, :3] = x
    for k in range(FREQ):
        for a in range(3):
            v = x[:, a].astype(np.float64) * (1 << k)
            f[:, 3 + 6 * k + 2 * a] = np.sin(np.pi * v)
            f[:, 3 + 6 * k + 2 * a + 1] = np.cos(np.pi * v)
    return f


def forward(P, x):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(P)
    h0 = h16(features(x))
    h1 = h16(np.maximum(h0 @ W1.T + b1, 0.0))
    h2 = h16(np.maximum(h1 @ W2.T + b2, 0.0))
    a3 = np.maximum(h2 @ W3.T + b3, 0.0).astype(np.float32)
    y = (a3 @ w4 + b4).astype(np.float32)
    dh = np.where(y > 20.0, y, np.log1p(np.exp(np.minimum(y, 20.0)))).astype(np.float32)
    return dict(h0=h0, h1=h1, h2=h2, a3=a3, y=y, dhat=dh)


def loss_and_grad(P, x, t):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(P)
    c = forward(P, x)
    t = np.asarray(t, np.float32)
    B = t.shape[0]
    r = np.log(c["dhat"] + EPS) - np.log(t + EPS)
    loss = float(np.mean(r * r))
    sig = 1.0 / (1.0 + np.exp(-c["y"]))
    gy = (2.0 * r / (c["dhat"] + EPS) * sig / B).astype(np.float32)
    dz3 = np.where(c["a3"] > 0, gy[:, None] * w4[None, :], 0.0).astype(np.float32)
    dz2 = np.where(c["h2"] > 0, dz3 @ W3, 0.0).astype(np.float32)
    dz1 = np.where(c["h1"] > 0, dz2 @ W2, 0.0).astype(np.float32)
    G = np.zeros(PARAMS, np.float32)
    G[OFF_W1:OFF_B1] = (dz1.T @ c["h0"]).reshape(-1)
    G[OFF_B1:OFF_W2] = dz1.sum(0)
    G[OFF_W2:OFF_B2] = (dz2.T @ c["h1"]).reshape(-1)
    G[OFF_B2:OFF_W3] = dz2.sum(0)
    G[OFF_W3:OFF_B3] = (dz3.T @ c["h2"]).reshape(-1)
    G[OFF_B3:OFF_W4] = dz3.sum(0)
    G[OFF_W4:OFF_B4] = gy @ c["a3"]
    G[OFF_B4] = gy.sum()
    return loss, G, c["dhat"]


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    P = np.zeros(PARAMS, np.float32)
    P[OFF_W1:OFF_B1] = (rng.uniform(-1, 1, (HID, IN)) * np.sqrt(6.0 / FEAT)).reshape(-1)
    P[OFF_W1:OFF_B1].reshape(HID, IN)[:, FEAT:] = 0.0
    P[OFF_B1:OFF_W2] = rng.uniform(-0.1, 0.1, HID)
    P[OFF_W2:OFF_B2] = (rng.uniform(-1, 1, (HID, HID)) * np.sqrt(6.0 / HID)).reshape(-1)
    P[OFF_B2:OFF_W3] = rng.uniform(-0.1, 0.1, HID)
    P[OFF_W3:OFF_B3] = (rng.uniform(-1, 1, (HID, HID)) * np.sqrt(6.0 / HID)).reshape(-1)
    P[OFF_B3:OFF_W4] = rng.uniform(-0.1, 0.1, HID)
    P[OFF_W4:OFF_B4] = rng.uniform(-1, 1, HID) * 0.3
    P[OFF_B4] = -0.5
    return P
