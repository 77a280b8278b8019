"""Learned search radius: GPU training kernels against the CPU reference of the network, the
tensor-core inference kernel against the same, and the certified search against the plain
unbounded search (bit-identical distances, plus what the network saves)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import mlp
from conftest import grid_of

pytestmark = pytest.mark.gpu


def _batch(seed, B=512):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (B, 3)).astype(np.float32)
    t = rng.uniform(0.0, 0.6, B).astype(np.float32)
    return x, t


def test_training_forward_and_gradient_match_cpu(gpu_ctx):
    P = mlp.init_params(3)
    x, t = _batch(4)
    dh, loss, grad = gpu_ctx.mlp_train_eval(P, x, t)
    loss_c, grad_c, dh_c = mlp.loss_and_grad(P, x, t)
    assert np.allclose(dh, dh_c, rtol=2e-3, atol=1e-4)
    assert loss == pytest.approx(loss_c, rel=2e-3)
    scale = np.abs(grad_c).max()
    assert np.abs(grad - grad_c).max() <= 2e-3 * scale
    # and against finite differences of the CPU loss on a few parameters of each layer
    for q in (mlp.OFF_W1 + 5, mlp.OFF_B2 + 7, mlp.OFF_W3 + 100, mlp.OFF_W4 + 3, mlp.OFF_B4):
        e = np.zeros_like(P)
        e[q] = 1e-2 if q >= mlp.OFF_B4 or (mlp.OFF_B1 <= q < mlp.OFF_W2) or (mlp.OFF_B2 <= q < mlp.OFF_W3) else 0.0
        if e[q] == 0.0:
            continue  # weights are FP16-rounded: finite differences only on FP32 biases
        fd = (mlp.loss_and_grad(P + e, x, t)[0] - mlp.loss_and_grad(P - e, x, t)[0]) / (2e-2)
        assert grad[q] == pytest.approx(fd, rel=5e-2, abs=1e-5)


def test_tensor_core_inference_matches_cpu(gpu_ctx):
    P = mlp.init_params(7)
    gpu_ctx.set_radius_params(P, np.array([0.0, 0.0, 0.0, 1.0]))
    x, _ = _batch(8, B=1000)
    got = gpu_ctx.radius_eval(x)
    ref = mlp.forward(P, x)["dhat"]
    assert np.allclose(got, ref, rtol=1e-2, atol=1e-3)
    P2, norm = gpu_ctx.radius_params()
    assert np.array_equal(P2, P.astype(np.float32)) and norm.tolist() == [0.0, 0.0, 0.0, 1.0]


def test_training_reduces_loss(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    gpu_ctx.set_mesh(X, IEN)
    l0 = gpu_ctx.train_radius(coarse_n=32, steps=0, batch=4096)
    l1 = gpu_ctx.train_radius(coarse_n=32, steps=600, batch=4096)
    assert l1 < 0.25 * l0


def test_learned_radius_is_exact_and_certifies(gpu_ctx, torus_mesh):
    """Certified search with the trained radius == plain unbounded search, bit for bit, and most
    nodes certify (the printed times show what the network saves; bench.py records it)."""
    X, IEN = torus_mesh
    g = grid_of(X, n_nodes_long_axis=96)
    gpu_ctx.set_mesh(X, IEN)
    gpu_ctx.train_radius(coarse_n=64, steps=1500, batch=8192)
    plain, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 2)
    t_plain = gpu_ctx.stats()["ms_distance"]
    learned, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 2, learned=True)
    st = gpu_ctx.stats()
    assert np.array_equal(plain, learned)
    assert st["certified_nodes"] + st["unbounded_fallbacks"] == g["ngp"]
    assert st["certified_nodes"] >= 0.5 * g["ngp"]
    print(f"plain {t_plain:.3f} ms, learned {st['ms_distance']:.3f} ms, certified "
          f"{st['certified_nodes'] / g['ngp']:.3f}, loss {st['radius_loss']:.4f}")
    nodes = np.sort(np.random.default_rng(5).choice(g["ngp"], 2000, replace=False))
    ref, _, _ = oracle.distances(X, IEN, g["origin"], g["h"], g["N"], mode=2, nodes=nodes)
    assert np.array_equal(learned[nodes], ref)


def test_tight_margin_falls_back_and_stays_exact(gpu_ctx, torus_mesh):
    """With no margin about half the nodes are not certified by their bounded search and search
    again; results still equal the plain unbounded search bit for bit."""
    X, IEN = torus_mesh
    g = grid_of(X, n_nodes_long_axis=64)
    gpu_ctx.set_mesh(X, IEN)
    gpu_ctx.train_radius(coarse_n=48, steps=600, batch=4096)
    plain, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 2)
    try:
        gpu_ctx.set_radius_margin(0.0, 0.0)
        learned, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 2, learned=True)
        st = gpu_ctx.stats()
    finally:
        gpu_ctx.set_radius_margin()
    assert np.array_equal(plain, learned)
    assert st["unbounded_fallbacks"] > 0.1 * g["ngp"]
    assert st["certified_nodes"] + st["unbounded_fallbacks"] == g["ngp"]
