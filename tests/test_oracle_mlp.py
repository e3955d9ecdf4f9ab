"""Pins the FP64 oracle of the leaf-value network (oracle/mlp_fp64.py)
before it checks the GPU kernels: analytic gradients against central finite
differences in float64, bfloat16 rounding against torch's conversion, and
the Adam step against its definition written out by hand."""
import numpy as np
import pytest

from oracle import mlp_fp64


def tiny_layers(rng, dims):
    return [(rng.normal(0, 1.0 / np.sqrt(k), (n, k)), rng.normal(0, 0.1, n)) for k, n in zip(dims[:-1], dims[1:])]


@pytest.mark.parametrize("masked", [False, True])
def test_gradients_match_finite_differences(masked):
    rng = np.random.default_rng(11)
    dims = [7, 9, 8, 5]
    layers = tiny_layers(rng, dims)
    x = rng.normal(size=(6, 7))
    t = rng.normal(size=(6, 5))
    mask = (rng.random((6, 5)) < 0.6).astype(np.float64) if masked else None
    loss, grads = mlp_fp64.loss_and_gradients(layers, x, t, mask)
    h = 1e-6
    worst = 0.0
    for l, (w, b) in enumerate(layers):
        for arr, g in ((w, grads[l][0]), (b, grads[l][1])):
            flat, gflat = arr.reshape(-1), g.reshape(-1)
            for i in range(flat.size):
                keep = flat[i]
                flat[i] = keep + h
                lp, _ = mlp_fp64.loss_and_gradients(layers, x, t, mask)
                flat[i] = keep - h
                lm, _ = mlp_fp64.loss_and_gradients(layers, x, t, mask)
                flat[i] = keep
                fd = (lp - lm) / (2 * h)
                worst = max(worst, abs(fd - gflat[i]) / max(1e-3, abs(fd)))
    assert worst < 1e-6, worst
    assert loss > 0


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(size=4096) * 10.0 ** rng.integers(-30, 30, 4096),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.005859375, 65504.0, 3.0e38])])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    got = mlp_fp64.bf16(x)
    assert np.array_equal(got, ref)


def test_adam_step_matches_definition():
    rng = np.random.default_rng(5)
    w, g = rng.normal(size=50), rng.normal(size=50)
    m, v = np.zeros(50), np.zeros(50)
    w1, m1, v1 = mlp_fp64.adam_step(w, g, m, v, 1, 1e-3)
    # Step 1 from zero moments: m/c1 = g and v/c2 = g^2, so the move is
    # lr * g / (|g| + eps).
    assert np.allclose(w1, w - 1e-3 * g / (np.abs(g) + 1e-8), rtol=0, atol=1e-15)
    w2, _, _ = mlp_fp64.adam_step(w1, g, m1, v1, 2, 1e-3)
    m2 = 0.9 * m1 + 0.1 * g
    v2 = 0.999 * v1 + 0.001 * g * g
    assert np.allclose(w2, w1 - 1e-3 * (m2 / (1 - 0.81)) / (np.sqrt(v2 / (1 - 0.999 ** 2)) + 1e-8), rtol=0,
                       atol=1e-15)
