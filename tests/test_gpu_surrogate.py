"""The calibration surrogate on the GPU (tcgen05 BF16 GEMMs with FP32
accumulation) against the CPU oracle with BF16 rounding at the same points.

Inference runs as one fused kernel (layers 1 and 4 on the CUDA cores, 2 and 3
on the tensor cores); training passes run one GEMM per layer.
Tolerances: the oracle accumulates in FP64 and evaluates erf/exp in double;
the GPU accumulates in FP32 and rounds the pre-activations it turns into BF16
from FP32, so a few BF16 values differ by one unit (2^-8 relative). Outputs
are compared to 1e-2 of their norm, gradients per parameter block to 3e-2 of
the block's norm.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _net(seed=7, capacity=4096):
    from mercurydpm_fork_b200.surrogate import Surrogate
    s = Surrogate(capacity=capacity, seed=seed)
    s.set_normalisation([0.45, 0.15, 0.6, 0.1], [0.2, 0.09, 0.17, 0.06], [30.0, 0.6, 0.05], [5.0, 0.02, 0.02])
    return s


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = np.column_stack([rng.uniform(0.1, 0.8, n), rng.uniform(0, 0.3, n), rng.uniform(0.3, 0.9, n),
                         rng.uniform(0, 0.2, n)])
    y = np.column_stack([20 + 25 * x[:, 0] + 10 * x[:, 1], 0.55 + 0.1 * x[:, 2] - 0.2 * x[:, 3],
                         0.03 + 0.04 * x[:, 2] * x[:, 0]])
    return x, y


@pytest.mark.parametrize("n", [1, 77, 300, 1024])
def test_forward_matches_oracle(gpu, n):
    s = _net()
    x, _ = _data(n)
    y = s.predict(x)
    yo, _ = M.forward(s.params().astype(np.float64), x, s.norm)
    yo = yo * s.norm[3] + s.norm[2]
    s.close()
    assert np.linalg.norm(y - yo) <= 1e-2 * np.linalg.norm(yo)


@pytest.mark.parametrize("n", [4097, 65536])
def test_fused_forward_at_size_matches_oracle(gpu, n):
    """Inference runs as one fused kernel (one CTA per SM over 128-sample
    tiles): several tiles per CTA, and a last tile that is not full."""
    s = _net(capacity=65536)
    x, _ = _data(n, seed=5)
    y = s.predict(x)
    yo, _ = M.forward(s.params().astype(np.float64), x, s.norm)
    yo = yo * s.norm[3] + s.norm[2]
    s.close()
    assert np.linalg.norm(y - yo) <= 1e-2 * np.linalg.norm(yo)
    assert np.all(np.isfinite(y))


@pytest.mark.parametrize("n", [64, 300, 1024])
def test_gradients_match_oracle(gpu, n):
    s = _net()
    x, t = _data(n, seed=n)
    loss, g = s.gradients(x, t)
    lo, go = M.loss_and_grad(s.params().astype(np.float64), x, t, s.norm)
    s.close()
    assert abs(loss - lo) <= 1e-2 * lo
    o = 0
    for name, shape in M.SHAPES:
        k = int(np.prod(shape))
        a, b = g[o:o + k], go[o:o + k]
        assert np.linalg.norm(a - b) <= 3e-2 * np.linalg.norm(b) + 1e-12, name
        o += k


def test_training_reduces_loss(gpu):
    s = _net()
    x, y = _data(4096, seed=3)
    s.fit_normalisation(x, y)
    hist = s.fit(x, y, epochs=60, batch=1024, lr=1e-3)
    xv, yv = _data(1024, seed=4)
    pred = s.predict(xv)
    s.close()
    assert hist[-1] < 0.1 * hist[0]
    rel = np.abs(pred - yv) / np.abs(yv).mean(0)
    assert rel.mean() < 0.05


def test_large_batch_inference_is_consistent(gpu):
    s = _net(capacity=65536)
    x, _ = _data(65536, seed=9)
    y = s.predict(x)
    y2 = np.concatenate([s.predict(x[a:a + 1000]) for a in range(0, 3000, 1000)])
    s.close()
    assert np.isfinite(y).all()
    np.testing.assert_array_equal(y[:3000], y2)


def test_surrogate_guided_calibration_beats_plain_search(gpu):
    """Batched DEM heaps generate the training data; at the same DEM budget
    (one round of 64 proposals) the surrogate's proposals land closer to a
    held-out target response than uniform proposals (plain batched DEM
    search)."""
    from mercurydpm_fork_b200 import calibration as cal
    from mercurydpm_fork_b200.surrogate import Surrogate

    def dem(p):
        return cal.heap_responses(p, n=300, steps=6000, trace_every=1000)

    rng = np.random.default_rng(0)
    X = cal.sample_params(rng, 576)
    Y = dem(X)
    assert np.isfinite(Y).all() and (Y[:, 0] > 0).all()
    s = Surrogate(capacity=65536, seed=1)
    s.fit_normalisation(X[:512], Y[:512])
    s.fit(X[:512], Y[:512], epochs=150, batch=128, lr=1e-3)
    gains = []
    for k in range(2):
        target = Y[512 + k]
        a = cal.calibrate(target, dem, surrogate=s, rounds=1, proposals=64, candidates=65536, seed=k, tol=0.0,
                          data=(X[:512], Y[:512]), retrain_epochs=1)
        b = cal.calibrate(target, dem, surrogate=None, rounds=1, proposals=64, seed=k, tol=0.0)
        gains.append((a["history"][0]["median_error"], b["history"][0]["median_error"]))
    # both targets at once: one batched DEM run judges both targets' proposals
    rb = cal.calibrate_batch(Y[512:514], dem, s, rounds=1, proposals=64, candidates=65536, seed=5, tol=0.0,
                             data=(X[:512], Y[:512]), retrain_epochs=1)
    assert len(rb) == 2
    for k, r in enumerate(rb):
        assert r["rounds"] == 1 and r["dem_runs"] == 64
        assert abs(cal.response_error(r["response"], Y[512 + k])[0] - r["best_error"]) < 1e-12
        assert r["history"][0]["median_error"] < 0.5 * gains[k][1], (r["history"], gains)
    s.close()
    for surr, plain in gains:
        assert surr < 0.5 * plain, gains
