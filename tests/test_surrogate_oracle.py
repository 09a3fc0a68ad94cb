"""CPU tests of the surrogate's oracle (oracle/mlp_oracle.py) and of the
surrogate library's exports. The reference has no surrogate; the oracle's
backward pass is pinned by central finite differences of its FP64 forward,
and its BF16 rounding by torch's BF16 conversion."""
import ctypes as C
import os
import re
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as M  # noqa: E402


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    a = np.concatenate([rng.normal(size=5000) * 10.0 ** rng.integers(-8, 8, 5000), [0.0, -0.0, 1.0, 3.0e38]])
    ref = torch.tensor(a.astype(np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)
    np.testing.assert_array_equal(M.bf16(a), ref)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = M.he_uniform(3) * 0.5
    x = rng.uniform(-1, 1, size=(12, 4))
    t = rng.normal(size=(12, 3))
    norm = (np.zeros(4), np.ones(4), np.zeros(3), np.ones(3))
    loss, g = M.loss_and_grad(p, x, t, norm, bf16_points=False)
    idx = rng.choice(M.NPARAMS, 60, replace=False)
    idx = np.concatenate([idx, [M.NPARAMS - 1, M.NPARAMS - 4, 0, 1024 + 5]])  # b4, W4, W1, b1 entries
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp = M.loss_and_grad(p + e, x, t, norm, bf16_points=False)[0]
        lm = M.loss_and_grad(p - e, x, t, norm, bf16_points=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_surrogate_library_exports_header():
    lib = C.CDLL(os.path.join(ROOT, "mercurydpm_fork_b200", "libdem_surrogate.so"))
    names = re.findall(r"\b(dem_mlp_\w+)\s*\(", open(os.path.join(ROOT, "include", "dem_surrogate.h")).read())
    assert len(names) >= 9
    for n in names:
        assert hasattr(lib, n), n
    assert M.NPARAMS == 133635
