"""Shared data generators and recall helpers for the tests (seeded, synthetic)."""
import numpy as np


def uniform(n, d, seed=0):
    return np.random.default_rng(seed).random((n, d), dtype=np.float32)


def gmm(n, d, n_clusters=100, center_std=10.0, seed=0):
    """Isotropic Gaussian mixture: centers ~ N(0, center_std^2 I), unit within-cluster std."""
    rng = np.random.default_rng(seed)
    centers = rng.normal(0.0, center_std, (n_clusters, d)).astype(np.float32)
    return (centers[rng.integers(0, n_clusters, n)] + rng.normal(0.0, 1.0, (n, d))).astype(np.float32)


def sin_fixture(n, d, scale=0.1):
    """core/index.rs:740-749 test data: sin((i*dim + j) * 0.1)."""
    i = np.arange(n * d, dtype=np.float32)
    return np.sin(i * np.float32(scale)).astype(np.float32).reshape(n, d)


def recall(found, truth):
    k = truth.shape[1]
    hits = 0
    for f, t in zip(found, truth):
        hits += len(set(f[f >= 0].tolist()) & set(t.tolist()))
    return hits / (truth.shape[0] * k)
