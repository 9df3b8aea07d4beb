"""Deterministic inputs shared by the configuration-size fixtures and tests.

integer_velocity(g) is a velocity field made from integer arithmetic only:
every value is a small integer divided by a power of two, so NumPy forms it
exactly, on any machine, and the transport run on it is reproducible bit for
bit without storing the field.  It is not a flow solution (its divergence is
not zero); the transport algorithm is the same function of any field, and
its C div(u) term is exercised too.

subsample(n, k, seed) picks k sorted voxel indices out of n, for fixtures
whose full fields are too large to commit.
"""

import hashlib

import numpy as np

PORE = 2


def integer_velocity(g):
    g = np.asarray(g)
    m = g == PORE
    idx = np.indices(g.shape)
    if g.ndim == 3:
        x, y, z = idx
    else:
        x, y = idx
        z = np.zeros_like(x)
    vx = (16 + (3 * x + 5 * y + 7 * z) % 11).astype(np.float32) / np.float32(16)
    vy = (((5 * x + 3 * y + z) % 9) - 4).astype(np.float32) / np.float32(32)
    vz = (((x + 7 * y + 3 * z) % 7) - 3).astype(np.float32) / np.float32(32)
    if g.ndim == 2:
        vz = np.zeros_like(vz)
    v = np.stack([vx, vy, vz]).astype(np.float32)
    v[:, ~m] = 0.0
    return v


def subsample(n, k, seed=0):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(k, n), replace=False)).astype(np.int64)


def digest(a):
    """sha256 of an array's bytes (C order), as a hex string."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def field_stats(v, m):
    """Per component over the mask: float64 sum, sum of squares, max |v|."""
    v = np.asarray(v, np.float64)
    out = []
    for c in range(v.shape[0]):
        a = v[c][m]
        out.append([a.sum(), (a * a).sum(), np.abs(a).max() if a.size else 0.0])
    return np.asarray(out, np.float64)
