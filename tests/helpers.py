"""Shared seeded input generators and error metrics for the tests."""

import numpy as np

E_EV = 6400.0
K64 = 2 * np.pi / (1.24 / E_EV)


def rng(seed):
    return np.random.Generator(np.random.Philox(seed))


def sphere(g, n, r):
    t = g.uniform(-1, 1, n)
    p = g.uniform(0, 2 * np.pi, n)
    u = r * g.uniform(0, 1, n) ** (1 / 3)
    s = np.sqrt(1 - t ** 2)
    return np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)


def atoms(pos, phase):
    return np.ascontiguousarray(np.concatenate([pos, np.reshape(phase, (-1, 1))], 1))


def rel_field_err(E, E_ref):
    """max |dE| / rms|E_ref| -- a field metric insensitive to speckle minima."""
    E = np.asarray(E)
    E_ref = np.asarray(E_ref)
    return float(np.abs(E - E_ref).max() / np.sqrt(np.mean(np.abs(E_ref) ** 2)))
