"""Shared helpers for the parity tests: seeded Fortran-layout inputs."""
import numpy as np

import oracle as O


def rand_spinor(L, rng, scale=1.0):
    a = O.spinor(L)
    a[1:-1, 1:-1, 1:-1, 1:-1, :] = scale * (rng.standard_normal(a[1:-1, 1:-1, 1:-1, 1:-1, :].shape)
                                             + 1j * rng.standard_normal(a[1:-1, 1:-1, 1:-1, 1:-1, :].shape))
    return O.update_halo_5(L, a)


def rand_theta(L, rng, beta=0.3):
    return np.asfortranarray(rng.standard_normal((L.lx, L.ly, L.lt, 3)) / np.sqrt(beta), dtype=np.float32)


def rand_links(L, rng, beta=0.3):
    """u = coef(theta) for Gaussian theta, antiperiodic in t."""
    return O.coef(L, rand_theta(L, rng, beta))


def interior(a):
    return a[1:-1, 1:-1, 1:-1, 1:-1, :]


def rel_err(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))
