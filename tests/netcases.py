"""Seeded inputs for the learned preconditioner's network tests."""
import numpy as np


def net_case(shape, seed=0):
    """(r, type, solid): a smooth random level set gives fluid (type 2), a
    few phi == 0 cells (type 1) and air; solid cells are a slab at x = 0."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    phi = (y - 0.6 * ny) + 1.5 * np.sin(0.7 * x) + rng.uniform(-0.4, 0.4, size=shape)
    type_ = np.where(phi < 0, 2, 0).astype(np.uint8)
    type_[rng.uniform(size=shape) < 0.01] = 1
    solid = np.zeros(shape, np.uint8)
    solid[0] = 1
    solid[type_ != 0] = 0
    r = (rng.standard_normal(shape) * (type_ != 0)).astype(np.float32)
    return r, type_, solid


def random_params(n, seed=1, scale=0.08):
    return (np.random.default_rng(seed).standard_normal(n) * scale).astype(np.float32)
