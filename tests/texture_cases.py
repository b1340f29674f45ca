"""Shared inputs of the rigid-texture tests, restated from the reference's own
texture tests (src/texture.rs, mod tests):

* ``shear_pair(gamma)`` -- 1500 round Gaussian blobs (width 4 px, peak 100)
  on 200 x 200 from the tests' 64-bit LCG (seed 777), each moved rigidly by
  u = gamma (y - 100) in the target (src/texture.rs:424-437);
* ``grid_centres()`` -- the 20 subset centres of solve_grid_with (:447-449);
* ``draw`` -- the blob intensity model (:285-287).
"""
import numpy as np

S = 4.0
MASK64 = (1 << 64) - 1


def lcg(seed, count):
    """Uniform [0, 1) draws of the tests' generator: state = state *
    6364136223846793005 + 1442695040888963407 (mod 2^64), value = (state >> 11) / 2^53."""
    out = np.empty(count)
    state = seed
    for k in range(count):
        state = (state * 6364136223846793005 + 1442695040888963407) & MASK64
        out[k] = (state >> 11) / float(1 << 53)
    return out


def draw(centres, n):
    """n x n image of 100 * sum exp(-|x - c|^2 / S^2) (rows = y, columns = x)."""
    ys, xs = np.mgrid[0:n, 0:n].astype(np.float64)
    img = np.zeros((n, n))
    for cx, cy in centres:
        img += np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / (S * S))
    return 100.0 * img


def shear_pair(gamma, n=200, count=1500):
    r = lcg(777, 2 * count).reshape(count, 2) * n
    moved = np.column_stack([r[:, 0] + gamma * (r[:, 1] - 100.0), r[:, 1]])
    return draw(r, n), draw(moved, n)


def grid_centres():
    return np.array([[55.0 + 22.5 * xi + 0.3, 62.0 + 25.0 * yi + 0.6] for yi in range(4) for xi in range(5)])


def grid_desc(gpv_mod, gamma, order):
    xy = grid_centres()
    p0 = np.zeros((len(xy), 12))
    p0[:, 0] = gamma * (xy[:, 1] - 100.0)
    return gpv_mod.make_desc(xy, 15, order, p0)
