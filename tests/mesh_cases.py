"""Mesh test fixtures shared by the CPU and GPU mesh-driver tests.

The images are those of the reference's own mesh tests: the three-wave
texture of make_synthetic_texture_mesh (src/mesh.rs:2906-2920), shifted
uniformly (shift_image_uniform, :2926-2941) or by a horizontal band
(shift_image_band, :2979-2995) with clamped linear resampling; the mesh is
the fixed structured grid of make_band_test_mesh_and_solve_inputs
(:3038-3062): 9 x 9 nodes 7.5 px apart over [20, 80], two triangles per cell.
A 6-node version adds one mid-side node per edge.
"""
from __future__ import annotations

import math

import numpy as np


def texture(size=100):
    img = np.zeros((size, size))
    for y in range(size):
        for x in range(size):
            v = math.sin(0.7 * x) * math.cos(0.5 * y) + math.sin(0.31 * x + 0.2 * y) + math.cos(0.13 * x - 0.42 * y)
            img[y, x] = 128.0 + 40.0 * v
    return img


def shift_rows(src, u_of_row):
    h, w = src.shape
    out = np.zeros_like(src)
    for y in range(h):
        u = u_of_row(y)
        for x in range(w):
            sx = x - u
            x0 = math.floor(sx)
            frac = sx - x0
            x0i = min(int(max(x0, 0.0)), w - 1)
            x1i = min(int(max(x0 + 1.0, 0.0)), w - 1)
            out[y, x] = src[y, x0i] * (1.0 - frac) + src[y, x1i] * frac
    return out


def shift_uniform(src, u):
    return shift_rows(src, lambda y: u)


def shift_band(src, split_row, u_top, u_bottom):
    return shift_rows(src, lambda y: u_top if y < split_row else u_bottom)


def grid_mesh(n_side=9, start=20.0, step=7.5):
    at = [start + step * k for k in range(n_side)]
    nodes = np.array([[at[i % n_side], at[i // n_side]] for i in range(n_side * n_side)])

    def node_id(c, r):
        return r * n_side + c
    el = []
    for r in range(n_side - 1):
        for c in range(n_side - 1):
            el.append([node_id(c, r), node_id(c + 1, r), node_id(c, r + 1)])
            el.append([node_id(c + 1, r), node_id(c + 1, r + 1), node_id(c, r + 1)])
    return nodes, np.array(el, dtype=np.int64)


def to_order2(nodes, elements):
    """6-node elements [c0, c1, c2, m01, m12, m20] with shared mid-side nodes."""
    nodes = [list(v) for v in nodes]
    mid = {}
    out = []
    for a, b, c in elements:
        row = [int(a), int(b), int(c)]
        for u, v in ((a, b), (b, c), (c, a)):
            key = (min(u, v), max(u, v))
            if key not in mid:
                mid[key] = len(nodes)
                nodes.append([(nodes[u][0] + nodes[v][0]) / 2.0, (nodes[u][1] + nodes[v][1]) / 2.0])
            row.append(mid[key])
        out.append(row)
    return np.array(nodes), np.array(out, dtype=np.int64)


def speckle_quadratic(size=256, seed=5):
    """A seeded speckle pair under a smooth field (translation + affine +
    quadratic terms about the centre) and that field."""
    from gpv import synth
    c = size / 2.0
    field = synth.make_field(xc=c, yc=c, t=(1.3, -0.7), a=(0.01, 0.004, -0.006, 0.008),
                             q=(2e-5, -1e-5, 1e-5, -2e-5, 1e-5, 3e-5))
    f, g = synth.pair(size, size, field, seed)
    return f.astype(np.float64), g.astype(np.float64), field


def oracle_solver(oracle, f, g, border, max_norm=1e-5, max_iterations=50, mask=None):
    """solver(desc, tolerance) over the FP64 oracle for images f, g."""
    Cf = oracle.get_c(np.asarray(f, dtype=np.float64), border)
    Cg = oracle.get_c(np.asarray(g, dtype=np.float64), border)

    def solve(desc, tolerance):
        return oracle.solve_batch(Cf, Cg, f.shape, border, desc, max_norm=max_norm, max_iterations=max_iterations,
                                  tolerance=tolerance, mask=mask)
    return solve
