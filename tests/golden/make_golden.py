"""Generates the golden vectors in this directory from closed forms and brute force
alone (no code of the oracle or of the library):

- can.npz: the reference's can test (crates/icam-core/src/solid3.rs:2044-2069): its
  2000 + 40 query points and the closed-form signed distance of the cylinder r 3,
  z in [0, 5];
- bump_box.npz: the reference's bump-box test (solid3.rs:2178-2210): its 200 query
  points, the analytic inside test, and the dense-sample distance bracket (300 x 300
  samples of every face);
- block_with_hole.npz: 4000 seeded points around the 100 x 60 x 40 block with a
  20 mm hole, with the brute-force signed distance over its seven trimmed faces
  (tests/brute.py) and point membership.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import brute  # noqa: E402


def can():
    t = np.arange(2000.0)
    pts = np.stack([6 * np.sin(t * 0.37), 6 * np.cos(t * 0.71), 2.5 + 5 * np.sin(t * 1.3)], 1)
    axis = np.stack([np.zeros(40), np.zeros(40), -2 + 9 * np.arange(40) / 39], 1)
    p = np.concatenate([pts, axis])
    rho = np.hypot(p[:, 0], p[:, 1])
    dr, dz = rho - 3.0, np.abs(p[:, 2] - 2.5) - 2.5
    inside = (dr <= 0) & (dz <= 0)
    d = np.where(inside, np.maximum(dr, dz), np.sqrt(np.maximum(dr, 0) ** 2 + np.maximum(dz, 0) ** 2))
    np.savez_compressed(os.path.join(HERE, "can.npz"), points=p, sdf=d)


def bump_top(x, y):
    zc = np.array([[5.0, 5.0, 5.0], [7.0, 9.0, 5.0], [5.0, 6.0, 5.0]])
    u, v = x / 10.0, y / 10.0
    bu = np.stack([(1 - u) ** 2, 2 * u * (1 - u), u * u], -1)
    bv = np.stack([(1 - v) ** 2, 2 * v * (1 - v), v * v], -1)
    return np.einsum("...i,...j,ij->...", bu, bv, zc)


def bump_box():
    n = 300
    A, B = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    A, B = A.ravel(), B.ravel()
    fx, fy = 10.0 * A / n, 10.0 * B / n
    s = [np.stack([fx, fy, bump_top(fx, fy)], 1), np.stack([fx, fy, 0 * fx], 1)]
    for px, py in [(fx, 0 * fx), (fx, 0 * fx + 10), (0 * fx, fx), (0 * fx + 10, fx)]:
        s.append(np.stack([px, py, bump_top(px, py) * B / n], 1))
    S = np.concatenate(s)
    t = np.arange(200.0)
    p = np.stack([5 + 8 * np.sin(t * 0.37), 5 + 8 * np.cos(t * 0.71), 4 + 6 * np.sin(t * 1.3)], 1)
    dense = np.empty(len(p))
    for i in range(len(p)):
        dense[i] = np.sqrt(((S - p[i]) ** 2).sum(1).min())
    inside = (p[:, 0] > 0) & (p[:, 0] < 10) & (p[:, 1] > 0) & (p[:, 1] < 10) & (p[:, 2] > 0) & (p[:, 2] < bump_top(p[:, 0], p[:, 1]))
    np.savez_compressed(os.path.join(HERE, "bump_box.npz"), points=p, dense=dense, inside=inside, h=10.0 / n)


def block_with_hole():
    rng = np.random.default_rng(20261203)
    p = rng.uniform([-10, -10, -10], [110, 70, 50], size=(4000, 3))
    d = brute.block_with_hole_sdf(p)
    np.savez_compressed(os.path.join(HERE, "block_with_hole.npz"), points=p, sdf=d)


if __name__ == "__main__":
    can()
    bump_box()
    block_with_hole()
    print("written to", HERE)
