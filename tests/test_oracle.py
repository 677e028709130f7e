"""The oracle pinned against the reference's own known-answer tests and an
independent brute force. CPU only.

- the can: |Exact - closed form| < 1e-9 at the reference's 2000 + 40 points, never
  unsure (crates/icam-core/src/solid3.rs:2044-2069);
- the bump box: sign equals the analytic inside test, |d| within the dense-sample
  bracket [dense - h, dense + 1e-9] (solid3.rs:2178-2210);
- the block with a hole: agreement with a brute force over its seven trimmed faces
  and point membership (tests/brute.py);
- the freeform top: the dense-sample bracket on its B-spline face.
"""
import numpy as np
import pytest
from scipy.spatial import cKDTree

import brute
from implicitcam_b200 import parts


def can_exact(p):
    rho = np.hypot(p[:, 0], p[:, 1])
    dr, dz = rho - 3.0, np.abs(p[:, 2] - 2.5) - 2.5
    inside = (dr <= 0) & (dz <= 0)
    return np.where(inside, np.maximum(dr, dz), np.sqrt(np.maximum(dr, 0) ** 2 + np.maximum(dz, 0) ** 2))


def can_points():
    t = np.arange(2000.0)
    pts = np.stack([6 * np.sin(t * 0.37), 6 * np.cos(t * 0.71), 2.5 + 5 * np.sin(t * 1.3)], 1)
    axis = np.stack([np.zeros(40), np.zeros(40), -2 + 9 * np.arange(40) / 39], 1)
    return np.concatenate([pts, axis])


def test_can_closed_form(oracle_mod):
    o = oracle_mod.Oracle(parts.can())
    p = can_points()
    d, _, _, _, unsure, _ = o.sdf(p)
    assert not unsure.any()
    assert np.abs(d - can_exact(p)).max() < 1e-9


def bump_samples(n=300):
    A, B = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    A, B = A.ravel(), B.ravel()
    fx, fy = 10.0 * A / n, 10.0 * B / n
    top = np.vectorize(parts.bump_box_top)
    s = [np.stack([fx, fy, top(fx, fy)], 1), np.stack([fx, fy, 0 * fx], 1)]
    for px, py in [(fx, 0 * fx), (fx, 0 * fx + 10), (0 * fx, fx), (0 * fx + 10, fx)]:
        s.append(np.stack([px, py, top(px, py) * B / n], 1))
    return np.concatenate(s), 10.0 / n


def test_bump_box_dense_bracket(oracle_mod):
    o = oracle_mod.Oracle(parts.bump_box())
    t = np.arange(200.0)
    p = np.stack([5 + 8 * np.sin(t * 0.37), 5 + 8 * np.cos(t * 0.71), 4 + 6 * np.sin(t * 1.3)], 1)
    d, _, _, _, unsure, _ = o.sdf(p)
    S, h = bump_samples()
    top = np.vectorize(parts.bump_box_top)
    inside = (p[:, 0] > 0) & (p[:, 0] < 10) & (p[:, 1] > 0) & (p[:, 1] < 10) & (p[:, 2] > 0) & (p[:, 2] < top(p[:, 0], p[:, 1]))
    dense = cKDTree(S).query(p)[0]
    assert not unsure.any()
    assert ((d < 0) == inside).all()
    assert (np.abs(d) <= dense + 1e-9).all()
    assert (np.abs(d) >= dense - h).all()


def test_block_with_hole_brute_force(oracle_mod):
    o = oracle_mod.Oracle(parts.block_with_hole())
    rng = np.random.default_rng(0)
    p = rng.uniform([-10, -10, -10], [110, 70, 50], size=(50000, 3))
    # points on the axes of symmetry, the faces and the hole's wall
    g = np.linspace(-5, 105, 23)
    p = np.concatenate([p, np.stack([g, 30 + 0 * g, 20 + 0 * g], 1), np.stack([50 + 0 * g, 30 + 0 * g, g * 0.4], 1)])
    d, _, _, _, unsure, _ = o.sdf(p)
    b = brute.block_with_hole_sdf(p)
    assert not unsure.any()
    assert np.abs(d - b).max() < 1e-9
    assert (np.sign(d) == np.sign(b)).all()


def test_freeform_top_dense_bracket(oracle_mod):
    b = parts.freeform_top(seed=0)
    o = oracle_mod.Oracle(b)
    patches = b.patches[0].reshape(13, 13, 4, 4, 4)
    # dense samples of the B-spline top: 40 x 40 per span
    s = np.linspace(0, 1, 41)
    B = np.stack([(1 - s) ** 3, 3 * (1 - s) ** 2 * s, 3 * (1 - s) * s * s, s ** 3], 1)
    H = np.einsum("ui,vj,abijc->abuvc", B, B, patches)
    S = (H[..., :3] / H[..., 3:]).reshape(-1, 3)
    h = 120.0 / 13 / 40 * 1.5
    rng = np.random.default_rng(1)
    xy = rng.uniform(5, 115, size=(300, 2))
    z = rng.uniform(48, 75, size=300)
    p = np.concatenate([xy, z[:, None]], 1)
    d, _, kind, fid, unsure, _ = o.sdf(p)
    dense = cKDTree(S).query(p)[0]
    top_face = (kind == 0) & (fid == 0)
    assert not unsure.any()
    assert top_face.sum() > 200
    assert (np.abs(d) <= dense + 1e-9).all()
    assert (np.abs(d[top_face]) >= dense[top_face] - h).all()
