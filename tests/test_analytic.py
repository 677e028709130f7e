"""Cones, spheres and tori: the three analytic surface kinds the other parts lack.

The oracle is pinned to closed forms first (CPU): a ball's |p| - r, a ring's torus
distance, and a frustum's distance in its (radius, height) half-plane. On a B200 the
library then agrees with the oracle: points within 1e-9 of the diagonal with the same
signs, level bakes bit-exact in double precision and within one i16 step in the mixed
form, and a batch of the three gives each the bake it gets alone. The ball and the
ring have one face and no edges or vertices at all.
"""
import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

TOL = 1e-9  # x diagonal
R0, HEIGHT, ANGLE = 2.0, 4.0, np.radians(20.0)


def ball_sdf(p, r=3.0):
    return np.linalg.norm(p, axis=1) - r


def ring_sdf(p, major=4.0, minor=1.5):
    return np.sqrt((np.hypot(p[:, 0], p[:, 1]) - major) ** 2 + p[:, 2] ** 2) - minor


def frustum_sdf(p):
    """Nearest of the bottom disc, the cone's side line and the top disc in the
    (radius, height) half-plane; inside between the discs and under the side."""
    q = np.stack([np.hypot(p[:, 0], p[:, 1]), p[:, 2]], 1)
    r1 = R0 + HEIGHT * np.tan(ANGLE)
    corners = np.array([[0.0, 0.0], [R0, 0.0], [r1, HEIGHT], [0.0, HEIGHT]])

    def seg(a, b):
        ab = b - a
        t = np.clip(((q - a) @ ab) / (ab @ ab), 0.0, 1.0)
        return np.linalg.norm(q - (a + t[:, None] * ab), axis=1)

    d = np.min([seg(corners[i], corners[i + 1]) for i in range(3)], axis=0)
    inside = (q[:, 1] > 0) & (q[:, 1] < HEIGHT) & (q[:, 0] < R0 + q[:, 1] * np.tan(ANGLE))
    return np.where(inside, -d, d)


KINDS = {
    "frustum": (parts.frustum, frustum_sdf, 0.125),
    "ball": (parts.ball, ball_sdf, 0.125),
    "ring": (parts.ring, ring_sdf, 0.125),
}


def sample(o, seed, n=4000, pad=2.0):
    lo, hi = o.bbox()
    return np.random.default_rng(seed).uniform(lo - pad, hi + pad, size=(n, 3))


@pytest.mark.parametrize("name", sorted(KINDS))
def test_oracle_closed_form(oracle_mod, name):
    make, closed, _ = KINDS[name]
    o = oracle_mod.Oracle(make())
    p = sample(o, 11)
    assert np.abs(o.sdf(p)[0] - closed(p)).max() < 1e-12


_cache = {}


def setup(name, oracle_mod):
    if name not in _cache:
        solid = KINDS[name][0]()
        o = oracle_mod.Oracle(solid)
        lo, hi = o.bbox()
        _cache[name] = (part_gpu.PartGpu(solid), o, lo, hi, float(np.linalg.norm(hi - lo)))
    return _cache[name]


@pytest.fixture(scope="module")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def level_of(o, lo, hi, h):
    l2 = lo - 2.0
    nb = np.ceil((hi - lo + 4.0) / (8 * h)).astype(np.int64)
    return l2, nb


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(KINDS))
def test_points(cuda, oracle_mod, name):
    g, o, lo, hi, diag = setup(name, oracle_mod)
    p = np.concatenate([sample(o, 5), np.zeros((1, 3)), np.asarray(hi)[None, :]])
    v, f = g.points(p)
    d = o.sdf(p)[0]
    assert (f == 0).all()
    assert np.abs(v - d).max() <= TOL * diag
    assert np.abs(v - KINDS[name][1](p)).max() <= TOL * diag
    off = np.abs(d) > 1e-9
    assert (np.sign(v[off]) == np.sign(d[off])).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(KINDS))
def test_level_bit_exact(cuda, oracle_mod, name):
    from test_gpu_parity import oracle_level

    g, o, lo, hi, diag = setup(name, oracle_mod)
    h = KINDS[name][2]
    l2, nb = level_of(o, lo, hi, h)
    clamp = h * np.sqrt(3)
    m, a, st = g.level(h, l2, nb, clamp)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, l2, nb, clamp)
    assert st["nodes_undecided"] == 0
    assert (m == om).all()
    assert a.shape == oa.shape and (a == oa).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(KINDS))
def test_mixed_level(cuda, oracle_mod, name):
    from test_gpu_parity import oracle_level

    g, o, lo, hi, diag = setup(name, oracle_mod)
    h = KINDS[name][2]
    l2, nb = level_of(o, lo, hi, h)
    m, a, st = g.level(h, l2, nb, 1.0, precision=part_gpu.MIXED)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, l2, nb, 1.0)
    assert (m == om).all()
    qg = part_gpu.unpack_atlas(a).astype(np.int64)
    qo = part_gpu.unpack_atlas(oa).astype(np.int64)
    assert qg.shape == qo.shape and np.abs(qg - qo).max() <= 1
    assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()


@pytest.mark.gpu
def test_batch_of_the_three(cuda, oracle_mod):
    names = sorted(KINDS)
    gs, levels = [], []
    for name in names:
        g, o, lo, hi, diag = setup(name, oracle_mod)
        h = KINDS[name][2]
        l2, nb = level_of(o, lo, hi, h)
        gs.append(g)
        levels.append((h, l2, nb, h * np.sqrt(3)))
    b = part_gpu.Batch(gs)
    try:
        st, res = b.bake(levels, precision=part_gpu.FP64)
        assert st["parts"] == 3 and st["nodes_undecided"] == 0
        for g, L, (m, a) in zip(gs, levels, res):
            m1, a1, _ = g.level(*L)
            assert np.array_equal(m, m1) and np.array_equal(a, a1)
    finally:
        b.close()
