"""Cones, spheres and tori: the analytic surface kinds the other parts lack, alone
(frustum, ball, ring) and in the analytic families of a batch (a boss with a torus
fillet, a block with a countersunk hole, a spherical dome).

The oracle is pinned to closed forms first (CPU): a ball's |p| - r, a ring's torus
distance, the solids of revolution's distance in their (radius, height) half-plane,
and the countersunk block's distance face by face. On a B200 the library then agrees
with the oracle: points within 1e-9 of the diagonal with the same signs, level bakes
bit-exact in double precision and within one i16 step in the mixed form, and a batch
of them gives each the bake it gets alone. The ball and the ring have one face and no
edges or vertices at all.
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


def _seg(q, a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    ab = b - a
    t = np.clip(((q - a) @ ab) / (ab @ ab), 0.0, 1.0)
    return np.linalg.norm(q - (a + t[:, None] * ab), axis=1)


def _arc(q, c, rad, a0, a1):
    """Distance to the arc of centre c and radius rad over angles [a0, a1]."""
    d = q - np.asarray(c, float)
    ang = np.arctan2(d[:, 1], d[:, 0])
    on = np.abs(np.linalg.norm(d, axis=1) - rad)
    e0 = np.linalg.norm(d - rad * np.array([np.cos(a0), np.sin(a0)]), axis=1)
    e1 = np.linalg.norm(d - rad * np.array([np.cos(a1), np.sin(a1)]), axis=1)
    return np.where((ang >= a0) & (ang <= a1), on, np.minimum(e0, e1))


def _rz(p):
    return np.stack([np.hypot(p[:, 0], p[:, 1]), p[:, 2]], 1)


def boss_sdf(p, r=3.0, h=5.0, f=1.0):
    q = _rz(p)
    d = np.min([_seg(q, [0, 0], [r, 0]), _seg(q, [r, 0], [r, h - f]), _arc(q, [r - f, h - f], f, 0, np.pi / 2),
                _seg(q, [r - f, h], [0, h])], axis=0)
    rho, z = q[:, 0], q[:, 1]
    fil = (rho < r - f) | ((rho - (r - f)) ** 2 + (z - (h - f)) ** 2 < f * f)
    inside = (z > 0) & (((z <= h - f) & (rho < r)) | ((z > h - f) & (z < h) & fil))
    return np.where(inside, -d, d)


def dome_sdf(p, r=3.0, h=4.0):
    q = _rz(p)
    d = np.min([_seg(q, [0, 0], [r, 0]), _seg(q, [r, 0], [r, h]), _arc(q, [0, h], r, 0, np.pi / 2)], axis=0)
    rho, z = q[:, 0], q[:, 1]
    inside = (z > 0) & (((z <= h) & (rho < r)) | ((z > h) & (rho ** 2 + (z - h) ** 2 < r * r)))
    return np.where(inside, -d, d)


def countersunk_sdf(p, X=40.0, Y=30.0, Z=20.0, cx=20.0, cy=15.0, r=4.0, sink=2.0, ang=np.radians(45.0)):
    """The nearest of the eight trimmed faces: the top and bottom rectangles less their
    discs, the four sides, the hole's wall and the countersink's cone."""
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    rt, zm = r + sink * np.tan(ang), Z - sink
    rho = np.hypot(x - cx, y - cy)

    def rect(u, v, U, V):
        du = np.maximum(np.maximum(-u, u - U), 0)
        dv = np.maximum(np.maximum(-v, v - V), 0)
        return np.hypot(du, dv), (u >= 0) & (u <= U) & (v >= 0) & (v <= V)

    def holed(dz, hole_r):
        d2, inr = rect(x, y, X, Y)
        return np.hypot(dz, np.where(inr & (rho < hole_r), hole_r - rho, d2))

    faces = [holed(z, r), holed(z - Z, rt)]
    for coord, val, u, U in ((y, 0, x, X), (y, Y, x, X), (x, 0, y, Y), (x, X, y, Y)):
        faces.append(np.hypot(coord - val, rect(u, z, U, Z)[0]))
    q = np.stack([rho, z], 1)
    faces += [_seg(q, [r, 0], [r, zm]), _seg(q, [r, zm], [rt, Z])]
    d = np.min(faces, axis=0)
    hole_r = np.where(z < zm, r, r + (z - zm) * np.tan(ang))
    inside = (x > 0) & (x < X) & (y > 0) & (y < Y) & (z > 0) & (z < Z) & (rho > hole_r)
    return np.where(inside, -d, d)


KINDS = {
    "frustum": (parts.frustum, frustum_sdf, 0.125),
    "ball": (parts.ball, ball_sdf, 0.125),
    "ring": (parts.ring, ring_sdf, 0.125),
    "boss": (parts.boss, boss_sdf, 0.125),
    "dome": (parts.dome, dome_sdf, 0.125),
    "countersunk_block": (parts.countersunk_block, countersunk_sdf, 0.25),
}


def sample(o, seed, n=4000, pad=2.0):
    lo, hi = o.bbox()
    return np.random.default_rng(seed).uniform(lo - pad, hi + pad, size=(n, 3))


def near_features(name, seed, n=4000):
    """Points crowded about the curved faces' edges (the fillet, the countersink)."""
    rng = np.random.default_rng(seed)
    if name == "countersunk_block":
        return rng.uniform([12.0, 7.0, 14.0], [28.0, 23.0, 22.0], size=(n, 3))
    if name == "boss":
        return rng.uniform([-4.0, -4.0, 3.0], [4.0, 4.0, 6.0], size=(n, 3))
    return np.zeros((0, 3))


@pytest.mark.parametrize("name", sorted(KINDS))
def test_oracle_closed_form(oracle_mod, name):
    make, closed, _ = KINDS[name]
    o = oracle_mod.Oracle(make())
    p = np.concatenate([sample(o, 11), near_features(name, 12)])
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
    p = np.concatenate([sample(o, 5), near_features(name, 6), np.zeros((1, 3)), np.asarray(hi)[None, :]])
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
def test_batch_of_the_analytic_parts(cuda, oracle_mod):
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
        assert st["parts"] == len(names) and st["nodes_undecided"] == 0
        for g, L, (m, a) in zip(gs, levels, res):
            m1, a1, _ = g.level(*L)
            assert np.array_equal(m, m1) and np.array_equal(a, a1)
    finally:
        b.close()
