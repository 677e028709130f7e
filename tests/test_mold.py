"""The mold cavity (parts.mold): 630 faces, 500 of them B-spline faces of 8 x 8 to
24 x 24 control points (5 to 21 spans a side) cut from the pocket's floor and joined along
shared B-spline edges, and 40 filleted bosses on the rim.

CPU: the oracle's distances over the rim's material away from the pocket's corners and
the bosses are the closed form (the nearest of six planes), and over the pocket never
exceed the distance to a dense sampling of the floor (which they equal where the floor
is nearest). B200: points agree with the oracle within 1e-9 of the diagonal with equal
signs, and level bakes over a corner (floor faces, two walls, two bosses) and over the
floor's middle are bit-exact (FP64) and within one i16 step (mixed).
"""
import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

TOL = 1e-9  # x diagonal
X, Y, Z, RIM = 250.0, 200.0, 80.0, 25.0

_cache = {}


def solid_and_oracle(oracle_mod):
    if "o" not in _cache:
        b = parts.mold()
        _cache["b"], _cache["o"] = b, oracle_mod.Oracle(b)
    return _cache["b"], _cache["o"]


def boss_centres(count=40):
    half, px, py = RIM / 2, X - RIM, Y - RIM
    per = 2 * (px + py)
    out = []
    for k in range(count):
        t = (k + 0.5) * per / count
        if t < px:
            out.append((half + t, half))
        elif t < px + py:
            out.append((X - half, half + (t - px)))
        elif t < 2 * px + py:
            out.append((X - half - (t - px - py), Y - half))
        else:
            out.append((half, Y - half - (t - 2 * px - py)))
    return np.array(out)


def test_rim_is_the_closed_form(oracle_mod):
    b, o = solid_and_oracle(oracle_mod)
    rng = np.random.default_rng(3)
    q = np.concatenate([rng.uniform([2, 30, 62], [23, 170, 78], (800, 3)),
                        rng.uniform([30, 2, 62], [220, 23, 78], (800, 3))])
    far = np.min(np.linalg.norm(q[:, None, :2] - boss_centres()[None], axis=2), axis=1) > 8.0
    q = q[far]
    x, y, z = q.T
    wall = np.where(x < RIM, RIM - x, RIM - y)  # the pocket wall the point faces
    closed = -np.minimum.reduce([Z - z, x, X - x, y, Y - y, wall, z])
    assert np.abs(o.sdf(q)[0] - closed).max() < 1e-9


def test_pocket_against_a_sampled_floor(oracle_mod):
    from scipy.spatial import cKDTree

    b, o = solid_and_oracle(oracle_mod)
    nets = np.concatenate([p.reshape(-1, 4, 4, 4) for p in b.patches])
    t = np.linspace(0.0, 1.0, 6)  # spans of ~0.6 mm: samples ~0.12 mm apart
    bern = np.stack([(1 - t) ** 3, 3 * t * (1 - t) ** 2, 3 * t ** 2 * (1 - t), t ** 3], 1)
    s = np.einsum("ai,bj,nijk->nabk", bern, bern, nets)
    tree = cKDTree((s[..., :3] / s[..., 3:]).reshape(-1, 3))
    rng = np.random.default_rng(4)
    q = rng.uniform([45, 45, 20], [205, 155, 75], (2000, 3))
    d = o.sdf(q)[0]
    ds, _ = tree.query(q)
    assert (np.abs(d) <= ds + 1e-9).all()
    # above the floor and nearer to it than to any wall (the rim's top and the bosses lie
    # beyond the walls), the floor is the nearest feature: equal within the sampling's
    # spacing (spans of ~0.6 mm sampled 5 times, steeper than 1:1 in places: < 0.2 mm)
    x, y = q[:, 0], q[:, 1]
    walls = np.minimum.reduce([x - RIM, X - RIM - x, y - RIM, Y - RIM - y])
    up = (d > 0) & (ds < walls - 0.05)
    assert up.sum() > 500
    assert (ds[up] - d[up]).max() < 0.2


@pytest.fixture(scope="module")
def gpu(oracle_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    b, o = solid_and_oracle(oracle_mod)
    g = part_gpu.PartGpu(b)
    lo, hi = o.bbox()
    yield g, o, float(np.linalg.norm(hi - lo))
    g.close()


@pytest.mark.gpu
def test_points(gpu, oracle_mod):
    g, o, diag = gpu
    rng = np.random.default_rng(5)
    p = np.concatenate([rng.uniform([-5, -5, -5], [X + 5, Y + 5, 100], (3000, 3)),
                        rng.uniform([25, 25, 30], [225, 175, 60], (3000, 3)),  # about the floor
                        np.concatenate([boss_centres(), np.full((40, 1), 84.0)], 1)])
    v, f = g.points(p)
    d = o.sdf(p)[0]
    assert (f == 0).all()
    assert np.abs(v - d).max() <= TOL * diag
    off = np.abs(d) > 1e-9
    assert (np.sign(v[off]) == np.sign(d[off])).all()


BOXES = {  # (lo, nb) at h = 0.25: a pocket corner with two walls, floor faces and two bosses
    "corner": (np.array([8.0, 8.0, 28.0]), np.array([16, 14, 30])),
    # the floor's middle: junctions of several one-span faces
    "floor": (np.array([100.0, 80.0, 20.0]), np.array([8, 8, 25])),
}


@pytest.mark.gpu
@pytest.mark.parametrize("box", sorted(BOXES))
def test_level_bit_exact(gpu, oracle_mod, box):
    from test_gpu_parity import oracle_level

    g, o, diag = gpu
    lo, nb = BOXES[box]
    h, clamp = 0.25, 1.0
    m, a, st = g.level(h, lo, nb, clamp)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, lo, nb, clamp)
    assert st["nodes_undecided"] == 0
    assert (m == om).all()
    assert a.shape == oa.shape and (a == oa).all()


@pytest.mark.gpu
@pytest.mark.parametrize("box", sorted(BOXES))
def test_mixed_level(gpu, oracle_mod, box):
    from test_gpu_parity import oracle_level

    g, o, diag = gpu
    lo, nb = BOXES[box]
    h, clamp = 0.25, 1.0
    m, a, st = g.level(h, lo, nb, clamp, precision=part_gpu.MIXED)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, lo, nb, clamp)
    assert (m == om).all()
    qg = part_gpu.unpack_atlas(a).astype(np.int64)
    qo = part_gpu.unpack_atlas(oa).astype(np.int64)
    assert qg.shape == qo.shape and np.abs(qg - qo).max() <= 1
    assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()
