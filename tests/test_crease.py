"""A crease inside a B-spline face (parts.ridge_box: a top folded along a knot of full
multiplicity, the reference's C0 knot line, crates/icam-core/src/solid3.rs:1821-1886).

CPU: the oracle's distances equal the closed form of the folded top (two planes meeting
at the ridge) above it, where the ridge itself is the nearest point, and below it inside
the solid; on a top that also waves along the ridge, they never exceed a dense sampling of
the top and equal it within the sampling where the top is nearest. B200: the library's
points agree with the oracle within 1e-9 of the diagonal with equal signs, and its levels
over the ridge are the oracle's (FP64 bit for bit; mixed within one i16 step, no sign flip).
"""
import numpy as np
import pytest

from implicitcam_b200 import parts

FOLD, SIZE, BASE = 0.3, 30.0, 13.0


def top(x):
    return BASE - FOLD * np.abs(x - SIZE / 2)


def tent_distance(x, z):
    """Distance in the (x, z) plane to the folded top's two segments."""
    a = np.array([[0.0, top(0.0)], [SIZE / 2, BASE], [SIZE, top(SIZE)]])
    best = np.full(len(x), np.inf)
    for p, q in ((a[0], a[1]), (a[1], a[2])):
        ab = q - p
        t = np.clip(((x - p[0]) * ab[0] + (z - p[1]) * ab[1]) / ab.dot(ab), 0.0, 1.0)
        best = np.minimum(best, np.hypot(x - p[0] - t * ab[0], z - p[1] - t * ab[1]))
    return best


@pytest.mark.parametrize("n", [7, 11])
def test_ridge_is_the_closed_form(oracle_mod, n):
    o = oracle_mod.Oracle(parts.ridge_box(fold=FOLD, size=SIZE, base=BASE, n=n))
    rng = np.random.default_rng(n)
    x, y = rng.uniform(3, 27, 3000), rng.uniform(8, 22, 3000)
    z = top(x) + rng.uniform(0.05, 4.0, 3000)  # above: the ridge nearest in a wedge over it
    d = o.sdf(np.stack([x, y, z], 1))[0]
    assert np.abs(d - tent_distance(x, z)).max() < 1e-9
    near = np.abs(x - SIZE / 2) < FOLD * (z - BASE)  # in the ridge's wedge
    assert near.sum() > 100
    xi, yi = rng.uniform(6, 24, 3000), rng.uniform(8, 22, 3000)
    zi = top(xi) - rng.uniform(0.05, 3.0, 3000)
    di = o.sdf(np.stack([xi, yi, zi], 1))[0]
    closed = -np.minimum.reduce([tent_distance(xi, zi), zi, xi, SIZE - xi, yi, SIZE - yi])
    assert np.abs(di - closed).max() < 1e-9


def test_waved_ridge_against_a_sampled_top(oracle_mod):
    from scipy.spatial import cKDTree

    b = parts.ridge_box(fold=FOLD, size=SIZE, base=BASE, wave=1.5, n=9)
    o = oracle_mod.Oracle(b)
    nets = np.concatenate([np.asarray(p).reshape(-1, 4, 4, 4) for p in b.patches])
    t = np.linspace(0.0, 1.0, 61)
    bern = np.stack([(1 - t) ** 3, 3 * t * (1 - t) ** 2, 3 * t ** 2 * (1 - t), t ** 3], 1)
    s = np.einsum("ai,bj,nijk->nabk", bern, bern, nets)
    tree = cKDTree((s[..., :3] / s[..., 3:]).reshape(-1, 3))
    rng = np.random.default_rng(2)
    q = np.stack([rng.uniform(4, 26, 3000), rng.uniform(6, 24, 3000), rng.uniform(14.6, 18.0, 3000)], 1)  # above the top (at most 14.5)
    d = o.sdf(q)[0]
    ds, _ = tree.query(q)
    assert (d > 0).all()
    assert (d <= ds + 1e-9).all()
    assert (ds - d).max() < 0.05  # spans of ~5 mm sampled 60 times


@pytest.mark.gpu
def test_ridge_on_the_gpu(oracle_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from implicitcam_b200 import part_gpu

    b = parts.ridge_box(fold=FOLD, size=SIZE, base=BASE, wave=1.5, n=9)
    o = oracle_mod.Oracle(b)
    lo, hi = map(np.asarray, o.bbox())
    diag = float(np.linalg.norm(hi - lo))
    h, clamp = 0.2, 1.0
    g = part_gpu.PartGpu(b, need=clamp + 4 * h * np.sqrt(3))
    try:
        rng = np.random.default_rng(5)
        p = np.stack([rng.uniform(-2, 32, 20000), rng.uniform(-2, 32, 20000), rng.uniform(-2, 20, 20000)], 1)
        p[:5000, 0] = SIZE / 2 + rng.uniform(-1.0, 1.0, 5000)  # about the ridge
        p[:5000, 2] = BASE + rng.uniform(-1.5, 2.0, 5000)
        v, f = g.points(p)
        d = o.sdf(p)[0]
        assert (f == 0).all()
        assert np.abs(v - d).max() < 1e-9 * diag
        assert (np.sign(v[np.abs(d) > 1e-9]) == np.sign(d[np.abs(d) > 1e-9])).all()
        l2 = lo - clamp
        nb = np.ceil((hi - lo + 2 * clamp) / (8 * h)).astype(np.int64)
        om, idx, _ = o.decide(h, l2, nb, clamp)
        idx = np.sort(idx)
        firsts = np.stack([l2[0] + 8 * h * (idx % nb[0]), l2[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                           l2[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
        _, _, kind, words = o.bricks(firsts, h, clamp)
        m0 = om.copy()
        atlas = []
        for j, bi in enumerate(idx):
            m0[bi] = part_gpu.AIR if kind[j] == 1 else (part_gpu.SOLID if kind[j] == 2 else len(atlas))
            if kind[j] == 0:
                atlas.append(words[j])
        oa = np.array(atlas, dtype=np.uint32).reshape(-1, 365)
        m, a, st = g.level(h, l2, nb, clamp, precision=part_gpu.FP64)
        assert st["nodes_undecided"] == 0
        assert (m == m0).all() and a.shape == oa.shape and (a == oa).all()
        m2, a2, _ = g.level(h, l2, nb, clamp, precision=part_gpu.MIXED)
        assert (m2 == m0).all()
        qg, qo = part_gpu.unpack_atlas(a2).astype(np.int64), part_gpu.unpack_atlas(oa).astype(np.int64)
        assert np.abs(qg - qo).max() <= 1
        assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()
    finally:
        g.close()
