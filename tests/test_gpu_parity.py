"""The CUDA library against the oracle and the golden vectors, on a B200.

Tolerances: signed distances in double precision agree within 1e-9 of the part's box
diagonal (the bar for the plain FP64 kernel); signs, flags, the brick map
and every packed atlas word agree exactly.
"""
import os

import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-9  # x diagonal


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


_cache = {}


def setup(name, oracle_mod, need=2.0):
    key = (name, need)
    if key not in _cache:
        b = parts.CONFIGS[name]()
        g = part_gpu.PartGpu(b, need=need)
        o = oracle_mod.Oracle(b)
        lo, hi = o.bbox()
        _cache[key] = (b, g, o, lo, hi, float(np.linalg.norm(hi - lo)))
    return _cache[key]


PARTS = ["can", "block_with_hole", "bump_box", "freeform_top"]


@pytest.mark.parametrize("name", ["can", "bump_box", "block_with_hole"])
def test_points_against_golden(torch_cuda, oracle_mod, name):
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    gold = np.load(os.path.join(GOLDEN, name + ".npz"))
    v, f = g.points(gold["points"])
    assert (f == 0).all()
    if name == "bump_box":
        assert ((v < 0) == gold["inside"]).all()
        assert (np.abs(v) <= gold["dense"] + 1e-9).all()
        assert (np.abs(v) >= gold["dense"] - float(gold["h"])).all()
    else:
        assert np.abs(v - gold["sdf"]).max() < 1e-9


@pytest.mark.parametrize("name", PARTS)
def test_points_against_oracle(torch_cuda, oracle_mod, name):
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    rng = np.random.default_rng(7)
    p = rng.uniform(lo - 10, hi + 10, size=(5000, 3))
    v, f = g.points(p)
    d = o.sdf(p)[0]
    assert (f == 0).all(), np.bincount(f)
    assert np.abs(v - d).max() <= TOL * diag
    assert (np.sign(v) == np.sign(d)).all()


@pytest.mark.parametrize("name", PARTS)
def test_points_on_features(torch_cuda, oracle_mod, name):
    """Points on the part's grid, faces, edges and vertices (round numbers land on
    loop lines and planes): distances agree, and signs wherever |d| is not zero."""
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    verts = np.asarray(b.verts)
    axes = [np.unique(np.concatenate([verts[:, k], [lo[k], hi[k], 0.5 * (lo[k] + hi[k])]])) for k in range(3)]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    mids = 0.5 * (verts[:, None, :] + verts[None, :, :]).reshape(-1, 3)
    p = np.concatenate([grid, mids, verts, verts + 1e-3, verts - 1e-3])
    v, f = g.points(p)
    d = o.sdf(p)[0]
    assert (f == 0).all()
    assert np.abs(np.abs(v) - np.abs(d)).max() <= TOL * diag
    far = np.abs(d) > 1e-9
    assert (np.sign(v[far]) == np.sign(d[far])).all()


@pytest.mark.parametrize("name", ["block_with_hole", "freeform_top"])
def test_capped_points(torch_cuda, oracle_mod, name):
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    rng = np.random.default_rng(3)
    p = rng.uniform(lo - 5, hi + 5, size=(5000, 3))
    clamp = 1.5
    v, f = g.points(p, clamp=clamp, capped=True)
    d = o.sdf(p)[0]
    assert (f != 2).all()
    assert ((f == 1) == (np.abs(d) >= clamp)).sum() >= len(d) - 2  # ties at |d| == clamp aside
    ex = f == 0
    assert np.abs(v[ex] - d[ex]).max() <= TOL * diag
    assert (v[f == 1] == clamp).all()


def level_params(lo, hi, h, pad=2.0):
    l2 = lo - pad
    nb = np.ceil((hi - lo + 2 * pad) / (8 * h)).astype(np.int64)
    return l2, nb


def oracle_level(o, oracle_mod, h, lo, nb, clamp):
    om, idx, dc = o.decide(h, lo, nb, clamp)
    order = np.argsort(idx)
    idx = idx[order]
    firsts = np.stack([lo[0] + 8 * h * (idx % nb[0]), lo[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                       lo[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
    f, q, kind, words = o.bricks(firsts, h, clamp)
    m = om.copy()
    atlas = []
    for j, bi in enumerate(idx):
        if kind[j] == 1:
            m[bi] = part_gpu.AIR
        elif kind[j] == 2:
            m[bi] = part_gpu.SOLID
        else:
            m[bi] = len(atlas)
            atlas.append(words[j])
    return m, np.array(atlas, dtype=np.uint32).reshape(-1, 365), firsts, f


@pytest.mark.parametrize("name", PARTS)
@pytest.mark.parametrize("h", [1.0, 0.5])
def test_level_bit_exact(torch_cuda, oracle_mod, name, h):
    """The level's map and every atlas word as the oracle's bake gives them
    (PartCache::level with the reference's clamp, a cell's diagonal)."""
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    if name in ("can", "bump_box"):
        h = h / 4
    l2, nb = level_params(lo, hi, h)
    clamp = h * np.sqrt(3)
    m, a, st = g.level(h, l2, nb, clamp)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, l2, nb, clamp)
    assert st["nodes_undecided"] == 0
    assert (m == om).all()
    assert a.shape == oa.shape and (a == oa).all()


def test_level_narrow_band_bit_exact(torch_cuda, oracle_mod):
    """The freeform part with the bench's band (clamp 2 mm) at h = 0.5 mm."""
    b, g, o, lo, hi, diag = setup("freeform_top", oracle_mod)
    h = 0.5
    l2, nb = level_params(lo, hi, h)
    m, a, st = g.level(h, l2, nb, 2.0)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, l2, nb, 2.0)
    assert (m == om).all()
    assert a.shape == oa.shape and (a == oa).all()


def test_level_far_from_the_part_is_air(torch_cuda, oracle_mod):
    b, g, o, lo, hi, diag = setup("block_with_hole", oracle_mod)
    m, a, st = g.level(1.0, hi + 50.0, np.array([4, 3, 2]))
    assert (m == part_gpu.AIR).all() and len(a) == 0


def test_level_inside_the_solid_is_solid(torch_cuda, oracle_mod):
    b, g, o, lo, hi, diag = setup("block_with_hole", oracle_mod)
    # the block's slab between x = 5 and x = 30, away from the hole and the faces
    m, a, st = g.level(0.5, np.array([5.0, 5.0, 5.0]), np.array([5, 12, 7]))
    assert (m == part_gpu.SOLID).all() and len(a) == 0


def test_level_of_one_brick(torch_cuda, oracle_mod):
    b, g, o, lo, hi, diag = setup("block_with_hole", oracle_mod)
    lo1, nb1 = np.array([-0.5, -0.5, -0.5]), np.array([1, 1, 1])
    m, a, st = g.level(0.25, lo1, nb1)
    om, oa, _, _ = oracle_level(o, oracle_mod, 0.25, lo1, nb1, 0.25 * np.sqrt(3))
    assert (m == om).all() and (a == oa).all()


@pytest.mark.parametrize("name", ["block_with_hole", "freeform_top"])
def test_bricks_values(torch_cuda, oracle_mod, name):
    """PartGpu::bricks' contract: exact values within the clamp, flag 1 past it."""
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    h = 0.5
    l2, nb = level_params(lo, hi, h)
    clamp = h * np.sqrt(3)
    _, _, firsts, f = oracle_level(o, oracle_mod, h, l2, nb, clamp)
    sel = firsts[:: max(1, len(firsts) // 300)]
    fo = f[:: max(1, len(firsts) // 300)]
    vals, d = g.bricks(sel, h, clamp)
    flag = vals[:, :, 1]
    assert (flag != 2).all()
    ex = flag == 0
    assert np.abs(d[ex] - fo[ex]).max() <= TOL * diag
    assert (np.abs(fo[flag == 1]) >= clamp * (1 - 1e-12)).all()


def test_bad_arguments(torch_cuda, oracle_mod):
    b, g, o, lo, hi, diag = setup("block_with_hole", oracle_mod)
    with pytest.raises(part_gpu.IcamError):
        g.level(-1.0, lo, np.array([2, 2, 2]))
    with pytest.raises(part_gpu.IcamError):
        g.level(1.0, lo, np.array([0, 2, 2]))
    with pytest.raises(part_gpu.IcamError):
        g.points(np.zeros((1, 3)), precision=9)


def test_full_size_bake_properties(torch_cuda, oracle_mod):
    """The bench's workload (freeform part, h = 0.1 mm, band 2 mm, ~0.9M bricks read),
    checked by properties that hold whatever its size: no node left undecided, two
    bakes identical, a sample of stored bricks bit-exact against the oracle's
    exact_brick, a sample of air and material entries on the right side."""
    import bench

    b, lo, nb = bench.workload(0)
    g = part_gpu.PartGpu(b, need=bench.BAND + 8 * bench.H * np.sqrt(3))
    o = oracle_mod.Oracle(b)
    h, band = bench.H, bench.BAND
    m1, a1, st = g.level(h, lo, nb, band)
    m2, a2, _ = g.level(h, lo, nb, band)
    assert st["nodes_undecided"] == 0
    assert (m1 == m2).all() and (a1 == a2).all()
    rng = np.random.default_rng(11)
    stored = np.where(m1 < 0xFFFFFFF0)[0]
    pick = rng.choice(stored, 40, replace=False)
    firsts = np.stack([lo[0] + 8 * h * (pick % nb[0]), lo[1] + 8 * h * ((pick // nb[0]) % nb[1]),
                       lo[2] + 8 * h * (pick // (nb[0] * nb[1]))], 1)
    _, _, kind, words = o.bricks(firsts, h, band)
    assert (kind == 0).all()
    assert (words == a1[m1[pick]]).all()
    for val in (part_gpu.AIR, part_gpu.SOLID):
        ids = rng.choice(np.where(m1 == val)[0], 200, replace=False)
        c = np.stack([lo[0] + 8 * h * (ids % nb[0]), lo[1] + 8 * h * ((ids // nb[0]) % nb[1]),
                      lo[2] + 8 * h * (ids // (nb[0] * nb[1]))], 1) + 4 * h
        d = o.sdf(c)[0]
        assert ((d > 0) == (val == part_gpu.AIR)).all()
    g.close()


@pytest.mark.parametrize("name", ["block_with_hole", "bump_box", "freeform_top"])
def test_mixed_level(torch_cuda, oracle_mod, name):
    """The mixed-precision bake: the brick map (active set and AIR/SOLID signs) exactly
    the oracle's, every stored value within one i16 step, no sign flip."""
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    h = 0.5 if name != "bump_box" else 0.125
    l2, nb = level_params(lo, hi, h)
    clamp = 2.0 if name == "freeform_top" else h * np.sqrt(3)
    m, a, st = g.level(h, l2, nb, clamp, precision=part_gpu.MIXED)
    om, oa, _, _ = oracle_level(o, oracle_mod, h, l2, nb, clamp)
    assert st["nodes_undecided"] == 0
    assert (m == om).all()
    qg = part_gpu.unpack_atlas(a).astype(np.int64)
    qo = part_gpu.unpack_atlas(oa).astype(np.int64)
    assert np.abs(qg - qo).max() <= 1
    assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()


@pytest.mark.parametrize("name", ["block_with_hole", "freeform_top"])
def test_mixed_brick_values(torch_cuda, oracle_mod, name):
    """Values of the mixed kernel within 1e-7 of the diagonal of the oracle's."""
    b, g, o, lo, hi, diag = setup(name, oracle_mod)
    h = 0.5
    l2, nb = level_params(lo, hi, h)
    clamp = 2.0
    _, _, firsts, f = oracle_level(o, oracle_mod, h, l2, nb, clamp)
    sel = firsts[:: max(1, len(firsts) // 300)]
    fo = f[:: max(1, len(firsts) // 300)]
    vals, d = g.bricks(sel, h, clamp, precision=part_gpu.MIXED)
    flag = vals[:, :, 1]
    ex = flag == 0
    assert (flag != 2).all()
    assert np.abs(d[ex] - fo[ex]).max() <= 1e-7 * diag
    assert (np.abs(fo[flag == 1]) >= clamp * (1 - 1e-12)).all()
