"""The batch workload's part families (parts.freeform_patches, parts.bodies_on_plate).

CPU: a freeform top cut along its knot lines into many B-spline faces is the same solid
as the top left whole (the oracle's distances agree to rounding, degree 2 and 3); a
dome's apex and a boss's cap on their plate are where their closed forms put them.
B200: the library's levels of a many-faced freeform top and of bosses and domes on a
plate are the oracle's (FP64 bit for bit; mixed within one i16 step, no sign flip).
"""
import numpy as np
import pytest

from implicitcam_b200 import parts


@pytest.mark.parametrize("degree,n,faces", [(3, 12, 4), (2, 9, 7), (3, 20, 17)])
def test_cut_top_is_the_whole_top(oracle_mod, degree, n, faces):
    kw = dict(seed=7, n=n, size=60.0, base=20.0, bumps=4, degree=degree)
    cut = parts.freeform_patches(faces=faces, **kw)
    whole = parts.freeform_patches(faces=1, **kw)
    assert cut.desc().n_faces == min(faces, n - degree) ** 2 + 5
    rng = np.random.default_rng(degree)
    p = rng.uniform([-3, -3, -3], [63, 63, 35], (3000, 3))
    a = oracle_mod.Oracle(cut).sdf(p)[0]
    b = oracle_mod.Oracle(whole).sdf(p)[0]
    assert np.abs(a - b).max() < 1e-11
    assert (np.sign(a) == np.sign(b)).all()


@pytest.mark.parametrize("kind", ["boss", "dome"])
def test_bodies_on_a_plate(oracle_mod, kind):
    b = parts.bodies_on_plate(seed=2, kind=kind, count=3, plate=(40.0, 14.0, 5.0))
    assert b.desc().n_faces == 6 + (3 if kind == "boss" else 2) * 3
    o = oracle_mod.Oracle(b)
    rng = np.random.default_rng(1)
    inside = rng.uniform([0.5, 0.5, 0.5], [39.5, 13.5, 4.5], (500, 3))
    assert (o.sdf(inside)[0] < 0).all()
    # straight above each body's axis the nearest point is its top: a cap plane (boss)
    # or the hemisphere's pole (dome), at the body's highest point
    top = o.bbox()[1][2]
    for cx in (40.0 * (k + 0.5) / 3 for k in range(3)):
        q = np.array([[cx, 7.0, top + 3.0]])
        d = o.sdf(q)[0][0]
        assert d > 0
        zt = top + 3.0 - d  # the body's top under the point
        assert zt <= top + 1e-9
    q = np.array([[40.0 * 0.5 / 3, 7.0, 30.0]])
    near = o.sdf(np.array([[40.0 * 0.5 / 3, 7.0, 5.0 + 1e-3]]))[0][0]
    assert near < 0  # just above the plate, inside the first body
    assert o.sdf(q)[0][0] > 0


def _oracle_level(o, h, lo, nb, clamp):
    from implicitcam_b200 import part_gpu

    om, idx, _ = o.decide(h, lo, nb, clamp)
    idx = np.sort(idx)
    m = om.copy()
    atlas = []
    if len(idx):
        firsts = np.stack([lo[0] + 8 * h * (idx % nb[0]), lo[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                           lo[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
        _, _, kind, words = o.bricks(firsts, h, clamp)
        for j, bi in enumerate(idx):
            m[bi] = part_gpu.AIR if kind[j] == 1 else (part_gpu.SOLID if kind[j] == 2 else len(atlas))
            if kind[j] == 0:
                atlas.append(words[j])
    return m, np.array(atlas, dtype=np.uint32).reshape(-1, 365)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["freeform_patches", "bosses", "domes"])
def test_family_levels_on_the_gpu(oracle_mod, name):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from implicitcam_b200 import part_gpu

    if name == "freeform_patches":
        b, h, clamp = parts.freeform_patches(seed=11, n=14, size=40.0, base=15.0, bumps=5, degree=2, faces=6), 0.25, 1.0
    else:
        b = parts.bodies_on_plate(seed=5, kind=name[:-2] if name == "bosses" else "dome", count=2,
                                  plate=(24.0, 12.0, 4.0))
        h, clamp = 0.2, 0.2 * np.sqrt(3)
    o = oracle_mod.Oracle(b)
    lo, hi = map(np.asarray, o.bbox())
    lo = lo - clamp
    nb = np.ceil((hi - lo + clamp) / (8 * h)).astype(np.int64)
    om, oa = _oracle_level(o, h, lo, nb, clamp)
    g = part_gpu.PartGpu(b, need=clamp + 4 * h * np.sqrt(3))
    try:
        m, a, st = g.level(h, lo, nb, clamp, precision=part_gpu.FP64)
        assert st["nodes_undecided"] == 0
        assert (m == om).all() and a.shape == oa.shape and (a == oa).all()
        m2, a2, _ = g.level(h, lo, nb, clamp, precision=part_gpu.MIXED)
        assert (m2 == om).all()
        qg = part_gpu.unpack_atlas(a2).astype(np.int64)
        qo = part_gpu.unpack_atlas(oa).astype(np.int64)
        assert np.abs(qg - qo).max() <= 1
        assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()
    finally:
        g.close()
