"""The headline arm (mixed precision with the seed network's Newton starts) and the
headline level against the oracle, on a B200.

Tolerances, as the mixed form is bound to them: the brick map (the active set and
every air / material sign) exactly the oracle's; every stored i16 value within one
step of the oracle's and no value of the opposite sign; distances before quantisation
within 1e-7 of the part's box diagonal, with the sign of every exact node the
oracle's. The plain FP64 kernel: the map, the words and the signs exactly, distances
within 1e-9 of the diagonal.
"""
import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-7  # x diagonal


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


_cache = {}


def trained(name, oracle_mod, need=2.0):
    """The part packed, its seed network trained (a short run: the starts are checked
    by the solves they start, so a weaker net changes the work, not the answers)."""
    key = (name, need)
    if key not in _cache:
        b = parts.CONFIGS[name]()
        g = part_gpu.PartGpu(b, need=need)
        g.seednet_train(1500, batch=2048, seed=3, need=need)
        o = oracle_mod.Oracle(b)
        lo, hi = o.bbox()
        _cache[key] = (b, g, o, np.asarray(lo), np.asarray(hi), float(np.linalg.norm(np.asarray(hi) - lo)))
    return _cache[key]


def oracle_level(o, h, lo, nb, clamp):
    om, idx, dc = o.decide(h, lo, nb, clamp)
    idx = np.sort(idx)
    firsts = np.stack([lo[0] + 8 * h * (idx % nb[0]), lo[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                       lo[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
    f, q, kind, words = o.bricks(firsts, h, clamp)
    m = om.copy()
    atlas = []
    for j, bi in enumerate(idx):
        m[bi] = part_gpu.AIR if kind[j] == 1 else (part_gpu.SOLID if kind[j] == 2 else len(atlas))
        if kind[j] == 0:
            atlas.append(words[j])
    return m, np.array(atlas, dtype=np.uint32).reshape(-1, 365), firsts, f


@pytest.mark.parametrize("name", ["bump_box", "freeform_top"])
def test_learned_level(torch_cuda, oracle_mod, name):
    """The learned bake: map exactly the oracle's, words within one step, no sign flip."""
    b, g, o, lo, hi, diag = trained(name, oracle_mod)
    h = 0.5 if name == "freeform_top" else 0.125
    l2 = lo - 2.0
    nb = np.ceil((hi - lo + 4.0) / (8 * h)).astype(np.int64)
    clamp = 2.0 if name == "freeform_top" else h * np.sqrt(3)
    m, a, st = g.level(h, l2, nb, clamp, precision=part_gpu.MIXED_LEARNED)
    om, oa, _, _ = oracle_level(o, h, l2, nb, clamp)
    assert st["nodes_undecided"] == 0
    assert (m == om).all()
    qg = part_gpu.unpack_atlas(a).astype(np.int64)
    qo = part_gpu.unpack_atlas(oa).astype(np.int64)
    assert np.abs(qg - qo).max() <= 1
    assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()


@pytest.mark.parametrize("name", ["bump_box", "freeform_top"])
def test_learned_brick_values(torch_cuda, oracle_mod, name):
    """Node values of the learned kernel within 1e-7 of the diagonal of the oracle's,
    signs equal, flag 1 only past the clamp."""
    b, g, o, lo, hi, diag = trained(name, oracle_mod)
    h = 0.5 if name == "freeform_top" else 0.125
    l2 = lo - 2.0
    nb = np.ceil((hi - lo + 4.0) / (8 * h)).astype(np.int64)
    clamp = 2.0
    _, _, firsts, f = oracle_level(o, h, l2, nb, clamp)
    sel = firsts[:: max(1, len(firsts) // 300)]
    fo = f[:: max(1, len(firsts) // 300)]
    vals, d = g.bricks(sel, h, clamp, precision=part_gpu.MIXED_LEARNED)
    flag = vals[:, :, 1]
    ex = flag == 0
    assert (flag != 2).all()
    assert np.abs(d[ex] - fo[ex]).max() <= TOL_MIXED * diag
    # signs wherever the distance is above double rounding (a node on the surface up to
    # rounding has a sign of rounding; the reference's verify compares signs only past
    # the i16 step of zero, partcache.rs:536-538)
    nz = ex & (np.abs(fo) > 1e-9)
    bad = nz & (np.sign(d) != np.sign(fo))
    assert not bad.any(), (fo[bad][:5], d[bad][:5])
    assert (np.abs(fo[flag == 1]) >= clamp * (1 - 1e-12)).all()


@pytest.fixture(scope="module")
def headline(torch_cuda, oracle_mod):
    """The bench's level (freeform part, h = 0.1 mm, band 2 mm), its pack with the seed
    network trained as the bench trains it, and the oracle's decision of the level."""
    import bench

    b, lo, nb = bench.workload(0)
    need = bench.BAND + 8 * bench.H * np.sqrt(3)
    g = part_gpu.PartGpu(b, need=need)
    g.seednet_train(bench.SEEDNET_STEPS, batch=bench.SEEDNET_BATCH, seed=0, need=need)
    o = oracle_mod.Oracle(b)
    om, oidx, odc = o.decide(bench.H, lo, nb, bench.BAND)
    yield bench, g, o, lo, nb, (om, np.sort(oidx), odc)
    g.close()


@pytest.mark.parametrize("precision", [part_gpu.FP64, part_gpu.MIXED, part_gpu.MIXED_LEARNED])
def test_headline_decision_is_the_oracles(headline, precision):
    """The whole decision of the bench's level (~0.64M box centres, ~0.9M bricks to
    read): every map entry and the read set exactly the oracle's."""
    bench, g, o, lo, nb, (om, oidx, odc) = headline
    m, idx, dc, st = g.decide(bench.H, lo, nb, bench.BAND, precision=precision)
    assert len(idx) == len(oidx) and (idx == oidx).all()
    assert (m == om).all()


@pytest.mark.parametrize("precision", [part_gpu.FP64, part_gpu.MIXED_LEARNED])
def test_headline_level_against_the_oracle(headline, precision):
    """The bench's level baked, checked as the reference's verify checks a level: the
    decided entries exactly the oracle's decision, stored bricks only among the bricks
    it reads, sampled nodes (every 29th of 1000 stored bricks, every node within an i16
    step of zero) exact (FP64) or within one step (learned) with no sign flip, sampled
    distances within the form's tolerance."""
    bench, g, o, lo, nb, (om, oidx, odc) = headline
    m, a, st = g.level(bench.H, lo, nb, bench.BAND, precision=precision)
    assert st["nodes_undecided"] == 0
    r = bench.verify_against_oracle(g, o, part_gpu, lo, nb, bench.H, bench.BAND, precision, m, a, decision=om)
    diag = float(np.linalg.norm(np.asarray(o.bbox()[1]) - np.asarray(o.bbox()[0])))
    assert r["decided_entries_differ"] == 0 and r["stored_outside_read_set"] == 0
    assert r["air_solid_centres_wrong"] == 0
    assert r["sign_flips"] == 0 and r["distance_sign_flips"] == 0
    assert r["flags_undecided"] == 0 and r["flags_past_clamp_ok"]
    if precision == part_gpu.FP64:
        assert r["i16_max_step_diff"] == 0
        assert r["distance_max_over_diag"] <= 1e-9
    else:
        assert r["i16_max_step_diff"] <= 1
        assert r["distance_max_over_diag"] <= TOL_MIXED
    # the learned bake's map is the plain kernel's, entry for entry
    if precision != part_gpu.FP64:
        m64, _, _ = g.level(bench.H, lo, nb, bench.BAND, precision=part_gpu.FP64, atlas=False)
        assert (m == m64).all()
    assert diag > 0
