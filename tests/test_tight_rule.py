"""The bake's box decision bounds a box by its own nodes' half diagonal.

The reference (partcache.rs:226-331) bounds a box of bricks by the half diagonal of the
box grown by the clamp. Every node of the box lies within its own nodes' half diagonal of
the centre, so a box that the tighter bound decides AIR (SOLID) holds only nodes past the
clamp: the reference reads those bricks and packs each as an AIR (SOLID) brick (on a
closed solid, whose signed distance changes by at most the distance moved). These CPU
tests run the oracle's decision under both bounds and read every brick each one lists:
the final maps and atlases are the same, and the tighter bound reads fewer bricks
(a freeform top, bosses, a creased ridge and a pointed pole).
"""
import numpy as np
import pytest

from implicitcam_b200 import parts

AIR, SOLID = 0xFFFFFFFF, 0xFFFFFFFE


def _final_level(o, h, lo, nb, clamp, tight):
    om, idx, _ = o.decide(h, lo, nb, clamp, tight=tight)
    idx = np.sort(idx)
    m = om.copy()
    atlas = []
    if len(idx):
        firsts = np.stack([lo[0] + 8 * h * (idx % nb[0]), lo[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                           lo[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
        _, _, kind, words = o.bricks(firsts, h, clamp)
        for j, bi in enumerate(idx):
            m[bi] = AIR if kind[j] == 1 else (SOLID if kind[j] == 2 else len(atlas))
            if kind[j] == 0:
                atlas.append(words[j])
    return m, np.array(atlas, dtype=np.uint32).reshape(-1, 365), len(idx)


def _bodies():
    yield "freeform_patches", parts.freeform_patches(seed=11, n=14, size=40.0, base=15.0, bumps=5, degree=2,
                                                     faces=6), 0.25, 1.0
    yield "bosses", parts.bodies_on_plate(seed=5, kind="boss", count=2, plate=(24.0, 12.0, 4.0)), 0.2, 0.2 * np.sqrt(3)
    yield "ridge", parts.ridge_box(fold=0.5, size=20.0, base=8.0, wave=0.4, n=7), 0.2, 0.6
    yield "pole", parts.nurbs_dome(3.0, 4.0, rise=2.0), 0.1, 0.5


@pytest.mark.parametrize("case", list(range(4)))
def test_tight_bound_gives_the_same_level(oracle_mod, case):
    name, b, h, clamp = list(_bodies())[case]
    o = oracle_mod.Oracle(b)
    lo, hi = map(np.asarray, o.bbox())
    lo = lo - clamp
    nb = np.ceil((hi - lo + clamp) / (8 * h)).astype(np.int64)
    m0, a0, n0 = _final_level(o, h, lo, nb, clamp, tight=False)
    m1, a1, n1 = _final_level(o, h, lo, nb, clamp, tight=True)
    assert (m0 == m1).all(), name
    assert a0.shape == a1.shape and (a0 == a1).all(), name
    assert n1 <= n0, name
    assert a0.shape[0] > 0, name
