"""Batches (icam_batch_*): uneven parts baked together give every part the map and atlas
of baking it alone, bit for bit (FP64) and in the mixed form; a second bake of the same
levels replays the captured graph; the tiling is one the autotuner timed; one part may
be baked at two resolutions in one batch; a bad level is refused."""
import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

pytestmark = pytest.mark.gpu


def uneven_parts():
    """Planes, cylinders and rational B-spline tops of uneven sizes and face counts, and a
    cap of revolution with a pole at its apex (its level's nodes kept off the axis)."""
    return [
        (parts.can(), 0.25, 0.25 * np.sqrt(3)),
        (parts.block_with_hole(), 1.0, np.sqrt(3)),
        (parts.block_with_hole(size=(40.0, 30.0, 20.0), center=(15.0, 12.0), r=6.0), 0.5, 1.0),
        (parts.bump_box(), 0.125, 0.125 * np.sqrt(3)),
        (parts.freeform_top(seed=3, n=8, size=40.0, base=20.0, bumps=4), 0.25, 1.0),
        (parts.freeform_top(seed=5, n=12, size=60.0, base=30.0, bumps=6), 0.4, 2.0),
        (parts.nurbs_dome(3.0, 4.0, rise=2.0), 0.1, 0.5, 0.0371),
    ]


@pytest.fixture(scope="module")
def batch(oracle_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    spec = uneven_parts()
    gs, levels = [], []
    for solid, h, clamp, *shift in spec:
        g = part_gpu.PartGpu(solid)
        lo, hi = oracle_mod.Oracle(solid).bbox()
        lo2 = np.asarray(lo) - 2.0 - (shift[0] if shift else 0.0)
        nb = np.ceil((np.asarray(hi) - np.asarray(lo) + 4.0) / (8 * h)).astype(np.int64)
        gs.append(g)
        levels.append((h, lo2, nb, clamp))
    b = part_gpu.Batch(gs)
    yield b, gs, levels
    b.close()
    for g in gs:
        g.close()


@pytest.mark.parametrize("precision", [part_gpu.FP64, part_gpu.MIXED])
def test_batch_equals_parts_alone(batch, precision):
    b, gs, levels = batch
    st, res = b.bake(levels, precision=precision)
    assert st["parts"] == len(gs) and st["nodes_undecided"] == 0
    assert st["warps"] in (1, 2, 4)
    for g, L, (m, a) in zip(gs, levels, res):
        m1, a1, _ = g.level(*L, precision=precision)
        assert np.array_equal(m, m1)
        if precision == part_gpu.FP64:
            assert np.array_equal(a, a1)
        else:  # the float answers: the same within one i16 step, no sign flip
            q, q1 = part_gpu.unpack_atlas(a).astype(int), part_gpu.unpack_atlas(a1).astype(int)
            assert q.shape == q1.shape and np.abs(q - q1).max() <= 1
    # the same levels again: the graph is replayed and the answers repeat
    st2, res2 = b.bake(levels, precision=precision)
    assert st2["graph_replayed"] == 1
    for (m, a), (m2, a2) in zip(res, res2):
        assert np.array_equal(m, m2) and np.array_equal(a, a2)


def test_one_part_at_two_resolutions(batch):
    """The same pack twice in a batch, at two cell sizes: each level as baked alone."""
    b0, gs, levels = batch
    g = gs[1]
    h, lo, nb, clamp = levels[1]
    two = [(h, lo, nb, clamp), (h / 2, lo, 2 * nb, clamp / 2)]
    b = part_gpu.Batch([g, g])
    try:
        st, res = b.bake(two)
        assert st["parts"] == 2 and st["nodes_undecided"] == 0
        for L, (m, a) in zip(two, res):
            m1, a1, _ = g.level(*L)
            assert np.array_equal(m, m1) and np.array_equal(a, a1)
    finally:
        b.close()


def test_bad_levels_are_refused(batch):
    b, gs, levels = batch
    bad = list(levels)
    h, lo, nb, clamp = bad[2]
    bad[2] = (h, lo, np.array([nb[0], 0, nb[2]]), clamp)
    with pytest.raises(part_gpu.IcamError):
        b.bake(bad)
    st, _ = b.bake(levels)  # the batch still bakes
    assert st["parts"] == len(gs)
