"""One level baked by several ranks (implicitcam_b200/shard.py): the plan covers the level
with disjoint boxes; ranks baking their boxes and exchanging them assemble the map and
atlas of one bake of the whole level, bit for bit.

CPU: the ranks are gloo processes whose boxes the f64 oracle bakes (its decision of the
box's level, then every brick it reads, as PartCache::level does, partcache.rs:433-506),
checked against the oracle's bake of the whole level. GPU: the boxes of a 4-rank plan
baked one after another by the CUDA library on one device and assembled, checked against
the library's bake of the whole level (the exchange is the CPU test's)."""
import os
import socket

import numpy as np
import pytest

from implicitcam_b200 import parts, shard

AIR, SOLID = 0xFFFFFFFF, 0xFFFFFFFE


def oracle_bake(o, h, lo, nb, clamp, origin=None):
    """The oracle's level: (map u32, atlas slots x 365 u32)."""
    m, idx, _ = o.decide(h, lo, nb, clamp, origin=origin)
    idx = np.sort(idx)
    m = m.copy()
    atlas = []
    if len(idx):
        firsts = np.stack([lo[0] + 8 * h * (idx % nb[0]), lo[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                           lo[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
        _, _, kind, words = o.bricks(firsts, h, clamp)
        for j, bi in enumerate(idx):
            m[bi] = AIR if kind[j] == 1 else (SOLID if kind[j] == 2 else len(atlas))
            if kind[j] == 0:
                atlas.append(words[j])
    return m, np.array(atlas, dtype=np.uint32).reshape(-1, 365)


def level_of(name, h, clamp=None):
    b = getattr(parts, name)()
    import icam_oracle

    o = icam_oracle.Oracle(b)
    lo, hi = map(np.asarray, o.bbox())
    clamp = h * np.sqrt(3.0) if clamp is None else clamp
    l2 = lo - clamp
    nb = np.ceil((hi - lo + 2 * clamp) / (8 * h)).astype(np.int64)
    return b, o, l2, nb, clamp


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7, 8, 64])
def test_plan_covers_the_level_once(world):
    """Every brick in exactly one box; the weight split near evenly when the tiles allow."""
    rng = np.random.default_rng(world)
    nb = np.array([37, 21, 13])
    size, start, dims = shard.tile_grid(0.1, np.zeros(3), nb, origin=np.array([0.35, -0.2, 0.05]))
    assert size == 8 and (start <= 0).all() and (start > -8).all()
    w = np.where(rng.random(dims[::-1]) < 0.3, 1.0, shard.EMPTY_WEIGHT)
    boxes = shard.plan(w, size, start, nb, world)
    assert len(boxes) == world
    cover = np.zeros(nb[::-1], np.int32)
    for b0, b1 in boxes:
        assert (b0 >= 0).all() and (b1 <= nb).all()
        if (b1 > b0).all():
            cover[b0[2]:b1[2], b0[1]:b1[1], b0[0]:b1[0]] += 1
    assert (cover == 1).all()


def test_boxes_assemble_to_the_level_on_one_process(oracle_mod):
    """Without an exchange: the oracle's bakes of a 5-box plan assembled equal its bake of
    the whole level (the block with a hole at h = 0.5 mm)."""
    import torch

    b, o, lo, nb, clamp = level_of("block_with_hole", 0.5)
    h = 0.5
    m, a = oracle_bake(o, h, lo, nb, clamp)
    size, start, dims = shard.tile_grid(h, lo, nb)
    w = shard.tile_weights(lambda p: o.sdf(p)[0], h, lo, nb, clamp)
    boxes = shard.plan(w, size, start, nb, 5)
    org = shard.level_origin(h, lo)
    maps, atlases = [], []
    for box in boxes:
        lo_r, nb_r = shard.sub_level(h, lo, box)
        if (nb_r > 0).all():
            mr, ar = oracle_bake(o, h, lo_r, nb_r, clamp, origin=org)
        else:
            mr, ar = np.zeros(0, np.uint32), np.zeros((0, 365), np.uint32)
        maps.append(torch.from_numpy(mr.view(np.int32).copy()))
        atlases.append(torch.from_numpy(ar.view(np.int32).copy()))
    M, A = shard.assemble(nb, boxes, maps, atlases)
    assert (M.numpy().astype(np.uint64) == m.astype(np.uint64)).all()
    assert A.shape == a.shape and (A.numpy().view(np.uint32) == a).all()
    assert len(a) > 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, h, clamp, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import icam_oracle

        icam_oracle.build()
        b, o, lo, nb, clamp = level_of(name, h, clamp)

        def bake_box(lo_r, nb_r, origin):
            mr, ar = oracle_bake(o, h, lo_r, nb_r, clamp, origin=origin)
            return torch.from_numpy(mr.view(np.int32).copy()), torch.from_numpy(ar.view(np.int32).copy())

        M, A, mine, boxes = shard.bake_sharded(dist, bake_box, lambda p: o.sdf(p)[0], h, lo, nb, clamp)
        out.put((rank, M.numpy().copy(), A.numpy().copy(), [(b0.tolist(), b1.tolist()) for b0, b1 in boxes]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,h,clamp,world", [("block_with_hole", 0.5, None, 2), ("bump_box", 0.125, 1.0, 2),
                                                ("block_with_hole", 1.0, None, 3)])
def test_ranks_bake_one_level_over_gloo(oracle_mod, name, h, clamp, world):
    """gloo ranks each bake their box with the oracle, exchange and assemble: every rank
    holds the oracle's map and atlas of the whole level."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, h, clamp, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    b, o, lo, nb, clamp = level_of(name, h, clamp)
    m, a = oracle_bake(o, h, lo, nb, clamp)
    for rank, M, A, boxes in got:
        assert (M.astype(np.uint64) == m.astype(np.uint64)).all()
        assert A.shape == a.shape and (A.view(np.uint32) == a).all()
        # every rank had bricks wherever the level has a tile for each
        size, start, dims = shard.tile_grid(h, lo, nb)
        busy = sum(1 for b0, b1 in boxes if all(x < y for x, y in zip(b0, b1)))
        assert busy == min(world, int(np.prod(dims)))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_boxes_baked_on_the_gpu_assemble_to_its_level(oracle_mod, precision):
    """The freeform part at h = 0.25 mm, band 2 mm: the CUDA library's bakes of a 4-box
    plan's boxes, assembled on the device, equal its bake of the whole level (map and
    atlas, FP64 and mixed)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from implicitcam_b200 import part_gpu

    b, o, lo, nb, clamp = level_of("freeform_top", 0.25, 2.0)
    h = 0.25
    g = part_gpu.PartGpu(b, need=clamp + 4 * h * np.sqrt(3))
    try:
        m, a, _ = g.level(h, lo, nb, clamp, precision=precision)
        size, start, dims = shard.tile_grid(h, lo, nb)
        w = shard.tile_weights(lambda p: g.points(p)[0], h, lo, nb, clamp)
        boxes = shard.plan(w, size, start, nb, 4)
        org = shard.level_origin(h, lo)
        maps, atlases = [], []
        for box in boxes:
            lo_r, nb_r = shard.sub_level(h, lo, box)
            mr, ar = g.level_torch(h, lo_r, nb_r, clamp, origin=org, precision=precision)
            maps.append(mr)
            atlases.append(ar)
        M, A = shard.assemble(nb, boxes, maps, atlases)
        assert M.is_cuda and A.is_cuda
        assert (M.cpu().numpy().astype(np.uint64) == m.astype(np.uint64)).all()
        assert tuple(A.shape) == a.shape and (A.cpu().numpy().view(np.uint32) == a).all()
        assert sum(1 for b0, b1 in boxes if (b1 > b0).all()) == 4
    finally:
        g.close()
