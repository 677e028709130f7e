"""One level of the brick cache baked by several GPUs, one process a GPU.

The reference bakes a level on one device (PartCache::level, crates/icam-sim/src/
partcache.rs:433-506). Here the level's bricks are cut into one box a rank:

- **Plan.** The level's bricks are grouped into tiles of the box decision's first boxes
  (S = 8 bricks a side, aligned on the level's origin grid as the decision aligns them,
  partcache.rs:250-259). A tile is weighted 1 when the surface may lie within its reach
  (its centre's distance within its half-diagonal plus the clamp: it may hold bricks to
  read) and `EMPTY_WEIGHT` otherwise (it is decided from one reading). The tiles are cut
  by a k-d bisection: the ranks are halved, the tile box is cut across its longest side
  where the weight splits in the same ratio, down to one rank a box. Every rank computes
  the same plan from the same centre distances.
- **Bake.** Each rank bakes its box as a level of its own, with the level's h, clamp and
  origin. A brick's entry does not depend on the boxes the decision reaches it through:
  its own reading decides it (a box that settles its bricks settles each of them as the
  brick's own reading would, its ball holding theirs), and a read brick's words are its
  nodes'. So the box's map and words are the level's restricted to the box.
- **Exchange.** One all-gather of the ranks' maps and one of their atlases (NCCL between
  GPUs; any torch.distributed backend), each padded to the largest rank's size.
- **Assembly.** Every rank places the maps into the level's map, numbers the stored
  bricks in the level's brick order (x fastest, partcache.rs:486) and gathers their words
  into an atlas in that order: the map and atlas of one GPU baking the whole level.

The functions are independent of how a box is baked (`bake_box`) and how a distance is
read (`distance`), so the same plan, exchange and assembly run over the CUDA library on
GPUs and over the oracle on CPU ranks (tests).
"""
from __future__ import annotations

import numpy as np

AIR, SOLID, READ = 0xFFFFFFFF, 0xFFFFFFFE, 0xFFFFFFF0
WORDS = 365
EMPTY_WEIGHT = 0.02  # a tile with no surface within reach: one box reading


def tile_grid(h, lo, nb, origin=None):
    """The decision's first boxes over the level (as the library's first_boxes):
    (S bricks a side, the first box's brick offset start[3] (<= 0), tiles a side dims[3])."""
    lo = np.asarray(lo, dtype=np.float64)
    nb = np.asarray(nb, dtype=np.int64)
    size = 1
    while size < int(nb.max()) and size < 8:
        size *= 2
    side = 8.0 * h
    o = lo if origin is None else np.asarray(origin, dtype=np.float64) - h
    start = np.zeros(3, np.int64)
    for k in range(3):
        g0 = int(round((lo[k] - o[k]) / side)) if origin is not None else 0
        q = g0 // size if g0 >= 0 else -((-g0 + size - 1) // size)
        start[k] = q * size - g0
    dims = (nb - start + size - 1) // size
    return size, start, dims


def tile_boxes(size, start, dims, nb):
    """Every tile's brick range, clipped to the level: (lo (n, 3), hi (n, 3)), tiles x fastest."""
    idx = np.stack(np.meshgrid(np.arange(dims[0]), np.arange(dims[1]), np.arange(dims[2]), indexing="ij"), -1)
    idx = idx.transpose(2, 1, 0, 3).reshape(-1, 3)  # x fastest
    b0 = np.maximum(start + size * idx, 0)
    b1 = np.minimum(start + size * (idx + 1), np.asarray(nb))
    return b0, b1


def tile_weights(distance, h, lo, nb, clamp, origin=None):
    """The tiles' weights (dims[2], dims[1], dims[0]) from their centres' signed
    distances (`distance`: (n, 3) points -> (n,) distances)."""
    size, start, dims = tile_grid(h, lo, nb, origin)
    b0, b1 = tile_boxes(size, start, dims, nb)
    lo = np.asarray(lo, dtype=np.float64)
    side = 8.0 * h
    c = lo + side * 0.5 * (b0 + b1)
    half = 0.5 * side * np.linalg.norm(b1 - b0, axis=1)
    d = np.asarray(distance(c), dtype=np.float64)
    w = np.where(np.abs(d) <= half + clamp, 1.0, EMPTY_WEIGHT)
    return w.reshape(dims[2], dims[1], dims[0])


def plan(weights, size, start, nb, world):
    """The ranks' brick boxes [(b0, b1)] (an empty box where a rank gets none), by k-d
    bisection of the tiles (weights indexed z, y, x) into `world` parts."""
    nb = np.asarray(nb, dtype=np.int64)
    dims = np.array(weights.shape[::-1], dtype=np.int64)
    out = [None] * world

    def split(t0, t1, ranks):
        if len(ranks) == 1:
            out[ranks[0]] = (t0, t1)
            return
        n1 = len(ranks) // 2
        ext = t1 - t0
        axis = int(np.argmax(ext))
        if ext[axis] <= 1:  # one tile left: the first rank takes it
            out[ranks[0]] = (t0, t1)
            for r in ranks[1:]:
                out[r] = (t0, t0.copy())
            return
        sub = weights[t0[2]:t1[2], t0[1]:t1[1], t0[0]:t1[0]]
        prof = sub.sum(axis=tuple(a for a in range(3) if a != 2 - axis))
        cum = np.cumsum(prof)
        target = cum[-1] * n1 / len(ranks)
        cut = 1 + int(np.argmin(np.abs(cum[:-1] - target)))
        m0, m1 = t1.copy(), t0.copy()
        m0[axis] = t0[axis] + cut
        m1[axis] = t0[axis] + cut
        split(t0, m0, ranks[:n1])
        split(m1, t1, ranks[n1:])

    split(np.zeros(3, np.int64), dims, list(range(world)))
    boxes = []
    for t0, t1 in out:
        b0 = np.clip(start + size * t0, 0, nb)
        b1 = np.clip(start + size * t1, 0, nb)
        if (t1 <= t0).any():
            b1 = b0.copy()
        boxes.append((b0, b1))
    return boxes


def sub_level(h, lo, box):
    """A box's level: its first node and bricks a side."""
    b0, b1 = box
    return np.asarray(lo, dtype=np.float64) + 8.0 * h * b0, (b1 - b0).astype(np.int64)


def level_origin(h, lo, origin=None):
    """The origin every box's level takes, so that its box grid is the level's."""
    return np.asarray(lo, dtype=np.float64) + h if origin is None else np.asarray(origin, dtype=np.float64)


def assemble(nb, boxes, maps, atlases):
    """The level from its boxes: maps[q] box q's map (its bricks, x fastest; any integer
    tensor holding the u32 entries), atlases[q] its atlas (slots x 365). Returns (map as
    int64 (nb[0] nb[1] nb[2]), atlas int32 (slots x 365)) on the maps' device."""
    import torch

    dev = maps[0].device if len(maps) else torch.device("cpu")
    nbl = [int(x) for x in nb]
    total = nbl[0] * nbl[1] * nbl[2]
    M = torch.full((nbl[2], nbl[1], nbl[0]), AIR, dtype=torch.int64, device=dev)
    owner = torch.full((nbl[2], nbl[1], nbl[0]), -1, dtype=torch.int64, device=dev)
    for q, (b0, b1) in enumerate(boxes):
        d = [int(b1[k] - b0[k]) for k in range(3)]
        if min(d) <= 0:
            continue
        m = maps[q].reshape(-1)[: d[0] * d[1] * d[2]].to(torch.int64) & 0xFFFFFFFF
        M[b0[2]:b1[2], b0[1]:b1[1], b0[0]:b1[0]] = m.view(d[2], d[1], d[0])
        owner[b0[2]:b1[2], b0[1]:b1[1], b0[0]:b1[0]] = q
    M = M.reshape(total)
    owner = owner.reshape(total)
    if bool((owner < 0).any()):
        raise ValueError("the boxes do not cover the level")
    stored = torch.nonzero(M < READ).reshape(-1)  # brick order
    base = [0]
    for a in atlases:
        base.append(base[-1] + int(a.shape[0]))
    flat = torch.cat([a.reshape(-1, WORDS).to(torch.int32) for a in atlases]) if atlases else \
        torch.zeros((0, WORDS), dtype=torch.int32, device=dev)
    base_t = torch.tensor(base[:-1], dtype=torch.int64, device=dev)
    rows = base_t[owner[stored]] + M[stored]
    A = flat[rows]
    M[stored] = torch.arange(len(stored), dtype=torch.int64, device=dev)
    return M, A


def exchange(dist, boxes, map_r, atlas_r):
    """Every rank's map and atlas on every rank (two all-gathers, padded): lists over ranks."""
    import torch

    world = dist.get_world_size()
    dev = map_r.device
    sizes = [int(np.prod(b1 - b0)) if (b1 > b0).all() else 0 for b0, b1 in boxes]
    mmax = max(max(sizes), 1)
    mp = torch.zeros(mmax, dtype=torch.int32, device=dev)
    mp[: map_r.numel()] = map_r.reshape(-1).to(torch.int32)
    got_m = [torch.empty_like(mp) for _ in range(world)]
    dist.all_gather(got_m, mp)
    n = torch.tensor([int(atlas_r.shape[0])], dtype=torch.int64, device=dev)
    counts = [torch.empty_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    counts = [int(c.item()) for c in counts]
    amax = max(max(counts), 1)
    ap = torch.zeros((amax, WORDS), dtype=torch.int32, device=dev)
    if atlas_r.shape[0]:
        ap[: atlas_r.shape[0]] = atlas_r.reshape(-1, WORDS).to(torch.int32)
    got_a = [torch.empty_like(ap) for _ in range(world)]
    dist.all_gather(got_a, ap)
    maps = [got_m[q][: sizes[q]] for q in range(world)]
    atlases = [got_a[q][: counts[q]] for q in range(world)]
    return maps, atlases


def bake_sharded(dist, bake_box, distance, h, lo, nb, clamp, origin=None, device="cpu"):
    """The level baked by the ranks of `dist` together: `bake_box(lo_r, nb_r, origin)`
    bakes this rank's box as a level ((map, atlas) tensors: map u32 entries as int32,
    atlas slots x 365 int32, on `device`, where the exchange runs); `distance` reads
    signed distances at points (every rank the same). A rank whose box is empty (more
    ranks than tiles) bakes nothing and still takes part in the exchange. Returns (map
    int64, atlas int32, this rank's box, every rank's box)."""
    import torch

    world = dist.get_world_size()
    rank = dist.get_rank()
    size, start, dims = tile_grid(h, lo, nb, origin)
    w = tile_weights(distance, h, lo, nb, clamp, origin)
    boxes = plan(w, size, start, nb, world)
    org = level_origin(h, lo, origin)
    lo_r, nb_r = sub_level(h, lo, boxes[rank])
    if (nb_r > 0).all():
        map_r, atlas_r = bake_box(lo_r, nb_r, org)
    else:
        map_r = torch.zeros(0, dtype=torch.int32, device=device)
        atlas_r = torch.zeros((0, WORDS), dtype=torch.int32, device=device)
    maps, atlases = exchange(dist, boxes, map_r, atlas_r)
    M, A = assemble(nb, boxes, maps, atlases)
    return M, A, boxes[rank], boxes
