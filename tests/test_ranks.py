"""The bench's multi-process path on CPU (gloo, two ranks, 127.0.0.1): each rank bakes
its own part (weak scaling: seed = rank, no collective on the data path), and the job's
figures are the slowest rank's time and the sum of the ranks' voxels (`over_ranks`)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        ms, vox = bench.over_ranks(dist, "cpu", 10.0 * (rank + 1), 100.0 * (rank + 1))
        e2e, none = bench.over_ranks(dist, "cpu", 5.0 + rank)
        # the rank's own part: its control net's checksum, gathered
        b, lo, nb = bench.workload(seed=rank)
        net = np.concatenate([np.asarray(p).reshape(-1) for p in b.patches])
        mine = torch.tensor([float(np.sum(net * np.arange(len(net)) % 7919))], dtype=torch.float64)
        every = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(every, mine)
        fams = [f for f, _ in bench.batch_parts(seed0=64 * rank, count=4)]
        out.put((rank, ms, vox, e2e, none, [float(x.item()) for x in every], tuple(nb.tolist()), fams))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    for rank, ms, vox, e2e, none, every, nb, fams in got:
        assert ms == 20.0 and vox == 300.0  # the slowest rank's time, all ranks' voxels
        assert e2e == 6.0 and none is None
        assert every[0] != every[1]  # each rank its own part
        assert fams == ["freeform_top", "boss", "countersunk_block", "dome"]
