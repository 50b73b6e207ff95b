"""Host-side multi-GPU logic on CPU: LPT tile sharding and the max-over-ranks
timing reduction, run as two gloo ranks (world_size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from image360_b200 import shard, synth


def test_lpt_assignment_covers_each_tile_once():
    cfg = synth.C1
    pano = synth.make_panorama(cfg, with_cfa=False)
    for world in (1, 2, 4, 8):
        shards = shard.assign_tiles(pano.tiles, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(pano.tiles)))
        assert shard.imbalance(pano.tiles, world) < 1.25


def test_uneven_tiles_balance():
    import numpy as np
    rng = np.random.default_rng(3)
    sides = [512, 768, 1024, 1536, 2048]
    tiles = [(0, 0, int(rng.choice(sides)), int(rng.choice(sides)), list(range(int(rng.integers(1, 8)))))
             for _ in range(256)]
    for world in (2, 4, 8):
        assert shard.imbalance(tiles, world) < 1.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pano = synth.make_panorama(synth.C1, with_cfa=False)
    mine, frames = shard.shard(pano.tiles, rank, world)
    ids = torch.zeros(len(pano.tiles), dtype=torch.int64)
    ids[mine] = 1
    dist.all_reduce(ids)                       # every tile claimed exactly once
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)    # max-over-ranks step time
    need = {c for i in mine for c in pano.tiles[i][4]}
    q.put((rank, ids.tolist(), float(t.item()), need == set(frames), len(frames)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ids, t, frames_ok, nframes in res:
        assert all(v == 1 for v in ids)
        assert t == 11.0
        assert frames_ok and 0 < nframes <= 24
