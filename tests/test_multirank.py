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
        bands = shard.assign_bands(pano.tiles, world)
        assert sorted(i for s in bands for i in s) == list(range(len(pano.tiles)))
        assert shard.imbalance(pano.tiles, world, "bands") < 1.35


def test_band_shards_of_the_scaled_panorama_balance_and_keep_frames_local():
    """The sharded bench mode's panorama (8 frame columns per rank): cost
    balance within 5 % and each rank holding well under all frames."""
    for world in (2, 4, 8):
        cfg = synth.PanoConfig(**{**synth.C1.__dict__, "cols": synth.C1.cols * world})
        pano = synth.make_panorama(cfg, with_cfa=False)
        assert shard.imbalance(pano.tiles, world, "bands") < 1.05
        for r in range(world):
            _, need = shard.shard(pano.tiles, r, world)
            assert len(need) <= 3 * 10  # its own 8 columns plus neighbours


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


def _sharded_worker(rank, world, port, q):
    """One panorama of 8 frame columns per rank (the sharded bench mode at
    small size): each rank makes only the frames its LPT tiles need and
    renumbers its tiles to them."""
    import hashlib

    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    base = synth.scaled(synth.C1, 0.02, tile=64)
    cfg = synth.PanoConfig(**{**base.__dict__, "cols": base.cols * world})
    geo = synth.make_panorama(cfg, with_cfa=False)
    mine, need = shard.shard(geo.tiles, rank, world)
    pano = synth.make_panorama(cfg, frames=need)
    local = shard.local_view(geo.tiles, mine, need)
    hashes = {f: hashlib.sha1(pano.cfa[f].numpy().tobytes()).hexdigest() for f in need}
    remap_ok = all([need[c] for c in lt[4]] == list(geo.tiles[i][4]) and lt[:4] == tuple(geo.tiles[i][:4])
                   for i, lt in zip(mine, local))
    absent_ok = all(pano.cfa[f] is None for f in range(len(geo.to_canvas)) if f not in need)
    info = {"rank": rank, "mine": mine, "need": need, "hashes": hashes, "remap_ok": remap_ok,
            "absent_ok": absent_ok, "px": sum(t[2] * t[3] for t in local)}
    gathered = [None] * world
    dist.all_gather_object(gathered, info)
    px = torch.tensor([float(info["px"])], dtype=torch.float64)
    dist.all_reduce(px)  # whole-job output pixels
    q.put((rank, gathered, float(px.item()), geo.canvas_w * geo.canvas_h, len(geo.tiles), len(geo.to_canvas)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_sharded_panorama_bookkeeping_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _, gathered, px, canvas_px, n_tiles, n_frames = res[0]
    assert n_frames == 3 * 16
    tiles = sorted(i for g in gathered for i in g["mine"])
    assert tiles == list(range(n_tiles))                      # every tile rendered once
    assert px == canvas_px                                    # the tiles cover the canvas exactly
    assert all(g["remap_ok"] and g["absent_ok"] for g in gathered)
    assert all(0 < len(g["need"]) < n_frames for g in gathered)  # no rank holds every frame
    shared = set(gathered[0]["need"]) & set(gathered[1]["need"])
    for f in shared:                                          # a frame made on two ranks is the same frame
        assert gathered[0]["hashes"][f] == gathered[1]["hashes"][f]
    loads = shard.loads(synth.make_panorama(synth.PanoConfig(**{**synth.scaled(synth.C1, 0.02, tile=64).__dict__,
                                                                "cols": 16}), with_cfa=False).tiles, 2)
    assert max(c for _, _, c in loads) / (sum(c for _, _, c in loads) / 2) < 1.25
