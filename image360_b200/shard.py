"""Multi-GPU partitioning of a panorama's output tiles.

Output tiles are independent: each re-warps its own contributors
(RenderExecutor.cpp:70-117) and no halo crosses a tile boundary, so the render
shards with no data-path collective.  Tiles are assigned to ranks on an area x
contributors cost, either as contiguous column bands of the canvas balanced by
cost ("bands": a rank's tiles, and so the frames it must hold, stay together)
or by LPT (longest processing time first: the tightest balance, for tile sets
without spatial locality).  Each rank then needs only the frames its tiles
reference, and renders them as a panorama of its own (local_view).  One
process per GPU.
"""
from __future__ import annotations

import heapq


def tile_cost(tile) -> int:
    x, y, w, h, contrib = tile[:5]
    return w * h * max(1, len(contrib))


def assign_tiles(tiles, world: int):
    """LPT assignment: returns a list of tile-index lists, one per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(tiles)), key=lambda i: (-tile_cost(tiles[i]), i))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + tile_cost(tiles[i]), r))
    return [sorted(s) for s in shards]


def assign_bands(tiles, world: int):
    """Contiguous runs of the tiles in column-major canvas order (x, then y),
    cut where the running cost passes each rank's share: returns a list of
    tile-index lists, one per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(tiles)), key=lambda i: (tiles[i][0], tiles[i][1], i))
    total = sum(tile_cost(tiles[i]) for i in order)
    shards = [[] for _ in range(world)]
    acc, r = 0, 0
    for i in order:
        c = tile_cost(tiles[i])
        while r < world - 1 and acc + c / 2 > total * (r + 1) / world:
            r += 1
        shards[r].append(i)
        acc += c
    return [sorted(s) for s in shards]


def shard(tiles, rank: int, world: int, method: str = "bands"):
    """(tile indices, frame indices needed) of `rank`."""
    mine = (assign_bands if method == "bands" else assign_tiles)(tiles, world)[rank]
    frames = sorted({c for i in mine for c in tiles[i][4]})
    return mine, frames


def imbalance(tiles, world: int, method: str = "lpt") -> float:
    """max rank load / mean rank load of an assignment."""
    loads = [sum(tile_cost(tiles[i]) for i in s) for s in (assign_bands if method == "bands" else assign_tiles)(tiles, world)]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0


def local_view(tiles, mine, frames):
    """The rank's share as a self-contained render: its tiles (canvas
    rectangles unchanged) with contributor lists renumbered to positions in
    `frames` (the frame indices it holds, ascending)."""
    pos = {f: i for i, f in enumerate(frames)}
    return [(x, y, w, h, [pos[c] for c in cs]) for (x, y, w, h, cs) in (tuple(tiles[i][:5]) for i in mine)]


def loads(tiles, world: int, method: str = "bands"):
    """Per rank: (tiles, frames needed, cost) of an assignment."""
    out = []
    for s in (assign_bands if method == "bands" else assign_tiles)(tiles, world):
        out.append((len(s), len({c for i in s for c in tiles[i][4]}), sum(tile_cost(tiles[i]) for i in s)))
    return out
