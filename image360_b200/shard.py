"""Multi-GPU partitioning of a panorama's output tiles.

Output tiles are independent: each re-warps its own contributors
(RenderExecutor.cpp:70-117) and no halo crosses a tile boundary, so the render
shards with no data-path collective.  Tiles are assigned to ranks by LPT
(longest processing time first) on an area x contributors cost; each rank then
needs only the frames its tiles reference.  One process per GPU.
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


def shard(tiles, rank: int, world: int):
    """(tile indices, frame indices needed) of `rank`."""
    mine = assign_tiles(tiles, world)[rank]
    frames = sorted({c for i in mine for c in tiles[i][4]})
    return mine, frames


def imbalance(tiles, world: int) -> float:
    """max rank load / mean rank load of the LPT assignment."""
    loads = [sum(tile_cost(tiles[i]) for i in s) for s in assign_tiles(tiles, world)]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0
