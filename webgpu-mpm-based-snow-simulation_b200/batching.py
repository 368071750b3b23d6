"""Batched scenes: sharding across ranks and the tile-size autotuner.

Independent scenes (config 3: 256 scenes of 2e3..2e5 particles) shard across
GPUs without any data-path collective: each rank advances its own subset in
one GpuMpmBatch.  `shard_scenes` balances the ranks by particle count
(longest-processing-time greedy bin packing, deterministic, so every rank
computes the same assignment without communicating).  `autotune_tile_edge`
times a few substeps of a batch at each supported tile edge and returns the
fastest; the tile edge sets both the shared-memory tile and the binning
bucket (one hash bucket per occupied tile).
"""
from __future__ import annotations

import heapq

import numpy as np

TILE_EDGES = (8, 12, 14, 16)


def shard_scenes(counts, world: int) -> list[list[int]]:
    """Scene indices per rank, heaviest scenes first onto the lightest rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(counts[i]), r))
    return [sorted(s) for s in out]


def shard_loads(counts, shards) -> np.ndarray:
    return np.array([sum(int(counts[i]) for i in s) for s in shards], np.int64)


def time_batch(batch, method, steps: int, warmup: int = 2) -> float:
    """Milliseconds per substep of a batch, CUDA events on its stream."""
    import torch

    for _ in range(warmup):
        batch.step(method, 1)
    batch.mpm.sync()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        batch.step(method, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def autotune_tile_edge(specs, method, *, edges=TILE_EDGES, steps: int = 3, device: int = 0):
    """(best tile edge, {edge: ms per substep}) for this set of scenes.  The
    batch is built on torch's current stream so the events see its work."""
    import torch

    from .pipeline import GpuMpmBatch

    times = {}
    for e in edges:
        b = GpuMpmBatch(specs, device=device, tile_edge=e, stream=torch.cuda.current_stream().cuda_stream)
        try:
            times[e] = time_batch(b, method, steps)
        finally:
            b.close()
    best = min(times, key=times.get)
    return best, times
