"""Batched scenes: sharding across ranks and the autotuner.

Independent scenes (config 3: 256 scenes of 2e3..2e5 particles) shard across
GPUs without any data-path collective: each rank advances its own subset in
one GpuMpmBatch (`run_sharded`), and only the per-scene aggregates are
gathered.  `shard_scenes` balances the ranks by particle count
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


def scene_aggregates(rec) -> list[float]:
    """Per-scene summary gathered from the ranks: centre of mass (3), net
    momentum (3), total absolute momentum, mean J_p (f64), from 192-byte
    records (or any record array with pos, vel, mass and a 3x3 Fp)."""
    m = np.asarray(rec["mass"], np.float64)
    v = np.asarray(rec["vel"], np.float64)
    com = (np.asarray(rec["pos"], np.float64) * m[:, None]).sum(0) / m.sum()
    mom = (v * m[:, None]).sum(0)
    abs_mom = float((np.linalg.norm(v, axis=1) * m).sum())
    Fp = np.asarray(rec["Fp"], np.float64)
    Fp = Fp.reshape(-1, 3, 3) if Fp.ndim == 2 else Fp[:, :, :3]
    jp = float(np.linalg.det(Fp).mean())
    return [*map(float, com), *map(float, mom), abs_mom, jp]


def advance_on_gpu(specs, method, steps: int, *, device: int = 0, tile_edge: int = 0, stream=None):
    """Final records of each scene after `steps` substeps, all scenes in one
    GpuMpmBatch on `device` (the per-rank work of a sharded run)."""
    from .pipeline import GpuMpmBatch

    b = GpuMpmBatch(specs, device=device, tile_edge=tile_edge, stream=stream)
    try:
        b.step(method, steps)
        status = b.mpm.sync()
        if status:
            raise RuntimeError(f"device status {status:#x}")
        rec = b.mpm.read_particles()
        return [b.scene_particles(i, rec).copy() for i in range(len(specs))]
    finally:
        b.close()


def run_sharded(specs, method, steps: int, *, rank: int = 0, world: int = 1, advance=None, group=None):
    """Advances this rank's shard of independent scenes (shard_scenes by
    particle count, the same assignment on every rank, no communication) and
    gathers the per-scene aggregates on every rank, the only exchange of a
    sharded run (host objects through torch.distributed; no data-path
    collective).  `advance(specs, method, steps)` returns each scene's final
    records (default: advance_on_gpu on the current device).  Returns
    {scene index: scene_aggregates}."""
    counts = [int(s.particles.shape[0]) for s in specs]
    mine = shard_scenes(counts, world)[rank]
    if advance is None:
        import torch

        def advance(sp, m, n):
            return advance_on_gpu(sp, m, n, device=torch.cuda.current_device())
    records = advance([specs[i] for i in mine], method, steps) if mine else []
    local = {i: scene_aggregates(r) for i, r in zip(mine, records)}
    if world == 1:
        return local
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for part in parts:
        merged.update(part)
    return merged


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


# schedules found by autotune_schedule, per (method, scene-count bucket,
# particle-count bucket): a batch of similar shape reuses the choice
SCHEDULE_CACHE: dict = {}


def schedule_bucket(specs, method) -> tuple:
    """Cache key of a batch: method, log2 buckets of the scene count and of the
    total particle count."""
    n = sum(int(s.particles.shape[0]) for s in specs)
    return (int(method), int(np.log2(max(len(specs), 1))), int(np.log2(max(n, 1))))


def autotune_schedule(specs, method, *, steps: int = 3, device: int = 0, cache: dict | None = SCHEDULE_CACHE):
    """Coordinate descent over the schedule knobs of a batch, each timed on a
    few substeps (time_batch): tile edge (8, 12, 14, 16; it sets the binning
    bucket and the shared-memory tile), threads per CTA of the explicit tile
    kernels (256, 128), the tile claim order (automatic; compact; Morton
    buckets of 4 or 5 bits per axis) and the tile hash capacity (the derived
    default, or 2 / 8 slots per occupied tile, rounded up to a power of two).
    Results do not depend on any knob.  Returns (schedule dict, {label: ms per
    substep}); the choice is cached per schedule_bucket."""
    import torch

    from .pipeline import GpuMpmBatch

    key = schedule_bucket(specs, method)
    if cache is not None and key in cache:
        return dict(cache[key]), {}
    times: dict = {}
    tiles: dict = {}

    def run(cfg):
        label = ",".join(f"{k}={v}" for k, v in cfg.items())
        if label not in times:
            b = GpuMpmBatch(specs, device=device, tile_edge=cfg["tile_edge"], tile_block=cfg["tile_block"],
                            order_mode=cfg["order_mode"], hash_capacity=cfg["hash_capacity"],
                            stream=torch.cuda.current_stream().cuda_stream)
            try:
                times[label] = time_batch(b, method, steps)
                tiles[cfg["tile_edge"]] = b.mpm.counts()[0]
            finally:
                b.close()
        return times[label]

    best = {"tile_edge": 16, "tile_block": 0, "order_mode": 0, "hash_capacity": 0}

    def descend(knob, values):
        cands = []
        for v in values:
            cfg = dict(best, **{knob: v})
            cands.append((run(cfg), v))
        best[knob] = min(cands)[1]

    descend("tile_edge", TILE_EDGES)
    if int(method) == 0:
        descend("tile_block", (0, 128))
    descend("order_mode", (0, 1, 4, 5))
    n_tiles = max(int(tiles.get(best["tile_edge"], 0)), 1)

    def cap(f):
        return max(4096, 1 << int(np.ceil(np.log2(f * n_tiles))))
    descend("hash_capacity", (0, cap(2), cap(8)))
    if cache is not None:
        cache[key] = dict(best)
    return dict(best), times


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
