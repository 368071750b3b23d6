"""Scene sharding for batched scenes (config 3) across ranks: balanced,
disjoint and covering, identical on every rank (checked with two gloo ranks
on the CPU, the same way the ranks of a multi-GPU run agree without a
data-path collective)."""
import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def test_shards_cover_scenes_once_and_balance(pkg):
    b = pkg.batching
    rng = np.random.default_rng(3)
    counts = np.floor(np.exp(rng.uniform(np.log(2e3), np.log(2e5), 256))).astype(int)
    for world in (1, 2, 3, 8):
        sh = b.shard_scenes(counts, world)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(256))
        loads = b.shard_loads(counts, sh)
        assert loads.max() - loads.min() <= counts.max()
        assert loads.max() <= counts.sum() / world + counts.max()


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import importlib
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    pkg = importlib.import_module("webgpu-mpm-based-snow-simulation_b200")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(7)
    counts = np.floor(np.exp(rng.uniform(np.log(2e3), np.log(2e5), 64))).astype(int)
    mine = pkg.batching.shard_scenes(counts, world)[rank]
    # per-scene metric gathered on the host, as a multi-GPU batched run reports it
    metric = [(i, int(counts[i])) for i in mine]
    gathered = [None] * world
    dist.all_gather_object(gathered, metric)
    if rank == 0:
        out.put(gathered)
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ids = sorted(i for part in gathered for i, _ in part)
    assert ids == list(range(64))
    assert not set(i for i, _ in gathered[0]) & set(i for i, _ in gathered[1])
