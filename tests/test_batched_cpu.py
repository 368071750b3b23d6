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


def _oracle_advance(specs, method, steps):
    """Test-only stand-in for a rank's GPU: each scene advanced by the f32 oracle."""
    import oracle

    out = []
    for spec in specs:
        p = spec.particles.copy()
        o = oracle.Oracle(p.shape[0], max_blocks=20000, hash_size=200003)
        for _ in range(steps):
            o.step(spec.uniforms.bytes(), spec.params, p, method)
        o.close()
        out.append(p)
    return out


def _small_batch(pkg):
    return pkg.scenes.c3_batched(n_scenes=5, seed=8, lo_count=200, hi_count=1500)


def _sharded_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import importlib
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    pkg = importlib.import_module("webgpu-mpm-based-snow-simulation_b200")
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    aggs = pkg.batching.run_sharded(_small_batch(pkg), 0, 3, rank=rank, world=world, advance=_oracle_advance)
    if rank == 0:
        out.put(aggs)
    dist.destroy_process_group()


def test_two_ranks_advance_their_shards(pkg, oracle_mod):
    """Each of two gloo ranks advances its own shard of a config-3 batch (the
    oracle standing in for the rank's GPU); the per-scene aggregates gathered
    on rank 0 equal a single-rank run of all scenes."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_sharded_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = _small_batch(pkg)
    single = pkg.batching.run_sharded(specs, 0, 3, advance=_oracle_advance)
    assert sorted(gathered) == list(range(len(specs)))
    for i in range(len(specs)):
        assert np.array_equal(np.array(gathered[i]), np.array(single[i])), i
    # both ranks worked: the shards are disjoint and non-empty
    counts = [s.particles.shape[0] for s in specs]
    sh = pkg.batching.shard_scenes(counts, 2)
    assert sh[0] and sh[1]


def _leaving_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import importlib
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    pkg = importlib.import_module("webgpu-mpm-based-snow-simulation_b200")
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)   # this rank leaves between steps, before the gather
    specs = _small_batch(pkg)
    try:
        pkg.batching.run_sharded(specs, 0, 1, rank=rank, world=world,
                                 advance=lambda sp, m, n: [s.particles for s in sp])
        out.put("gathered")
    except Exception as e:  # the peer is gone: the collective ends with an error
        out.put("error: " + type(e).__name__)


def test_rank_leaving_ends_the_gather_with_an_error():
    """A rank that exits between steps: the other rank's gather ends with an
    error within the process group's short timeout instead of waiting for
    good (host-side failure; no GPU involved)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29300 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_leaving_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert res.startswith("error"), res
    assert procs[1].exitcode == 3
