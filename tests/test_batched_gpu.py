"""Batched scenes (config 3) on the GPU: many independent scenes advanced by
the same launches give each scene exactly the states it gets alone."""
import numpy as np
import pytest

from helpers import GpuScene, compare_states, run_oracle

pytestmark = pytest.mark.gpu


def _solo(gpu, spec, steps):
    g = GpuScene(gpu, spec)
    assert g.step(steps) == 0
    rec = g.particles()
    g.close()
    return rec


def test_batched_explicit_scenes_equal_solo_runs(gpu):
    specs = gpu.scenes.c3_batched(n_scenes=6, seed=5, lo_count=300, hi_count=4000)
    b = gpu.GpuMpmBatch(specs)
    b.step(gpu.GpuSimulationMethodType.ExplicitMpm, 4)
    assert b.mpm.sync() == 0
    rec = b.mpm.read_particles()
    for i, spec in enumerate(specs):
        compare_states(b.scene_particles(i, rec), _solo(gpu, spec, 4))
    b.close()


@pytest.mark.parametrize("tile_edge", [8, 14, 16])
def test_batched_pbmpm_scenes_with_colliders_equal_solo_runs(gpu, tile_edge):
    specs = [gpu.scenes.parity_scene(kind="pbmpm", n_side=n, seed=s, with_collider=True)
             for n, s in ((8, 40), (12, 41), (10, 42))]
    b = gpu.GpuMpmBatch(specs, tile_edge=tile_edge)
    b.step(gpu.GpuSimulationMethodType.Pbmpm, 3)
    assert b.mpm.sync() == 0
    rec = b.mpm.read_particles()
    for i, spec in enumerate(specs):
        compare_states(b.scene_particles(i, rec), _solo(gpu, spec, 3))
    b.close()


@pytest.mark.parametrize("method", [0, 1])
def test_batch_with_empty_scenes(gpu, oracle_mod, method):
    """Scenes with no particles (first, middle and last in the buffer) leave
    the others unchanged: each populated scene equals the f32 oracle's run of
    it alone, bit for bit."""
    import dataclasses

    kind = "pbmpm" if method else "explicit"
    full = [gpu.scenes.parity_scene(kind=kind, n_side=n, seed=s, with_collider=(method == 1))
            for n, s in ((9, 50), (11, 51))]
    empty = dataclasses.replace(full[0], particles=full[0].particles[:0].copy())
    specs = [empty, full[0], empty, full[1], empty]
    b = gpu.GpuMpmBatch(specs)
    b.step(method, 3)
    assert b.mpm.sync() == 0
    rec = b.mpm.read_particles()
    assert rec.shape[0] == sum(int(f.particles.shape[0]) for f in full)
    for i, spec in ((1, full[0]), (3, full[1])):
        o, want = run_oracle(oracle_mod, spec, n_steps=3)
        o.close()
        compare_states(b.scene_particles(i, rec), want)
    assert b.scene_particles(0, rec).shape[0] == 0 and b.scene_particles(4, rec).shape[0] == 0
    b.close()


@pytest.mark.parametrize("order_mode,tile_block,hash_factor", [(1, 128, 2), (5, 0, 8), (4, 128, 0)])
def test_schedule_knobs_leave_results_unchanged(gpu, oracle_mod, order_mode, tile_block, hash_factor):
    """Claim order, CTA size of the explicit tile kernels and hash capacity
    change the schedule only: each scene still equals the f32 oracle."""
    from helpers import run_oracle

    specs = gpu.scenes.c3_batched(n_scenes=5, seed=9, lo_count=400, hi_count=5000)
    cap = 0
    if hash_factor:
        probe = gpu.GpuMpmBatch(specs, tile_edge=8)
        probe.step(gpu.GpuSimulationMethodType.ExplicitMpm, 1)
        n_tiles = probe.mpm.counts()[0]
        probe.close()
        cap = max(4096, 1 << int(np.ceil(np.log2(hash_factor * n_tiles))))
    b = gpu.GpuMpmBatch(specs, tile_edge=8, order_mode=order_mode, tile_block=tile_block, hash_capacity=cap)
    b.step(gpu.GpuSimulationMethodType.ExplicitMpm, 3)
    assert b.mpm.sync() == 0
    rec = b.mpm.read_particles()
    for i, spec in enumerate(specs):
        _, want = run_oracle(oracle_mod, spec, n_steps=3)
        compare_states(b.scene_particles(i, rec), want)
    b.close()


def test_schedule_autotuner(gpu):
    specs = gpu.scenes.c3_batched(n_scenes=4, seed=6, lo_count=500, hi_count=3000)
    cache = {}
    sched, times = gpu.batching.autotune_schedule(specs, gpu.GpuSimulationMethodType.ExplicitMpm, steps=2,
                                                  cache=cache)
    assert sched["tile_edge"] in (8, 12, 14, 16) and sched["tile_block"] in (0, 128)
    assert sched["order_mode"] in (0, 1, 4, 5) and sched["hash_capacity"] >= 0
    assert len(times) >= 8 and all(t > 0 for t in times.values())
    again, t2 = gpu.batching.autotune_schedule(specs, gpu.GpuSimulationMethodType.ExplicitMpm, cache=cache)
    assert again == sched and t2 == {}   # served from the cache


def test_autotuner_picks_a_supported_edge(gpu):
    specs = gpu.scenes.c3_batched(n_scenes=4, seed=6, lo_count=500, hi_count=3000)
    best, times = gpu.batching.autotune_tile_edge(specs, gpu.GpuSimulationMethodType.ExplicitMpm, steps=2)
    assert best in (8, 12, 14, 16) and set(times) == {8, 12, 14, 16}
    assert all(t > 0 for t in times.values())
