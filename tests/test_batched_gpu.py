"""Batched scenes (config 3) on the GPU: many independent scenes advanced by
the same launches give each scene exactly the states it gets alone."""
import numpy as np
import pytest

from helpers import GpuScene, compare_states

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


def test_autotuner_picks_a_supported_edge(gpu):
    specs = gpu.scenes.c3_batched(n_scenes=4, seed=6, lo_count=500, hi_count=3000)
    best, times = gpu.batching.autotune_tile_edge(specs, gpu.GpuSimulationMethodType.ExplicitMpm, steps=2)
    assert best in (8, 12, 14, 16) and set(times) == {8, 12, 14, 16}
    assert all(t > 0 for t in times.values())
