"""Committed golden fixtures (tests/golden/*.npz, written by
tests/golden/make_golden.py from the oracle).

The reference ships no golden vectors and its WGSL cannot run without a
graphics stack, so these fixtures pin the oracle against regressions (CPU
test) and give the CUDA path a fixed expected output that does not depend
on the live oracle (GPU test).  Both comparisons are bit for bit: particle
records (computed fields) and the dense fixed-point grid.
"""
import glob
import json
import os

import numpy as np
import pytest

from helpers import GpuScene, bits_equal, compare_states

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load_fixture(pkg, path):
    z = np.load(path)
    meta = json.loads(bytes(z["meta"]).decode())
    params = json.loads(bytes(z["params"]).decode())
    u = pkg.GpuUniformsBufferManager()
    u.buffer[:] = bytes(z["uniforms"])
    p_in = z["particles_in"].view(pkg.PARTICLE_DTYPE).copy()
    p_out = z["particles_out"].view(pkg.PARTICLE_DTYPE).copy()
    mesh = None
    if z["mesh_indices"].size:
        mesh = (z["mesh_vertices"].astype(np.float32), z["mesh_indices"].astype(np.uint32))
    spec = pkg.scenes.SceneSpec(os.path.basename(path)[:-4], u, params, p_in, int(meta["method"]), int(meta["steps"]),
                                mesh, tuple(meta["res"]))
    return spec, p_out, z["grid"]


def test_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in FIXTURES}
    assert {"explicit_plain", "explicit_collider", "pbmpm_plain", "pbmpm_collider_interaction"} <= names


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_reproduces_fixture(pkg, oracle_mod, path):
    spec, want, grid_want = load_fixture(pkg, path)
    o = oracle_mod.Oracle(spec.particles.shape[0], max_blocks=20000, hash_size=200003)
    if spec.mesh is not None:
        o.set_collider(*spec.mesh)
    p = spec.particles.copy()
    for _ in range(spec.n_steps):
        o.step(spec.uniforms.bytes(), spec.params, p, spec.method)
    compare_states(p, want)
    assert bits_equal(o.dense_grid(spec.uniforms.bytes()), grid_want)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_gpu_reproduces_fixture(gpu, path):
    spec, want, grid_want = load_fixture(gpu, path)
    g = GpuScene(gpu, spec)
    assert g.step(spec.n_steps) == 0
    compare_states(g.particles(), want)
    grid = g.grid(apply_update=(spec.method == 0))
    assert np.array_equal(grid, grid_want), f"{np.count_nonzero(grid != grid_want)} grid words differ"
    g.close()
