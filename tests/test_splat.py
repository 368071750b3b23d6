"""Renderer splats (calculateGridMass.wgsl, mcDensity.cs.wgsl): the oracle
conserves mass on the CPU; the CUDA kernels equal the oracle bit for bit on
the GPU, for particles inside, on the edges of and outside the domain."""
import numpy as np
import pytest

from helpers import GpuScene


def _records(pkg, n=3000, seed=0, lo=-0.05, hi=1.05):
    rng = np.random.default_rng(seed)
    p = pkg.new_particles(n)
    p["pos"] = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    p["mass"] = rng.uniform(1e-6, 4e-6, n).astype(np.float32)
    p["pos"][0] = [0.0, 0.0, 0.0]                  # the grid's minimum corner
    p["pos"][1] = [1.0, 0.5, 0.5]                  # on the maximum face: excluded
    p["pos"][2] = np.nextafter(np.float32([1.0, 1.0, 1.0]), np.float32(0))
    return p


def test_oracle_splats_conserve_interior_mass(pkg, oracle_mod):
    rng = np.random.default_rng(1)
    p = pkg.new_particles(2000)
    p["pos"] = rng.uniform(0.2, 0.8, (2000, 3)).astype(np.float32)
    p["mass"] = np.float32(3e-6)
    scale = 2.0 ** 30
    for kind, res in (("mass", (32, 32, 32)), ("density", (16, 16, 16))):
        g = oracle_mod.splat(kind, p, [0, 0, 0], [1, 1, 1], res, scale)
        total = float(g.astype(np.float64).sum())
        want = 2000 * 3e-6 * scale
        # eight truncations per particle lose at most 8 units each
        assert want - 8 * 2000 <= total <= want * (1 + 1e-6), (kind, total, want)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mass", "density"])
def test_splats_bit_exact(gpu, oracle_mod, kind):
    spec = gpu.scenes.parity_scene(kind="explicit", with_collider=True)
    g = GpuScene(gpu, spec)
    assert g.step(3) == 0
    rec = g.particles()
    res = spec.res if kind == "mass" else tuple(r // 2 for r in spec.res)
    out = (g.buf.calculate_grid_mass(res) if kind == "mass" else g.buf.calculate_density(res)).cpu().numpy()
    u = np.frombuffer(spec.uniforms.bytes(), np.uint8)
    scale = float(np.frombuffer(u[4:8].tobytes(), "<f4")[0])
    want = oracle_mod.splat(kind, rec, [0, 0, 0], [1, 1, 1], res, scale)
    assert want.sum() > 0
    assert np.array_equal(out.view(np.uint32), want)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mass", "density"])
def test_splats_edges_and_outside(gpu, oracle_mod, kind):
    p = _records(gpu)
    spec = gpu.scenes.parity_scene(kind="explicit")
    buf = gpu.GpuMpmBufferManager(n_particles=p.shape[0])
    buf.write_particles(p)
    pipe = gpu.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms)
    res = (32, 32, 32) if kind == "mass" else (15, 16, 17)
    if kind == "mass":
        spec.uniforms.write_grid_resolution(res)
        pipe.push_uniforms()
    out = (buf.calculate_grid_mass(res) if kind == "mass" else buf.calculate_density(res)).cpu().numpy()
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    want = oracle_mod.splat(kind, p, [0, 0, 0], [1, 1, 1], res, scale)
    assert np.array_equal(out.view(np.uint32), want)
    buf.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mass", "density"])
def test_splats_coarse_grid_aggregated(gpu, oracle_mod, kind):
    # fewer cells than particles: the warp-aggregated form of the adds
    p = _records(gpu, n=5000, seed=4, lo=0.1, hi=0.9)
    spec = gpu.scenes.parity_scene(kind="explicit")
    buf = gpu.GpuMpmBufferManager(n_particles=p.shape[0])
    buf.write_particles(p)
    pipe = gpu.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms)
    res = (6, 5, 7)
    if kind == "mass":
        spec.uniforms.write_grid_resolution(res)
        pipe.push_uniforms()
    out = (buf.calculate_grid_mass(res) if kind == "mass" else buf.calculate_density(res)).cpu().numpy()
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    want = oracle_mod.splat(kind, p, [0, 0, 0], [1, 1, 1], res, scale)
    assert want.sum() > 0
    assert np.array_equal(out.view(np.uint32), want)
    buf.close()
