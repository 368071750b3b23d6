"""Particle initialisation (scatterParticles, particleScatter.cs.wgsl): the
oracle puts the particles inside the mesh (CPU); the CUDA kernel writes the
same records as the oracle, bit for bit (GPU), for meshes that fit one
shared-memory chunk of triangles and meshes that take several."""
import numpy as np
import pytest


def _mesh(pkg, kind):
    sc = pkg.scenes
    if kind == "box":
        v, f = sc.box_mesh((0.3, 0.4, 0.35), (0.7, 0.6, 0.65))
    elif kind == "sphere320":
        v, f = sc.icosphere(2, 0.15, (0.5, 0.5, 0.5))
    else:
        v, f = sc.icosphere(3, 0.2, (0.45, 0.55, 0.5))   # 1,280 triangles: three chunks
    return pkg.GpuMeshBufferManager(vertices=v, indices=f)


def test_oracle_scatter_fills_the_mesh(pkg, oracle_mod):
    mesh = _mesh(pkg, "sphere320")
    rec = oracle_mod.scatter(mesh.vertices, mesh.min_coords, mesh.max_coords, 2000).view(pkg.PARTICLE_DTYPE).reshape(-1)
    r = np.linalg.norm(rec["pos"] - 0.5, axis=1)
    assert (r < 0.15 + 0.05 * np.sqrt(3)).all()      # inside, plus the jitter of at most 0.05 per axis
    assert (r < 0.15).mean() > 0.8
    assert np.all((rec["mass"] >= 0) & (rec["mass"] < 1))
    assert np.all(rec["Fe"][:, :, :3] == np.eye(3, dtype=np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["box", "sphere320", "sphere1280"])
def test_scatter_bit_exact(gpu, oracle_mod, kind):
    mesh = _mesh(gpu, kind)
    n = 3000
    buf = gpu.GpuMpmBufferManager(n_particles=n)
    u = gpu.GpuUniformsBufferManager()
    init = gpu.GpuParticleInitializePipelineManager(mpm_manager=buf, mesh_manager=mesh, uniforms_manager=u)
    init.add_dispatch(n_particles=n)
    got = buf.read_particles(n)
    want = oracle_mod.scatter(mesh.vertices, mesh.min_coords, mesh.max_coords, n)
    assert np.array_equal(got.view(np.uint8).reshape(n, 192), want)
    buf.close()
