"""Collider BVH built on the GPU (mpm_build_bvh_device): node for node and
bit for bit the tree of the host build, which restates the reference's
(GpuColliderBufferManager.ts:222-350), on meshes with many centroid ties, on
the 130,050-triangle terrain of the large workload, on ragged small counts and
on an empty mesh; a collider installed from device buffers gives the same
simulation as the host-installed one."""
import numpy as np
import pytest

from helpers import GpuScene


def _meshes(pkg):
    rng = np.random.default_rng(5)
    out = {"icosphere": pkg.scenes.icosphere(3, 0.1, (0.5, 0.2, 0.5)),
           "terrain_256": pkg.scenes.fbm_terrain(n=256)}
    vq = (rng.integers(-2, 3, (400, 3)).astype(np.float32) * 0.25)
    vq[rng.random(vq.shape) < 0.1] = -0.0                  # signed zeros on the bounds
    out["ties"] = (vq, rng.integers(0, 400, (3000, 3)).astype(np.uint32))
    # degenerate triangles: repeated vertices and zero-area slivers, equal centroids
    vd = rng.random((50, 3)).astype(np.float32)
    fd = rng.integers(0, 50, (600, 3)).astype(np.uint32)
    fd[::3, 1] = fd[::3, 0]
    fd[::5] = fd[0]
    out["degenerate"] = (vd, fd)
    for n in (1, 4, 5, 9, 17, 1000):
        out[f"soup_{n}"] = (rng.random((3 * n, 3)).astype(np.float32), np.arange(3 * n, dtype=np.uint32).reshape(n, 3))
    return out


def test_node_count_matches_host_build(pkg):
    for n in (0, 1, 4, 5, 8, 9, 100, 1281, 130050):
        v = np.random.default_rng(n).random((3 * max(n, 1), 3)).astype(np.float32)
        f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
        nodes, _ = pkg.build_bvh(v, f)
        assert pkg.load().mpm_bvh_node_count(n) == nodes.shape[0]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["icosphere", "terrain_256", "ties", "degenerate", "soup_1", "soup_4", "soup_5",
                                  "soup_9", "soup_17", "soup_1000"])
def test_device_build_equals_host_build(gpu, name):
    import torch

    v, f = _meshes(gpu)[name]
    v = np.asarray(v, np.float32).reshape(-1, 3)
    f = np.asarray(f, np.uint32).reshape(-1, 3)
    want_nodes, want_order = gpu.build_bvh(v, f)
    vd = torch.from_numpy(v.copy()).cuda()
    fd = torch.from_numpy(f.astype(np.int32)).cuda()
    nodes, order = gpu.build_bvh_device(vd, fd)
    torch.cuda.synchronize()
    assert np.array_equal(nodes.cpu().numpy().view(np.uint32), want_nodes)
    assert np.array_equal(order.cpu().numpy().view(np.uint32), want_order)


@pytest.mark.gpu
def test_device_build_empty_and_bad_index(gpu):
    import torch

    nodes, order = gpu.build_bvh_device(torch.zeros((0, 3), dtype=torch.float32, device="cuda"),
                                        torch.zeros(0, dtype=torch.int32, device="cuda"))
    want, _ = gpu.build_bvh(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32))
    assert np.array_equal(nodes.cpu().numpy().view(np.uint32), want)
    v = torch.rand((5, 3), device="cuda")
    f = torch.tensor([0, 1, 2, 2, 3, 5], dtype=torch.int32, device="cuda")   # 5 is out of range
    with pytest.raises(gpu.MpmError):
        gpu.build_bvh_device(v, f)


@pytest.mark.gpu
def test_device_installed_collider_same_simulation(gpu):
    import torch

    spec = gpu.scenes.parity_scene(kind="explicit", with_collider=True)
    a = GpuScene(gpu, spec)
    assert a.step(5) == 0
    want = a.particles()
    a.close()
    buf = gpu.GpuMpmBufferManager(n_particles=spec.particles.shape[0])
    buf.write_particles(spec.particles)
    from helpers import make_params
    pipe = gpu.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms,
                                     params=make_params(gpu, spec.params))
    v, f = spec.mesh
    pipe.set_collider_mesh_device(torch.from_numpy(np.asarray(v, np.float32).copy()).cuda(),
                                  torch.from_numpy(np.asarray(f, np.int32).reshape(-1).copy()).cuda())
    for _ in range(5):
        pipe.step(gpu.GpuSimulationMethodType(spec.method), 1)
    assert buf.sync() == 0
    got = buf.read_particles()
    buf.close()
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
