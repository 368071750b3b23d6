"""Volumetric ray march (volumetricRaymarch.cs.wgsl): the oracle against a
closed form on the CPU (empty grid: only the ground is lit); the CUDA kernel
equal to the oracle bit for bit on the GPU (RGBA8 image, colour before
quantisation, depth), on a synthetic density field and through the whole
chain simulation -> calculateGridMass -> ray march."""
import numpy as np
import pytest

from helpers import GpuScene


def inv_view_proj(eye, target, width, height):
    from conftest import import_pkg

    return import_pkg().scenes.camera_inv_view_proj(eye, target, width, height)


def _blob_grid(res, seed=0):
    """u32 mass grid with a few dense Gaussian blobs, fixed point 2^28."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.arange(r) + 0.5 for r in res[::-1]), indexing="ij")
    g = np.zeros(res[::-1])
    for _ in range(4):
        c = rng.uniform(0.25, 0.75, 3) * np.array(res)
        r = rng.uniform(0.08, 0.18) * res[0]
        g += np.exp(-(((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * r * r)))
    cell_vol = 1.0 / (res[0] * res[1] * res[2])
    mass = g * 600.0 * cell_vol      # ~600 kg/m^3 at the blob centres
    return np.floor(mass * 2.0 ** 28).astype(np.uint32)


def test_oracle_empty_grid_lights_only_the_ground(oracle_mod):
    w, h = 24, 16
    M = inv_view_proj((0.5, -1.2, 1.4), (0.5, 0.5, 0.0), w, h)
    grid = np.zeros((8, 8, 8), np.uint32)
    rgba, depth, color = oracle_mod.raymarch(grid, [0, 0, 0], [1, 1, 1], 2.0 ** 28, M, 7, w, h)
    ld = np.array([0.2, 0.18, 0.9])
    ld /= np.linalg.norm(ld)
    lc = np.array([0.95, 0.995, 1.0]) * 5
    ground = np.array([0.0, 0.1, 0.2]) + 0.05 * lc * ld[2]     # unshadowed: nothing in the grid
    want = ground ** (1 / 2.2)
    hit = color[..., 3] > 0
    assert hit.sum() > 30                                        # the camera sees the ground
    np.testing.assert_allclose(color[hit][:, :3], np.broadcast_to(want, (hit.sum(), 3)), rtol=2e-6)
    assert np.all(color[hit][:, 3] == 1.0)
    # depth of a ground hit: distance along the ray to z = 0
    assert np.all(depth[hit] > 0) and np.all(depth[hit] < 5)
    # the other rays: zero colour; depth 1e20 where the ray crossed the empty
    # grid, untouched (-1 here) where it missed the grid's box
    other = depth[~hit]
    assert np.all(rgba[~hit] == 0)
    assert np.all((other == -1.0) | (other == np.float32(1e20)))
    assert (other == -1.0).any() and (other == np.float32(1e20)).any()


@pytest.mark.gpu
def test_raymarch_bit_exact_synthetic(gpu, oracle_mod):
    import torch

    spec = gpu.scenes.parity_scene(kind="pbmpm")
    res = (24, 20, 28)
    spec.uniforms.write_grid_resolution(res)
    w, h = 64, 48
    M = inv_view_proj((1.6, -0.9, 1.3), (0.5, 0.5, 0.4), w, h)
    spec.uniforms.write_view_proj_inv_mat(M.reshape(4, 4))
    spec.uniforms.write_time(12345)
    g = GpuScene(gpu, spec)
    vol = gpu.GpuVolumetricBufferManager(grid_resolution=res, screen_dims=(w, h))
    grid = _blob_grid(res)
    vol.mass_grid.copy_(torch.from_numpy(grid.view(np.int32)))
    vol.depth.fill_(-1.0)
    torch.cuda.synchronize()
    rp = gpu.GpuVolumetricRenderPipelineManager(mpm_manager=g.buf, volumetric_manager=vol)
    rp.add_raymarch_dispatch()
    g.buf.sync()
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    want_rgba, want_depth, want_color = oracle_mod.raymarch(grid, [0, 0, 0], [1, 1, 1], scale, M, 12345, w, h)
    got_color = vol.color.cpu().numpy()
    assert (want_color[..., 3] > 0.05).sum() > 100                # the blobs are in view
    assert np.array_equal(got_color.view(np.uint32), want_color.view(np.uint32))
    assert np.array_equal(vol.output.cpu().numpy(), want_rgba)
    assert np.array_equal(vol.depth.cpu().numpy().view(np.uint32), want_depth.view(np.uint32))
    g.close()


@pytest.mark.gpu
def test_raymarch_chain_after_simulation(gpu, oracle_mod):
    spec = gpu.scenes.parity_scene(kind="explicit", with_collider=True)
    w, h = 40, 32
    M = inv_view_proj((0.5, -0.8, 0.9), (0.5, 0.5, 0.35), w, h)
    spec.uniforms.write_view_proj_inv_mat(M.reshape(4, 4))
    spec.uniforms.write_time(3)
    g = GpuScene(gpu, spec)
    assert g.step(3) == 0
    vol = gpu.GpuVolumetricBufferManager(grid_resolution=spec.res, screen_dims=(w, h))
    rp = gpu.GpuVolumetricRenderPipelineManager(mpm_manager=g.buf, volumetric_manager=vol)
    vol.depth.fill_(-1.0)
    import torch

    torch.cuda.synchronize()
    rp.add_prerender_passes()
    g.buf.sync()
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    grid = oracle_mod.splat("mass", g.particles(), [0, 0, 0], [1, 1, 1], spec.res, scale)
    assert np.array_equal(vol.mass_grid.cpu().numpy().view(np.uint32), grid)
    want_rgba, want_depth, want_color = oracle_mod.raymarch(grid, [0, 0, 0], [1, 1, 1], scale, M, 3, w, h)
    assert (want_color[..., 3] > 0.05).sum() > 20                 # the snow block is in view
    assert np.array_equal(vol.color.cpu().numpy().view(np.uint32), want_color.view(np.uint32))
    assert np.array_equal(vol.output.cpu().numpy(), want_rgba)
    assert np.array_equal(vol.depth.cpu().numpy().view(np.uint32), want_depth.view(np.uint32))
    g.close()


@pytest.mark.gpu
def test_raymarch_camera_inside_grid(gpu, oracle_mod):
    import torch

    spec = gpu.scenes.parity_scene(kind="pbmpm")
    res = (20, 20, 20)
    spec.uniforms.write_grid_resolution(res)
    w, h = 32, 24
    M = inv_view_proj((0.5, 0.1, 0.45), (0.5, 0.9, 0.4), w, h)    # eye inside the unit box
    spec.uniforms.write_view_proj_inv_mat(M.reshape(4, 4))
    spec.uniforms.write_time(77)
    g = GpuScene(gpu, spec)
    vol = gpu.GpuVolumetricBufferManager(grid_resolution=res, screen_dims=(w, h))
    grid = _blob_grid(res, seed=5)
    vol.mass_grid.copy_(torch.from_numpy(grid.view(np.int32)))
    vol.depth.fill_(-1.0)
    torch.cuda.synchronize()
    gpu.GpuVolumetricRenderPipelineManager(mpm_manager=g.buf, volumetric_manager=vol).add_raymarch_dispatch()
    g.buf.sync()
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    want_rgba, want_depth, want_color = oracle_mod.raymarch(grid, [0, 0, 0], [1, 1, 1], scale, M, 77, w, h)
    assert (want_color[..., 3] > 0.05).sum() > 50
    assert np.array_equal(vol.color.cpu().numpy().view(np.uint32), want_color.view(np.uint32))
    assert np.array_equal(vol.output.cpu().numpy(), want_rgba)
    assert np.array_equal(vol.depth.cpu().numpy().view(np.uint32), want_depth.view(np.uint32))
    g.close()
