"""The allocation-free substep (mpm_step_noalloc) against the handle-based step.

mpm_step_noalloc serves callers that cannot allocate device memory while
they run: a host that gives the library a fixed device budget and owns every
allocation itself, or a real-time frame loop that cannot take cudaMalloc's
implicit device-wide synchronisation.  Its intermediate buffers live in one
static device array; the caller passes only the particle records and the
collider arrays.  Two substeps in a row through it must give the same
particle records, bit for bit, as two substeps through a libmpm handle (the
bar of every parity test here), so the shared array's leftovers from the
first call must not leak into the second.

This file is named to be collected last: the other tests have run by the
time a failure here stops a run at its first failure.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import GpuScene, compare_states, make_params

pytestmark = pytest.mark.gpu


def _device_copy(torch, arr):
    a = np.ascontiguousarray(arr)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()


def _noalloc_step(lib, spec, params, dev_particles, n, col):
    import torch

    ub = spec.uniforms.bytes()
    status = C.c_uint32(0)
    err = C.create_string_buffer(256)
    if col is None:
        cd_ptr, cd_words, n_idx, nodes_ptr, n_nodes = None, 0, 0, None, 0
    else:
        cd, nodes, n_idx = col
        cd_ptr, cd_words = C.c_void_p(cd.data_ptr()), cd.numel() // 4
        nodes_ptr, n_nodes = C.c_void_p(nodes.data_ptr()), nodes.numel() // 32
    rc = lib.mpm_step_noalloc(0, C.c_void_p(torch.cuda.current_stream().cuda_stream), C.c_void_p(dev_particles.data_ptr()),
                              n, spec.method, ub, len(ub), C.byref(params), cd_ptr, cd_words, n_idx, nodes_ptr,
                              n_nodes, C.byref(status), err, len(err))
    assert rc == 0, f"mpm_step_noalloc returned {rc}: {err.value.decode()} (status {status.value:#x})"
    assert status.value == 0


@pytest.mark.parametrize("kind,collider,interaction", [("explicit", True, False), ("pbmpm", True, True),
                                                        ("pbmpm", False, False)])
def test_noalloc_matches_handle_step_twice(gpu, kind, collider, interaction):
    import torch

    lib = gpu.load()
    spec = gpu.scenes.parity_scene(kind=kind, n_side=16, with_collider=collider, interaction=interaction)
    n = spec.particles.shape[0]
    g = GpuScene(gpu, spec)  # also writes colliderNumIndices into spec.uniforms
    col = None
    if spec.mesh is not None:
        cm = gpu.GpuColliderBufferManager(vertices=spec.mesh[0], indices=spec.mesh[1])
        col = (_device_copy(torch, cm.collider_data), _device_copy(torch, cm.bvh_nodes), cm.num_indices)
    params = make_params(gpu, spec.params)
    dev = _device_copy(torch, spec.particles)
    for call in range(2):
        assert g.step(1) == 0
        want = g.particles()
        _noalloc_step(lib, spec, params, dev, n, col)
        torch.cuda.synchronize()
        got = dev.cpu().numpy().view(spec.particles.dtype)
        compare_states(got, want)
        assert np.isfinite(got["pos"]).all(), f"call {call}"
    g.close()


def test_noalloc_rejects_more_particles_than_its_limit(gpu):
    import torch

    lib = gpu.load()
    spec = gpu.scenes.parity_scene(kind="explicit", n_side=4)
    params = make_params(gpu, spec.params)
    ub = spec.uniforms.bytes()
    dev = _device_copy(torch, spec.particles)
    err = C.create_string_buffer(256)
    too_many = 65536 + 1
    rc = lib.mpm_step_noalloc(0, None, C.c_void_p(dev.data_ptr()), too_many, 0, ub, len(ub), C.byref(params), None, 0,
                              0, None, 0, None, err, len(err))
    assert rc == -3, rc  # MPM_ERR_CAPACITY, before any device work
    assert b"65536" in err.value


def test_noalloc_reports_tile_overflow(gpu):
    """More occupied 8^3-cell tiles than the array holds (512): the call
    returns MPM_ERR_DEVICE_STATUS with status bit 0x2 (a status the host
    reads; nothing faults), and the scratch array is left usable: a normal
    call right after it matches the handle step again."""
    import torch

    lib = gpu.load()
    spec = gpu.scenes.parity_scene(kind="explicit", n_side=13, res=256)
    rng = np.random.default_rng(17)
    n = spec.particles.shape[0]
    spec.particles["pos"] = rng.uniform(0.05, 0.95, size=(n, 3)).astype(np.float32)
    params = make_params(gpu, spec.params)
    ub = spec.uniforms.bytes()
    dev = _device_copy(torch, spec.particles)
    status = C.c_uint32(0)
    err = C.create_string_buffer(256)
    rc = lib.mpm_step_noalloc(0, C.c_void_p(torch.cuda.current_stream().cuda_stream), C.c_void_p(dev.data_ptr()), n,
                              0, ub, len(ub), C.byref(params), None, 0, 0, None, 0, C.byref(status), err, len(err))
    assert rc == -5, (rc, err.value)  # MPM_ERR_DEVICE_STATUS
    assert status.value & 0x2, status.value
    assert b"512" in err.value
    # the next call starts from a clean array
    spec2 = gpu.scenes.parity_scene(kind="explicit", n_side=12)
    g = GpuScene(gpu, spec2)
    assert g.step(1) == 0
    want = g.particles()
    g.close()
    dev2 = _device_copy(torch, spec2.particles)
    _noalloc_step(lib, spec2, make_params(gpu, spec2.params), dev2, spec2.particles.shape[0], None)
    torch.cuda.synchronize()
    compare_states(dev2.cpu().numpy().view(spec2.particles.dtype), want)


def test_noalloc_without_status_does_not_wait(gpu):
    """With status_out NULL the call only enqueues work; after the caller
    synchronises, the records equal the handle step's."""
    import torch

    lib = gpu.load()
    spec = gpu.scenes.parity_scene(kind="pbmpm", n_side=12, with_collider=False)
    n = spec.particles.shape[0]
    g = GpuScene(gpu, spec)
    assert g.step(1) == 0
    want = g.particles()
    g.close()
    params = make_params(gpu, spec.params)
    ub = spec.uniforms.bytes()
    dev = _device_copy(torch, spec.particles)
    err = C.create_string_buffer(256)
    rc = lib.mpm_step_noalloc(0, C.c_void_p(torch.cuda.current_stream().cuda_stream), C.c_void_p(dev.data_ptr()), n,
                              spec.method, ub, len(ub), C.byref(params), None, 0, 0, None, 0, None, err, len(err))
    assert rc == 0, err.value
    torch.cuda.synchronize()
    compare_states(dev.cpu().numpy().view(spec.particles.dtype), want)
