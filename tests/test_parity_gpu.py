"""Parity of the CUDA step (through the C ABI) with the CPU oracle.

Bar: the fixed-point grid is compared bit for bit, and so are the particle
fields, because the CUDA path evaluates the oracle's canonical operation
order (the same fused multiply-adds, reciprocal products for substep-constant
divisors, the same f64 exp/log).  Where a
test states a tolerance it is the relative bound 1e-5 on single-step fields.
"""
import numpy as np
import pytest

from helpers import GpuScene, bits_equal, compare_states, make_params, run_oracle

pytestmark = pytest.mark.gpu


def test_device_arithmetic_selftest(gpu):
    """On 2^28 random operand pairs the folded fixed-point encoding equals the
    two-product one after i32 conversion and the device reciprocal equals the
    IEEE quotient 1/d; f32->i32 saturates with NaN -> 0."""
    import ctypes as C
    a, b, nanv = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
    assert gpu.load().mpm_selftest(0, 1 << 28, 12345, C.byref(a), C.byref(b), C.byref(nanv)) == 0
    assert a.value == 0, f"{a.value} identity mismatches"
    assert b.value == 0, f"conversion mismatch code {b.value}"


def _scene(pkg, **kw):
    return pkg.scenes.parity_scene(**kw)


@pytest.mark.parametrize("kind,interaction", [("explicit", False), ("pbmpm", False), ("pbmpm", True)])
def test_p2g_grid_bit_exact(gpu, oracle_mod, kind, interaction):
    spec = _scene(gpu, kind=kind, interaction=interaction)
    g = GpuScene(gpu, spec)
    assert g.p2g_only() == 0
    grid_gpu = g.grid()
    o, _ = run_oracle(oracle_mod, spec, stop_after=1)
    grid_ref = o.dense_grid(spec.uniforms.bytes())
    assert np.count_nonzero(grid_ref[..., 0]) > 100
    assert np.array_equal(grid_gpu, grid_ref), f"{np.count_nonzero(grid_gpu != grid_ref)} cells differ"
    g.close()


@pytest.mark.parametrize("kind,collider,interaction", [
    ("explicit", False, False), ("explicit", True, False), ("pbmpm", False, False), ("pbmpm", True, True)])
def test_one_step_bit_exact(gpu, oracle_mod, kind, collider, interaction):
    spec = _scene(gpu, kind=kind, with_collider=collider, interaction=interaction)
    g = GpuScene(gpu, spec)
    assert g.step(1) == 0
    got = g.particles()
    o, want = run_oracle(oracle_mod, spec, n_steps=1)
    compare_states(got, want)
    grid_gpu = g.grid(apply_update=(kind == "explicit"))
    grid_ref = o.dense_grid(spec.uniforms.bytes())
    assert np.array_equal(grid_gpu, grid_ref)
    g.close()


@pytest.mark.parametrize("tile_edge", [16, 8])
@pytest.mark.parametrize("use_graphs", [True, False])
@pytest.mark.parametrize("n_iter", [1, 2, 4, 5])
def test_pbmpm_iteration_counts_bit_exact(gpu, oracle_mod, n_iter, use_graphs, tile_edge):
    """PBMPM with 1 (no constraint iteration: the first transfer feeds G2P
    directly), 2, 4 and 5 iterations, captured in graphs and launched eagerly,
    at tile edge 16 and at edge 8 (where this small scene's few tiles run the
    512-thread tile kernels): particles after two substeps and the last
    transfer's grid (which of the ping-pong buffers holds it depends on the
    count's parity) equal the oracle's bit for bit."""
    spec = _scene(gpu, kind="pbmpm", with_collider=True, n_iter=n_iter)
    g = GpuScene(gpu, spec, tile_edge=tile_edge, use_graphs=use_graphs)
    assert g.step(2) == 0
    got = g.particles()
    o, want = run_oracle(oracle_mod, spec, n_steps=2)
    compare_states(got, want)
    grid_gpu = g.grid()
    grid_ref = o.dense_grid(spec.uniforms.bytes())
    assert np.count_nonzero(grid_ref[..., 0]) > 100
    assert np.array_equal(grid_gpu, grid_ref), f"{np.count_nonzero(grid_gpu != grid_ref)} cells differ"
    o.close()
    g.close()


@pytest.mark.parametrize("kind", ["explicit", "pbmpm"])
def test_multi_step_bit_exact_and_aggregates(gpu, oracle_mod, kind):
    spec = _scene(gpu, kind=kind, with_collider=True, n_side=12)
    n = 20
    g = GpuScene(gpu, spec)
    assert g.step(n) == 0
    got = g.particles()
    _, want = run_oracle(oracle_mod, spec, n_steps=n)
    compare_states(got, want)
    # aggregates against the f64 oracle: centre of mass relative to its
    # magnitude, net momentum relative to the total absolute momentum, mean J_p
    # relative to itself, each within 1e-3
    _, w64 = run_oracle(oracle_mod, spec, n_steps=n, fp64=True)
    m32, m64 = got["mass"].astype(np.float64), w64["mass"]
    v32, v64 = got["vel"].astype(np.float64), w64["vel"]
    c32 = oracle_mod.aggregates(got["pos"], got["vel"], got["mass"], got["Fp"][:, :, :3].reshape(-1, 9))
    c64 = oracle_mod.aggregates(w64["pos"], w64["vel"], w64["mass"], w64["Fp"])
    abs_mom = float((np.linalg.norm(v64, axis=1) * m64).sum())
    assert np.abs(c32[0] - c64[0]).max() <= 1e-3 * np.abs(c64[0]).max()
    assert np.abs((v32 * m32[:, None]).sum(0) - (v64 * m64[:, None]).sum(0)).max() <= 1e-3 * abs_mom
    assert abs(c32[2] - c64[2]) <= 1e-3 * abs(c64[2])
    g.close()


@pytest.mark.parametrize("kind,interaction", [("explicit", False), ("pbmpm", True)])
def test_non_power_of_two_scale_bit_exact(gpu, oracle_mod, kind, interaction):
    """A fixed-point scale that is not a power of two takes the unfolded
    encoding i32((x * RN(1/dt)) * scale); it matches the oracle as well."""
    spec = _scene(gpu, kind=kind, with_collider=True, interaction=interaction)
    spec.uniforms.write_fixed_point_scale(3.0 * 2.0 ** 26)
    g = GpuScene(gpu, spec)
    assert g.step(2) == 0
    _, want = run_oracle(oracle_mod, spec, n_steps=2)
    compare_states(g.particles(), want)
    g.close()


@pytest.mark.parametrize("n", [1, 7, 255, 257])
def test_small_and_ragged_counts(gpu, oracle_mod, n):
    spec = _scene(gpu, kind="explicit", n_side=8)
    spec.particles = spec.particles[:n].copy()
    g = GpuScene(gpu, spec)
    assert g.step(2) == 0
    _, want = run_oracle(oracle_mod, spec, n_steps=2)
    compare_states(g.particles(), want)
    g.close()


@pytest.mark.parametrize("kind", ["explicit", "pbmpm"])
def test_coincident_particles_bit_exact(gpu, oracle_mod, kind):
    """Half of the particles stacked on one point and a quarter on another
    (every lane of a warp adding to the same grid cells): two substeps equal
    the oracle bit for bit."""
    spec = _scene(gpu, kind=kind, with_collider=(kind == "pbmpm"))
    p = spec.particles
    n = p.shape[0]
    p["pos"][: n // 2] = p["pos"][0]
    p["pos"][n // 2: 3 * n // 4] = p["pos"][n - 1]
    g = GpuScene(gpu, spec)
    assert g.step(2) == 0
    got = g.particles()
    o, want = run_oracle(oracle_mod, spec, n_steps=2)
    o.close()
    compare_states(got, want)
    g.close()


@pytest.mark.parametrize("kind", ["pbmpm", "explicit"])
def test_tile_edges_agree(gpu, oracle_mod, kind):
    spec = _scene(gpu, kind=kind, with_collider=True)
    outs = []
    for e in (8, 12, 14, 16):
        g = GpuScene(gpu, spec, tile_edge=e)
        assert g.step(3) == 0
        outs.append(g.particles())
        g.close()
    for o in outs[1:]:
        compare_states(o, outs[0])
    _, want = run_oracle(oracle_mod, spec, n_steps=3)
    compare_states(outs[0], want)


def test_graph_and_eager_agree(gpu):
    spec = _scene(gpu, kind="explicit", with_collider=True)
    outs = []
    for use_graphs in (True, False):
        g = GpuScene(gpu, spec, use_graphs=use_graphs)
        assert g.step(4) == 0
        outs.append(g.particles())
        g.close()
    compare_states(outs[0], outs[1])


def test_particles_outside_domain(gpu, oracle_mod):
    """Particles below the grid minimum and far outside it: the oracle and the
    GPU both reflect them back to the boundary."""
    spec = _scene(gpu, kind="explicit", n_side=8)
    p = spec.particles
    p["pos"][0] = [-0.01, 0.5, 0.5]
    p["pos"][1] = [0.5, -3.0, 0.5]
    p["pos"][2] = [0.5, 0.5, 7.0]
    g = GpuScene(gpu, spec)
    assert g.step(1) == 0
    _, want = run_oracle(oracle_mod, spec, n_steps=1)
    compare_states(g.particles(), want)
    g.close()


def test_tile_overflow_reports_status(gpu):
    """Capacity overflow sets a status bit instead of dropping work silently."""
    spec = gpu.scenes.c0_explicit_snow(n_side=16)
    g = GpuScene(gpu, spec, tile_edge=8, max_tiles=2)
    with pytest.raises(gpu.MpmError) as ei:
        g.step(1)
    assert ei.value.status & 0x2
    g.close()


@pytest.mark.parametrize("kind,res,n_side,min_tiles", [
    ("explicit", 128, 16, 1024), ("pbmpm", 128, 16, 1024), ("pbmpm", 256, 20, 4096)])
def test_many_tiles_bit_exact(gpu, oracle_mod, kind, res, n_side, min_tiles):
    """Sparse scenes with thousands of occupied tiles (above the 256 below
    which the tile kernels keep the compact tile order; the last case above
    the 4,096 where the order's Morton bucket widens), so the tiles are
    claimed in Morton order, alternating direction between passes: results
    stay bit-exact against the oracle."""
    spec = _scene(gpu, kind=kind, res=res, n_side=n_side)
    rng = np.random.default_rng(31)
    n = spec.particles.shape[0]
    spec.particles["pos"] = rng.uniform(0.05, 0.95, size=(n, 3)).astype(np.float32)
    g = GpuScene(gpu, spec, tile_edge=8)
    assert g.step(2) == 0
    n_tiles, _ = g.buf.counts()
    assert n_tiles > min_tiles, n_tiles
    got = g.particles()
    o, want = run_oracle(oracle_mod, spec, n_steps=2)
    compare_states(got, want)
    if res <= 128:
        assert np.array_equal(g.grid(apply_update=(kind == "explicit")), o.dense_grid(spec.uniforms.bytes()))
    g.close()


def test_permutation_invariance(gpu):
    """Results per particle do not depend on the record order."""
    spec = _scene(gpu, kind="pbmpm", with_collider=True)
    g = GpuScene(gpu, spec)
    assert g.step(2) == 0
    a = g.particles()
    g.close()
    perm = np.random.default_rng(5).permutation(spec.particles.shape[0])
    spec.particles = spec.particles[perm].copy()
    g = GpuScene(gpu, spec)
    assert g.step(2) == 0
    b = g.particles()
    g.close()
    inv = np.argsort(perm)
    compare_states(b[inv], a)


def test_bound_device_buffer_updated_after_each_step(gpu, oracle_mod):
    """Zero-copy binding (mpm_bind_particles_device): the library advances
    its own tile-ordered copy of the state and writes the caller's buffer
    back, in the caller's order, at the end of every step call."""
    import torch

    spec = _scene(gpu, kind="pbmpm", with_collider=True)
    n = spec.particles.shape[0]
    dev = torch.from_numpy(spec.particles.view(np.uint8).reshape(-1).copy()).cuda()
    g = GpuScene(gpu, spec)
    g.buf.bind_particles_device(dev.data_ptr(), n)
    for steps in (1, 3):
        assert g.step(1 if steps == 1 else 2) == 0
        torch.cuda.synchronize()
        got = dev.cpu().numpy().view(spec.particles.dtype)
        _, want = run_oracle(oracle_mod, spec, n_steps=steps)
        compare_states(got, want)
    g.close()


def test_reading_between_steps_changes_nothing(gpu):
    """Reading the records (which brings the caller-order copy up to date)
    between substeps leaves the state the substeps advance untouched."""
    spec = _scene(gpu, kind="explicit", with_collider=True)
    a = GpuScene(gpu, spec)
    assert a.step(4) == 0
    want = a.particles()
    a.close()
    b = GpuScene(gpu, spec)
    for _ in range(4):
        assert b.step(1) == 0
        b.particles()
    compare_states(b.particles(), want)
    b.close()


def test_device_upload_and_pointer(gpu, oracle_mod):
    """Records uploaded from device memory, read back into device memory,
    and the device pointer the library hands out: all hold the current
    records in the caller's order."""
    import ctypes as C

    import torch

    spec = _scene(gpu, kind="explicit", n_side=10)
    n = spec.particles.shape[0]
    nbytes = n * spec.particles.dtype.itemsize
    src = torch.from_numpy(spec.particles.view(np.uint8).reshape(-1).copy()).cuda()
    g = GpuScene(gpu, spec)
    g.buf.write_particles_device(src.data_ptr(), n)
    assert g.step(2) == 0
    _, want = run_oracle(oracle_mod, spec, n_steps=2)
    out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    lib = gpu.load()
    assert lib.mpm_get_particles(g.buf.handle, C.c_void_p(out.data_ptr()), n, 1) == 0
    torch.cuda.synchronize()
    compare_states(out.cpu().numpy().view(spec.particles.dtype), want)
    ptr = lib.mpm_particles_device_ptr(g.buf.handle)
    assert ptr
    assert g.buf.sync() == 0

    class _Raw:  # a view of the library's record buffer for torch
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}

    recs = torch.as_tensor(_Raw(), device="cuda").clone()
    compare_states(recs.cpu().numpy().view(spec.particles.dtype), want)
    # readback into pinned host memory without waiting (dst_is_device = 2)
    assert g.step(1) == 0
    _, want3 = run_oracle(oracle_mod, spec, n_steps=3)
    pinned = torch.zeros(nbytes, dtype=torch.uint8, pin_memory=True)
    assert lib.mpm_get_particles(g.buf.handle, C.c_void_p(pinned.data_ptr()), n, 2) == 0
    assert g.buf.sync() == 0
    compare_states(pinned.numpy().view(spec.particles.dtype), want3)
    g.close()


@pytest.mark.parametrize("max_tiles,hash_capacity,bit", [(64, 0, 0x2), (8192, 4096, 0x1)])
def test_capacity_overflow_keeps_every_particle(gpu, max_tiles, hash_capacity, bit):
    """When tiles do not fit the tile storage (status 0x2) or the tile hash
    table is full (0x1), the particles no tile kernel advances are carried
    over unchanged: after the step every particle is still present once, at
    its own caller index (masses, which a substep never changes, are all
    distinct here), and the unadvanced ones keep their records bit for bit."""
    spec = _scene(gpu, kind="explicit", res=256, n_side=20)
    n = spec.particles.shape[0]
    rng = np.random.default_rng(41)
    spec.particles["pos"] = rng.uniform(0.05, 0.95, size=(n, 3)).astype(np.float32)
    spec.particles["mass"] = (np.float32(1e-6) * (1.0 + np.arange(n) / n)).astype(np.float32)
    buf = gpu.GpuMpmBufferManager(n_particles=n, tile_edge=8, max_tiles=max_tiles, hash_capacity=hash_capacity)
    buf.write_particles(spec.particles)
    pipe = gpu.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms,
                                     params=make_params(gpu, spec.params))
    pipe.add_explicit_mpm_dispatches(n_particles=n)
    with pytest.raises(gpu.MpmError) as ei:
        buf.sync()
    assert ei.value.status & bit, ei.value.status
    gpu.load().mpm_clear_status(buf.handle)
    got = buf.read_particles()
    assert np.array_equal(got["mass"].view(np.uint32), spec.particles["mass"].view(np.uint32))
    same = np.all(got["pos"] == spec.particles["pos"], axis=1)
    assert 0 < same.sum() < n, same.sum()
    kept = got[same]
    for f in ("vel", "Fe", "Fp", "dxp", "D"):
        assert np.array_equal(kept[f].view(np.uint32), spec.particles[same][f].view(np.uint32)), f
    buf.close()
