"""Marching cubes (mcListBlocks, mcVertexDensity, mcGenerate): the library's
case table is the reference's (the oracle reads the same table and restates
the reference's edge endpoints), consistent with the reference's separate
per-case triangle counts; the CUDA passes equal the oracle's restatement
vertex for vertex on the GPU, on a synthetic density field with partial
blocks, with a vertex cap, and through the chain simulation ->
calculateDensity -> mesh."""
from collections import Counter

import numpy as np
import pytest

from helpers import GpuScene


def _blobs(res, seed=0, scale=2.0 ** 28):
    """u32 density grid [z][y][x] of Gaussian blobs, zero on the border."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.arange(r) + 0.5 for r in res[::-1]), indexing="ij")
    g = np.zeros(res[::-1])
    for _ in range(5):
        c = rng.uniform(0.3, 0.7, 3) * np.array(res)
        r = rng.uniform(0.08, 0.16) * min(res)
        g += np.exp(-(((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * r * r)))
    g[0, :, :] = g[-1, :, :] = g[:, 0, :] = g[:, -1, :] = g[:, :, 0] = g[:, :, -1] = 0
    return np.floor(g * 0.6 * scale).astype(np.uint32)


def test_tables_are_the_reference_table(pkg, oracle_mod):
    tri, cnt, ev = pkg.pipeline.mc_tables()
    otri, ocnt, oev = oracle_mod.mc_tables()
    assert np.array_equal(tri, otri) and np.array_equal(cnt, ocnt)
    # the library derives the edge endpoints from the numbering; the oracle
    # restates the reference's MC_EDGE_V0 / MC_EDGE_V1
    assert np.array_equal(ev, oev)
    assert cnt[0] == 0 and cnt[255] == 0 and cnt.max() <= 5
    # first cases of MC_TRI_TABLE (triTable.wgsl:6-9)
    assert tri[1][:3].tolist() == [0, 8, 4] and tri[2][:3].tolist() == [0, 5, 9]
    assert tri[3][:6].tolist() == [8, 4, 9, 9, 4, 5]
    for c in range(256):
        # the reference's per-case counts (MC_TRI_COUNTS) equal its triangle lists
        used = tri[c][: 3 * cnt[c]]
        assert np.all(used >= 0) and np.all(tri[c][3 * cnt[c]:] == -1)
        # every triangle edge index is a cut edge of the case
        for e in used:
            a, b = ev[e]
            assert ((c >> a) & 1) != ((c >> b) & 1)
    # the total number of triangles over all cases
    assert int(cnt.sum()) == int((tri >= 0).sum()) // 3


def test_oracle_mesh_is_closed_and_oriented(oracle_mod):
    res = (20, 17, 23)
    dens = _blobs(res, seed=3)
    mres = (19, 21, 16)
    verts, n = oracle_mod.marching_cubes(dens, [0, 0, 0], [1, 1, 1], 2.0 ** 28, mres)
    assert n > 300 and n % 3 == 0
    key = [tuple(v) for v in np.ascontiguousarray(verts[:, :3]).view(np.uint32).reshape(-1, 3).tolist()]
    directed = Counter()
    for t in range(0, n, 3):
        tri = key[t:t + 3]
        for i in range(3):
            directed[(tri[i], tri[(i + 1) % 3])] += 1
    # a closed, consistently oriented surface uses every edge once in each direction
    # (degenerate slivers, where two cut points coincide, are skipped)
    bad = [(a, b) for (a, b), k in directed.items() if a != b and directed.get((b, a), 0) != k]
    assert not bad, len(bad)
    nrm = verts[:, 3:]
    lens = np.linalg.norm(nrm, axis=1)
    assert np.all((np.abs(lens - 1) < 1e-4) | (lens == 0))


@pytest.mark.gpu
@pytest.mark.parametrize("cap", [None, 999])
def test_mc_bit_exact_synthetic(gpu, oracle_mod, cap):
    import torch

    spec = gpu.scenes.parity_scene(kind="pbmpm")
    g = GpuScene(gpu, spec)
    res = (26, 22, 30)
    mres = (37, 29, 44)          # partial 8^3 blocks on every axis
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    dens = _blobs(res, seed=1, scale=scale)
    want, n_want = oracle_mod.marching_cubes(dens, [0, 0, 0], [1, 1, 1], scale, mres)
    assert n_want > 1000
    max_v = n_want + 10 if cap is None else cap
    out = torch.zeros((max_v, 6), dtype=torch.float32, device="cuda")
    d_dev = torch.from_numpy(dens.view(np.int32)).cuda()
    import ctypes as C
    lib = gpu.load()
    dres = (C.c_uint32 * 3)(res[0], res[1], res[2])
    mr = (C.c_uint32 * 3)(*mres)
    cnt, gen = C.c_uint32(0), C.c_uint32(0)
    torch.cuda.synchronize()
    gpu._lib.check(lib.mpm_marching_cubes(g.buf.handle, 0, C.c_void_p(d_dev.data_ptr()), dres, mr,
                                          C.c_void_p(out.data_ptr()), max_v, C.byref(cnt), C.byref(gen)), g.buf.handle)
    assert gen.value == n_want
    assert cnt.value == min(n_want, max_v)
    got = out[: cnt.value].cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want[: cnt.value].view(np.uint32))
    g.close()


@pytest.mark.gpu
def test_mc_chain_after_simulation(gpu, oracle_mod):
    spec = gpu.scenes.parity_scene(kind="explicit", with_collider=True)
    g = GpuScene(gpu, spec)
    assert g.step(3) == 0
    # a coarse density grid (8^3 cells of the unit box): the snow block's mass per
    # cell exceeds the isovalue 0.15 there; the MC grid is finer (24^3)
    mc = gpu.GpuMarchingCubesBufferManager(grid_resolution=(16, 16, 16), mc_grid_resolution=(24, 24, 24),
                                           max_vertices=400_000)
    rp = gpu.GpuMarchingCubesRenderPipelineManager(mpm_manager=g.buf, mc_manager=mc)
    n = rp.add_mesh_generation_pass()
    scale = float(np.frombuffer(spec.uniforms.bytes()[4:8], "<f4")[0])
    dens = oracle_mod.splat("density", g.particles(), [0, 0, 0], [1, 1, 1], mc.density_grid_resolution, scale)
    assert np.array_equal(mc.density_grid.cpu().numpy().view(np.uint32), dens)
    want, n_want = oracle_mod.marching_cubes(dens, [0, 0, 0], [1, 1, 1], scale, mc.mc_grid_resolution)
    assert n == n_want and n > 30
    assert np.array_equal(mc.vertices[:n].cpu().numpy().view(np.uint32), want.view(np.uint32))
    g.close()


@pytest.mark.gpu
def test_mc_empty_density_gives_no_vertices(gpu):
    import ctypes as C

    import torch

    spec = gpu.scenes.parity_scene(kind="explicit")
    g = GpuScene(gpu, spec)
    d_dev = torch.zeros((9, 10, 11), dtype=torch.int32, device="cuda")
    out = torch.zeros((16, 6), dtype=torch.float32, device="cuda")
    cnt, gen = C.c_uint32(7), C.c_uint32(7)
    gpu._lib.check(gpu.load().mpm_marching_cubes(g.buf.handle, 0, C.c_void_p(d_dev.data_ptr()),
                                                 (C.c_uint32 * 3)(11, 10, 9), (C.c_uint32 * 3)(20, 17, 13),
                                                 C.c_void_p(out.data_ptr()), 16, C.byref(cnt), C.byref(gen)),
                   g.buf.handle)
    assert cnt.value == 0 and gen.value == 0
    g.close()
