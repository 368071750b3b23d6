"""The benchmark scenes in their own mode, against the oracle.

The benchmark configurations run the step with constants that differ from the
reference's: y-up gravity (0, -9.8, 0), hardening 10, a grid-side sticky
ground layer with slip walls (boundary mode 1), collider margins scaled to the
cell size, and fixed-point scales of 2^34 (config 0), 2^39 (config 1) and 2^45
(config 2).  Each scene here is advanced on the GPU through the C ABI and by
the f32 oracle from the same initial records, in that mode.

Bar: the fixed-point grid and every particle field bit for bit after one
substep, the particle fields bit for bit after 20 substeps; against the f64
oracle, after 100 substeps of config 0, the centre of mass (relative to its
own magnitude), the net momentum (relative to the total absolute momentum) and
the mean J_p (relative to itself) each within 1e-3.
"""
import numpy as np
import pytest

from helpers import GpuScene, compare_states, make_params

pytestmark = pytest.mark.gpu

AGG_TOL = 1e-3


def _oracle(oracle_mod, spec, n_steps, fp64=False, stop_after=0):
    """Oracle context and records after n_steps substeps (capacities sized for
    the large slab's ~3e5 reference blocks)."""
    p = spec.particles.copy()
    if fp64:
        p = oracle_mod.to_fp64(p)
    o = oracle_mod.Oracle(p.shape[0], max_blocks=600000, hash_size=2000003, fp64=fp64)
    if spec.mesh is not None:
        o.set_collider(*spec.mesh)
    for _ in range(n_steps):
        o.step(spec.uniforms.bytes(), spec.params, p, spec.method, stop_after)
    return o, p


def _aggregates(rec):
    """(centre of mass, net momentum, total |momentum|, mean J_p) in f64, for
    192-byte records or the f64 oracle's records."""
    m = rec["mass"].astype(np.float64)
    v = rec["vel"].astype(np.float64)
    com = (rec["pos"].astype(np.float64) * m[:, None]).sum(0) / m.sum()
    mom = (v * m[:, None]).sum(0)
    abs_mom = float((np.linalg.norm(v, axis=1) * m).sum())
    Fp = rec["Fp"]
    Fp = Fp.reshape(-1, 3, 3) if Fp.ndim == 2 else Fp[:, :, :3]
    jp = float(np.linalg.det(Fp.astype(np.float64)).mean())
    return com, mom, abs_mom, jp


def _agg_errors(got, ref64):
    a, b = _aggregates(got), _aggregates(ref64)
    return {"centre_of_mass": float(np.abs(a[0] - b[0]).max() / np.abs(b[0]).max()),
            "momentum": float(np.abs(a[1] - b[1]).max() / max(b[2], 1e-30)),
            "mean_jp": float(abs(a[3] - b[3]) / abs(b[3]))}


def _config_mode(spec):
    """The scene really runs in the benchmark mode (guards the fixtures)."""
    p = spec.params
    assert p["boundary_mode"] == 1 and p["ground_axis"] == 1
    assert list(p["gravity"]) == [0.0, -9.8, 0.0]
    assert p["hardening_explicit"] == 10.0 and p["hardening_pbmpm"] == 10.0


def _c0(gpu):
    return gpu.scenes.c0_explicit_snow()


def _c1(gpu):
    return gpu.scenes.c1_pbmpm_spheres()


def _c2_block(gpu):
    return gpu.scenes.c2_large_pbmpm(counts=(128, 32, 128))


SCENES = {"c0": _c0, "c1": _c1, "c2_block": _c2_block}


@pytest.mark.parametrize("name", list(SCENES))
def test_config_one_substep_grid_and_particles_bit_exact(gpu, oracle_mod, name):
    spec = SCENES[name](gpu)
    _config_mode(spec)
    g = GpuScene(gpu, spec)
    assert g.step(1) == 0
    got = g.particles()
    o, want = _oracle(oracle_mod, spec, 1)
    compare_states(got, want)
    if max(spec.res) <= 128:
        grid_gpu = g.grid(apply_update=(spec.method == 0))
        grid_ref = o.dense_grid(spec.uniforms.bytes())
        assert np.count_nonzero(grid_ref[..., 0]) > 1000
        assert np.array_equal(grid_gpu, grid_ref), f"{np.count_nonzero(grid_gpu != grid_ref)} cells differ"
    o.close()
    g.close()


def test_config2_block_p2g_grid_bit_exact(gpu, oracle_mod):
    """The large slab's first transfer at its 512^3 grid and 2^45 scale: the
    dense grid is compared over the slab's bounding box of cells."""
    spec = _c2_block(gpu)
    _config_mode(spec)
    g = GpuScene(gpu, spec)
    assert g.p2g_only() == 0
    grid_gpu = g.grid()
    o, _ = _oracle(oracle_mod, spec, 1, stop_after=1)
    grid_ref = o.dense_grid(spec.uniforms.bytes())
    occupied = np.count_nonzero(grid_ref[..., 0])
    assert occupied > 1_000_000, occupied
    assert np.array_equal(grid_gpu, grid_ref), f"{np.count_nonzero(grid_gpu != grid_ref)} cells differ"
    o.close()
    g.close()


@pytest.mark.parametrize("name", list(SCENES))
def test_config_twenty_substeps_bit_exact(gpu, oracle_mod, name):
    spec = SCENES[name](gpu)
    g = GpuScene(gpu, spec)
    assert g.step(20) == 0
    got = g.particles()
    o, want = _oracle(oracle_mod, spec, 20)
    compare_states(got, want)
    o.close()
    g.close()


def test_config0_hundred_substeps_against_fp64(gpu, oracle_mod):
    """Config 0 as specified (100 substeps): bit-exact against the f32 oracle,
    and each aggregate within 1e-3 of the f64 oracle."""
    spec = _c0(gpu)
    g = GpuScene(gpu, spec)
    assert g.step(100) == 0
    got = g.particles()
    g.close()
    o, want = _oracle(oracle_mod, spec, 100)
    o.close()
    compare_states(got, want)
    o, w64 = _oracle(oracle_mod, spec, 100, fp64=True)
    o.close()
    err = _agg_errors(got, w64)
    assert all(v <= AGG_TOL for v in err.values()), err


def test_config1_aggregates_against_fp64(gpu, oracle_mod):
    """Config 1 (two spheres colliding, PBMPM x6, box + icosphere collider),
    20 substeps: aggregates within 1e-3 of the f64 oracle."""
    spec = _c1(gpu)
    g = GpuScene(gpu, spec)
    assert g.step(20) == 0
    got = g.particles()
    g.close()
    o, w64 = _oracle(oracle_mod, spec, 20, fp64=True)
    o.close()
    err = _agg_errors(got, w64)
    assert all(v <= AGG_TOL for v in err.values()), err


def test_config2_full_size_substep_bit_exact(gpu, oracle_mod):
    """One substep of the full 4,194,304-particle slab (the benchmark
    workload) against the f32 oracle, every particle field bit for bit."""
    spec = gpu.scenes.c2_large_pbmpm()
    assert spec.particles.shape[0] == 4_194_304
    g = GpuScene(gpu, spec)
    assert g.step(1) == 0
    got = g.particles()
    g.close()
    o, want = _oracle(oracle_mod, spec, 1)
    o.close()
    compare_states(got, want)


def test_config3_batch_scenes_against_oracle(gpu, oracle_mod):
    """A small batch of config-3 scenes (explicit, each with its own E,
    theta_c and dx) in one handle: each scene equals the f32 oracle's run of
    that scene alone, bit for bit."""
    specs = gpu.scenes.c3_batched(n_scenes=5, seed=8, lo_count=500, hi_count=6000)
    for s in specs:
        _config_mode(s)
    b = gpu.GpuMpmBatch(specs)
    b.step(gpu.GpuSimulationMethodType.ExplicitMpm, 5)
    assert b.mpm.sync() == 0
    rec = b.mpm.read_particles()
    for i, spec in enumerate(specs):
        o, want = _oracle(oracle_mod, spec, 5)
        o.close()
        compare_states(b.scene_particles(i, rec), want)
    b.close()


def _tiles_at(gpu, spec, edge):
    """Occupied tiles of the scene's first substep at a fixed tile edge."""
    g = GpuScene(gpu, spec, tile_edge=edge)
    assert g.step(1) == 0
    n = g.buf.counts()[0]
    g.close()
    return n


def _rule(n_st, n_sms, usable=(True, True, True)):
    """The library's choice over edges (16, 12, 8): among the edges with at
    least two occupied tiles per SM, the fewest halo cells ((E+2)^3 per tile;
    a smaller edge only below 9/10 of the current choice's), else the edge
    with the most tiles."""
    edges = (16, 12, 8)
    halo = [n * (e + 2) ** 3 for e, n in zip(edges, n_st)]
    pick = None
    for i in range(3):
        if usable[i] and n_st[i] >= 2 * n_sms and (pick is None or 10 * halo[i] < 9 * halo[pick]):
            pick = i
    if pick is None:
        pick = max((i for i in range(3) if usable[i]), key=lambda i: n_st[i])
    return edges[pick]


@pytest.mark.parametrize("name", ["c1", "c2_block"])
def test_automatic_tile_edge_follows_occupancy_and_stays_bit_exact(gpu, oracle_mod, name):
    """tile_edge 0: the first step picks the edge from the occupied tiles (two
    spheres of config 1 fill 60 tiles of 16^3 and run at edge 8; the 524,288-
    particle slab fills 676, whose halos hold fewer cells than its 1,620 tiles
    of 12^3 or 4,732 of 8^3, and stays at 16); the substeps then equal the f32
    oracle bit for bit."""
    import torch

    spec = SCENES[name](gpu)
    n_sms = torch.cuda.get_device_properties(0).multi_processor_count
    n_st = [_tiles_at(gpu, spec, e) for e in (16, 12, 8)]
    g = GpuScene(gpu, spec, tile_edge=0)
    assert g.buf.tile_edge == 16          # nothing chosen before the first step
    assert g.step(5) == 0
    edge = g.buf.tile_edge
    assert edge == _rule(n_st, n_sms), (n_st, edge)
    assert edge == (8 if name == "c1" else 16)
    got = g.particles()
    g.close()
    o, want = _oracle(oracle_mod, spec, 5)
    o.close()
    compare_states(got, want)


def test_automatic_tile_edge_respects_fixed_max_tiles(gpu, oracle_mod):
    """With a fixed tile capacity, an edge whose occupied tiles exceed it is
    not a candidate: config 1 with room for 200 tiles runs at edge 12 (~100
    tiles) instead of 8 (~240), bit-exact."""
    import torch

    spec = _c1(gpu)
    n_sms = torch.cuda.get_device_properties(0).multi_processor_count
    n_st = [_tiles_at(gpu, spec, e) for e in (16, 12, 8)]
    cap = 200
    usable = [n <= cap for n in n_st]
    g = GpuScene(gpu, spec, tile_edge=0, max_tiles=cap)
    assert g.step(3) == 0
    assert g.buf.tile_edge == _rule(n_st, n_sms, usable)
    got = g.particles()
    g.close()
    o, want = _oracle(oracle_mod, spec, 3)
    o.close()
    compare_states(got, want)


@pytest.mark.parametrize("tile_edge,edges", [(0, (8, 16)), (8, (8, 8))])
def test_new_particle_count_sizes_the_handle_again(gpu, oracle_mod, tile_edge, edges):
    """One handle first runs config 1, then is given the 524,288-particle slab
    (a new particle count): the next step sizes the tile storage again (at
    edge 8 the slab fills 4,732 tiles, against 248 for config 1) and, with
    tile_edge 0, picks the edge again (8, then 16, the tile buffers growing to
    the larger halo); no capacity status is raised and the slab's substeps
    equal the f32 oracle bit for bit."""
    c1, slab = _c1(gpu), _c2_block(gpu)
    n = max(c1.particles.shape[0], slab.particles.shape[0])
    buf = gpu.GpuMpmBufferManager(n_particles=n, tile_edge=tile_edge)
    try:
        for spec, want_edge, steps in ((c1, edges[0], 2), (slab, edges[1], 3)):
            buf.write_particles(spec.particles)
            col = None
            if spec.mesh is not None:
                col = gpu.GpuColliderBufferManager(vertices=spec.mesh[0], indices=spec.mesh[1])
            pipe = gpu.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms,
                                             collider_manager=col, params=make_params(gpu, spec.params))
            for _ in range(steps):
                pipe.add_pbmpm_dispatches(n_particles=buf.n_particles)
            assert buf.sync() == 0
            assert buf.tile_edge == want_edge
            got = buf.read_particles()
            o, want = _oracle(oracle_mod, spec, steps)
            o.close()
            compare_states(got, want)
    finally:
        buf.close()


def test_edge8_tile_kernel_widths_bit_exact(gpu, oracle_mod):
    """At tile edge 8 the tile kernels run 512-thread CTAs when the occupied
    tiles number fewer than two per SM (config 1: 248 tiles; config 0: 80) and
    their usual widths otherwise (the 524,288-particle slab: 4,732 tiles),
    for PBMPM (first transfer, iterations, G2P) and explicit MPM (P2G, G2P);
    every case equals the f32 oracle bit for bit after two substeps."""
    import ctypes as C
    import dataclasses

    import torch

    lib = gpu.load()
    names = gpu.kernel_names()
    K = lib.mpm_kernel_count()
    n_sms = torch.cuda.get_device_properties(0).multi_processor_count
    slab = _c2_block(gpu)
    cases = [(_c1(gpu), ("pbmpm_first", 2), ("pbmpm_iter", 2 * 5), ("g2p_pbmpm_integrate", 2)),
             (slab, ("pbmpm_first", 2), ("pbmpm_iter", 2 * 5), ("g2p_pbmpm_integrate", 2)),
             (_c0(gpu), ("p2g_explicit", 2), ("g2p_explicit_integrate", 2)),
             (dataclasses.replace(slab, method=0), ("p2g_explicit", 2), ("g2p_explicit_integrate", 2))]
    for spec, *expect in cases:
        g = GpuScene(gpu, spec, tile_edge=8)
        lib.mpm_enable_kernel_timing(g.buf.handle, 1)
        assert g.step(2) == 0
        kms, kcnt = (C.c_float * K)(), (C.c_uint32 * K)()
        lib.mpm_kernel_times(g.buf.handle, kms, kcnt, K)
        launches = {names[i]: kcnt[i] for i in range(K) if kcnt[i]}
        wide = g.buf.counts()[0] < 2 * n_sms
        for k, n in expect:
            used, unused = (k + "_wide", k) if wide else (k, k + "_wide")
            assert launches.get(used, 0) == n and unused not in launches, (spec.name, launches)
        got = g.particles()
        g.close()
        o, want = _oracle(oracle_mod, spec, 2)
        o.close()
        compare_states(got, want)


def test_edge8_width_follows_the_tile_count_at_sync(gpu, oracle_mod):
    """The CTA width at tile edge 8 follows the occupied tiles at each sync:
    a handle with fixed tile storage starts at the usual width, turns wide
    after the first sync of config 1 (248 tiles), and back after the sync that
    follows new records spread over the whole domain (thousands of tiles);
    the spread particles' substeps equal the f32 oracle bit for bit."""
    import ctypes as C

    lib = gpu.load()
    names = gpu.kernel_names()
    K = lib.mpm_kernel_count()

    def launches(h):
        kms, kcnt = (C.c_float * K)(), (C.c_uint32 * K)()
        lib.mpm_kernel_times(h, kms, kcnt, K)
        lib.mpm_enable_kernel_timing(h, 1)     # and start counting again
        return {names[i]: kcnt[i] for i in range(K) if kcnt[i]}

    spec = _c1(gpu)
    g = GpuScene(gpu, spec, tile_edge=8, max_tiles=8192)
    h = g.buf.handle
    lib.mpm_enable_kernel_timing(h, 1)
    assert g.step(1) == 0
    assert launches(h).get("pbmpm_iter") == 5
    assert g.step(1) == 0
    assert launches(h).get("pbmpm_iter_wide") == 5
    spread = spec.particles.copy()
    rng = np.random.default_rng(3)
    spread["pos"] = rng.uniform(0.05, 0.95, spread["pos"].shape).astype(np.float32)
    g.buf.write_particles(spread)
    assert g.step(1) == 0
    assert launches(h).get("pbmpm_iter_wide") == 5
    import torch
    assert g.buf.counts()[0] >= 3 * torch.cuda.get_device_properties(0).multi_processor_count
    assert g.step(2) == 0
    last = launches(h)
    assert last.get("pbmpm_iter") == 10 and "pbmpm_iter_wide" not in last, last
    got = g.particles()
    g.close()
    o = oracle_mod.Oracle(spread.shape[0], max_blocks=600000, hash_size=2000003)
    o.set_collider(*spec.mesh)
    want = spread.copy()
    for _ in range(3):
        o.step(spec.uniforms.bytes(), spec.params, want, spec.method)
    o.close()
    compare_states(got, want)
