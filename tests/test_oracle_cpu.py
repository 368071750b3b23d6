"""Known-answer and self-consistency tests of the CPU oracle (no GPU).

The reference ships no golden vectors for the step, so the oracle is pinned
by (a) known answers of its building blocks derived independently here in
Python, (b) agreement of its f32 instantiation with its f64 one, (c) physical
invariants of the transfer, and (d) the committed fixtures in tests/golden/.
"""
import math
import os
import struct

import numpy as np
import pytest

from helpers import compare_states, run_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def hash3_py(x, y, z):
    """xxHash32-style mix of randomNumberGenerators.wgsl:24-38, in Python."""
    M = 0xFFFFFFFF
    p2, p3, p4, p5 = 2246822519, 3266489917, 668265263, 374761393
    rot = lambda v: ((v << 17) | (v >> 15)) & M
    h = (z + p5 + x * p3) & M
    h = (p4 * rot(h)) & M
    h = (h + y * p3) & M
    h = (p4 * rot(h)) & M
    h = (p2 * (h ^ (h >> 15))) & M
    h = (p3 * (h ^ (h >> 13))) & M
    return h ^ (h >> 16)


def f32(x):
    return struct.unpack("<f", struct.pack("<f", x))[0]


def test_hash3_known_answers(oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(0)
    for _ in range(200):
        x, y, z = (int(v) for v in rng.integers(0, 2 ** 32, 3, dtype=np.uint64))
        assert L.or_hash3(x, y, z) == hash3_py(x, y, z)
    # negative block coordinates are hashed through their u32 bit pattern
    assert L.or_hash3((-1) & 0xFFFFFFFF, 0, 5) == hash3_py(0xFFFFFFFF, 0, 5)


@pytest.mark.parametrize("x", [-30.0, -5.0, -0.7, -1e-3, 0.0, 1e-6, 0.3, 1.0, 2.5, 10.0, 40.0])
def test_exp_correctly_rounded(oracle_mod, x):
    got = oracle_mod.lib().or_expf(x)
    assert got == f32(math.exp(f32(x)))


def test_exp_pow_error_bound(oracle_mod):
    L = oracle_mod.lib()
    xs = np.linspace(-80, 80, 4001).astype(np.float32)
    for x in xs:
        e = math.exp(float(x))
        g = L.or_expf(float(x))
        if e < 1e-37 or e > 3e38:
            continue
        assert abs(g - e) <= 0.51 * np.spacing(np.float32(e)) + 1e-45
    ys = np.float32(-0.3333333)
    for v in np.geomspace(1e-3, 1e3, 2001).astype(np.float32):
        want = math.exp(float(ys) * math.log(float(v)))
        g = L.or_powf(float(v), float(ys))
        assert abs(g - want) <= 0.51 * np.spacing(np.float32(want))


def test_pow_matches_exact_rounding(oracle_mod):
    """or_powf (table-driven f64 log/exp) returns the f32 nearest the exact
    power on a sample spanning normal and subnormal bases, and keeps the
    special cases: NaN for a negative or NaN base, pow(+inf, y<0) = 0,
    pow(0, y<0) = +inf, pow(0, 0) = 1."""
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    L = oracle_mod.lib()
    rng = np.random.default_rng(7)
    xs = np.concatenate([np.exp(rng.uniform(-90.0, 88.0, 1500)), rng.uniform(0.5, 2.0, 500),
                         [1.0, 2.0, 0.5, 1e-40, 1.4e-45, 1.1754942e-38, 3e38]]).astype(np.float32)
    for y in (f32(-0.3333333), f32(1.5), f32(1.0 / 2.2)):
        for x in xs:
            x = float(x)
            ex = (Decimal(y) * Decimal(x).ln()).exp()
            want = float("inf") if ex > Decimal("3.4028236e38") else f32(float(ex))
            assert L.or_powf(x, y) == want, (x, y)
    assert math.isnan(L.or_powf(float("nan"), -0.3)) and math.isnan(L.or_powf(-1.0, 0.5))
    assert L.or_powf(float("inf"), -0.3) == 0.0 and L.or_powf(float("inf"), 0.5) == float("inf")
    assert L.or_powf(0.0, -1.0) == float("inf") and L.or_powf(0.0, 0.0) == 1.0 and L.or_powf(0.0, 2.0) == 0.0


def test_pow_tables_current():
    """The committed pow tables are what gen_pow_tables.py writes."""
    import importlib.util
    path = os.path.join(ROOT, "webgpu-mpm-based-snow-simulation_b200", "csrc", "gen_pow_tables.py")
    spec = importlib.util.spec_from_file_location("gen_pow_tables", path)
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    with open(gen.OUT) as f:
        assert f.read() == gen.render()


def test_f2i_saturates_and_truncates(oracle_mod):
    L = oracle_mod.lib()
    assert L.or_f2i(2.9) == 2 and L.or_f2i(-2.9) == -2
    assert L.or_f2i(3e9) == 2 ** 31 - 1 and L.or_f2i(-3e9) == -(2 ** 31)
    assert L.or_f2i(float("nan")) == 0 and L.or_f2i(float("inf")) == 2 ** 31 - 1


def _mat(m):
    return np.ascontiguousarray(np.asarray(m, np.float32).reshape(9))


def test_inverse_and_identity_fallback(oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(1)
    for _ in range(50):
        m = (np.eye(3) + 0.3 * rng.normal(size=(3, 3))).astype(np.float32)
        out = np.zeros(9, np.float32)
        L.orf_inverse(_mat(m).ctypes.data, out.ctypes.data)
        # column-major storage: out[c*3+r] = inv[r][c]; m stored m[c*3+r]
        M = m.reshape(3, 3).T
        Inv = out.reshape(3, 3).T
        assert np.allclose(M @ Inv, np.eye(3), atol=1e-4)
    out = np.zeros(9, np.float32)
    L.orf_inverse(np.zeros(9, np.float32).ctypes.data, out.ctypes.data)
    assert np.array_equal(out.reshape(3, 3), np.eye(3))


def test_polar_rotation_is_orthogonal(oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(2)
    for _ in range(50):
        m = (np.eye(3) + 0.1 * rng.normal(size=(3, 3))).astype(np.float32)
        out = np.zeros(9, np.float32)
        L.orf_polar(_mat(m).ctypes.data, out.ctypes.data)
        R = out.reshape(3, 3).T
        assert np.allclose(R.T @ R, np.eye(3), atol=2e-3)
        assert np.linalg.det(R) > 0


def test_plasticity_clamp(oracle_mod):
    L = oracle_mod.lib()
    ext = oracle_mod.make_ext({})
    # stretch beyond theta_s along x: the singular value is clamped to 1+theta_s
    Fe = _mat(np.diag([1.05, 1.0, 1.0]))
    Fp = _mat(np.eye(3))
    L.orf_plasticity(oracle_mod.C.byref(ext) if hasattr(oracle_mod, "C") else __import__("ctypes").byref(ext),
                     Fe.ctypes.data, Fp.ctypes.data)
    assert abs(Fe[0] - f32(1.0075)) < 1e-6
    # the total deformation Fe*Fp is preserved
    assert abs(Fe[0] * Fp[0] - 1.05) < 1e-5
    # inside the band nothing changes
    Fe2 = _mat(np.diag([1.001, 0.99, 1.0]))
    Fp2 = _mat(np.eye(3))
    before = Fe2.copy()
    L.orf_plasticity(__import__("ctypes").byref(ext), Fe2.ctypes.data, Fp2.ctypes.data)
    assert np.array_equal(Fe2, before)


def test_bspline_partition_of_unity_mass(pkg, oracle_mod):
    """The P2G mass of every particle sums to its mass: the grid total equals
    the particle total up to the fixed-point truncation of each add."""
    spec = pkg.scenes.parity_scene(kind="explicit")
    o, _ = run_oracle(oracle_mod, spec, stop_after=1)
    grid = o.dense_grid(spec.uniforms.bytes())
    scale = 2.0 ** 28
    total = grid[..., 0].astype(np.float64).sum() / scale
    pm = spec.particles["mass"].astype(np.float64).sum()
    n = spec.particles.shape[0]
    assert abs(total - pm) <= 27 * n / scale + 1e-6 * pm


@pytest.mark.parametrize("kind", ["explicit", "pbmpm"])
def test_f32_oracle_tracks_f64(pkg, oracle_mod, kind):
    spec = pkg.scenes.parity_scene(kind=kind, with_collider=True)
    _, p32 = run_oracle(oracle_mod, spec, n_steps=3)
    _, p64 = run_oracle(oracle_mod, spec, n_steps=3, fp64=True)
    dv = np.abs(p32["vel"].astype(np.float64) - p64["vel"])
    vmax = np.abs(p64["vel"]).max()
    assert np.median(dv) < 1e-4 * max(vmax, 1.0)


def test_oracle_threads_deterministic(pkg, oracle_mod):
    spec = pkg.scenes.parity_scene(kind="pbmpm", with_collider=True)
    L = oracle_mod.lib()
    L.orf_set_threads(1)
    _, a = run_oracle(oracle_mod, spec, n_steps=2)
    L.orf_set_threads(4)
    _, b = run_oracle(oracle_mod, spec, n_steps=2)
    compare_states(a, b)


def test_bvh_builders_agree(pkg, oracle_mod):
    """The product's host BVH builder and the oracle's restatement of the
    reference builder (GpuColliderBufferManager.ts:222-350) emit identical
    nodes and triangle order."""
    for mesh in (pkg.scenes.box_mesh((0, 0, 0), (1, 1, 1)),
                 pkg.scenes.merge_meshes(pkg.scenes.box_mesh((0, 0, 0), (1, 1, 1)),
                                         pkg.scenes.icosphere(3, 0.1, (0.5, 0.2, 0.5))),
                 pkg.scenes.fbm_terrain(64, 0.1, 2)):
        v, f = mesh
        n1, o1 = pkg.build_bvh(v, f)
        n2, o2 = oracle_mod.bvh_build(v, f)
        assert np.array_equal(n1, n2)
        assert np.array_equal(o1, o2)
    n, _ = pkg.build_bvh(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32))
    assert n.shape == (1, 8) and n[0, 7] == 0x80000000


def test_bvh_leaves_cover_all_triangles(pkg):
    v, f = pkg.scenes.icosphere(3, 0.1, (0.5, 0.2, 0.5))
    nodes, order = pkg.build_bvh(v, f)
    leaf = (nodes[:, 7] & 0x80000000) != 0
    cnt = nodes[leaf, 7] & 0x7FFFFFFF
    assert cnt.max() <= 4 and cnt.sum() == f.size // 3
    assert sorted(order.tolist()) == list(range(f.size // 3))


def test_svd_return_map_matches_numpy_svd(oracle_mod):
    """The SVD return map (return_map 1, an option of this library): the f64
    oracle equals a numpy SVD clamp of the singular values (Fe' = U clamp(S)
    V^T, Fp' = Fe'^-1 Fe Fp) to 1e-8 (four Jacobi sweeps converge well below
    f32 rounding); the f32 oracle is within 2e-6 of it;
    states whose singular values are all inside the band come back unchanged
    bit for bit."""
    rng = np.random.default_rng(11)
    n = 2000
    Fe = np.eye(3)[None] + rng.normal(0.0, 0.03, (n, 3, 3))
    Fp = np.eye(3)[None] + rng.normal(0.0, 0.01, (n, 3, 3))
    prm = {"theta_c": 2.5e-2, "theta_s": 7.5e-3, "return_map": 1}
    smin, smax = 1 - 2.5e-2, 1 + 7.5e-3
    # 9 stored entries per matrix are column-major: entry 3c + r = M[r][c]
    col = lambda M: np.ascontiguousarray(np.transpose(M, (0, 2, 1))).reshape(-1, 9)
    uncol = lambda m: np.transpose(m.reshape(-1, 3, 3), (0, 2, 1))
    fe64, fp64 = oracle_mod.return_map(col(Fe), col(Fp), prm, fp64=True)
    U, S, Vt = np.linalg.svd(Fe)
    Sc = np.clip(S, smin, smax)
    want_fe = U @ (Sc[:, :, None] * Vt)
    want_fp = np.linalg.inv(want_fe) @ Fe @ Fp
    inside = np.all((S >= smin) & (S <= smax), axis=1)
    got_fe, got_fp = uncol(fe64), uncol(fp64)
    assert np.max(np.abs(got_fe - want_fe)) < 1e-8
    assert np.max(np.abs(got_fp[~inside] - want_fp[~inside])) < 1e-8
    fe32, fp32 = oracle_mod.return_map(col(Fe).astype(np.float32), col(Fp).astype(np.float32), prm)
    assert np.max(np.abs(uncol(fe32).astype(np.float64) - want_fe)) < 2e-6
    # a state well inside the band: unchanged, bit for bit
    F0 = (np.eye(3) * 1.001).astype(np.float32).reshape(1, 9)
    P0 = np.eye(3, dtype=np.float32).reshape(1, 9)
    f, p = oracle_mod.return_map(F0, P0, prm)
    assert np.array_equal(f.view(np.uint32), F0.view(np.uint32)) and np.array_equal(p.view(np.uint32), P0.view(np.uint32))
    # the reference map (return_map 0) differs from the SVD clamp on sheared states
    fr, _ = oracle_mod.return_map(col(Fe), col(Fp), dict(prm, return_map=0), fp64=True)
    assert np.max(np.abs(uncol(fr) - want_fe)) > 1e-4
