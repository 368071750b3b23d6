"""The benchmark scenes match the configurations they stand for: particle
counts, method, iteration count, grid and time step, and the config-mode
constants (y-up gravity, hardening 10, boundary mode 1).  Host-side only."""
import numpy as np


def _mode(spec):
    p = spec.params
    assert p["boundary_mode"] == 1 and p["ground_axis"] == 1
    assert list(p["gravity"]) == [0.0, -9.8, 0.0]
    assert p["hardening_explicit"] == 10.0 and p["hardening_pbmpm"] == 10.0


def test_config0_explicit_snow(pkg):
    s = pkg.scenes.c0_explicit_snow()
    assert s.particles.shape[0] == 32_768 and s.method == 0 and s.n_steps == 100
    assert tuple(s.res) == (64, 64, 64)
    _mode(s)


def test_config1_colliding_spheres(pkg):
    s = pkg.scenes.c1_pbmpm_spheres()
    assert s.particles.shape[0] == 262_144 and s.method == 1 and int(s.params["n_iter"]) == 6
    assert s.mesh is not None and s.mesh[1].size // 3 == 1_292
    v = s.particles["vel"]
    assert np.isclose(v[:, 0].max(), 2.0) and np.isclose(v[:, 0].min(), -2.0)   # +-2 m/s
    _mode(s)


def test_config2_block_shape(pkg):
    """The 524,288-particle block of the slab (the full 4,194,304-particle
    slab is the same lattice at 256 x 64 x 256)."""
    s = pkg.scenes.c2_large_pbmpm(counts=(128, 32, 128))
    assert s.particles.shape[0] == 128 * 32 * 128 and s.method == 1 and int(s.params["n_iter"]) == 6
    assert tuple(s.res) == (512, 512, 512)
    assert s.mesh is not None and s.mesh[1].size // 3 == 130_050
    _mode(s)


def test_config3_scene_distribution(pkg):
    specs = pkg.scenes.c3_batched(n_scenes=12, seed=3)
    counts = [s.particles.shape[0] for s in specs]
    assert all(2_000 <= c < 200_000 for c in counts)
    for s in specs:
        assert s.method == 0 and tuple(s.res) in ((64, 64, 64), (128, 128, 128))
        _mode(s)
    # the full batch's first scenes are these (same seed)
    first = pkg.scenes.c3_batched(n_scenes=3, seed=3)
    assert [f.particles.shape[0] for f in first] == counts[:3]
