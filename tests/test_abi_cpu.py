"""The C ABI library loads on a machine without a GPU and exports every symbol
include/mpm.h declares; the host-side layouts match the reference's."""
import os
import re

import numpy as np

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), f"libmpm.so lacks {n}"
    from importlib import import_module
    sigs = import_module(pkg.__name__ + "._lib").SIGNATURES
    assert set(names) == set(sigs), set(names) ^ set(sigs)


def test_default_params_are_reference_constants(pkg):
    p = pkg.default_params()
    assert list(p.gravity) == [0.0, 0.0, np.float32(-9.81)]
    assert p.youngs_modulus == np.float32(1.4e5) and p.poissons_ratio == np.float32(0.2)
    assert p.hardening_explicit == 5.0 and p.hardening_pbmpm == 20.0
    assert p.n_iter == 3 and p.force_divisor == 3.0
    assert p.collider_margin == np.float32(0.05) and p.collider_friction == np.float32(0.1)
    assert p.pbmpm_volume_exponent == np.float32(-0.3333333)


def test_particle_layout_is_192_bytes(pkg):
    dt = pkg.PARTICLE_DTYPE
    assert dt.itemsize == 192
    offs = {k: dt.fields[k][1] for k in dt.names}
    # shaderPrelude/mpmOps.wgsl:1-12 with std430 mat3x3f columns of 16 bytes
    assert offs == {"pos": 0, "hom": 12, "vel": 16, "mass": 28, "Fe": 32, "Fp": 80, "dxp": 128, "pad": 140, "D": 144}


def test_uniform_writer_offsets(pkg):
    u = pkg.GpuUniformsBufferManager()
    u.write_simulation_timestep_s(0.5)
    u.write_fixed_point_scale(65536.0)
    u.write_grid_min_coords([-5, -5, -5])
    u.write_grid_resolution([256, 128, 64])
    u.write_collider_num_indices(36)
    u.write_grid_cell_dims([0.25, 0.5, 1.0])
    u.write_interaction_strength(1000.0)
    b = u.bytes()
    assert len(b) == 37376
    f = np.frombuffer(b, "<f4")
    i = np.frombuffer(b, "<u4")
    assert f[0] == 0.5 and f[1] == 65536.0
    assert list(f[4:7]) == [-5, -5, -5]
    assert list(i[52:55]) == [256, 128, 64]   # offset 208
    assert i[87] == 36                          # offset 348
    assert list(f[88:91]) == [0.25, 0.5, 1.0]   # offset 352
    assert f[127] == 1000.0                     # offset 508


def test_create_fails_cleanly_without_gpu_or_bad_args(pkg):
    """Bad arguments are rejected with an error, never a crash."""
    import ctypes as C
    lib = pkg.load()
    cfg = pkg.MpmConfig(max_particles=0, max_scenes=1, tile_edge=16)
    h = C.c_void_p()
    rc = lib.mpm_create(C.byref(cfg), C.byref(h))
    assert rc != 0
    assert b"max_particles" in lib.mpm_last_error(h)
    lib.mpm_destroy(h)
    cfg = pkg.MpmConfig(max_particles=10, max_scenes=1, tile_edge=13)
    rc = lib.mpm_create(C.byref(cfg), C.byref(h))
    assert rc != 0
    assert b"tile_edge" in lib.mpm_last_error(h)
    lib.mpm_destroy(h)


def test_kernel_names(pkg):
    names = pkg.kernel_names()
    assert "p2g_explicit" in names and "pbmpm_iter" in names and "g2p_pbmpm_integrate" in names
