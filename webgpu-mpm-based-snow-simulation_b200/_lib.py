"""ctypes binding of libmpm.so (include/mpm.h).

The library is the only compute path: if it is missing or fails to load,
every call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB_PATH

MPM_OK = 0
MPM_ERR_DEVICE_STATUS = -5
METHOD_EXPLICIT = 0
METHOD_PBMPM = 1

STATUS_BITS = {
    0x1: "tile hash table full",
    0x2: "tile capacity overflow",
    0x4: "BVH stack overflow",
    0x8: "particle outside every scene range",
    0x10: "learned plasticity fallback",
    0x20: "learned plasticity tensor-core wait ran out",
    0x40: "halo bulk-copy wait ran out",
}

PLASTICITY_INLINE = 0
PLASTICITY_EXACT = 1
PLASTICITY_COLLECT = 2
PLASTICITY_LEARNED = 3
MLP_INPUTS = 12
MLP_OUTPUTS = 11
MLP_TARGETS = 10
MLP_PARAMS = 9867


class MpmConfig(C.Structure):
    _fields_ = [
        ("max_particles", C.c_uint32),
        ("max_scenes", C.c_uint32),
        ("max_tiles", C.c_uint32),
        ("hash_capacity", C.c_uint32),
        ("tile_edge", C.c_uint32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
    ]


class MpmParams(C.Structure):
    _fields_ = [
        ("gravity", C.c_float * 3),
        ("youngs_modulus", C.c_float),
        ("poissons_ratio", C.c_float),
        ("hardening_explicit", C.c_float),
        ("hardening_pbmpm", C.c_float),
        ("theta_c", C.c_float),
        ("theta_s", C.c_float),
        ("density", C.c_float),
        ("n_iter", C.c_uint32),
        ("force_divisor", C.c_float),
        ("boundary_mode", C.c_uint32),
        ("restitution", C.c_float),
        ("bc_cells", C.c_uint32),
        ("ground_axis", C.c_uint32),
        ("collider_margin", C.c_float),
        ("collider_surface_margin", C.c_float),
        ("collider_threshold", C.c_float),
        ("collider_friction", C.c_float),
        ("collider_vel_scale", C.c_float),
        ("pbmpm_blend", C.c_float),
        ("pbmpm_volume_exponent", C.c_float),
        ("return_map", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name == "gravity" else v
        return d


class MpmMlpTrainConfig(C.Structure):
    _fields_ = [("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float), ("lr_final", C.c_float),
                ("unc_weight", C.c_float), ("seed", C.c_uint32)]


class MpmPlasticityStats(C.Structure):
    _fields_ = [("candidates", C.c_uint64), ("learned", C.c_uint64), ("fallback_domain", C.c_uint64),
                ("fallback_uncertain", C.c_uint64), ("fallback_det", C.c_uint64), ("audited", C.c_uint64),
                ("audit_max_err", C.c_float), ("audit_mean_err", C.c_float), ("pairs_collected", C.c_uint32),
                ("pad", C.c_uint32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


# exported symbols and their signatures: (restype, argtypes)
_H = C.c_void_p
SIGNATURES = {
    "mpm_default_params": (C.c_int, [C.POINTER(MpmParams)]),
    "mpm_create": (C.c_int, [C.POINTER(MpmConfig), C.POINTER(C.c_void_p)]),
    "mpm_destroy": (C.c_int, [_H]),
    "mpm_last_error": (C.c_char_p, [_H]),
    "mpm_set_uniforms": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_size_t]),
    "mpm_set_params": (C.c_int, [_H, C.c_uint32, C.POINTER(MpmParams)]),
    "mpm_set_scene_range": (C.c_int, [_H, C.c_uint32, C.c_uint32, C.c_uint32]),
    "mpm_set_scene_count": (C.c_int, [_H, C.c_uint32]),
    "mpm_set_particles": (C.c_int, [_H, C.c_void_p, C.c_uint32, C.c_int]),
    "mpm_get_particles": (C.c_int, [_H, C.c_void_p, C.c_uint32, C.c_int]),
    "mpm_bind_particles_device": (C.c_int, [_H, C.c_void_p, C.c_uint32]),
    "mpm_particles_device_ptr": (C.c_void_p, [_H]),
    "mpm_set_collider": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_size_t, C.c_uint32, C.c_void_p, C.c_uint32]),
    "mpm_build_bvh": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_uint32)]),
    "mpm_step": (C.c_int, [_H, C.c_int, C.c_uint32]),
    "mpm_add_explicit_mpm_dispatches": (C.c_int, [_H, C.c_uint32]),
    "mpm_add_pbmpm_dispatches": (C.c_int, [_H, C.c_uint32]),
    "mpm_sync": (C.c_int, [_H, C.POINTER(C.c_uint32)]),
    "mpm_clear_status": (C.c_int, [_H]),
    "mpm_step_p2g_only": (C.c_int, [_H, C.c_int]),
    "mpm_get_grid_dense": (C.c_int, [_H, C.c_uint32, C.c_int, C.c_void_p, C.c_size_t]),
    "mpm_get_counts": (C.c_int, [_H, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "mpm_get_tile_edge": (C.c_int, [_H, C.POINTER(C.c_uint32)]),
    "mpm_enable_kernel_timing": (C.c_int, [_H, C.c_int]),
    "mpm_set_schedule": (C.c_int, [_H, C.c_uint32, C.c_uint32]),
    "mpm_kernel_times": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_uint32]),
    "mpm_kernel_name": (C.c_char_p, [C.c_uint32]),
    "mpm_kernel_count": (C.c_uint32, []),
    "mpm_use_graphs": (C.c_int, [_H, C.c_int]),
    "mpm_selftest": (C.c_int, [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                               C.POINTER(C.c_uint64)]),
    "mpm_scatter_particles": (C.c_int, [_H, C.c_void_p, C.c_uint32, C.c_uint32]),
    "mpm_grid_mass": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_int]),
    "mpm_mc_density": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int]),
    "mpm_marching_cubes": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                     C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "mpm_mc_tables": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mpm_bvh_node_count": (C.c_uint32, [C.c_uint32]),
    "mpm_build_bvh_device": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_uint32), C.c_void_p]),
    "mpm_set_collider_mesh_device": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "mpm_volumetric_raymarch": (C.c_int, [_H, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    "mpm_mlp_init_params": (C.c_int, [C.c_uint32, C.c_void_p]),
    "mpm_mlp_create": (C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_void_p)]),
    "mpm_mlp_destroy": (C.c_int, [C.c_void_p]),
    "mpm_mlp_last_error": (C.c_char_p, [C.c_void_p]),
    "mpm_mlp_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mpm_mlp_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mpm_mlp_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mpm_mlp_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "mpm_mlp_gradient": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p,
                                   C.c_void_p]),
    "mpm_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(MpmMlpTrainConfig),
                                C.c_void_p]),
    "mpm_set_plasticity": (C.c_int, [_H, C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_float]),
    "mpm_set_pair_buffer": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_uint32]),
    "mpm_get_plasticity_stats": (C.c_int, [_H, C.POINTER(MpmPlasticityStats), C.c_int]),
    "mpm_step_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_size_t,
                                   C.POINTER(MpmParams), C.c_void_p, C.c_size_t, C.c_uint32, C.c_void_p, C.c_uint32,
                                   C.POINTER(C.c_uint32), C.c_char_p, C.c_size_t]),
}

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load libmpm.so (built in-tree by build.py) and declare its signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libmpm.so not found at {p}; run the build (python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


class MpmError(RuntimeError):
    def __init__(self, code: int, msg: str, status: int = 0):
        super().__init__(f"libmpm error {code}: {msg}")
        self.code = code
        self.status = status


def check(code: int, handle=None, status: int = 0) -> None:
    if code != MPM_OK:
        lib = load()
        msg = lib.mpm_last_error(handle).decode() if handle else "error"
        raise MpmError(code, msg, status)


def default_params() -> MpmParams:
    p = MpmParams()
    check(load().mpm_default_params(C.byref(p)))
    return p
