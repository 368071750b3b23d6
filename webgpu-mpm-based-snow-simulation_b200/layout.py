"""Byte layouts shared with the reference: the 192-byte particle record and the
37,376-byte uniform block, plus a mirror of the reference's uniform writer.

References:
  ParticleData          src/lib/gpu/shaderPrelude/mpmOps.wgsl:1-12
  particle buffer size  src/lib/gpu/mpm/GpuMpmBufferManager.ts:22-26 (N x 192 B)
  Uniforms struct       src/lib/gpu/shaderPrelude/uniforms.wgsl:1-56
  uniform writers       src/lib/gpu/uniforms/GpuUniformsBufferManager.ts:54-182
"""
from __future__ import annotations

import numpy as np

UNIFORMS_BYTES = 37376
PARTICLE_BYTES = 192
BVH_NODE_BYTES = 32
MAX_COLLIDER_OBJECTS = 1024

# mat3x3f in a storage buffer: 3 columns of vec3f, each padded to 16 bytes
PARTICLE_DTYPE = np.dtype(
    {
        "names": ["pos", "hom", "vel", "mass", "Fe", "Fp", "dxp", "pad", "D"],
        "formats": ["<3f4", "<f4", "<3f4", "<f4", ("<f4", (3, 4)), ("<f4", (3, 4)), "<3f4", "<f4", ("<f4", (3, 4))],
        "offsets": [0, 12, 16, 28, 32, 80, 128, 140, 144],
        "itemsize": PARTICLE_BYTES,
    }
)

# The fields the step computes; padding words are not part of the state.
STATE_FIELDS = ("pos", "vel", "mass", "Fe", "Fp", "dxp", "D")


def mat_cols(rec_field: np.ndarray) -> np.ndarray:
    """(n, 3, 4) padded column storage -> (n, 3, 3) with m[:, c, r]."""
    return np.ascontiguousarray(rec_field[..., :3])


def new_particles(n: int) -> np.ndarray:
    """Zeroed records with F_e = F_p = I and _hom = 1, as the scatter kernel
    initialises them (particleInitialize/particleScatter.cs.wgsl:73-83)."""
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    eye = np.zeros((3, 4), np.float32)
    eye[0, 0] = eye[1, 1] = eye[2, 2] = 1.0
    p["Fe"] = eye
    p["Fp"] = eye
    p["hom"] = 1.0
    return p


class GpuUniformsBufferManager:
    """Host-side mirror of the reference uniform writer: every write_* puts the
    value at the byte offset the reference uses
    (GpuUniformsBufferManager.ts:54-182).  `buffer` is the raw block handed to
    mpm_set_uniforms."""

    def __init__(self) -> None:
        self.buffer = bytearray(UNIFORMS_BYTES)

    def _f32(self, off: int, vals) -> None:
        a = np.asarray(vals, dtype="<f4").ravel()
        self.buffer[off : off + 4 * a.size] = a.tobytes()

    def _u32(self, off: int, vals) -> None:
        a = np.asarray(vals, dtype="<u4").ravel()
        self.buffer[off : off + 4 * a.size] = a.tobytes()

    def write_simulation_timestep_s(self, t: float) -> None:
        self._f32(0, [t])

    def write_fixed_point_scale(self, s: float) -> None:
        self._f32(4, [s])

    def write_use_pbmpm(self, use: bool) -> None:
        self._u32(8, [1 if use else 0])

    def write_time(self, t: int) -> None:
        self._u32(12, [t & 0xFFFFFFFF])

    def write_grid_min_coords(self, v) -> None:
        self._f32(16, v)

    def write_grid_max_coords(self, v) -> None:
        self._f32(32, v)

    def write_view_proj_mat(self, m) -> None:
        self._f32(48, np.asarray(m, np.float32).reshape(16))

    def write_view_proj_inv_mat(self, m) -> None:
        self._f32(112, np.asarray(m, np.float32).reshape(16))

    def write_mesh_min_coords(self, v) -> None:
        self._f32(176, v)

    def write_mesh_max_coords(self, v) -> None:
        self._f32(192, v)

    def write_grid_resolution(self, r) -> None:
        self._u32(208, r)

    def write_collider_min_coords(self, v) -> None:
        self._f32(224, v)

    def write_collider_max_coords(self, v) -> None:
        self._f32(240, v)

    def write_collider_transform_mat(self, m) -> None:
        """m: 16 floats, column-major (wgpu-matrix Mat4 layout)."""
        self._f32(256, np.asarray(m, np.float32).reshape(16))

    def write_collider_vel(self, v) -> None:
        self._f32(320, v)

    def write_camera_pos(self, v) -> None:
        self._f32(336, v)

    def write_grid_cell_dims(self, v) -> None:
        self._f32(352, v)

    def write_collider_num_indices(self, n: int) -> None:
        self._u32(348, [n])

    def write_collider_num_objects(self, n: int) -> None:
        self._u32(364, [n])

    def write_light_view_proj_mat(self, m) -> None:
        self._f32(368, np.asarray(m, np.float32).reshape(16))

    def write_collider_transform_inv(self, m) -> None:
        self._f32(432, np.asarray(m, np.float32).reshape(16))

    def write_interaction_pos(self, v) -> None:
        self._f32(496, v)

    def write_interaction_strength(self, s: float) -> None:
        self._f32(508, [s])

    def write_interaction_radius(self, r: float) -> None:
        self._f32(512, [r])

    def write_is_interacting(self, b: bool) -> None:
        self._u32(516, [1 if b else 0])

    def write_interaction_mode(self, m: int) -> None:
        self._u32(520, [m])

    def write_interaction_dir(self, v) -> None:
        self._f32(528, v)

    def write_collider_objects(self, objects) -> None:
        """objects: iterable of dicts with min, max, startIndex, countIndices
        (GpuUniformsBufferManager.ts:162-182)."""
        objs = list(objects)[:MAX_COLLIDER_OBJECTS]
        raw = np.zeros((len(objs), 8), dtype="<u4")
        f = raw.view("<f4")
        for i, o in enumerate(objs):
            f[i, 0:3] = o["min"]
            raw[i, 3] = o["startIndex"]
            f[i, 4:7] = o["max"]
            raw[i, 7] = o["countIndices"]
        self.buffer[544 : 544 + raw.nbytes] = raw.tobytes()

    def bytes(self) -> bytes:
        return bytes(self.buffer)


def identity_mat4() -> np.ndarray:
    return np.eye(4, dtype=np.float32).reshape(16)
