"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle (liboracle.so,
built from mpm_oracle.c / bvh_oracle.c / mlp_oracle.c / splat_oracle.c /
scatter_oracle.c by oracle/Makefile).

The oracle restates the reference MPM step (WGSL under src/lib/gpu/mpm/ and
src/lib/gpu/shaderPrelude/, scheduled by GpuMpmPipelineManager.ts:327-521).
Parity status: UNPINNED -- the reference ships no golden vectors and its
WGSL cannot run here.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
UNIFORMS_BYTES = 37376


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("mpm_oracle.c", "mpm_oracle.h", "bvh_oracle.c", "mlp_oracle.c", "splat_oracle.c",
                                             "scatter_oracle.c", "raymarch_oracle.c", "mc_oracle.c", "Makefile")]
    srcs.append(os.path.join(HERE, "..", "webgpu-mpm-based-snow-simulation_b200", "csrc", "mpm_mc_table.h"))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB


class OrExt(C.Structure):
    _fields_ = [
        ("gravity", C.c_float * 3), ("youngs_modulus", C.c_float), ("poissons_ratio", C.c_float),
        ("hardening_explicit", C.c_float), ("hardening_pbmpm", C.c_float), ("theta_c", C.c_float),
        ("theta_s", C.c_float), ("density", C.c_float), ("n_iter", C.c_uint32), ("force_divisor", C.c_float),
        ("boundary_mode", C.c_uint32), ("restitution", C.c_float), ("bc_cells", C.c_uint32),
        ("ground_axis", C.c_uint32), ("collider_margin", C.c_float), ("collider_surface_margin", C.c_float),
        ("collider_threshold", C.c_float), ("collider_friction", C.c_float), ("collider_vel_scale", C.c_float),
        ("pbmpm_blend", C.c_float), ("pbmpm_volume_exponent", C.c_float), ("return_map", C.c_uint32),
    ]


class OrCollider(C.Structure):
    _fields_ = [("data", C.c_void_p), ("data_words", C.c_uint32), ("nodes", C.c_void_p), ("n_nodes", C.c_uint32)]


D_DTYPE = np.dtype([("pos", "<3f8"), ("vel", "<3f8"), ("mass", "<f8"), ("Fe", "<9f8"), ("Fp", "<9f8"),
                    ("dxp", "<3f8"), ("D", "<9f8")])

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        V, U32, I32 = C.c_void_p, C.c_uint32, C.c_int
        sig = {
            "or_default_ext": (None, [V]),
            "orf_create": (V, [U32, U32, U32]), "orf_destroy": (None, [V]), "orf_status": (U32, [V]),
            "orf_set_threads": (None, [I32]),
            "orf_step": (I32, [V, V, V, V, U32, V, I32, I32]), "orf_dense_grid": (I32, [V, V, V]),
            "orf_n_blocks": (U32, [V]),
            "ord_create": (V, [U32, U32, U32]), "ord_destroy": (None, [V]), "ord_status": (U32, [V]),
            "ord_step": (I32, [V, V, V, V, U32, V, I32, I32]), "ord_dense_grid": (I32, [V, V, V]),
            "or_hash3": (U32, [U32, U32, U32]), "or_expf": (C.c_float, [C.c_float]),
            "or_powf": (C.c_float, [C.c_float, C.c_float]), "or_f2i": (C.c_int32, [C.c_float]),
            "orf_inverse": (None, [V, V]), "orf_polar": (None, [V, V]), "orf_det": (C.c_float, [V]),
            "orf_plasticity": (None, [V, V, V]),
            "orf_plasticity_n": (None, [V, V, V, U32]), "ord_plasticity_n": (None, [V, V, V, U32]),
            "or_bvh_build": (U32, [V, U32, V, U32, V, V]),
            "or_mlp_forward": (None, [V, V, U32, I32, V]),
            "or_mlp_gradient": (C.c_double, [V, V, V, U32, C.c_float, I32, V]),
            "or_mlp_features": (I32, [V, V, C.c_float, C.c_float, V]),
            "or_mlp_targets": (None, [V, V, V, V, V]),
            "or_cert_elastic": (I32, [C.c_float, C.c_float, V]),
            "or_grid_mass": (None, [V, U32, V, V, V, C.c_float, V]),
            "or_mc_density": (None, [V, U32, V, V, V, C.c_float, V]),
            "or_scatter": (None, [V, U32, V, V, U32, V]),
            "or_raymarch": (None, [V, V, V, V, C.c_float, V, U32, U32, U32, V, V, V]),
            "or_marching_cubes": (None, [V, V, V, V, V, C.c_float, V, V, V, V, U32, V]),
            "or_mc_tables": (None, [V, V, V]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
    return _lib


def make_ext(params: dict) -> OrExt:
    e = OrExt()
    lib().or_default_ext(C.byref(e))
    for k, v in params.items():
        if k == "gravity":
            e.gravity[:] = [float(x) for x in v]
        else:
            setattr(e, k, v)
    return e


def bvh_build(vertices, indices):
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    nt = i.size // 3
    nodes = np.zeros((2 * nt + 1, 8), np.uint32)
    order = np.zeros(max(nt, 1), np.uint32)
    n = lib().or_bvh_build(v.ctypes.data, v.size // 3, i.ctypes.data, i.size, nodes.ctypes.data, order.ctypes.data)
    return nodes[:n].copy(), order[:nt].copy()


def collider_buffers(vertices, indices):
    """Packed [indices in BVH order | vertices] and nodes, built by the oracle."""
    nodes, order = bvh_build(vertices, indices)
    tri = np.asarray(indices, np.uint32).reshape(-1, 3)
    data = np.concatenate([tri[order].reshape(-1), np.asarray(vertices, np.float32).reshape(-1).view(np.uint32)])
    return np.ascontiguousarray(data, np.uint32), nodes


class Oracle:
    """One oracle context (f32 with fixed-point grid, or f64)."""

    def __init__(self, n_particles: int, max_blocks: int = 200000, hash_size: int = 2000003, fp64: bool = False,
                 threads: int = 0):
        self.fp64 = fp64
        L = lib()
        if threads:
            L.orf_set_threads(threads)
        self.ctx = (L.ord_create if fp64 else L.orf_create)(hash_size, max_blocks, max(n_particles, 1))
        if not self.ctx:
            raise MemoryError("oracle context allocation failed")
        self._col = None

    def close(self):
        if self.ctx:
            (lib().ord_destroy if self.fp64 else lib().orf_destroy)(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_collider(self, vertices, indices):
        if vertices is None:
            self._col = None
            return
        data, nodes = collider_buffers(vertices, indices)
        self._col_keep = (data, nodes)
        self._col = OrCollider(data.ctypes.data, data.size, nodes.ctypes.data, nodes.shape[0])

    def step(self, uniforms: bytes, params: dict, particles: np.ndarray, method: int, stop_after: int = 0) -> None:
        """Advances `particles` in place (f32 records, or D_DTYPE for fp64)."""
        ub = np.frombuffer(bytes(uniforms).ljust(UNIFORMS_BYTES, b"\0"), np.uint8)
        ext = make_ext(params)
        assert particles.flags["C_CONTIGUOUS"]
        fn = lib().ord_step if self.fp64 else lib().orf_step
        col = C.byref(self._col) if self._col is not None else None
        rc = fn(self.ctx, ub.ctypes.data, C.byref(ext), particles.ctypes.data, particles.shape[0], col, method,
                stop_after)
        if rc != 0:
            raise RuntimeError(f"oracle step failed: {rc}")

    def status(self) -> int:
        return (lib().ord_status if self.fp64 else lib().orf_status)(self.ctx)

    def dense_grid(self, uniforms: bytes) -> np.ndarray:
        ub = np.frombuffer(bytes(uniforms).ljust(UNIFORMS_BYTES, b"\0"), np.uint8)
        res = np.frombuffer(ub[208:220].tobytes(), "<u4")
        out = np.zeros((res[2], res[1], res[0], 4), np.float64 if self.fp64 else np.int32)
        (lib().ord_dense_grid if self.fp64 else lib().orf_dense_grid)(self.ctx, ub.ctypes.data, out.ctypes.data)
        return out


def to_fp64(records: np.ndarray) -> np.ndarray:
    d = np.zeros(records.shape[0], D_DTYPE)
    d["pos"] = records["pos"]
    d["vel"] = records["vel"]
    d["mass"] = records["mass"]
    d["Fe"] = records["Fe"][:, :, :3].reshape(-1, 9)
    d["Fp"] = records["Fp"][:, :, :3].reshape(-1, 9)
    d["dxp"] = records["dxp"]
    d["D"] = records["D"][:, :, :3].reshape(-1, 9)
    return d


def aggregates(pos, vel, mass, Fp9):
    """Centre of mass, total momentum and mean J_p = det(F_p) (f64)."""
    m = np.asarray(mass, np.float64)
    pos = np.asarray(pos, np.float64)
    vel = np.asarray(vel, np.float64)
    F = np.asarray(Fp9, np.float64).reshape(-1, 3, 3)
    com = (pos * m[:, None]).sum(0) / m.sum()
    mom = (vel * m[:, None]).sum(0)
    jp = np.linalg.det(F).mean()
    return com, mom, jp


# ---- learned-plasticity network reference (mlp_oracle.c) --------------
MLP_PARAMS = 9867


def mlp_forward(params, x, bf16=True):
    """Network outputs [n, 11] (f64) of inputs x [n, 12]."""
    p = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    y = np.zeros((xx.shape[0], 11), np.float64)
    lib().or_mlp_forward(p.ctypes.data, xx.ctypes.data, xx.shape[0], 1 if bf16 else 0, y.ctypes.data)
    return y


def mlp_gradient(params, x, t, unc_weight=0.1, bf16=True):
    """(loss, gradient [MLP_PARAMS] f64) of the batch loss."""
    p = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    tt = np.ascontiguousarray(t, np.float32)
    g = np.zeros(MLP_PARAMS, np.float64)
    loss = lib().or_mlp_gradient(p.ctypes.data, xx.ctypes.data, tt.ctypes.data, xx.shape[0], unc_weight,
                                 1 if bf16 else 0, g.ctypes.data)
    return loss, g


def mlp_pair(Fe, Fp, dt, theta_c, theta_s, return_map=0):
    """(in_domain, x[12], t[10], Fe', Fp') of one trial state through the exact
    map (return_map 0: applyPlasticity; 1: the SVD clamp)."""
    fe = np.ascontiguousarray(Fe, np.float32).reshape(9)
    fp = np.ascontiguousarray(Fp, np.float32).reshape(9)
    x = np.zeros(12, np.float32)
    ok = lib().or_mlp_features(fe.ctypes.data, fp.ctypes.data, dt, theta_c, x.ctypes.data)
    e = make_ext({"theta_c": theta_c, "theta_s": theta_s, "return_map": return_map})
    fe2, fp2 = fe.copy(), fp.copy()
    lib().orf_plasticity(C.byref(e), fe2.ctypes.data, fp2.ctypes.data)
    t = np.zeros(10, np.float32)
    lib().or_mlp_targets(fe.ctypes.data, fp.ctypes.data, fe2.ctypes.data, fp2.ctypes.data, t.ctypes.data)
    return bool(ok), x, t, fe2, fp2


def return_map(Fe, Fp, params: dict, fp64: bool = False):
    """The selected return map (params["return_map"]: 0 applyPlasticity, 1 the
    SVD clamp) on states Fe, Fp [n, 3, 3] stored as 9 column-major entries:
    (Fe', Fp')."""
    dt = np.float64 if fp64 else np.float32
    fe = np.ascontiguousarray(np.asarray(Fe, dt).reshape(-1, 9)).copy()
    fp = np.ascontiguousarray(np.asarray(Fp, dt).reshape(-1, 9)).copy()
    e = make_ext(params)
    (lib().ord_plasticity_n if fp64 else lib().orf_plasticity_n)(C.byref(e), fe.ctypes.data, fp.ctypes.data,
                                                                fe.shape[0])
    return fe, fp


def cert_elastic(Fe, theta_c, theta_s):
    fe = np.ascontiguousarray(Fe, np.float32).reshape(9)
    smin, smax = np.float32(1.0 - float(np.float32(theta_c))), np.float32(1.0 + float(np.float32(theta_s)))
    return bool(lib().or_cert_elastic(float(smin), float(smax), fe.ctypes.data))


# ---- renderer splats (splat_oracle.c) ---------------------------------
def splat(kind, records, grid_min, grid_max, res, scale):
    """calculateGridMass (kind 'mass') or calculateDensity (kind 'density'):
    u32 grid [res_z][res_y][res_x]."""
    rec = np.ascontiguousarray(records)
    gmin = np.ascontiguousarray(grid_min, np.float32)
    gmax = np.ascontiguousarray(grid_max, np.float32)
    r = np.ascontiguousarray(res, np.uint32)
    out = np.zeros((int(r[2]), int(r[1]), int(r[0])), np.uint32)
    f = lib().or_grid_mass if kind == "mass" else lib().or_mc_density
    f(rec.ctypes.data, rec.shape[0], gmin.ctypes.data, gmax.ctypes.data, r.ctypes.data, float(np.float32(scale)),
      out.ctypes.data)
    return out


# ---- particle scatter (scatter_oracle.c) --------------------------------
def scatter(vertices4, mesh_min, mesh_max, n):
    """scatterParticles: n 192-byte records (as raw bytes reshaped [n, 192])."""
    v = np.ascontiguousarray(vertices4, np.float32)
    mn = np.ascontiguousarray(mesh_min, np.float32)
    mx = np.ascontiguousarray(mesh_max, np.float32)
    out = np.zeros((n, 192), np.uint8)
    lib().or_scatter(v.ctypes.data, v.shape[0] // 3, mn.ctypes.data, mx.ctypes.data, n, out.ctypes.data)
    return out


# ---- volumetric ray march (raymarch_oracle.c) ---------------------------
def raymarch(mass_grid, grid_min, grid_max, scale, inv_view_proj, time, width, height, depth_init=None):
    """doVolumetricRaymarch over a width x height image: (rgba [h][w][4] u8,
    depth [h][w] f32, color [h][w][4] f32).  mass_grid is the u32
    calculateGridMass grid [res_z][res_y][res_x]; inv_view_proj the 16
    column-major floats of viewProjInvMat."""
    m = np.ascontiguousarray(mass_grid, np.uint32)
    res = np.array([m.shape[2], m.shape[1], m.shape[0]], np.uint32)
    gmin = np.ascontiguousarray(grid_min, np.float32)
    gmax = np.ascontiguousarray(grid_max, np.float32)
    M = np.ascontiguousarray(np.asarray(inv_view_proj, np.float32).reshape(16))
    rgba = np.zeros((height, width, 4), np.uint8)
    depth = (np.full((height, width), np.float32(-1.0), np.float32) if depth_init is None
             else np.ascontiguousarray(depth_init, np.float32).copy())
    color = np.zeros((height, width, 4), np.float32)
    lib().or_raymarch(m.ctypes.data, res.ctypes.data, gmin.ctypes.data, gmax.ctypes.data, float(np.float32(scale)),
                      M.ctypes.data, int(time), int(width), int(height), rgba.ctypes.data, depth.ctypes.data,
                      color.ctypes.data)
    return rgba, depth, color


# ---- marching cubes (mc_oracle.c) and its triangulation table -----------
def mc_tables():
    """The reference's marching-cubes case table (marchingCubes/triTable.wgsl,
    prelude.wgsl MC_TRI_COUNTS) and edge endpoints (prelude.wgsl:45-46), from
    mc_oracle.c.  Returns (tri int8 [256, 16] padded with -1, counts uint8
    [256], edge endpoints uint8 [12, 2])."""
    tri = np.zeros((256, 16), np.int8)
    cnt = np.zeros(256, np.uint8)
    ev = np.zeros((12, 2), np.uint8)
    lib().or_mc_tables(tri.ctypes.data, cnt.ctypes.data, ev.ctypes.data)
    return tri, cnt, ev


def marching_cubes(density, grid_min, grid_max, scale, mc_res, tables=None, max_vertices=None):
    """Mesh of a u32 density grid [dz][dy][dx]: vertices [n, 6] f32 (position,
    normal) in block, cell, table order."""
    tri, cnt, ev = mc_tables() if tables is None else tables
    d = np.ascontiguousarray(density, np.uint32)
    dres = np.array([d.shape[2], d.shape[1], d.shape[0]], np.uint32)
    mres = np.ascontiguousarray(mc_res, np.uint32)
    gmin = np.ascontiguousarray(grid_min, np.float32)
    gmax = np.ascontiguousarray(grid_max, np.float32)
    tri = np.ascontiguousarray(tri, np.int8)
    cnt = np.ascontiguousarray(cnt, np.uint8)
    ev = np.ascontiguousarray(ev, np.uint8)
    n = C.c_uint32(0)
    lib().or_marching_cubes(d.ctypes.data, dres.ctypes.data, mres.ctypes.data, gmin.ctypes.data, gmax.ctypes.data,
                            float(np.float32(scale)), tri.ctypes.data, cnt.ctypes.data, ev.ctypes.data, None, 0,
                            C.byref(n))
    cap = n.value if max_vertices is None else int(max_vertices)
    out = np.zeros((max(cap, 1), 6), np.float32)
    lib().or_marching_cubes(d.ctypes.data, dres.ctypes.data, mres.ctypes.data, gmin.ctypes.data, gmax.ctypes.data,
                            float(np.float32(scale)), tri.ctypes.data, cnt.ctypes.data, ev.ctypes.data,
                            out.ctypes.data, cap, C.byref(n))
    return out[: min(cap, n.value)], n.value
