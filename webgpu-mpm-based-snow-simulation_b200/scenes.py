"""Seeded synthetic scenes: the benchmark configurations and the parity cases.

No public dataset is involved: the reference's own scenes are glTF meshes
(one of them missing from the mirror), so every workload here is procedural
geometry with the sizes, spacings and time steps of the configurations it
stands for.  All generators are deterministic given their seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .layout import GpuUniformsBufferManager, identity_mat4, new_particles


# ----------------------------------------------------------------------
# geometry
# ----------------------------------------------------------------------
def jittered_lattice(lo, counts, spacing, rng, jitter=0.5):
    """Lattice points lo + (ijk + 0.5 + U(-jitter, jitter)) * spacing, x fastest."""
    nx, ny, nz = counts
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ijk = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    u = rng.uniform(-jitter, jitter, size=ijk.shape)
    return (np.asarray(lo, np.float64) + (ijk + 0.5 + u) * spacing).astype(np.float32)


def sphere_lattice(center, radius, n, spacing, rng):
    """First n points of a jittered lattice that fall inside the sphere."""
    m = int(np.ceil(2 * radius / spacing)) + 2
    lo = np.asarray(center) - m * spacing / 2
    pts = jittered_lattice(lo, (m, m, m), spacing, rng)
    inside = np.sum((pts.astype(np.float64) - np.asarray(center)) ** 2, axis=1) <= radius * radius
    pts = pts[inside]
    if pts.shape[0] < n:
        raise ValueError(f"sphere lattice too sparse: {pts.shape[0]} < {n}")
    return pts[:n]


def box_mesh(lo, hi):
    """12-triangle axis-aligned box, outward winding."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    f = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [3, 6, 2], [3, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.uint32)
    return v, f.reshape(-1)


def icosphere(subdivisions, radius, center):
    """Icosahedron subdivided `subdivisions` times (20 * 4^s triangles)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    v = (np.array(verts) * radius + np.asarray(center)).astype(np.float32)
    return v, np.array(faces, np.uint32).reshape(-1)


def _value_noise_2d(x, z, seed):
    """Seeded value noise on the integer lattice, smoothstep interpolation."""
    def h(ix, iz):
        u = (ix.astype(np.uint64) * np.uint64(73856093)) ^ (iz.astype(np.uint64) * np.uint64(19349663)) ^ np.uint64(seed * 83492791 + 1)
        u = (u ^ (u >> np.uint64(13))) * np.uint64(0x5bd1e995)
        u = u ^ (u >> np.uint64(15))
        return (u & np.uint64(0xFFFFFF)).astype(np.float64) / float(0xFFFFFF)

    x0, z0 = np.floor(x), np.floor(z)
    fx, fz = x - x0, z - z0
    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
    ix, iz = x0.astype(np.int64), z0.astype(np.int64)
    a, b = h(ix, iz), h(ix + 1, iz)
    c, d = h(ix, iz + 1), h(ix + 1, iz + 1)
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def fbm_terrain(n=256, amplitude=0.1, seed=2, base=0.25, octaves=4, freq=4.0, axis_up=1):
    """n x n vertex heightfield over [0,1]^2, 2*(n-1)^2 triangles; height
    base + amplitude * (fbm - 0.5) along axis_up."""
    g = np.linspace(0.0, 1.0, n)
    X, Z = np.meshgrid(g, g, indexing="xy")
    hgt = np.zeros_like(X)
    amp, f = 0.5, freq
    for o in range(octaves):
        hgt += amp * _value_noise_2d(X * f, Z * f, seed + 101 * o)
        amp *= 0.5
        f *= 2.0
    hgt = base + amplitude * (hgt / (1.0 - 0.5 ** octaves) - 0.5)
    if axis_up == 1:
        v = np.stack([X.ravel(), hgt.ravel(), Z.ravel()], axis=1)
    else:
        v = np.stack([X.ravel(), Z.ravel(), hgt.ravel()], axis=1)
    i = np.arange(n - 1)
    I, J = np.meshgrid(i, i, indexing="xy")
    a = (J * n + I).ravel()
    b, c, d = a + 1, a + n, a + n + 1
    tris = np.stack([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], 1).reshape(-1, 3)
    return v.astype(np.float32), tris.astype(np.uint32).reshape(-1)


def merge_meshes(*meshes):
    vs, fs, off = [], [], 0
    for v, f in meshes:
        vs.append(v)
        fs.append(f + off)
        off += v.shape[0]
    return np.concatenate(vs).astype(np.float32), np.concatenate(fs).astype(np.uint32)


# ----------------------------------------------------------------------
# scenes
# ----------------------------------------------------------------------
@dataclass
class SceneSpec:
    name: str
    uniforms: GpuUniformsBufferManager
    params: dict
    particles: np.ndarray
    method: int                      # 0 explicit, 1 PBMPM
    n_steps: int
    mesh: tuple | None = None        # (vertices, indices) of the collider
    res: tuple = (64, 64, 64)
    notes: dict = field(default_factory=dict)


def make_uniforms(grid_min, grid_max, res, dt, fp_scale, mesh=None, interaction=None):
    u = GpuUniformsBufferManager()
    gmin = np.asarray(grid_min, np.float32)
    gmax = np.asarray(grid_max, np.float32)
    u.write_simulation_timestep_s(dt)
    u.write_fixed_point_scale(fp_scale)
    u.write_grid_min_coords(gmin)
    u.write_grid_max_coords(gmax)
    u.write_grid_resolution(res)
    # GpuSnowPipelineRunner.svelte.ts:136-140: (max - min) / res
    u.write_grid_cell_dims([(float(gmax[i]) - float(gmin[i])) / res[i] for i in range(3)])
    u.write_collider_transform_mat(identity_mat4())
    u.write_collider_transform_inv(identity_mat4())
    u.write_collider_vel([0.0, 0.0, 0.0])
    if mesh is not None:
        v, f = mesh
        u.write_collider_min_coords(v.min(axis=0))
        u.write_collider_max_coords(v.max(axis=0))
        u.write_collider_num_objects(1)
        u.write_collider_objects([{"min": v.min(axis=0), "max": v.max(axis=0), "startIndex": 0,
                                   "countIndices": int(f.size)}])
        u.write_collider_num_indices(int(f.size))
    if interaction is not None:
        u.write_is_interacting(True)
        u.write_interaction_pos(interaction["pos"])
        u.write_interaction_strength(interaction["strength"])
        u.write_interaction_radius(interaction["radius"])
        u.write_interaction_mode(interaction.get("mode", 0))
    return u


def reference_params(**over):
    """The reference's hard-coded constants (MpmParams defaults)."""
    p = dict(gravity=[0.0, 0.0, -9.81], youngs_modulus=1.4e5, poissons_ratio=0.2, hardening_explicit=5.0,
             hardening_pbmpm=20.0, theta_c=2.5e-2, theta_s=7.5e-3, density=400.0, n_iter=3, force_divisor=3.0,
             boundary_mode=0, restitution=-0.5, bc_cells=2, ground_axis=2, collider_margin=0.05,
             collider_surface_margin=0.05, collider_threshold=0.05, collider_friction=0.1, collider_vel_scale=0.2,
             pbmpm_blend=0.95, pbmpm_volume_exponent=-0.3333333)
    p.update(over)
    return p


def config_params(dx, **over):
    """Snow material of the benchmark configurations: y up, gravity -9.8,
    xi = 10, sticky ground plane + slip walls, collider margins scaled to the
    cell size (the reference's 0.05 m margins assume its 10 m domain)."""
    p = reference_params(gravity=[0.0, -9.8, 0.0], hardening_explicit=10.0, hardening_pbmpm=10.0,
                         boundary_mode=1, bc_cells=2, ground_axis=1, collider_margin=2 * dx,
                         collider_surface_margin=dx, collider_threshold=2 * dx)
    p.update(over)
    return p


def _particles_from(pos, mass, vel, pbmpm_dt=None):
    """Particle records at rest shape (F_e = F_p = I).  PBMPM's first transfer
    carries momentum from the displacement field (pbmpm.wgsl:67), not from
    the velocity, so a PBMPM scene passes its timestep and the initial
    velocity is also written as the displacement v * dt."""
    p = new_particles(pos.shape[0])
    p["pos"] = pos
    p["mass"] = mass
    p["vel"] = np.asarray(vel, np.float32)
    if pbmpm_dt is not None:
        p["dxp"] = p["vel"] * np.float32(pbmpm_dt)
    return p


def c0_explicit_snow(n_side=32, seed=0, parity=False):
    """Plain explicit MPM snow: n_side^3 jittered lattice at spacing 0.0125 in a
    0.4 cube centred at (0.5, 0.7, 0.5), v = (0,-1,0), unit box, dx = 1/64,
    dt = 1e-4, 100 steps.  parity=True switches to the reference constants
    (z up, g = -9.81, xi = 5, particle reflect only)."""
    rng = np.random.default_rng(seed)
    spacing = 0.4 / 32
    lo = np.array([0.5, 0.7, 0.5]) - 0.5 * n_side * spacing
    pos = jittered_lattice(lo, (n_side,) * 3, spacing, rng)
    mass = np.float32(400.0 * spacing ** 3)
    res = (64, 64, 64)
    u = make_uniforms([0, 0, 0], [1, 1, 1], res, 1e-4, 2.0 ** 34)
    if parity:
        params = reference_params()
        vel = (0.0, 0.0, -1.0)
    else:
        params = config_params(1 / 64)
        vel = (0.0, -1.0, 0.0)
    return SceneSpec("c0_explicit_snow" + ("_parity" if parity else ""), u, params, _particles_from(pos, mass, vel),
                     0, 100, None, res, {"spacing": spacing, "ppc": (1 / 64) ** 3 / spacing ** 3})


def c1_pbmpm_spheres(n_per_sphere=131072, seed=1, n_iter=6, parity=False, with_collider=True):
    """Two jittered-lattice spheres of radius 0.15 colliding at +-2 m/s, dx =
    1/128, dt = 2e-4, PBMPM; collider = unit box (12 tris) + icosphere (1280
    tris, r = 0.1 at (0.5, 0.2, 0.5))."""
    rng = np.random.default_rng(seed)
    r = 0.15
    spacing = (4.0 / 3.0 * np.pi * r ** 3 / n_per_sphere) ** (1 / 3) * 0.98
    a = sphere_lattice((0.3, 0.5, 0.5), r, n_per_sphere, spacing, rng)
    b = sphere_lattice((0.7, 0.5, 0.5), r, n_per_sphere, spacing, rng)
    pos = np.concatenate([a, b])
    vel = np.zeros((pos.shape[0], 3), np.float32)
    vel[:n_per_sphere, 0] = 2.0
    vel[n_per_sphere:, 0] = -2.0
    mass = np.float32(400.0 * spacing ** 3)
    res = (128, 128, 128)
    mesh = merge_meshes(box_mesh((0, 0, 0), (1, 1, 1)), icosphere(3, 0.1, (0.5, 0.2, 0.5))) if with_collider else None
    u = make_uniforms([0, 0, 0], [1, 1, 1], res, 2e-4, 2.0 ** 39, mesh=mesh)
    params = reference_params(n_iter=n_iter, force_divisor=float(n_iter)) if parity else \
        config_params(1 / 128, n_iter=n_iter, force_divisor=float(n_iter))
    return SceneSpec("c1_pbmpm_spheres", u, params, _particles_from(pos, mass, vel, pbmpm_dt=2e-4), 1, 100, mesh, res,
                     {"spacing": spacing})


def c2_large_pbmpm(counts=(256, 64, 256), seed=2, n_iter=6, terrain_n=256):
    """Snow slab 0.8 x 0.2 x 0.8 (256 x 64 x 256 jittered lattice, spacing
    0.003125) over a 256^2 fBm terrain (130,050 triangles); sparse grid at
    512^3 virtual resolution, dt = 5e-5, PBMPM, 200 substeps."""
    rng = np.random.default_rng(seed)
    spacing = 0.003125
    pos = jittered_lattice((0.1, 0.6, 0.1), counts, spacing, rng)
    mass = np.float32(400.0 * spacing ** 3)
    res = (512, 512, 512)
    mesh = fbm_terrain(terrain_n, 0.1, seed) if terrain_n else None
    u = make_uniforms([0, 0, 0], [1, 1, 1], res, 5e-5, 2.0 ** 45, mesh=mesh)
    params = config_params(1 / 512, n_iter=n_iter, force_divisor=float(n_iter))
    return SceneSpec("c2_large_pbmpm", u, params, _particles_from(pos, mass, (0.0, 0.0, 0.0)), 1, 200, mesh, res,
                     {"spacing": spacing, "ppc": (1 / 512) ** 3 / spacing ** 3})


def c4_prestrained(counts=(256, 64, 256), seed=4, n_iter=6, youngs_modulus=1.4e5, theta_c=2.5e-2, prestrain=0.01):
    """The large PBMPM scene with its return map active: c2_large_pbmpm (same
    slab, grid, dt, terrain) with pre-compacted snow, each particle's F_e
    drawn as I + N(0, prestrain^2) per entry, so most particles start beyond
    the elastic band and, once clamped, sit on the yield surface.  (With the
    reference's transfers the deformation rate is measured in cell units, so
    at dx = 1/512 the deformation of c2_large_pbmpm itself stays inside the
    elastic band and its return map never acts.)  Used to generate the
    learned plasticity's training pairs, with randomised E and theta_c, and
    to time the learned form where it does work."""
    spec = c2_large_pbmpm(counts=counts, seed=seed, n_iter=n_iter)
    rng = np.random.default_rng(seed + 1000)
    n = spec.particles.shape[0]
    Fe = np.eye(3, dtype=np.float32)[None] + rng.normal(0.0, prestrain, (n, 3, 3)).astype(np.float32)
    spec.particles["Fe"][:, :, :3] = Fe
    spec.params.update(youngs_modulus=youngs_modulus, theta_c=theta_c)
    spec.name = "c4_prestrained"
    spec.notes.update({"E": youngs_modulus, "theta_c": theta_c, "prestrain": prestrain})
    return spec


def c3_batched(n_scenes=256, seed=3, lo_count=2000, hi_count=200000):
    """Independent scenes with log-uniform particle counts in [2e3, 2e5], box
    or sphere emitters, E ~ U[5e4, 3e5], theta_c ~ U[1.5e-2, 3.5e-2],
    dx in {1/64, 1/128}; explicit, 100 substeps."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_scenes):
        n = int(np.floor(np.exp(rng.uniform(np.log(lo_count), np.log(hi_count)))))
        dx = 1 / 64 if rng.uniform() < 0.5 else 1 / 128
        res = (int(round(1 / dx)),) * 3
        spacing = dx / 2
        E = float(rng.uniform(5e4, 3e5))
        tc = float(rng.uniform(1.5e-2, 3.5e-2))
        sphere = rng.uniform() < 0.5
        side = (n * spacing ** 3) ** (1 / 3)
        c = np.array([0.5, 0.55, 0.5]) + rng.uniform(-0.05, 0.05, 3)
        if sphere:
            r = (3 * n * spacing ** 3 / (4 * np.pi)) ** (1 / 3) * 1.02
            pos = sphere_lattice(c, r, n, spacing * 0.99, rng)
        else:
            m = int(np.ceil(side / spacing))
            pos = jittered_lattice(c - m * spacing / 2, (m, m, m), spacing, rng)[:n]
        mass = np.float32(400.0 * spacing ** 3)
        u = make_uniforms([0, 0, 0], [1, 1, 1], res, 1e-4, 2.0 ** 36)
        params = config_params(dx, youngs_modulus=E, theta_c=tc)
        out.append(SceneSpec(f"c3_scene{s}", u, params, _particles_from(pos, mass, (0.0, -1.0, 0.0)), 0, 100, None,
                             res, {"dx": dx, "sphere": bool(sphere)}))
    return out


def parity_scene(kind="explicit", n_side=16, seed=10, res=32, with_collider=False, interaction=False, n_iter=3):
    """Small scenes in the reference's own conventions (z up, g = -9.81,
    reference constants) for bit-exact comparison with the oracle."""
    rng = np.random.default_rng(seed)
    spacing = 0.5 / res
    lo = np.array([0.5, 0.5, 0.35]) - 0.5 * n_side * spacing
    pos = jittered_lattice(lo, (n_side,) * 3, spacing, rng, jitter=0.45)
    mass = np.float32(400.0 * spacing ** 3)
    vel = rng.normal(0.0, 0.5, size=(pos.shape[0], 3)).astype(np.float32)
    vel[:, 2] -= 1.0
    p = _particles_from(pos, mass, vel)
    # a little initial deformation so stress and plasticity are exercised
    Fe = np.tile(np.eye(3, dtype=np.float32), (pos.shape[0], 1, 1)) + rng.normal(0, 0.02, (pos.shape[0], 3, 3)).astype(np.float32)
    p["Fe"][:, :, :3] = Fe
    p["D"][:, :, :3] = rng.normal(0, 0.01, (pos.shape[0], 3, 3)).astype(np.float32)
    p["dxp"] = vel * np.float32(1e-3)
    mesh = None
    if with_collider:
        mesh = icosphere(2, 0.12, (0.5, 0.5, 0.12))
    inter = {"pos": [res / 2, res / 2, res * 0.3], "strength": 50.0, "radius": res * 0.2, "mode": 0} if interaction else None
    res3 = (res, res, res)
    u = make_uniforms([0, 0, 0], [1, 1, 1], res3, 1e-3 if kind == "pbmpm" else 2e-4, 2.0 ** 28, mesh=mesh,
                      interaction=inter)
    params = reference_params(n_iter=n_iter, force_divisor=3.0, collider_margin=0.05)
    return SceneSpec(f"parity_{kind}", u, params, p, 1 if kind == "pbmpm" else 0, 1, mesh, res3)

def camera_inv_view_proj(eye, target, width: int, height: int, up=(0, 0, 1), fovy_deg: float = 50.0,
                         near: float = 0.05, far: float = 20.0) -> np.ndarray:
    """viewProjInvMat of a look-at camera with a WebGPU perspective projection
    (clip depth in [0, 1]), as the 16 column-major f32 the uniform block holds
    at byte 112 (GpuUniformsBufferManager.write_view_proj_inv_mat)."""
    eye, target, up = (np.asarray(v, np.float64) for v in (eye, target, up))
    f = target - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = s, u, -f
    view[:3, 3] = -view[:3, :3] @ eye
    t = 1.0 / np.tan(np.radians(fovy_deg) / 2)
    proj = np.zeros((4, 4))
    proj[0, 0], proj[1, 1] = t / (width / height), t
    proj[2, 2], proj[2, 3] = far / (near - far), near * far / (near - far)
    proj[3, 2] = -1.0
    return np.linalg.inv(proj @ view).T.reshape(16).astype(np.float32)
