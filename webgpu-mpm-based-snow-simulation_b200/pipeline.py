"""Host-side mirror of the reference's MPM plugin surface.

The reference drives its step from TypeScript through three managers:
  GpuMpmBufferManager      src/lib/gpu/mpm/GpuMpmBufferManager.ts:2-80
  GpuColliderBufferManager src/lib/gpu/collider/GpuColliderBufferManager.ts:42-351
  GpuMpmPipelineManager    src/lib/gpu/mpm/GpuMpmPipelineManager.ts:20-521
and the enum GpuSimulationMethodType (src/lib/gpu/GpuSimulationMethod.ts:1-4).
The classes below keep those names, arguments and call order; every call
lands in libmpm.so (include/mpm.h).  Errors raise MpmError (the reference
surfaces none: WebGPU validation is asynchronous and capacity overflow is
silently dropped, see mapAffectedBlocks.wgsl:27-31).
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum

import numpy as np

from . import _lib
from ._lib import MpmConfig, MpmParams, check, load
from .layout import PARTICLE_BYTES, PARTICLE_DTYPE, GpuUniformsBufferManager


class GpuSimulationMethodType(IntEnum):
    ExplicitMpm = 0
    Pbmpm = 1


def build_bvh(vertices: np.ndarray, indices: np.ndarray):
    """Reference-format BVH (GpuColliderBufferManager.ts:222-350) built by
    libmpm on the host.  Returns (nodes u32 (n, 8), triangle order)."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
    idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    nt = idx.size // 3
    nodes = np.zeros((2 * nt + 1, 8), dtype=np.uint32)
    order = np.zeros(max(nt, 1), dtype=np.uint32)
    n = C.c_uint32(0)
    check(load().mpm_build_bvh(v.ctypes.data, v.size // 3, idx.ctypes.data, idx.size, nodes.ctypes.data,
                               order.ctypes.data, C.byref(n)))
    return nodes[: n.value].copy(), order[:nt].copy()


def build_bvh_device(vertices, indices, stream: int | None = None):
    """The same BVH built on the GPU from device-resident torch tensors
    (vertices f32 [nv, 3], indices int32/uint32 [n_tris * 3]).  Returns (nodes
    int32 CUDA tensor [n, 8] holding the 32-byte nodes, triangle order)."""
    import torch

    v = vertices.contiguous().view(-1)
    idx = indices.contiguous().view(-1)
    if v.dtype != torch.float32 or idx.dtype not in (torch.int32, torch.uint32) or not v.is_cuda or not idx.is_cuda:
        raise TypeError("vertices: float32 CUDA tensor, indices: int32 CUDA tensor")
    nt = idx.numel() // 3
    lib = load()
    n_nodes = lib.mpm_bvh_node_count(nt)
    nodes = torch.empty((n_nodes, 8), dtype=torch.int32, device=v.device)
    order = torch.empty(max(nt, 1), dtype=torch.int32, device=v.device)
    n = C.c_uint32(0)
    s = torch.cuda.current_stream(v.device).cuda_stream if stream is None else stream
    check(lib.mpm_build_bvh_device(C.c_void_p(v.data_ptr()), v.numel() // 3, C.c_void_p(idx.data_ptr()), idx.numel(),
                                   C.c_void_p(nodes.data_ptr()), C.c_void_p(order.data_ptr()), C.byref(n),
                                   C.c_void_p(s)))
    return nodes[: n.value], order[:nt]


class GpuColliderBufferManager:
    """Packs a collider mesh the way the reference does: one u32 buffer
    [indices in BVH leaf order | vertices f32x3 | normals | uvs | material
    indices] plus 32-byte BVH nodes (GpuColliderBufferManager.ts:96-220)."""

    def __init__(self, *, vertices, indices, normals=None, uvs=None, material_indices=None):
        v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
        idx = np.asarray(indices, dtype=np.uint32).reshape(-1)
        if v.size:
            self.min_coords = v.min(axis=0).astype(np.float32)
            self.max_coords = v.max(axis=0).astype(np.float32)
        else:
            self.min_coords = np.full(3, np.inf, np.float32)
            self.max_coords = np.full(3, -np.inf, np.float32)
        self.num_indices = int(idx.size)
        nodes, order = build_bvh(v, idx)
        self.bvh_nodes = nodes
        self.num_bvh_nodes = int(nodes.shape[0])
        tri = idx.reshape(-1, 3)
        reordered = tri[order[: tri.shape[0]]].reshape(-1) if tri.size else idx
        parts = [reordered.astype(np.uint32), v.reshape(-1).view(np.uint32)]
        for extra in (normals, uvs):
            if extra is not None:
                parts.append(np.asarray(extra, dtype=np.float32).reshape(-1).view(np.uint32))
        if material_indices is not None:
            parts.append(np.asarray(material_indices, dtype=np.uint32).reshape(-1))
        self.collider_data = np.ascontiguousarray(np.concatenate(parts)) if parts else np.zeros(0, np.uint32)
        self.indices_offset = 0
        self.vertices_offset = 4 * self.num_indices


class GpuMpmBufferManager:
    """Owns the libmpm handle and, through it, the particle buffer and the
    sparse grid storage (GpuMpmBufferManager.ts:15-80).  The grid capacity is
    sized from the particle count here instead of the reference's fixed
    500,000 blocks / 2,000,003 hash entries."""

    def __init__(self, *, n_particles: int, device: int = 0, max_scenes: int = 1, tile_edge: int = 0,
                 max_tiles: int = 0, hash_capacity: int = 0, stream: int | None = None):
        lib = load()
        cfg = MpmConfig(max_particles=n_particles, max_scenes=max_scenes, max_tiles=max_tiles,
                        hash_capacity=hash_capacity, tile_edge=tile_edge, device=device,
                        stream=C.c_void_p(stream) if stream else None)
        h = C.c_void_p()
        rc = lib.mpm_create(C.byref(cfg), C.byref(h))
        self.handle = h
        if rc != _lib.MPM_OK:
            msg = lib.mpm_last_error(h).decode() if h.value else "mpm_create failed"
            if h.value:
                lib.mpm_destroy(h)
            self.handle = None
            raise _lib.MpmError(rc, msg)
        self.n_particles = n_particles
        self.device = device
        self._lib = lib

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mpm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # particle buffer (device.queue.writeBuffer / mapAsync equivalents)
    def write_particles(self, records: np.ndarray) -> None:
        rec = np.ascontiguousarray(records)
        assert rec.dtype.itemsize == PARTICLE_BYTES
        check(self._lib.mpm_set_particles(self.handle, rec.ctypes.data, rec.shape[0], 0), self.handle)
        self.n_particles = rec.shape[0]

    def write_particles_device(self, dev_ptr: int, n: int) -> None:
        check(self._lib.mpm_set_particles(self.handle, C.c_void_p(dev_ptr), n, 1), self.handle)
        self.n_particles = n

    def read_particles(self, n: int | None = None) -> np.ndarray:
        n = self.n_particles if n is None else n
        out = np.zeros(n, dtype=PARTICLE_DTYPE)
        check(self._lib.mpm_get_particles(self.handle, out.ctypes.data, n, 0), self.handle)
        return out

    def bind_particles_device(self, dev_ptr: int, n: int) -> None:
        check(self._lib.mpm_bind_particles_device(self.handle, C.c_void_p(dev_ptr), n), self.handle)
        self.n_particles = n

    def sync(self) -> int:
        st = C.c_uint32(0)
        rc = self._lib.mpm_sync(self.handle, C.byref(st))
        check(rc, self.handle, st.value)
        return st.value

    def counts(self):
        a, b = C.c_uint32(0), C.c_uint32(0)
        check(self._lib.mpm_get_counts(self.handle, C.byref(a), C.byref(b)), self.handle)
        return a.value, b.value

    @property
    def tile_edge(self) -> int:
        """The tile edge the substeps run with (tile_edge 0 at construction:
        chosen by the first step, and again after the particle count changes,
        from the occupied tiles; see mpm.h)."""
        e = C.c_uint32(0)
        check(self._lib.mpm_get_tile_edge(self.handle, C.byref(e)), self.handle)
        return e.value

    def calculate_grid_mass(self, res, scene: int = 0, out=None):
        """calculateGridMass (GpuVolumetricRenderPipelineManager.ts): the mass
        splat on the simulation grid, a torch u32-as-int32 CUDA tensor [z][y][x]."""
        import torch

        rx, ry, rz = (int(r) for r in res)
        out = torch.zeros((rz, ry, rx), dtype=torch.int32, device=f"cuda:{self.device}") if out is None else out
        check(self._lib.mpm_grid_mass(self.handle, scene, C.c_void_p(out.data_ptr()), 0), self.handle)
        return out

    def calculate_density(self, density_res, scene: int = 0, out=None):
        """calculateDensity (GpuMarchingCubesRenderPipelineManager.ts): the
        marching-cubes density splat, a torch u32-as-int32 CUDA tensor [z][y][x]."""
        import torch

        rx, ry, rz = (int(r) for r in density_res)
        out = torch.zeros((rz, ry, rx), dtype=torch.int32, device=f"cuda:{self.device}") if out is None else out
        res = (C.c_uint32 * 3)(rx, ry, rz)
        check(self._lib.mpm_mc_density(self.handle, scene, res, C.c_void_p(out.data_ptr()), 0), self.handle)
        return out

    def dense_grid(self, res, scene: int = 0, apply_grid_update: bool = False) -> np.ndarray:
        rx, ry, rz = (int(r) for r in res)
        out = np.zeros((rz, ry, rx, 4), dtype=np.int32)
        check(self._lib.mpm_get_grid_dense(self.handle, scene, 1 if apply_grid_update else 0, out.ctypes.data,
                                           rx * ry * rz), self.handle)
        return out


class GpuMpmPipelineManager:
    """The step's plugin surface (GpuMpmPipelineManager.ts:42-521).

    Construction wires the uniform block, the extension parameters and the
    collider into the handle; add_explicit_mpm_dispatches /
    add_pbmpm_dispatches enqueue one substep each, as the reference's two
    methods encode one substep's dispatches into a compute pass."""

    def __init__(self, *, mpm_manager: GpuMpmBufferManager, uniforms_manager: GpuUniformsBufferManager,
                 collider_manager: GpuColliderBufferManager | None = None, params: MpmParams | None = None,
                 scene: int = 0):
        self.mpm = mpm_manager
        self.uniforms = uniforms_manager
        self.scene = scene
        self._lib = load()
        self.params = params if params is not None else _lib.default_params()
        check(self._lib.mpm_set_params(self.mpm.handle, scene, C.byref(self.params)), self.mpm.handle)
        if collider_manager is not None:
            # GpuMpmPipelineManager.ts:80
            uniforms_manager.write_collider_num_indices(collider_manager.num_indices)
            cd = collider_manager.collider_data
            nodes = collider_manager.bvh_nodes
            check(self._lib.mpm_set_collider(self.mpm.handle, scene, cd.ctypes.data, cd.size,
                                             collider_manager.num_indices, nodes.ctypes.data, nodes.shape[0]),
                  self.mpm.handle)
        self._last_uniforms = None
        self.push_uniforms()

    def set_collider_mesh_device(self, vertices, indices) -> None:
        """Installs a device-resident collider mesh (torch CUDA tensors): BVH
        built and indices reordered on the GPU (mpm_set_collider_mesh_device).
        Collider bounds and transform stay the uniform writer's business, as
        with GpuColliderBufferManager."""
        import torch

        torch.cuda.current_stream().synchronize()
        v = vertices.contiguous().view(-1)
        idx = indices.contiguous().view(-1)
        self.uniforms.write_collider_num_indices(idx.numel())
        check(self._lib.mpm_set_collider_mesh_device(self.mpm.handle, self.scene, C.c_void_p(v.data_ptr()),
                                                     v.numel() // 3, C.c_void_p(idx.data_ptr()), idx.numel()),
              self.mpm.handle)
        self.push_uniforms()

    def push_uniforms(self) -> None:
        b = self.uniforms.bytes()
        if b != self._last_uniforms:
            check(self._lib.mpm_set_uniforms(self.mpm.handle, self.scene, b, len(b)), self.mpm.handle)
            self._last_uniforms = b

    def set_params(self, params: MpmParams) -> None:
        self.params = params
        check(self._lib.mpm_set_params(self.mpm.handle, self.scene, C.byref(params)), self.mpm.handle)

    def add_explicit_mpm_dispatches(self, *, n_particles: int, hash_map_size: int | None = None,
                                    n_blocks_in_hash_map: int | None = None) -> None:
        """GpuMpmPipelineManager.ts:327-428.  hash_map_size and
        n_blocks_in_hash_map are accepted for signature parity; capacities are
        fixed when the buffer manager is created."""
        self.uniforms.write_use_pbmpm(False)
        self.push_uniforms()
        check(self._lib.mpm_add_explicit_mpm_dispatches(self.mpm.handle, n_particles), self.mpm.handle)

    def add_pbmpm_dispatches(self, *, n_particles: int, n_blocks_in_hash_map: int | None = None,
                             hash_map_size: int | None = None) -> None:
        """GpuMpmPipelineManager.ts:431-521."""
        self.uniforms.write_use_pbmpm(True)
        self.push_uniforms()
        check(self._lib.mpm_add_pbmpm_dispatches(self.mpm.handle, n_particles), self.mpm.handle)

    def step(self, method: GpuSimulationMethodType, n_substeps: int = 1) -> None:
        self.uniforms.write_use_pbmpm(method == GpuSimulationMethodType.Pbmpm)
        self.push_uniforms()
        check(self._lib.mpm_step(self.mpm.handle, int(method), n_substeps), self.mpm.handle)


class GpuMeshBufferManager:
    """The closed mesh particles are scattered into (GpuMeshBufferManager.ts:1-46):
    a triangle soup of vertices padded to 4 floats, and its bounding box."""

    def __init__(self, *, vertices, indices=None):
        v = np.asarray(vertices, np.float32).reshape(-1, 3)
        if indices is not None:
            v = v[np.asarray(indices, np.int64).reshape(-1)]
        self.vertices = np.zeros((v.shape[0], 4), np.float32)
        self.vertices[:, :3] = v
        self.num_vertices = v.shape[0]
        self.min_coords = v.min(0)
        self.max_coords = v.max(0)


class GpuParticleInitializePipelineManager:
    """scatterParticles (GpuParticleInitializePipelineManager.ts:88-104):
    writes the mesh box into the uniforms and fills the particle buffer."""

    def __init__(self, *, mpm_manager: GpuMpmBufferManager, mesh_manager: GpuMeshBufferManager,
                 uniforms_manager: GpuUniformsBufferManager):
        self.mpm = mpm_manager
        self.mesh = mesh_manager
        self.uniforms = uniforms_manager
        self._lib = load()

    def add_dispatch(self, *, n_particles: int) -> None:
        self.uniforms.write_mesh_min_coords(self.mesh.min_coords)
        self.uniforms.write_mesh_max_coords(self.mesh.max_coords)
        b = self.uniforms.bytes()
        check(self._lib.mpm_set_uniforms(self.mpm.handle, 0, b, len(b)), self.mpm.handle)
        v = self.mesh.vertices
        check(self._lib.mpm_scatter_particles(self.mpm.handle, v.ctypes.data, v.shape[0], n_particles),
              self.mpm.handle)
        self.mpm.n_particles = n_particles


class GpuVolumetricBufferManager:
    """Device buffers of the volumetric renderer (GpuVolumetricBufferManager.ts:1-74),
    headless: the u32 mass grid on the simulation grid, the rgba8unorm output
    image and the r32float depth image as torch CUDA tensors, plus the f32
    colour before quantisation."""

    def __init__(self, *, grid_resolution, screen_dims, device: int = 0, mass_grid=None):
        """mass_grid: an existing int32 CUDA tensor [z][y][x] to render from
        (e.g. the result of GpuMpmBufferManager.calculate_grid_mass)."""
        import torch

        self.grid_resolution = tuple(int(r) for r in grid_resolution)
        self.device = device
        rx, ry, rz = self.grid_resolution
        dev = f"cuda:{device}"
        if mass_grid is not None and tuple(mass_grid.shape) != (rz, ry, rx):
            raise ValueError(f"mass grid shape {tuple(mass_grid.shape)} != {(rz, ry, rx)}")
        self.mass_grid = torch.zeros((rz, ry, rx), dtype=torch.int32, device=dev) if mass_grid is None else mass_grid
        self._alloc(*screen_dims)

    def _alloc(self, width: int, height: int) -> None:
        import torch

        dev = f"cuda:{self.device}"
        self.width, self.height = int(width), int(height)
        self.output = torch.zeros((self.height, self.width, 4), dtype=torch.uint8, device=dev)
        self.depth = torch.zeros((self.height, self.width), dtype=torch.float32, device=dev)
        self.color = torch.zeros((self.height, self.width, 4), dtype=torch.float32, device=dev)

    def resize(self, width: int, height: int) -> None:
        self._alloc(width, height)


class GpuVolumetricRenderPipelineManager:
    """The volumetric renderer's compute passes (GpuVolumetricRenderPipelineManager.ts:325-356):
    clear the mass grid, calculateGridMass, doVolumetricRaymarch, all on the
    handle's stream.  The composite draw (a full-screen triangle strip) has no
    headless counterpart: the output image is the result."""

    def __init__(self, *, mpm_manager: GpuMpmBufferManager, volumetric_manager: GpuVolumetricBufferManager,
                 scene: int = 0):
        self.mpm = mpm_manager
        self.vol = volumetric_manager
        self.scene = scene
        self._lib = load()

    def add_mass_calculation_dispatch(self, clear: bool = True) -> None:
        """calculateGridMass; clear=True also clears the grid first, on the same
        stream (the pass's clearBuffer)."""
        check(self._lib.mpm_grid_mass(self.mpm.handle, self.scene, C.c_void_p(self.vol.mass_grid.data_ptr()),
                                      0 if clear else 1), self.mpm.handle)

    def add_raymarch_dispatch(self) -> None:
        v = self.vol
        check(self._lib.mpm_volumetric_raymarch(self.mpm.handle, self.scene, C.c_void_p(v.mass_grid.data_ptr()),
                                                v.width, v.height, C.c_void_p(v.output.data_ptr()),
                                                C.c_void_p(v.depth.data_ptr()), C.c_void_p(v.color.data_ptr())),
              self.mpm.handle)

    def add_prerender_passes(self) -> None:
        """clearBuffer(massGrid), mass calculation, ray march (:345-356); read
        the images after the handle's sync()."""
        self.add_mass_calculation_dispatch(clear=True)
        self.add_raymarch_dispatch()


N_MAX_MC_VERTICES = 10_500_000   # GpuMarchingCubesBufferManager.ts:1-2 (3.5 M triangles)


class GpuMarchingCubesBufferManager:
    """Device buffers of the marching-cubes renderer (GpuMarchingCubesBufferManager.ts),
    headless: the u32 density grid (half the simulation resolution by default),
    the vertex buffer (6 f32 per vertex: position, normal) and the vertex
    count the draw would use."""

    def __init__(self, *, grid_resolution, mc_grid_resolution=None, device: int = 0,
                 max_vertices: int = N_MAX_MC_VERTICES):
        import torch

        gx, gy, gz = (int(r) for r in grid_resolution)
        self.density_grid_resolution = (gx // 2, gy // 2, gz // 2)
        self.mc_grid_resolution = tuple(int(r) for r in mc_grid_resolution) if mc_grid_resolution is not None \
            else (gx // 2, gy // 2, gz // 2)
        self.device = device
        dx, dy, dz = self.density_grid_resolution
        dev = f"cuda:{device}"
        self.density_grid = torch.zeros((dz, dy, dx), dtype=torch.int32, device=dev)
        self.max_vertices = int(max_vertices)
        self.vertices = torch.zeros((self.max_vertices, 6), dtype=torch.float32, device=dev)
        self.vertex_count = 0
        self.vertices_generated = 0


class GpuMarchingCubesRenderPipelineManager:
    """addMeshGenerationPass (GpuMarchingCubesRenderPipelineManager.ts:587-633):
    clear + calculateDensity, then listBlocks, computeVertexDensity,
    generateMesh and the draw-count clamp.  The mesh draw and shading passes
    are graphics work with no headless counterpart: the vertex buffer is the
    result."""

    def __init__(self, *, mpm_manager: GpuMpmBufferManager, mc_manager: GpuMarchingCubesBufferManager,
                 scene: int = 0):
        self.mpm = mpm_manager
        self.mc = mc_manager
        self.scene = scene
        self._lib = load()

    def add_density_dispatch(self) -> None:
        m = self.mc
        res = (C.c_uint32 * 3)(*m.density_grid_resolution)
        check(self._lib.mpm_mc_density(self.mpm.handle, self.scene, res, C.c_void_p(m.density_grid.data_ptr()), 0),
              self.mpm.handle)

    def add_mesh_dispatches(self) -> int:
        m = self.mc
        dres = (C.c_uint32 * 3)(*m.density_grid_resolution)
        mres = (C.c_uint32 * 3)(*m.mc_grid_resolution)
        cnt, gen = C.c_uint32(0), C.c_uint32(0)
        check(self._lib.mpm_marching_cubes(self.mpm.handle, self.scene, C.c_void_p(m.density_grid.data_ptr()), dres,
                                           mres, C.c_void_p(m.vertices.data_ptr()), m.max_vertices, C.byref(cnt),
                                           C.byref(gen)), self.mpm.handle)
        m.vertex_count, m.vertices_generated = cnt.value, gen.value
        return cnt.value

    def add_mesh_generation_pass(self) -> int:
        """Density splat and mesh generation; returns the vertex count."""
        self.add_density_dispatch()
        return self.add_mesh_dispatches()


def mc_tables():
    """(triangle table int8 [256, 16], counts uint8 [256], edge endpoints uint8 [12, 2])."""
    tri = np.zeros((256, 16), np.int8)
    cnt = np.zeros(256, np.uint8)
    ev = np.zeros((12, 2), np.uint8)
    check(load().mpm_mc_tables(tri.ctypes.data, cnt.ctypes.data, ev.ctypes.data))
    return tri, cnt, ev


class GpuMpmBatch:
    """Many independent scenes advanced by the same launches: one handle, one
    scene table, particles concatenated in scene order.  Each scene keeps its
    own uniform block, extension parameters, grid and collider (a
    GpuMpmPipelineManager per scene sets them up); a substep bins every
    scene's particles into one tile table keyed by (scene, tile) and runs each
    kernel once over all tiles, captured in one CUDA graph.  The reference
    runs one scene per device; this is the batched form of its step."""

    def __init__(self, specs, *, device: int = 0, tile_edge: int = 0, stream: int | None = None,
                 hash_capacity: int = 0, order_mode: int = 0, tile_block: int = 0):
        lib = load()
        self.specs = list(specs)
        counts = [int(s.particles.shape[0]) for s in self.specs]
        n = int(sum(counts))
        self.mpm = GpuMpmBufferManager(n_particles=n, device=device, max_scenes=len(self.specs),
                                       tile_edge=tile_edge, stream=stream, hash_capacity=hash_capacity)
        h = self.mpm.handle
        check(lib.mpm_set_schedule(h, order_mode, tile_block), h)
        check(lib.mpm_set_scene_count(h, len(self.specs)), h)
        self.ranges = []
        first = 0
        for i, c in enumerate(counts):
            check(lib.mpm_set_scene_range(h, i, first, c), h)
            self.ranges.append((first, c))
            first += c
        self.pipes = []
        for i, spec in enumerate(self.specs):
            col = None
            if spec.mesh is not None:
                col = GpuColliderBufferManager(vertices=spec.mesh[0], indices=spec.mesh[1])
            prm = _lib.default_params()
            for k, v in spec.params.items():
                if k == "gravity":
                    prm.gravity[:] = [float(x) for x in v]
                else:
                    setattr(prm, k, v)
            self.pipes.append(GpuMpmPipelineManager(mpm_manager=self.mpm, uniforms_manager=spec.uniforms,
                                                    collider_manager=col, params=prm, scene=i))
        self.mpm.write_particles(np.concatenate([s.particles for s in self.specs]))
        self._lib = lib

    @property
    def n_particles(self) -> int:
        return self.mpm.n_particles

    def step(self, method: GpuSimulationMethodType, n_substeps: int = 1) -> None:
        for p in self.pipes:
            p.uniforms.write_use_pbmpm(method == GpuSimulationMethodType.Pbmpm)
            p.push_uniforms()
        check(self._lib.mpm_step(self.mpm.handle, int(method), n_substeps), self.mpm.handle)

    def scene_particles(self, i: int, records: np.ndarray | None = None) -> np.ndarray:
        rec = self.mpm.read_particles() if records is None else records
        a, c = self.ranges[i]
        return rec[a:a + c]

    def close(self) -> None:
        self.mpm.close()


def kernel_names() -> list[str]:
    lib = load()
    return [lib.mpm_kernel_name(i).decode() for i in range(lib.mpm_kernel_count())]
