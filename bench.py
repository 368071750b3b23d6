"""Benchmark of the MPM substep on B200.

Workload (the configuration the headline metric is quoted on): a snow slab of
4,194,304 particles (256 x 64 x 256 jittered lattice, spacing 0.003125) over a
256^2 fBm terrain collider (130,050 triangles, BVH), sparse grid at 512^3
virtual resolution, dt = 5e-5, PBMPM with 6 constraint iterations.  Inputs
are seeded synthetic data of those shapes; the particle buffer (805 MB) is
larger than L2, so no flush is needed between timed steps.

`python bench.py [--gpus N --steps K --warmup W]` prints one JSON line.
Under torchrun each rank advances its own replica (weak scaling).
`--impl reference` times the CPU restatement of the reference step (the
oracle; the reference itself is WGSL that needs a graphics stack) on the
host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "webgpu-mpm-based-snow-simulation_b200"

METRIC = "particle-substeps/s at 4M (plain vs surrogate, agg err<=1e-3); P2G/G2P HBM GB/s"
# learned plasticity: predicted-error threshold above which the exact map is used
SURROGATE_UNC_THRESHOLD = 0.05
# independent particle states in flight in the end-to-end measurement
E2E_STATES = 3
WORKLOAD = "c2_large_pbmpm: 4,194,304-particle snow slab on 130,050-tri fBm terrain, 512^3 sparse grid, PBMPM x6, dt 5e-5"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms; start()
    returns once the first sample arrived, begin()/end() mark the timed
    region, and stop() summarises the samples that arrived inside it (all
    samples when none did, with samples_in_region 0)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self._t = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        deadline = time.monotonic() + 3.0
        while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def begin(self):
        self.t0 = time.monotonic()

    def end(self):
        self.t1 = time.monotonic()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, mx, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = [ln for t, ln in self.lines
                  if self.t0 is not None and self.t1 is not None and self.t0 <= t <= self.t1 + 0.05]
        for ln in inside or [ln for _, ln in self.lines]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "samples_in_region": len(inside),
                "reasons": sorted(reasons)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel: str):
    """DRAM bytes per full-size launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_c2.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def build_scene(pkg, counts=(256, 64, 256)):
    return pkg.scenes.c2_large_pbmpm(counts=counts)


def make_params(pkg, d):
    p = pkg.default_params()
    for k, v in d.items():
        if k == "gravity":
            p.gravity[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


# ----------------------------------------------------------------------
# reference arm: the CPU restatement on the host cores
# ----------------------------------------------------------------------
def bench_config(counts, steps, world):
    """The workload definition both arms report (run statistics such as the
    occupied tiles go elsewhere, so the two arms' configs compare equal)."""
    full = tuple(counts) == (256, 64, 256)
    return {"workload": WORKLOAD if full else
            f"reduced slab {counts[0]}x{counts[1]}x{counts[2]} of: {WORKLOAD}",
            "particles_per_gpu": int(counts[0]) * int(counts[1]) * int(counts[2]), "substeps_timed": steps,
            "method": "pbmpm", "n_iter": 6, "l2": "inputs larger than L2 (805 MB particle buffer)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def cpu_reference(steps, warmup, sample_counts=(256, 64, 256)):
    """Particle-substeps/s of the f32 oracle on every host core, `warmup`
    untimed then `steps` timed substeps of the scene (by default the full
    4,194,304-particle workload, about 6 s per substep on 16 threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the CPU restatement of the reference step (timed CPU baseline)

    pkg = importlib.import_module(PKG)
    spec = build_scene(pkg, counts=sample_counts)
    threads = os.cpu_count() or 1
    oracle.lib().orf_set_threads(threads)
    n = spec.particles.shape[0]
    o = oracle.Oracle(n, max_blocks=600000, hash_size=2000003)
    o.set_collider(*spec.mesh)
    p = spec.particles.copy()
    ub = spec.uniforms.bytes()
    for _ in range(warmup):
        o.step(ub, spec.params, p, 1)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(ub, spec.params, p, 1)
    dt = time.perf_counter() - t0
    o.close()
    rate = n * steps / dt
    if tuple(sample_counts) == (256, 64, 256):
        sample = (f"the full workload ({n:,} particles, 130,050-tri terrain, PBMPM x6): {warmup} untimed + "
                  f"{steps} timed substeps")
    else:
        sample = (f"{n:,}-particle block of the same slab ({sample_counts[0]}x{sample_counts[1]}x{sample_counts[2]} "
                  f"lattice, same spacing, grid, dt, terrain and PBMPM x6), {warmup} untimed + {steps} timed substeps")
    return rate, threads, sample, dt / steps


# ----------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------
def gpu_run(args, rank, world, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    pkg = importlib.import_module(PKG)
    lib = pkg.load()
    spec = build_scene(pkg, counts=args.counts)
    n = spec.particles.shape[0]
    # the library enqueues on this stream; the timing events are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    buf = pkg.GpuMpmBufferManager(n_particles=n, device=local, tile_edge=args.tile_edge, stream=stream.cuda_stream)
    buf.write_particles(spec.particles)
    col = pkg.GpuColliderBufferManager(vertices=spec.mesh[0], indices=spec.mesh[1])
    pipe = pkg.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms, collider_manager=col,
                                     params=make_params(pkg, spec.params))
    method = pkg.GpuSimulationMethodType.Pbmpm
    n_iter = int(spec.params["n_iter"])

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # warm-up (also sizes the tile storage from the first binning)
    for _ in range(args.warmup):
        pipe.step(method, 1)
    buf.sync()
    n_tiles, n_binned = buf.counts()

    # ---- timed region: K substeps, graphs on, events on the launch stream
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    clocks.begin()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        pipe.step(method, 1)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    status = buf.sync()
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * n * args.steps / (ms * 1e-3)

    # ---- per-kernel times (CUDA events around each launch, same stream)
    lib.mpm_enable_kernel_timing(buf.handle, 1)
    kt_steps = max(3, min(args.steps, 10))
    for _ in range(kt_steps):
        pipe.step(method, 1)
    K = lib.mpm_kernel_count()
    kms = (C.c_float * K)()
    kcnt = (C.c_uint32 * K)()
    lib.mpm_kernel_times(buf.handle, kms, kcnt, K)
    lib.mpm_enable_kernel_timing(buf.handle, 0)
    names = pkg.kernel_names()
    kernels = {names[i]: {"ms_per_launch": kms[i] / kcnt[i], "launches_per_step": kcnt[i] // kt_steps}
               for i in range(K) if kcnt[i]}
    # the 512-thread variants (`*_wide`: tile edge 8 with few tiles) under their base names
    by_base = {k.removesuffix("_wide"): v for k, v in kernels.items()}

    # active cells after the last P2G (grid cells with nonzero mass)
    grid = buf.dense_grid(spec.res, apply_grid_update=False)
    n_cells = int((grid[..., 0] != 0).sum())
    del grid

    # ---- roofline of the dominant kernel (PBMPM iteration: G2P + constraints + P2G)
    # algorithmic bytes per launch: per particle the fields it needs (pos 12,
    # mass 4, F_e 36, F_p 36) and its sorted index (4); per active cell one
    # 16-byte read of the previous grid and one 16-byte write of the new one.
    peak, peak_kind = measured_peak_hbm()
    dom = "pbmpm_iter"
    per_particle, per_cell = 92, 32
    alg_bytes = n * per_particle + n_cells * per_cell
    t_launch = by_base[dom]["ms_per_launch"] * 1e-3
    achieved = alg_bytes / t_launch / 1e9
    traffic = profile_traffic(dom)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "kernel": dom,
                "algorithmic_bytes_per_launch": alg_bytes, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    # P2G / G2P halves quoted by the metric: first P2G and the final G2P+integrate
    p2g_bytes = n * (12 + 4 + 36 + 36 + 12 + 36 + 4) + n_cells * 16
    g2p_bytes = n_cells * 16 + n * (4 + 88 + 144)
    p2g_gbs = p2g_bytes / (by_base["pbmpm_first"]["ms_per_launch"] * 1e-3) / 1e9
    g2p_gbs = g2p_bytes / (by_base["g2p_pbmpm_integrate"]["ms_per_launch"] * 1e-3) / 1e9

    # ---- explicit method on the same state (extra line item)
    ex = pkg.GpuSimulationMethodType.ExplicitMpm
    for _ in range(2):
        pipe.step(ex, 1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ex_steps = max(5, args.steps)
    for _ in range(ex_steps):
        pipe.step(ex, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    ex_rate = n * ex_steps / (e0.elapsed_time(e1) * 1e-3)

    # ---- renderer passes of the final state.  The step's fixed-point scale
    # (2^45, sized for the momentum sums) would wrap the renderers' u32 mass
    # sums, so they run with a scale of 2^20, restored afterwards.
    u_bytes = spec.uniforms.bytes()
    step_scale = float(np.frombuffer(bytes(u_bytes[4:8]), "<f4")[0])
    spec.uniforms.write_fixed_point_scale(2.0 ** 20)
    pipe.push_uniforms()
    # ---- renderer splats (calculateGridMass.wgsl, mcDensity.cs.wgsl)
    rx, ry, rz = spec.res
    mass_grid = torch.zeros((rz, ry, rx), dtype=torch.int32, device="cuda")
    dens_grid = torch.zeros((rz // 2, ry // 2, rx // 2), dtype=torch.int32, device="cuda")
    splats = {}
    for name, fn in (("grid_mass", lambda: buf.calculate_grid_mass(spec.res, out=mass_grid)),
                     ("mc_density", lambda: buf.calculate_density((rx // 2, ry // 2, rz // 2), out=dens_grid))):
        fn()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(5):
            fn()
        s1.record(stream)
        torch.cuda.synchronize()
        ms_s = s0.elapsed_time(s1) / 5
        splats[name] = {"ms": round(ms_s, 4), "particles_per_s": n / (ms_s * 1e-3)}
    del dens_grid
    # ---- volumetric ray march of the final state (volumetricRaymarch.cs.wgsl), 1280 x 720
    rw, rh = 1280, 720
    spec.uniforms.write_view_proj_inv_mat(pkg.scenes.camera_inv_view_proj((0.5, -0.9, 1.2), (0.5, 0.5, 0.3), rw, rh))
    spec.uniforms.write_time(1)
    pipe.push_uniforms()
    vol = pkg.GpuVolumetricBufferManager(grid_resolution=spec.res, screen_dims=(rw, rh), device=local,
                                         mass_grid=mass_grid)
    rpipe = pkg.GpuVolumetricRenderPipelineManager(mpm_manager=buf, volumetric_manager=vol)
    rpipe.add_raymarch_dispatch()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(3):
        rpipe.add_raymarch_dispatch()
    s1.record(stream)
    torch.cuda.synchronize()
    ms_r = s0.elapsed_time(s1) / 3
    splats["volumetric_raymarch"] = {"ms": round(ms_r, 4), "pixels": rw * rh,
                                     "covered": int((vol.output[..., 3] > 0).sum().item())}
    del vol, rpipe, mass_grid
    # ---- marching cubes of the final state: 256^3 MC grid over an 8^3 density
    # grid (cells of 1/8: the slab's mass per cell, up to ~0.57, crosses the
    # isovalue 0.15; at fine density grids it stays below it, the mesh is empty)
    mcb = pkg.GpuMarchingCubesBufferManager(grid_resolution=(16, 16, 16), mc_grid_resolution=(256, 256, 256),
                                            device=local, max_vertices=6_000_000)
    mcp = pkg.GpuMarchingCubesRenderPipelineManager(mpm_manager=buf, mc_manager=mcb)
    mcp.add_mesh_generation_pass()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        mcp.add_mesh_generation_pass()
    mc_ms = (time.perf_counter() - t0) / 3 * 1e3
    splats["marching_cubes"] = {"ms_wall": round(mc_ms, 3), "mc_res": list(mcb.mc_grid_resolution),
                                "vertices": mcb.vertices_generated}
    del mcp, mcb
    spec.uniforms.write_fixed_point_scale(step_scale)
    pipe.push_uniforms()
    # ---- collider BVH of the terrain (130,050 triangles): GPU build vs the host build
    tv, tf = spec.mesh
    tv_d = torch.from_numpy(np.ascontiguousarray(tv, np.float32)).cuda()
    tf_d = torch.from_numpy(np.ascontiguousarray(tf, np.int32).reshape(-1)).cuda()
    pkg.build_bvh_device(tv_d, tf_d, stream=stream.cuda_stream)
    t0 = time.perf_counter()
    for _ in range(3):
        pkg.build_bvh_device(tv_d, tf_d, stream=stream.cuda_stream)
    gpu_bvh_ms = (time.perf_counter() - t0) / 3 * 1e3
    t0 = time.perf_counter()
    pkg.build_bvh(tv, tf)
    host_bvh_ms = (time.perf_counter() - t0) * 1e3
    splats["bvh_build"] = {"triangles": int(np.asarray(tf).size // 3), "gpu_ms": round(gpu_bvh_ms, 3),
                           "host_ms": round(host_bvh_ms, 3)}
    del tv_d, tf_d
    # ---- particle initialisation (scatterParticles) into a 1,280-triangle icosphere, 262,144 particles
    v_ico, f_ico = pkg.scenes.icosphere(3, 0.15, (0.5, 0.5, 0.5))
    mesh = pkg.GpuMeshBufferManager(vertices=v_ico, indices=f_ico)
    sbuf = pkg.GpuMpmBufferManager(n_particles=262144, device=local, stream=stream.cuda_stream)
    sinit = pkg.GpuParticleInitializePipelineManager(mpm_manager=sbuf, mesh_manager=mesh,
                                                     uniforms_manager=pkg.GpuUniformsBufferManager())
    sinit.add_dispatch(n_particles=262144)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    sinit.add_dispatch(n_particles=262144)
    s1.record(stream)
    torch.cuda.synchronize()
    splats["scatter_particles"] = {"ms": round(s0.elapsed_time(s1), 4), "particles": 262144, "triangles": 1280}
    sbuf.close()

    # ---- end to end through the public API with host buffers.  Each step
    # uploads a state's 192-byte records from pinned host memory
    # (mpm_set_particles), advances it one substep and reads the records back
    # (mpm_get_particles).  E2E_STATES states on their own streams take turns,
    # so one state's upload overlaps the others' readbacks and substeps (PCIe
    # copies run both directions at once); the serial chain of one state is
    # timed beside it.
    e2e_steps = max(3, min(args.steps, 10))
    hosts, states = [], []
    for k in range(E2E_STATES):
        host = torch.empty(n * 192, dtype=torch.uint8, pin_memory=True)
        host.numpy()[:] = np.frombuffer(spec.particles.tobytes(), np.uint8)
        hosts.append(host)
        if k == 0:
            states.append((buf, pipe, stream))
        else:
            s2 = torch.cuda.Stream()
            b2 = pkg.GpuMpmBufferManager(n_particles=n, device=local, tile_edge=args.tile_edge, stream=s2.cuda_stream)
            b2.write_particles(spec.particles)
            c2 = pkg.GpuColliderBufferManager(vertices=spec.mesh[0], indices=spec.mesh[1])
            p2 = pkg.GpuMpmPipelineManager(mpm_manager=b2, uniforms_manager=spec.uniforms, collider_manager=c2,
                                           params=make_params(pkg, spec.params))
            states.append((b2, p2, s2))

    def e2e_issue(k, wait):
        b, pp, _ = states[k]
        hp = C.c_void_p(hosts[k].data_ptr())
        pkg._lib.check(lib.mpm_set_particles(b.handle, hp, n, 0), b.handle)
        pp.step(method, 1)
        pkg._lib.check(lib.mpm_get_particles(b.handle, hp, n, 0 if wait else 2), b.handle)

    for k in range(E2E_STATES):
        e2e_issue(k, True)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for k in range(E2E_STATES):
            e2e_issue(k, False)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_issue(0, True)
    torch.cuda.synchronize()
    e2e_serial_s = time.perf_counter() - t0
    for b_, _, _ in states[1:]:
        b_.close()
    del hosts, states
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_s, e2e_serial_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s, e2e_serial_s = (float(v) for v in t.tolist())
    e2e_rate = world * n * E2E_STATES * e2e_steps / e2e_s
    e2e_serial = world * n * e2e_steps / e2e_serial_s

    launches_per_step = sum(v["launches_per_step"] for v in kernels.values())
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "particle-substeps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (fixed-point i32 grid)",
        "data": "synthetic (seeded procedural slab + fBm terrain; no dataset)",
        "config": bench_config(args.counts, args.steps, world),
        "run": {"tile_edge": buf.tile_edge, "occupied_tiles": n_tiles, "active_cells": n_cells,
                "n_iter": n_iter},
        "roofline": roofline,
        "p2g_gbs": round(p2g_gbs, 1),
        "g2p_gbs": round(g2p_gbs, 1),
        "explicit_value": ex_rate,
        "splats": splats,
        "kernels": {k: round(v["ms_per_launch"], 4) for k, v in kernels.items()},
        "e2e": {"value": e2e_rate, "unit": "particle-substeps/s", "h2d_bytes_per_step": n * 192,
                "d2h_bytes_per_step": n * 192, "states_in_flight": E2E_STATES, "serial_one_state": e2e_serial},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
        "device_status": status,
    }
    return out


# ----------------------------------------------------------------------
# extra legs at N = 1: learned plasticity (config 4) and batched scenes (config 3)
# ----------------------------------------------------------------------
def _events(torch, stream):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _pipeline(pkg, spec, tile_edge, stream, local, max_tiles=0):
    buf = pkg.GpuMpmBufferManager(n_particles=spec.particles.shape[0], device=local, tile_edge=tile_edge,
                                  stream=stream.cuda_stream, max_tiles=max_tiles)
    buf.write_particles(spec.particles)
    col = None
    if spec.mesh is not None:
        col = pkg.GpuColliderBufferManager(vertices=spec.mesh[0], indices=spec.mesh[1])
    pipe = pkg.GpuMpmPipelineManager(mpm_manager=buf, uniforms_manager=spec.uniforms, collider_manager=col,
                                     params=make_params(pkg, spec.params))
    return buf, pipe


def _agg(rec):
    """Centre of mass, total momentum, total absolute momentum, mean J_p."""
    import numpy as np
    m = rec["mass"].astype(np.float64)
    v = rec["vel"].astype(np.float64)
    com = (rec["pos"].astype(np.float64) * m[:, None]).sum(0) / m.sum()
    mom = (v * m[:, None]).sum(0)
    abs_mom = float((np.linalg.norm(v, axis=1) * m).sum())
    F = rec["Fp"][:, :, :3].astype(np.float64)
    jp = float(np.linalg.det(F).mean())
    return com, mom, abs_mom, jp


def _agg_rel_err(a, b):
    """Relative deviation of a from b: centre of mass over its own magnitude,
    momentum over the total absolute momentum, mean J_p over itself."""
    import numpy as np
    return {"centre_of_mass": float(np.abs(a[0] - b[0]).max() / np.abs(b[0]).max()),
            "momentum": float(np.abs(a[1] - b[1]).max() / max(b[2], 1e-30)),
            "mean_jp": float(abs(a[3] - b[3]) / abs(b[3]))}


def _timed_run(pkg, torch, spec, mode, net, tile_edge, stream, local, warmup, steps):
    """(particle-substeps/s, final records, plasticity stats) of `steps`
    graph-replayed PBMPM substeps from the scene's initial state."""
    # fixed tile storage: the pre-compacted snow spreads while it relaxes
    buf, pipe = _pipeline(pkg, spec, tile_edge, stream, local, max_tiles=6 * 4732)
    ctl = pkg.learned.PlasticityController(buf)
    ctl.set_mode(mode, net, unc_threshold=SURROGATE_UNC_THRESHOLD, det_threshold=1e-3, audit_fraction=0.01)
    method = pkg.GpuSimulationMethodType.Pbmpm
    for _ in range(warmup):
        pipe.step(method, 1)
    buf.sync()
    ctl.stats(reset=True)
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    for _ in range(steps):
        pipe.step(method, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    rate = spec.particles.shape[0] * steps / (e0.elapsed_time(e1) * 1e-3)
    st = ctl.stats()
    buf.sync()
    rec = buf.read_particles()
    buf.close()
    return rate, rec, st


def _collect_pairs(pkg, args, local, stream, return_map, seed, rollouts=5, substeps=80, sample=0.12):
    """Training pairs (x, t) from COLLECT-mode rollouts of the config-2 slab
    geometry with pre-compacted snow (524,288 particles, the terrain, dt
    5e-5, PBMPM x6), E ~ U[5e4, 3e5] and theta_c ~ U[1.5e-2, 3.5e-2] per
    rollout; the targets are the scene's return map (return_map)."""
    import numpy as np
    import torch

    L = pkg._lib
    rng = np.random.default_rng(seed)
    xs, ts, mats = [], [], []
    for r in range(rollouts):
        E, tc = float(rng.uniform(5e4, 3e5)), float(rng.uniform(1.5e-2, 3.5e-2))
        spec = pkg.scenes.c4_prestrained(counts=(128, 32, 128), seed=50 + r, youngs_modulus=E, theta_c=tc)
        spec.params["return_map"] = return_map
        buf, pipe = _pipeline(pkg, spec, args.tile_edge, stream, local, max_tiles=6 * 1183)
        ctl = pkg.learned.PlasticityController(buf)
        ctl.set_mode(L.PLASTICITY_COLLECT, audit_fraction=sample)
        x, t = ctl.collect_into(3_500_000, device=local)
        for k in range(substeps):
            pipe.step(pkg.GpuSimulationMethodType.Pbmpm, 1)
        n = min(ctl.stats()["pairs_collected"], x.shape[0])
        xs.append(x[:n].clone())
        ts.append(t[:n].clone())
        mats.append({"E": round(E, 1), "theta_c": round(tc, 5), "pairs": int(n)})
        buf.close()
        del x, t
    return torch.cat(xs), torch.cat(ts), mats


def _max_err(errs):
    return {k: max(e[k] for e in errs) for k in errs[0]}


def surrogate_leg(pkg, args, local, stream):
    """Learned plasticity (config 4).  Two networks: one trained on the
    reference's return map, one on the SVD clamp (the option this library
    adds); each is timed against the exact map it replaces on the 4.19 M
    pre-compacted slab, with the aggregate deviation from the exact run, the
    scene's chaos floor (the exact run again from states nudged by one ulp,
    three nudges, largest deviation) and, on the 524,288-particle block, the
    deviation of the exact and the learned runs from the f64 oracle."""
    import dataclasses

    import numpy as np
    import torch

    L = pkg._lib
    out = {}
    nets = {}
    for rmap, name in ((0, "reference_map"), (1, "svd_map")):
        t0 = time.perf_counter()
        x, t, mats = _collect_pairs(pkg, args, local, stream, rmap, seed=41 + rmap)
        torch.cuda.synchronize()
        collect_s = time.perf_counter() - t0
        net = pkg.learned.PlasticityNet(device=local, seed=7 + rmap)
        net.set_stream(stream.cuda_stream)
        t0 = time.perf_counter()
        epochs = 24
        hist = net.train(x, t, epochs=epochs, batch=8192, lr=3e-3, lr_final=2e-5, unc_weight=0.1, seed=3)
        train_s = time.perf_counter() - t0
        nets[rmap] = net
        out[f"train_{name}"] = {"pairs": int(x.shape[0]), "rollouts": mats, "collect_s": round(collect_s, 2),
                                "train_s": round(train_s, 2), "epochs": epochs, "batch": 8192,
                                "loss_first_epoch": float(hist[0]), "loss_last_epoch": float(hist[-1])}
        if rmap == 0:
            # network throughput on 4,194,304 rows (tensor-core forward alone)
            rows = 4194304
            xr = x[torch.randint(0, x.shape[0], (rows,), device=x.device)].contiguous()
            net.forward(xr)
            torch.cuda.synchronize()
            e0, e1 = _events(torch, stream)
            e0.record(stream)
            for _ in range(5):
                net.forward(xr)
            e1.record(stream)
            torch.cuda.synchronize()
            fwd_ms = e0.elapsed_time(e1) / 5
            flops = 2.0 * (12 * 64 + 64 * 64 * 2 + 64 * 11) * rows
            out["mlp_forward"] = {"rows": rows, "ms": round(fwd_ms, 4),
                                  "tflops": round(flops / (fwd_ms * 1e-3) / 1e12, 2)}
            del xr
        del x, t
    steps, warm = max(10, min(args.steps, 40)), 3

    def nudged(spec, axis):
        p = spec.particles.copy()
        p["pos"][:, axis] = np.nextafter(p["pos"][:, axis], np.float32(np.inf))
        return dataclasses.replace(spec, particles=p)

    cases = (("c2_large_pbmpm", build_scene(pkg, counts=args.counts), 0, L.PLASTICITY_INLINE),
             ("c4_prestrained", pkg.scenes.c4_prestrained(counts=args.counts), 0, L.PLASTICITY_INLINE),
             ("c4_prestrained_svd_map", pkg.scenes.c4_prestrained(counts=args.counts), 1, L.PLASTICITY_EXACT))
    for name, spec, rmap, exact_mode in cases:
        spec.params["return_map"] = rmap
        r_exact, rec_p, _ = _timed_run(pkg, torch, spec, exact_mode, None, args.tile_edge, stream, local, warm, steps)
        r_learn, rec_l, st = _timed_run(pkg, torch, spec, L.PLASTICITY_LEARNED, nets[rmap], args.tile_edge, stream,
                                        local, warm, steps)
        floor = []
        for axis in range(3):
            _, rec_n, _ = _timed_run(pkg, torch, nudged(spec, axis), exact_mode, None, args.tile_edge, stream, local,
                                     warm, steps)
            floor.append(_agg_rel_err(_agg(rec_n), _agg(rec_p)))
            del rec_n
        st = {k: (int(v) if isinstance(v, int) else float(v)) for k, v in st.items()}
        out[name] = {"substeps": warm + steps, "return_map": "svd" if rmap else "reference",
                     "exact": r_exact, "learned": r_learn, "learned_vs_exact": r_learn / r_exact,
                     "agg_rel_err_vs_exact": _agg_rel_err(_agg(rec_l), _agg(rec_p)),
                     "chaos_floor_1ulp_vs_exact": _max_err(floor), "stats": st}
        del rec_p, rec_l
    # against the f64 oracle: the 524,288-particle block of the pre-compacted slab
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the f64 error reference

    oracle.lib().orf_set_threads(os.cpu_count() or 1)
    spec = pkg.scenes.c4_prestrained(counts=(128, 32, 128))
    n_blk = warm + steps
    recs = {}
    for label, mode in (("exact", L.PLASTICITY_INLINE), ("learned", L.PLASTICITY_LEARNED)):
        buf, pipe = _pipeline(pkg, spec, args.tile_edge, stream, local, max_tiles=6 * 1183)
        ctl = pkg.learned.PlasticityController(buf)
        ctl.set_mode(mode, nets[0] if mode == L.PLASTICITY_LEARNED else None,
                     unc_threshold=SURROGATE_UNC_THRESHOLD, det_threshold=1e-3, audit_fraction=0.01)
        pipe.step(pkg.GpuSimulationMethodType.Pbmpm, n_blk)
        buf.sync()
        recs[label] = buf.read_particles()
        buf.close()
    o = oracle.Oracle(spec.particles.shape[0], max_blocks=600000, hash_size=2000003, fp64=True)
    o.set_collider(*spec.mesh)
    p64 = oracle.to_fp64(spec.particles.copy())
    for _ in range(n_blk):
        o.step(spec.uniforms.bytes(), spec.params, p64, 1)
    o.close()
    ref = _agg_any(p64)
    out["c4_block_vs_f64"] = {"particles": int(spec.particles.shape[0]), "substeps": n_blk,
                              "exact_f32": _agg_rel_err(_agg(recs["exact"]), ref),
                              "learned": _agg_rel_err(_agg(recs["learned"]), ref)}
    for net in nets.values():
        net.close()
    return out


def batched_leg(pkg, args, local, stream):
    import torch

    specs = pkg.scenes.c3_batched()
    method = pkg.GpuSimulationMethodType.ExplicitMpm
    n_total = int(sum(s.particles.shape[0] for s in specs))
    sched, times = pkg.batching.autotune_schedule(specs, method, steps=3, device=local)
    b = pkg.GpuMpmBatch(specs, device=local, stream=stream.cuda_stream, **sched)
    steps = max(10, min(args.steps, 30))
    ms = pkg.batching.time_batch(b, method, steps, warmup=3)
    b.close()
    # the plain per-scene loop: one handle per scene (each at the tile edge the
    # library picks for it), launched one after another
    handles = []
    for spec in specs:
        buf, pipe = _pipeline(pkg, spec, 0, stream, local)
        handles.append((buf, pipe))
    for buf, pipe in handles:
        pipe.step(method, 2)
    torch.cuda.synchronize()
    loop_steps = 5
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    for _ in range(loop_steps):
        for buf, pipe in handles:
            pipe.step(method, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1) / loop_steps
    for buf, _ in handles:
        buf.close()
    return {"workload": f"c3_batched: {len(specs)} scenes, {n_total:,} particles, explicit, dx 1/64 or 1/128",
            "schedule_autotuned": sched, "autotune_ms_per_substep": {str(k): round(v, 4) for k, v in times.items()},
            "batched_ms_per_substep": round(ms, 4), "batched_value": n_total / (ms * 1e-3),
            "per_scene_loop_ms_per_substep": round(loop_ms, 4), "per_scene_loop_value": n_total / (loop_ms * 1e-3),
            "batched_vs_loop": loop_ms / ms, "unit": "particle-substeps/s"}


def batched_sharded(args, rank, world, local):
    """Config 3 sharded by scene over the ranks (`--batched`): each rank
    advances its shard of the 256 scenes (shard_scenes: balanced by particle
    count, the same on every rank, no communication) in one GpuMpmBatch;
    CUDA events around K substeps, the max over ranks; the per-scene
    aggregates are gathered on rank 0 afterwards (host objects, outside the
    timed region).  The total work is fixed as N grows: strong scaling."""
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    pkg = importlib.import_module(PKG)
    specs = pkg.scenes.c3_batched()
    counts = [int(s.particles.shape[0]) for s in specs]
    mine = pkg.batching.shard_scenes(counts, world)[rank]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    method = pkg.GpuSimulationMethodType.ExplicitMpm
    b = pkg.GpuMpmBatch([specs[i] for i in mine], device=local, tile_edge=args.tile_edge, stream=stream.cuda_stream)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        b.step(method, 1)
    b.mpm.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    clocks.begin()
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    for _ in range(args.steps):
        b.step(method, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    status = b.mpm.sync()
    rec = b.mpm.read_particles()
    local_aggs = {i: pkg.batching.scene_aggregates(b.scene_particles(j, rec)) for j, i in enumerate(mine)}
    b.close()
    aggs = local_aggs
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        parts = [None] * world
        dist.all_gather_object(parts, local_aggs)
        aggs = {}
        for part in parts:
            aggs.update(part)
    total = int(sum(counts))
    return {
        "metric": "particle-substeps/s, config 3 (256 independent scenes, sharded by scene)",
        "value": total * args.steps / (ms * 1e-3), "unit": "particle-substeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32 (fixed-point i32 grid)",
        "data": "synthetic (seeded procedural scenes; no dataset)",
        "config": {"workload": f"c3_batched: {len(specs)} scenes, {total:,} particles, explicit, dx 1/64 or 1/128",
                   "tile_edge": args.tile_edge, "parallelism": f"scenes sharded x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (2.2 GB of particle records)"},
        "shard_particles_rank0": int(sum(counts[i] for i in mine)) if rank == 0 else None,
        "scenes_gathered": len(aggs),
        "aggregate_checksum": float(np.sum([v[0] + v[1] + v[2] for v in aggs.values()])),
        "clocks": clk, "device_status": status,
    }


def f64_leg(pkg, args, local, stream, steps=3):
    """The full workload (config 2 at 4,194,304 particles) against the f64
    oracle: the GPU state after `steps` substeps from the initial records and
    the f64 oracle's after the same substeps (the f64 oracle is the error
    reference only; it runs on the host cores, outside any timed region)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the f64 error reference

    spec = build_scene(pkg, counts=args.counts)
    buf, pipe = _pipeline(pkg, spec, args.tile_edge, stream, local)
    pipe.step(pkg.GpuSimulationMethodType.Pbmpm, steps)
    status = buf.sync()
    rec = buf.read_particles()
    buf.close()
    oracle.lib().orf_set_threads(os.cpu_count() or 1)
    o = oracle.Oracle(spec.particles.shape[0], max_blocks=600000, hash_size=2000003, fp64=True)
    o.set_collider(*spec.mesh)
    p64 = oracle.to_fp64(spec.particles.copy())
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(spec.uniforms.bytes(), spec.params, p64, 1)
    oracle_s = time.perf_counter() - t0
    o.close()
    return {"particles": int(spec.particles.shape[0]), "substeps": steps, "device_status": status,
            "agg_rel_err_vs_f64": _agg_rel_err(_agg(rec), _agg_any(p64)), "f64_oracle_s": round(oracle_s, 1)}


def _agg_any(rec):
    """_agg for 192-byte records or the f64 oracle's records."""
    import numpy as np
    if "Fe" in rec.dtype.names and rec["Fp"].ndim == 2:     # f64 oracle layout (9 entries per matrix)
        m = rec["mass"].astype(np.float64)
        v = rec["vel"].astype(np.float64)
        com = (rec["pos"] * m[:, None]).sum(0) / m.sum()
        mom = (v * m[:, None]).sum(0)
        abs_mom = float((np.linalg.norm(v, axis=1) * m).sum())
        jp = float(np.linalg.det(rec["Fp"].reshape(-1, 3, 3)).mean())
        return com, mom, abs_mom, jp
    return _agg(rec)


def results_table(local):
    """Rows of the results table: configs 0-2 on the GPU (CUDA-event
    particle-substeps/s, P2G/G2P algorithmic GB/s), the f32 oracle on all host
    cores over the same substeps (bit-exactness of the GPU result against it),
    and the aggregate deviation of the GPU result from the f64 oracle."""
    import numpy as np
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # CPU restatement: the timed CPU baseline and the f64 error reference

    torch.cuda.set_device(local)
    pkg = importlib.import_module(PKG)
    lib = pkg.load()
    threads = os.cpu_count() or 1
    oracle.lib().orf_set_threads(threads)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    rows = []
    # (name, scene, timed GPU substeps, substeps compared bit for bit with the f32
    # oracle, substeps after which the aggregates are compared with the f64 oracle:
    # each configuration's own substep count, on the 524,288-particle block for config 2)
    def computed(r, f):   # matrices are three padded columns: compare the 3x3 part
        a = r[f][:, :, :3] if f in ("Fe", "Fp", "D") else r[f]
        return np.ascontiguousarray(a).view(np.uint32)

    cases = [("C0", pkg.scenes.c0_explicit_snow(), 100, 100, 100),
             ("C1", pkg.scenes.c1_pbmpm_spheres(), 100, 10, 100),
             ("C2 block", pkg.scenes.c2_large_pbmpm(counts=(128, 32, 128)), 60, 5, 200)]
    for name, spec, gpu_steps, cmp_steps, agg_steps in cases:
        n = spec.particles.shape[0]
        method = spec.method
        # GPU throughput (state advanced by warm-up, graphs on)
        buf, pipe = _pipeline(pkg, spec, 0, stream, local)
        for _ in range(3):
            pipe.step(method, 1)
        buf.sync()
        e0, e1 = _events(torch, stream)
        e0.record(stream)
        for _ in range(gpu_steps):
            pipe.step(method, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        gpu_rate = n * gpu_steps / (e0.elapsed_time(e1) * 1e-3)
        lib.mpm_enable_kernel_timing(buf.handle, 1)
        for _ in range(5):
            pipe.step(method, 1)
        K = lib.mpm_kernel_count()
        kms, kcnt = (C.c_float * K)(), (C.c_uint32 * K)()
        lib.mpm_kernel_times(buf.handle, kms, kcnt, K)
        lib.mpm_enable_kernel_timing(buf.handle, 0)
        kn = pkg.kernel_names()
        # the 512-thread variants (`*_wide`, tile edge 8 with few tiles) under their base names
        kt = {kn[i].removesuffix("_wide"): kms[i] / kcnt[i] for i in range(K) if kcnt[i]}
        grid = buf.dense_grid(spec.res, apply_grid_update=False)
        cells = int((grid[..., 0] != 0).sum())
        del grid
        edge = buf.tile_edge
        buf.close()
        if method == 0:
            p2g = (n * (128 + 4) + cells * 16) / (kt["p2g_explicit"] * 1e-3) / 1e9
            g2p = (cells * 16 + n * (4 + 88 + 144)) / (kt["g2p_explicit_integrate"] * 1e-3) / 1e9
        else:
            p2g = (n * (12 + 4 + 36 + 36 + 12 + 36 + 4) + cells * 16) / (kt["pbmpm_first"] * 1e-3) / 1e9
            g2p = (cells * 16 + n * (4 + 88 + 144)) / (kt["g2p_pbmpm_integrate"] * 1e-3) / 1e9
        # GPU result after cmp_steps substeps from the initial state
        buf, pipe = _pipeline(pkg, spec, 0, stream, local)
        for _ in range(cmp_steps):
            pipe.step(method, 1)
        status = buf.sync()
        got = buf.read_particles()
        buf.close()
        # f32 oracle over the same substeps: timed CPU baseline and bit-exactness
        o = oracle.Oracle(n, max_blocks=600000, hash_size=2000003)
        if spec.mesh is not None:
            o.set_collider(*spec.mesh)
        p32 = spec.particles.copy()
        t0 = time.perf_counter()
        for _ in range(cmp_steps):
            o.step(spec.uniforms.bytes(), spec.params, p32, method)
        cpu_s = time.perf_counter() - t0
        o.close()
        exact = all(np.array_equal(computed(got, f), computed(p32, f))
                    for f in ("pos", "vel", "mass", "Fe", "Fp", "dxp", "D"))
        # GPU state after the configuration's own substep count, against the f64 oracle
        if agg_steps != cmp_steps:
            buf, pipe = _pipeline(pkg, spec, 0, stream, local)
            for _ in range(agg_steps):
                pipe.step(method, 1)
            status |= buf.sync()
            got = buf.read_particles()
            buf.close()
        o = oracle.Oracle(n, max_blocks=600000, hash_size=2000003, fp64=True)
        if spec.mesh is not None:
            o.set_collider(*spec.mesh)
        p64 = oracle.to_fp64(spec.particles.copy())
        for _ in range(agg_steps):
            o.step(spec.uniforms.bytes(), spec.params, p64, method)
        o.close()
        err = _agg_rel_err(_agg(got), _agg_any(p64))
        rows.append({"config": name, "workload": spec.name, "particles": n, "method": "pbmpm" if method else "explicit",
                     "gpu_value": gpu_rate, "gpu_steps": gpu_steps, "tile_edge": edge, "p2g_gbs": round(p2g, 1), "g2p_gbs": round(g2p, 1),
                     "kernels_ms": {k: round(v, 4) for k, v in kt.items()}, "active_cells": cells,
                     "cpu_value": n * cmp_steps / cpu_s, "cpu_threads": threads, "cpu_steps": cmp_steps,
                     "bit_exact_vs_f32_oracle": bool(exact), "agg_steps": agg_steps, "agg_rel_err_vs_f64": err,
                     "device_status": status})
        print(json.dumps(rows[-1]), flush=True)
    # config 3: a sample of 8 of its 256 scenes as one batch, 100 substeps,
    # each scene against the f32 oracle (bit for bit) and the f64 oracle
    specs = pkg.scenes.c3_batched()[:8]
    batch = pkg.GpuMpmBatch(specs, tile_edge=8, stream=stream.cuda_stream)
    batch.step(pkg.GpuSimulationMethodType.ExplicitMpm, 100)
    status = batch.mpm.sync()
    rec = batch.mpm.read_particles()
    errs, exact = [], True
    for i, spec in enumerate(specs):
        got = batch.scene_particles(i, rec)
        o = oracle.Oracle(spec.particles.shape[0], max_blocks=200000, hash_size=2000003)
        p32 = spec.particles.copy()
        for _ in range(100):
            o.step(spec.uniforms.bytes(), spec.params, p32, 0)
        o.close()
        exact = exact and all(np.array_equal(computed(got, f), computed(p32, f))
                              for f in ("pos", "vel", "mass", "Fe", "Fp", "dxp", "D"))
        o = oracle.Oracle(spec.particles.shape[0], max_blocks=200000, hash_size=2000003, fp64=True)
        p64 = oracle.to_fp64(spec.particles.copy())
        for _ in range(100):
            o.step(spec.uniforms.bytes(), spec.params, p64, 0)
        o.close()
        errs.append(_agg_rel_err(_agg(got), _agg_any(p64)))
    batch.close()
    rows.append({"config": "C3 sample", "workload": "c3_batched, scenes 0-7 as one batch",
                 "particles": int(sum(s.particles.shape[0] for s in specs)), "method": "explicit",
                 "agg_steps": 100, "bit_exact_vs_f32_oracle": bool(exact),
                 "agg_rel_err_vs_f64_max_over_scenes": {k: max(e[k] for e in errs) for k in errs[0]},
                 "device_status": status})
    print(json.dumps(rows[-1]), flush=True)
    return rows


def step_case(args, local):
    """The substep alone (the profiling case of the step's kernels): builds the
    slab of --counts, runs --warmup then --steps PBMPM substeps through the
    public API and prints the CUDA-event time per substep; no other leg."""
    import torch

    torch.cuda.set_device(local)
    pkg = importlib.import_module(PKG)
    spec = pkg.scenes.c1_pbmpm_spheres() if args.scene == "c1" else build_scene(pkg, counts=args.counts)
    n = spec.particles.shape[0]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    buf, pipe = _pipeline(pkg, spec, args.tile_edge, stream, local)
    method = pkg.GpuSimulationMethodType.Pbmpm
    for _ in range(args.warmup):
        pipe.step(method, 1)
    status = buf.sync()
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    for _ in range(args.steps):
        pipe.step(method, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    # per-kernel CUDA-event times over a few more substeps
    lib = pkg.load()
    lib.mpm_enable_kernel_timing(buf.handle, 1)
    kt_steps = max(3, min(args.steps, 10))
    for _ in range(kt_steps):
        pipe.step(method, 1)
    K = lib.mpm_kernel_count()
    kms, kcnt = (C.c_float * K)(), (C.c_uint32 * K)()
    lib.mpm_kernel_times(buf.handle, kms, kcnt, K)
    lib.mpm_enable_kernel_timing(buf.handle, 0)
    names = pkg.kernel_names()
    kernels = {names[i]: round(kms[i] / kcnt[i], 4) for i in range(K) if kcnt[i]}
    print(json.dumps({"case": "step", "particles": n, "tiles": buf.counts()[0], "tile_edge": buf.tile_edge,
                      "ms_per_substep": ms,
                      "value": n / (ms * 1e-3), "kernels_ms": kernels, "device_status": status}), flush=True)
    buf.close()


def mlp_case(local):
    """The network alone (the profiling case of its kernels): forward passes over
    1,048,576 random rows and one training epoch over 65,536 random pairs;
    prints the forward throughput."""
    import numpy as np
    import torch

    pkg = importlib.import_module(PKG)
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    net = pkg.learned.PlasticityNet(device=local, seed=1)
    net.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(0)
    n = 1 << 20
    x = torch.from_numpy(rng.normal(0, 1, (n, 12)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.normal(0, 1, (n, 10)).astype(np.float32)).cuda()
    for _ in range(3):
        net.forward(x)
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    for _ in range(5):
        net.forward(x)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    net.train(x[:65536].contiguous(), t[:65536].contiguous(), epochs=1, batch=8192)
    torch.cuda.synchronize()
    flops = 2.0 * (12 * 64 + 64 * 64 * 2 + 64 * 11) * n
    print(json.dumps({"case": "mlp", "rows": n, "forward_ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}), flush=True)
    net.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--tile-edge", type=int, default=0,
                    help="grid tile edge 8, 12, 14 or 16; 0 lets the library choose from the occupied tiles")
    ap.add_argument("--cpu-steps", type=int, default=2,
                    help="timed substeps of the in-line CPU baseline (after one untimed substep)")
    ap.add_argument("--mlp-case", action="store_true",
                    help="run only the learned-plasticity network on random rows (profiling case of its kernels)")
    ap.add_argument("--results-table", action="store_true",
                    help="measure configs 0-2 against the f32 and f64 oracles (one JSON line per config)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the learned-plasticity and batched-scene legs (they run at N = 1 only)")
    ap.add_argument("--step-only", action="store_true",
                    help="run only warm-up + timed substeps of the slab (profiling case of the step's kernels)")
    ap.add_argument("--scene", default="c2", choices=["c2", "c1"],
                    help="--step-only: the slab (c2, default) or the two colliding spheres (c1)")
    ap.add_argument("--batched", action="store_true",
                    help="config 3 instead: 256 independent scenes sharded by scene over the ranks")
    ap.add_argument("--counts", default="256,64,256",
                    help="slab lattice size x,y,z (default: the full 4,194,304-particle workload; smaller "
                         "lattices give the small cases used for profiling)")
    args = ap.parse_args()
    args.counts = tuple(int(v) for v in args.counts.split(","))
    if args.mlp_case:
        mlp_case(dist_env()[2])
        return
    if args.results_table:
        results_table(dist_env()[2])
        return
    if args.step_only:
        step_case(args, dist_env()[2])
        return
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return
        # each step is one substep of the full workload (about 6 s on 16 host threads)
        rate, cores, sample, s_step = cpu_reference(max(1, args.steps), args.warmup, args.counts)
        line = {"metric": METRIC, "value": rate, "unit": "particle-substeps/s", "n_gpus": args.gpus,
                "steps": max(1, args.steps), "warmup": args.warmup, "ms_per_step": s_step * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fixed-point i32 grid)",
                "data": "synthetic", "impl": "reference",
                "config": bench_config(args.counts, max(1, args.steps), args.gpus),
                "cpu_baseline": {"value": rate, "unit": "particle-substeps/s", "cores": cores, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": rate, "unit": "particle-substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.batched:
        if args.tile_edge == 0:
            args.tile_edge = 8   # the edge the autotuner picks for these scenes
        out = batched_sharded(args, rank, world, local)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    out = gpu_run(args, rank, world, local)
    if world == 1 and not args.no_extra:
        import torch
        stream = torch.cuda.current_stream()
        out["surrogate"] = surrogate_leg(importlib.import_module(PKG), args, local, stream)
        out["batched"] = batched_leg(importlib.import_module(PKG), args, local, stream)
        out["full_size_vs_f64"] = f64_leg(importlib.import_module(PKG), args, local, stream)
    if rank == 0:
        rate, cores, sample, _ = cpu_reference(args.cpu_steps, 1, args.counts)
        out["cpu_baseline"] = {"value": rate, "unit": "particle-substeps/s", "cores": cores, "kind": "port",
                               "sample": sample}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
