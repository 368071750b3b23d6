"""Helpers shared by the parity tests: run a scene through libmpm (the product
path, via the C ABI) and through the oracle, and compare."""
from __future__ import annotations

import numpy as np

from conftest import import_pkg

STATE_FIELDS = ("pos", "vel", "mass", "Fe", "Fp", "dxp", "D")


def state_view(rec: np.ndarray) -> dict:
    """The computed fields of particle records (padding words excluded)."""
    return {
        "pos": rec["pos"], "vel": rec["vel"], "mass": rec["mass"],
        "Fe": rec["Fe"][:, :, :3], "Fp": rec["Fp"][:, :, :3], "dxp": rec["dxp"], "D": rec["D"][:, :, :3],
    }


def bits_equal(a: np.ndarray, b: np.ndarray) -> bool:
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def compare_states(got: np.ndarray, want: np.ndarray, rtol: float = 0.0):
    """Returns {field: max abs diff}; with rtol == 0 requires identical bits."""
    g, w = state_view(got), state_view(want)
    out = {}
    for k in STATE_FIELDS:
        a, b = np.asarray(g[k], np.float64), np.asarray(w[k], np.float64)
        out[k] = float(np.max(np.abs(a - b))) if a.size else 0.0
        if rtol == 0.0:
            assert bits_equal(np.asarray(g[k]), np.asarray(w[k])), f"{k}: max |diff| {out[k]:.3e}"
        else:
            scale = np.maximum(np.abs(b), 1.0)
            assert np.all(np.abs(a - b) <= rtol * scale), f"{k}: max |diff| {out[k]:.3e} > rtol {rtol}"
    return out


def make_params(pkg, d: dict):
    p = pkg.default_params()
    for k, v in d.items():
        if k == "gravity":
            p.gravity[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


class GpuScene:
    """One scene in one libmpm handle, through the reference-mirror classes."""

    def __init__(self, pkg, spec, tile_edge=16, max_tiles=0, use_graphs=True):
        self.pkg = pkg
        self.spec = spec
        n = spec.particles.shape[0]
        self.buf = pkg.GpuMpmBufferManager(n_particles=max(n, 1), tile_edge=tile_edge, max_tiles=max_tiles)
        self.buf.write_particles(spec.particles)
        col = None
        if spec.mesh is not None:
            v, f = spec.mesh
            col = pkg.GpuColliderBufferManager(vertices=v, indices=f)
        self.pipe = pkg.GpuMpmPipelineManager(mpm_manager=self.buf, uniforms_manager=spec.uniforms,
                                              collider_manager=col, params=make_params(pkg, spec.params))
        if not use_graphs:
            pkg.load().mpm_use_graphs(self.buf.handle, 0)

    def step(self, n=1, method=None):
        m = self.spec.method if method is None else method
        for _ in range(n):
            if m == 0:
                self.pipe.add_explicit_mpm_dispatches(n_particles=self.buf.n_particles)
            else:
                self.pipe.add_pbmpm_dispatches(n_particles=self.buf.n_particles)
        return self.buf.sync()

    def p2g_only(self, method=None):
        m = self.spec.method if method is None else method
        self.pipe.push_uniforms()
        self.pkg._lib.check(self.pkg.load().mpm_step_p2g_only(self.buf.handle, m), self.buf.handle)
        return self.buf.sync()

    def particles(self):
        return self.buf.read_particles()

    def grid(self, apply_update=False):
        return self.buf.dense_grid(self.spec.res, apply_grid_update=apply_update)

    def close(self):
        self.buf.close()


def run_oracle(oracle_mod, spec, n_steps=1, stop_after=0, fp64=False, particles=None):
    p = spec.particles.copy() if particles is None else particles
    if fp64:
        p = oracle_mod.to_fp64(p)
    o = oracle_mod.Oracle(p.shape[0], max_blocks=200000, hash_size=2000003, fp64=fp64)
    if spec.mesh is not None:
        o.set_collider(*spec.mesh)
    for _ in range(n_steps):
        o.step(spec.uniforms.bytes(), spec.params, p, spec.method, stop_after)
    return o, p
