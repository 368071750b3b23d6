"""Generates the golden fixtures of the MPM step parity tests.

The reference (WGSL on WebGPU) ships no golden vectors and cannot run
without a graphics stack, so these fixtures are produced by the CPU oracle
(oracle/mpm_oracle.c, a restatement of the reference shaders).  They pin the
oracle against regressions and give the GPU tests a fixed expected output
independent of the live oracle.  Each fixture stores the input particle
records, the uniform block, the extension parameters, the collider mesh and
the oracle's output after n substeps (particle records and the dense grid).

    python tests/golden/make_golden.py
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = [
    # name, scene kwargs, substeps
    ("explicit_plain", dict(kind="explicit", n_side=6, res=16, seed=21), 3),
    ("explicit_collider", dict(kind="explicit", n_side=6, res=16, seed=22, with_collider=True), 3),
    ("pbmpm_plain", dict(kind="pbmpm", n_side=6, res=16, seed=23), 2),
    ("pbmpm_collider_interaction", dict(kind="pbmpm", n_side=6, res=16, seed=24, with_collider=True,
                                        interaction=True), 2),
]


def run_case(pkg, oracle, kw, steps):
    spec = pkg.scenes.parity_scene(**kw)
    p_in = spec.particles.copy()
    o = oracle.Oracle(p_in.shape[0], max_blocks=20000, hash_size=200003)
    if spec.mesh is not None:
        o.set_collider(*spec.mesh)
    p = p_in.copy()
    for _ in range(steps):
        o.step(spec.uniforms.bytes(), spec.params, p, spec.method)
    grid = o.dense_grid(spec.uniforms.bytes())
    return spec, p_in, p, grid


def main():
    pkg = importlib.import_module("webgpu-mpm-based-snow-simulation_b200")
    import oracle

    oracle.build()
    for name, kw, steps in CASES:
        spec, p_in, p_out, grid = run_case(pkg, oracle, kw, steps)
        mesh_v = spec.mesh[0] if spec.mesh is not None else np.zeros((0, 3), np.float32)
        mesh_f = spec.mesh[1] if spec.mesh is not None else np.zeros(0, np.uint32)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            particles_in=p_in.view(np.uint8), particles_out=p_out.view(np.uint8),
            uniforms=np.frombuffer(spec.uniforms.bytes(), np.uint8), grid=grid,
            mesh_vertices=mesh_v, mesh_indices=mesh_f,
            params=np.frombuffer(json.dumps(spec.params).encode(), np.uint8),
            meta=np.frombuffer(json.dumps({"method": spec.method, "steps": steps, "res": list(spec.res)}).encode(),
                               np.uint8))
        print(name, p_in.shape[0], "particles,", steps, "substeps, nonzero cells", int((grid[..., 0] != 0).sum()))


if __name__ == "__main__":
    main()
