"""B200-native (sm_100a) MPM snow simulation step.

Drop-in for the step of luoluobuli/WebGPU-MPM-based-Snow-Simulation: the
reference's 192-byte particle records and uniform block go in, the same
records come out.  Compute runs in libmpm.so (include/mpm.h); this package is
the host-side mirror of the reference's TypeScript managers plus scene
generators.
"""
from . import _lib, batching, layout, learned, scenes
from ._lib import METHOD_EXPLICIT, METHOD_PBMPM, MpmConfig, MpmError, MpmParams, default_params, load
from .layout import PARTICLE_DTYPE, GpuUniformsBufferManager, new_particles
from .pipeline import (GpuColliderBufferManager, GpuMarchingCubesBufferManager,
                       GpuMarchingCubesRenderPipelineManager, GpuMeshBufferManager, GpuMpmBatch, GpuMpmBufferManager,
                       GpuMpmPipelineManager, GpuParticleInitializePipelineManager, GpuSimulationMethodType,
                       GpuVolumetricBufferManager, GpuVolumetricRenderPipelineManager, build_bvh, build_bvh_device,
                       kernel_names)

__all__ = [
    "METHOD_EXPLICIT", "METHOD_PBMPM", "MpmConfig", "MpmError", "MpmParams", "default_params", "load",
    "PARTICLE_DTYPE", "GpuUniformsBufferManager", "new_particles", "GpuColliderBufferManager",
    "GpuMpmBufferManager", "GpuMpmBatch", "GpuMpmPipelineManager", "GpuMeshBufferManager",
    "GpuParticleInitializePipelineManager", "GpuSimulationMethodType", "GpuVolumetricBufferManager",
    "GpuVolumetricRenderPipelineManager", "GpuMarchingCubesBufferManager", "GpuMarchingCubesRenderPipelineManager",
    "build_bvh", "build_bvh_device", "kernel_names",
    "layout", "scenes", "learned", "batching",
]
