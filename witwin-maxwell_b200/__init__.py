"""B200-native FDTD time-stepping hot path with the witwin-maxwell solver interface.

Modules:
    scene       scene description and compilation into solver-scene tensors
    solver      B200FDTD: the fused sm_100a step engine behind the FDTD solve contract;
                B200Batch: independent scenes stepped together (graph-captured blocks)
    backend     NativeFDTDModule-compatible per-op surface (camelCase kernel names)
    simulation  Simulation.fdtd(...).run() -> Result facade
    adjoint     reverse-time adjoint: dL/deps_r of a design region (torch.autograd.Function)
    _lib        ctypes binding of libfdtd_b200.so (C ABI in include/fdtd_b200.h)
"""
from . import scene, workloads
from .scene import (
    BOUNDARY_BLOCH,
    BOUNDARY_NONE,
    BOUNDARY_PEC,
    BOUNDARY_PERIODIC,
    BOUNDARY_PMC,
    BOUNDARY_PML,
    CW,
    Box,
    CustomSourceTime,
    GaussianBeam,
    GaussianPulse,
    MaterialRegion,
    Medium,
    PlaneMonitor,
    PlaneSource,
    PlaneWaveTFSF,
    PointDipole,
    PointMonitor,
    VolumeMonitor,
    Scene,
    Sphere,
    Structure,
    closed_box_monitor,
    compile_scene,
    flux_monitor,
)

__version__ = "0.1.0"


def __getattr__(name):
    # Lazily import the CUDA-backed modules so that scene compilation and the
    # library's symbol table can be used on machines without a GPU.
    if name in ("solver", "backend", "simulation", "adjoint", "distributed", "postprocess", "_lib"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    if name == "B200FDTD":
        from .solver import B200FDTD

        return B200FDTD
    if name == "B200Batch":
        from .solver import B200Batch

        return B200Batch
    if name in ("Simulation", "TimeConfig", "SpectralSampler"):
        from . import simulation

        return getattr(simulation, name)
    raise AttributeError(name)
