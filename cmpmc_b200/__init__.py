"""cmpmc_b200 -- CMPMC's phonon / charge transport path on NVIDIA B200 (sm_100a).

The public API mirrors the reference's C++ API (run_events, SimulationEngine,
CrystalLattice, DetectorModel, ...); the work runs in hand-written CUDA kernels behind
the C ABI in include/cmpmc_gpu.h.
"""
from .api import (AluminumFilm, CmpmcError, ElectrodePad, ElectrodePatternMask, CrystalConfig, CrystalLattice, CylinderSolid, DetectorModel,
                  EventInput, ExcitationType, IsotropicAMMInterface, IsotropicMedium, KaplanFilm,
                  KaplanSurrogateLUT, PackedEvents, PhononMode, Rng, RunOptions, RunResult,
                  SimStats, SimulationEngine, SuperconductorFilmConfig, SurfaceId, SurfaceProperty,
                  TriLinearMesh3D, BiLinearMesh2D, UniformElectricField, UnvalidatedModuleError, Workload, materials, run_events, units, workloads)
from .partition import (EmpiricalNIELParams, EnergyPartition, HitMerger, NIELModel, PartitionOptions, PartitionResult,
                        PrimaryStepInput, partition_deposits_on_device, physics)
from .adjoint import AdjointResult, HistogramAdjoint, THETA_NAMES, default_theta

__all__ = [
    "AdjointResult", "AluminumFilm", "CmpmcError", "ElectrodePad", "ElectrodePatternMask", "CrystalConfig", "CrystalLattice", "CylinderSolid", "DetectorModel", "EventInput",
    "ExcitationType", "IsotropicAMMInterface", "IsotropicMedium", "KaplanFilm",
    "KaplanSurrogateLUT", "PackedEvents", "PhononMode", "Rng", "RunOptions", "RunResult", "SimStats",
    "SimulationEngine", "SuperconductorFilmConfig", "SurfaceId", "SurfaceProperty", "TriLinearMesh3D", "BiLinearMesh2D",
    "UniformElectricField",
    "UnvalidatedModuleError", "Workload", "materials", "run_events", "units", "workloads", "HistogramAdjoint",
    "THETA_NAMES", "default_theta", "EmpiricalNIELParams", "EnergyPartition", "HitMerger", "NIELModel",
    "PartitionOptions", "PartitionResult", "PrimaryStepInput", "partition_deposits_on_device", "physics",
]
