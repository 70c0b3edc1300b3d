"""Shared helpers of the test suite: fixture paths and the canonical workloads."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def detector_for(workload: str):
    """The canonical detector of each fixture workload (mirrors oracle/ref_driver.cpp)."""
    import cmpmc_b200 as cm
    det = cm.DetectorModel()
    if workload == "c2":
        det.e_field = cm.UniformElectricField.from_bias(4.0, 2.54 * cm.units.cm)
        det.luke_sample_fraction = 0.0
    elif workload == "c3s":
        det.mesh_field_3d = recoil_mesh()
        det.luke_sample_fraction = 0.05
    elif workload in ("tp", "tpl", "tpm", "tpd", "tpe", "tp2"):
        det.e_field = cm.UniformElectricField.from_bias(2.0, 2.54 * cm.units.cm)
        if workload == "tp2":
            det.mesh_field_2d = axisym_mesh(det)
        det.luke_sample_fraction = 1.0 if workload == "tpl" else 0.02
        det.charge_release = {"tpd": 1, "tpe": 2}.get(workload, 0)
    elif workload in ("pub", "pubc"):
        det = cm.DetectorModel.published_benchmark(0.0 if workload == "pub" else 4.0,
                                                   1.0 if workload == "pub" else 0.0)
    if workload in ("tps", "tpt"):
        det.e_field = cm.UniformElectricField.from_bias(2.0, 2.54 * cm.units.cm)
        det.luke_sample_fraction = 0.02
        det.charge_stepping = 1 if workload == "tps" else 0
    if workload == "c0r":
        det.russian_roulette_bounces = 64
    if workload == "c0a":
        amm = cm.IsotropicAMMInterface(cm.IsotropicMedium(5323.0, 5324.2077, 3258.7879),
                                       cm.IsotropicMedium(2700.0, 6420.0, 3040.0))
        for f in (0, 1):
            det.surfaces[f].amm_interface = amm
    if workload in ("c0m", "tpm"):
        for f in (0, 1):
            det.surfaces[f].electrode_mask = cm.ElectrodePatternMask.supercdms_qet_mask(det.solid.radius, 0.8)
    return det


def lattice_for(workload: str, default_lattice):
    """The lattice of a fixture workload: the shared Ge lattice, or a Ge lattice in the
    Exact (c0x) or Bilinear (c0b) kinematics mode."""
    import dataclasses
    import cmpmc_b200 as cm
    if workload == "tpt":  # every trapping and trap-ionisation channel on (oracle/ref_driver.cpp)
        return cm.CrystalLattice(dataclasses.replace(
            cm.materials.Germanium(), e_trapping_mfp_m=0.02, h_trapping_mfp_m=0.03, e_trap_ion_d0_mfp_m=0.04,
            e_trap_ion_a_mfp_m=0.05, h_trap_ion_d_mfp_m=0.045, h_trap_ion_a0_mfp_m=0.06))
    if workload not in ("c0x", "c0b"):
        return default_lattice
    lat = cm.CrystalLattice(cm.materials.Germanium())
    lat.set_kinematics_mode(cm.CrystalLattice.Exact if workload == "c0x" else cm.CrystalLattice.Bilinear)
    return lat


_MESH = []


def axisym_mesh(det):
    """The tp2 field: BiLinearMesh2D.build_grid(0, R, -h, h, 40, 40) in (r, z) of
    V = 2 (z + h) / 2h + 0.3 (r / R)^2 (z / h)."""
    import cmpmc_b200 as cm
    R, h = det.solid.radius, det.solid.half_z
    return cm.BiLinearMesh2D.build_grid(0.0, R, -h, h, 40, 40,
                                        lambda r, z: 2.0 * (z + h) / (2.0 * h) + 0.3 * (r / R) * (r / R) * (z / h),
                                        True)


def planar_mesh(det):
    """A planar (x, y) BiLinearMesh2D.build_grid(-R, R, -R, R, 32, 32) of
    V = 3 (x + R) / 2R + 0.5 (y / R)^2."""
    import cmpmc_b200 as cm
    R = det.solid.radius
    return cm.BiLinearMesh2D.build_grid(-R, R, -R, R, 32, 32,
                                        lambda x, y: 3.0 * (x + R) / (2.0 * R) + 0.5 * (y / R) * (y / R), False)


def recoil_mesh():
    """The recoil workloads' field mesh (built once per test process)."""
    import cmpmc_b200 as cm
    if not _MESH:
        _MESH.append(cm.TriLinearMesh3D.recoil_mesh(cm.DetectorModel()))
    return _MESH[0]


WORKLOAD_SEED = {"c0": 42, "c1": 7, "c2": 11, "c4": 17, "tp": 77, "tpl": 77, "c3s": 13, "c0m": 42, "tpm": 77, "c0a": 42,
                 "tpd": 77, "tpe": 77, "c0x": 42, "c0b": 42, "tp2": 77, "c0r": 42, "tps": 77, "tpt": 77,
                 "pub": 12345, "pubc": 12345}


def workload_of(name: str):
    import cmpmc_b200 as cm
    return {"c0": cm.workloads.single_l_origin, "c1": cm.workloads.mixed_energy, "c2": cm.workloads.pair_drift,
            "c4": cm.workloads.single_l_volume, "tp": cm.workloads.test_parallel,
            "tpl": cm.workloads.test_parallel, "c3s": cm.workloads.recoil_light,
            "c0m": cm.workloads.single_l_origin, "tpm": cm.workloads.test_parallel,
            "c0a": cm.workloads.single_l_origin, "tpd": cm.workloads.test_parallel,
            "tpe": cm.workloads.test_parallel, "c0x": cm.workloads.single_l_origin,
            "c0b": cm.workloads.single_l_origin, "tp2": cm.workloads.test_parallel,
            "c0r": cm.workloads.single_l_origin, "tps": cm.workloads.test_parallel,
            "tpt": cm.workloads.test_parallel, "pub": cm.workloads.published_phonon,
            "pubc": cm.workloads.published_pair}[name]


def has_gpu() -> bool:
    try:
        from cmpmc_b200 import _ffi
        import ctypes
        n = ctypes.c_int32(0)
        return _ffi.load().cmpmc_gpu_device_count(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False
