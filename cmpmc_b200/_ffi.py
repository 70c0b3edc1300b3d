"""ctypes binding of the C ABI declared in include/cmpmc_gpu.h.

The library is the in-tree ``cmpmc_b200/_lib/libcmpmc_b200.so`` (built by
``python -m cmpmc_b200.build``). Loading fails loudly when it is missing: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcmpmc_b200.so")

ABI_VERSION = 1

OK, ERR_INVALID, ERR_CUDA, ERR_UNVALIDATED, ERR_CAPACITY, ERR_DEVICE, ERR_NO_DEVICE = range(7)
FORM_PLAIN_FP64, FORM_BATCHED_FP32, FORM_BATCHED_FP32_INLINE = 0, 1, 2
WL_SINGLE_L_ORIGIN, WL_MIXED_ENERGY, WL_PAIR_DRIFT, WL_SINGLE_L_VOLUME, WL_TEST_PARALLEL = 0, 1, 2, 4, 5
WL_RECOIL, WL_RECOIL_LIGHT = 3, 6
WL_PUBLISHED_PHONON, WL_PUBLISHED_PAIR = 7, 8

MAX_VALLEYS, MAX_IV, MAX_POLY = 8, 4, 8

# numpy views of the record layouts (byte-compatible with the reference's types)
PHONON_DTYPE = np.dtype([("pos", "<f8", 3), ("k_dir", "<f8", 3), ("vg_dir", "<f8", 3), ("energy", "<f8"),
                         ("vg_mag", "<f8"), ("time", "<f8"), ("weight", "<f8"), ("bounces", "<u4"),
                         ("mode", "u1"), ("_pad", "u1", 19)])
CHARGE_DTYPE = np.dtype([("pos", "<f8", 3), ("p_eV", "<f8", 3), ("ekin", "<f8"), ("time", "<f8"),
                         ("weight", "<f8"), ("valley", "<u2"), ("type", "u1"), ("alive", "u1"),
                         ("_pad", "u1", 52)])
HIT_DTYPE = np.dtype([("pos", "<f8", 3), ("time", "<f8"), ("edep", "<f8"), ("incident_energy", "<f8"),
                      ("surface_id", "u1"), ("excitation", "u1"), ("mode", "u1"), ("_pad", "u1"),
                      ("channel_id", "<i4")])
STATS_FIELDS = [
    ("total_steps", "u8"), ("isotope_scatters", "u8"), ("polycrystal_scatters", "u8"),
    ("decays_L_to_TT", "u8"), ("decays_L_to_LT", "u8"), ("surface_refls", "u8"),
    ("surface_downconversions", "u8"), ("sensor_hits", "u8"), ("killed_tracks", "u8"),
    ("charge_steps", "u8"), ("luke_phonons_emitted", "u8"), ("intervalley_scatters", "u8"),
    ("charges_trapped", "u8"), ("trap_ionizations", "u8"), ("charge_surface_refls", "u8"),
    ("charges_collected", "u8"), ("total_luke_phonon_eV", "f8"), ("charge_recomb_edep_eV", "f8"),
    ("sc_pair_breakings", "u8"), ("qp_diffusion_steps", "u8"), ("qp_phonons_radiated", "u8"),
    ("qp_recombinations", "u8"), ("qp_local_traps", "u8"), ("total_injected_eV", "f8"),
    ("total_deposited_eV", "f8"), ("escaped_or_killed_eV", "f8"),
]
STATS_DTYPE = np.dtype([(n, "<" + t) for n, t in STATS_FIELDS])

_u8, _i32, _u32, _u64, _f64 = C.c_uint8, C.c_int32, C.c_uint32, C.c_uint64, C.c_double


class SimStatsC(C.Structure):
    _fields_ = [(n, _u64 if t == "u8" else _f64) for n, t in STATS_FIELDS]


class CrystalConfigC(C.Structure):
    _fields_ = [
        ("group", _i32), ("has_custom_C", _i32), ("density", _f64),
        ("C11", _f64), ("C12", _f64), ("C13", _f64), ("C14", _f64), ("C16", _f64), ("C33", _f64),
        ("C44", _f64), ("C66", _f64), ("C_custom", (_f64 * 6) * 6),
        ("beta", _f64), ("gamma", _f64), ("lambda_", _f64), ("mu", _f64),
        ("B_iso", _f64), ("A_anh", _f64), ("fTT_frac", _f64), ("polycrystal_mfp_m", _f64),
        ("fLDOS", _f64), ("fSTDOS", _f64), ("fFTDOS", _f64),
        ("debye_freq", _f64), ("v_sound", _f64), ("v_trans", _f64),
        ("bandgap", _f64), ("pair_energy", _f64), ("fano_factor", _f64), ("epsilon_rel", _f64),
        ("neutral_impurity_cm3", _f64), ("alpha_nonparabolic", _f64), ("h_mass_ratio", _f64),
        ("e_mass_tensor", _f64 * 3), ("n_valleys", _i32), ("iv_model", _i32),
        ("valley_dirs", (_f64 * 3) * MAX_VALLEYS), ("ac_deform_e", _f64), ("ac_deform_h", _f64),
        ("n_iv", _i32), ("_pad0", _i32), ("iv_deform_eV_m", _f64 * MAX_IV), ("iv_energy_eV", _f64 * MAX_IV),
        ("iv_min_energy", _f64), ("iv_quad_rate", _f64), ("iv_quad_field", _f64), ("iv_quad_power", _f64),
        ("iv_lin_rate0", _f64), ("iv_lin_rate1", _f64), ("iv_lin_power", _f64),
        ("e_trapping_mfp_m", _f64), ("h_trapping_mfp_m", _f64), ("e_trap_ion_d0_mfp_m", _f64),
        ("e_trap_ion_a_mfp_m", _f64), ("h_trap_ion_d_mfp_m", _f64), ("h_trap_ion_a0_mfp_m", _f64),
        ("orient", (_f64 * 3) * 3), ("atomic_Z", _f64), ("atomic_A", _f64),
    ]


class ElectrodePadC(C.Structure):
    _fields_ = [("shape", _i32), ("channel_id", _i32), ("cx", _f64), ("cy", _f64), ("r_min", _f64), ("r_max", _f64),
                ("phi_min", _f64), ("phi_max", _f64), ("fill_fraction", _f64)]


class FilmConfigC(C.Structure):
    _fields_ = [
        ("film_absorption", _f64), ("film_thickness", _f64), ("v_sound", _f64), ("gap_energy", _f64),
        ("phonon_lifetime", _f64), ("phonon_lifetime_slope", _f64), ("low_qp_limit", _f64),
        ("high_qp_limit", _f64), ("subgap_absorption", _f64), ("absorber_gap", _f64), ("absorber_eff", _f64),
        ("absorber_eff_slope", _f64), ("temperature", _f64), ("keep_all_phonons", _i32), ("loss_model", _i32),
        ("phonon_loss_time", _f64),
    ]


class SurfaceC(C.Structure):
    _fields_ = [
        ("prob_abs", _f64), ("prob_refl", _f64), ("refl_cutoff", _f64), ("anh_cutoff", _f64),
        ("prob_charge_abs", _f64), ("prob_charge_spec", _f64), ("min_k_elec", _f64), ("min_k_hole", _f64),
        ("spec_prob_const", _f64), ("n_spec", _i32), ("n_diff", _i32), ("n_anh", _i32), ("demo_values", _i32),
        ("spec_coeffs", _f64 * MAX_POLY), ("diff_coeffs", _f64 * MAX_POLY), ("anh_coeffs", _f64 * MAX_POLY),
        ("has_film", _i32), ("has_amm", _i32), ("has_mask", _i32), ("_pad0", _i32), ("film", FilmConfigC),
        ("amm_substrate", _f64 * 3), ("amm_film", _f64 * 3),
    ]


class DetectorC(C.Structure):
    _fields_ = [
        ("radius", _f64), ("half_z", _f64), ("e_field", _f64 * 3), ("surfaces", SurfaceC * 3),
        ("max_bounces", _u32), ("russian_roulette_bounces", _u32), ("russian_roulette_survival", _f64),
        ("min_phonon_eV", _f64), ("luke_sample_fraction", _f64), ("charge_max_dk_frac", _f64),
        ("charge_dt_cap_s", _f64), ("charge_sampling_dk_frac", _f64), ("charge_stepping", _i32),
        ("charge_release", _i32), ("fermi_level_above_Ev_eV", _f64), ("electrode_seed_max_gap", _f64),
        ("allow_unvalidated", _i32), ("jump_to_ballistic", _i32), ("kinematics_mode", _i32), ("_pad0", _i32),
    ]


class RunDescC(C.Structure):
    _fields_ = [
        ("n_events", _u64), ("first_event", _u64), ("rng_state", C.c_void_p), ("injected_eV", C.c_void_p),
        ("phonon_offsets", C.c_void_p), ("phonons", C.c_void_p), ("charge_offsets", C.c_void_p),
        ("charges", C.c_void_p), ("keep_hits", _i32), ("form", _i32), ("inputs_on_device", _i32),
        ("outputs_on_device", _i32), ("seed", _u64), ("want_event_stats", _i32), ("kaplan_surrogate", _i32),
    ]


class RunOutC(C.Structure):
    _fields_ = [
        ("stats", SimStatsC), ("n_hits", _u64), ("hits", C.c_void_p), ("hit_offsets", C.c_void_p),
        ("event_stats", C.c_void_p), ("kernel_ms", _f64), ("total_ms", _f64), ("device_error", _u32),
        ("kernel_launches", _u32),
    ]


ADJ_MAX_BINS = 256


class AdjointDescC(C.Structure):
    _fields_ = [
        ("n_events", _u64), ("first_event", _u64), ("seed", _u64), ("phonon_offsets", C.c_void_p),
        ("phonons", C.c_void_p), ("inputs_on_device", _i32), ("n_bins", _i32), ("t_min", _f64), ("t_max", _f64),
        ("theta", _f64 * 4), ("bin_weight", C.c_void_p), ("per_primary", C.c_void_p),
        ("per_primary_on_device", _i32), ("_pad0", _i32),
    ]


class AdjointOutC(C.Structure):
    _fields_ = [
        ("hist", _f64 * ADJ_MAX_BINS), ("value", _f64), ("grad", _f64 * 4), ("value_var", _f64),
        ("grad_var", _f64 * 4), ("stats", SimStatsC), ("n_primaries", _u64), ("kernel_ms", _f64),
        ("total_ms", _f64), ("device_error", _u32), ("kernel_launches", _u32),
    ]


# double (*)(const double p[3], void* user): node potential of cmpmc_mesh_build_cartesian
POTENTIAL_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p)

# double (*)(double u, double v, void* user): node potential of cmpmc_mesh2d_build_grid
POTENTIAL2D_FN = C.CFUNCTYPE(C.c_double, C.c_double, C.c_double, C.c_void_p)

TUNE_MAX = 16


class TuneResultC(C.Structure):
    _fields_ = [
        ("threads_per_block", _i32), ("blocks_per_sm", _i32), ("queue_capacity", _u64), ("phase_steps", _u32),
        ("_pad1", _u32), ("best_ms", _f64),
        ("first_ms", _f64), ("n_tried", _i32), ("_pad0", _i32), ("tried_tpb", _i32 * TUNE_MAX),
        ("tried_bps", _i32 * TUNE_MAX), ("tried_queue", _u64 * TUNE_MAX), ("tried_ms", _f64 * TUNE_MAX),
    ]


DEPOSIT_DTYPE = np.dtype([("pos", "<f8", 3), ("time_s", "<f8"), ("edep_eV", "<f8"), ("is_nuclear_recoil", "<i4"),
                          ("_pad", "<i4")])


class PartitionOptionsC(C.Structure):
    _fields_ = [("niel_model", _i32), ("use_fano_fluctuations", _i32), ("use_charge_cloud", _i32),
                ("max_sampled_pairs", _u32), ("max_sampled_phonons", _u32), ("emp_energy_dependent_k", _i32),
                ("emp_k_fixed", _f64), ("emp_k_low", _f64), ("emp_k_high", _f64), ("emp_e_low_eV", _f64),
                ("emp_e_high_eV", _f64)]


class PartitionResultC(C.Structure):
    _fields_ = [("total_edep_eV", _f64), ("ionizing_eV", _f64), ("niel_eV", _f64), ("lindhard_yield", _f64),
                ("n_pairs_true", _u64), ("n_pairs_sampled", _u64), ("n_phonons_true", _u64),
                ("n_phonons_sampled", _u64), ("charge_weight", _f64), ("phonon_weight", _f64),
                ("prompt_phonon_eV", _f64)]


class PrimaryStepC(C.Structure):
    _fields_ = [("track_id", _i32), ("is_charged", _i32), ("start_pos", _f64 * 3), ("end_pos", _f64 * 3),
                ("time_s", _f64), ("edep_eV", _f64), ("eniel_eV", _f64), ("hit_boundary", _i32),
                ("track_stopped", _i32)]


_U64x4 = _u64 * 4

_SIG = {
    "cmpmc_abi_sizes": (_i32, [C.POINTER(C.c_size_t), _i32]),
    "cmpmc_crystal_config_germanium": (None, [C.POINTER(CrystalConfigC)]),
    "cmpmc_detector_default": (None, [C.POINTER(DetectorC)]),
    "cmpmc_film_aluminum": (None, [C.POINTER(FilmConfigC)]),
    "cmpmc_lattice_create": (_i32, [C.POINTER(CrystalConfigC), C.POINTER(C.c_void_p)]),
    "cmpmc_lattice_destroy": (None, [C.c_void_p]),
    "cmpmc_lattice_tables": (_i32, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "cmpmc_lattice_set_kinematics_mode": (_i32, [C.c_void_p, _i32]),
    "cmpmc_lattice_kinematics_mode": (_i32, [C.c_void_p]),
    "cmpmc_lattice_map_k_to_vg": (_i32, [C.c_void_p, _i32, C.POINTER(_f64), C.POINTER(_f64), C.POINTER(_f64)]),
    "cmpmc_make_track": (_i32, [C.c_void_p, C.POINTER(_f64), C.POINTER(_f64), _i32, _f64, _f64, _f64, C.c_void_p]),
    "cmpmc_make_charge": (_i32, [C.c_void_p, _i32, C.POINTER(_f64), C.POINTER(_f64), _f64, _i32, _f64,
                                 C.c_void_p]),
    "cmpmc_rng_for_stream": (None, [_u64, _u64, C.POINTER(_u64)]),
    "cmpmc_rng_next_u64": (_u64, [C.POINTER(_u64)]),
    "cmpmc_rng_uniform": (_f64, [C.POINTER(_u64)]),
    "cmpmc_generate": (_i32, [C.c_void_p, C.POINTER(DetectorC), _i32, _u64, _u64, _u64, _i32, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, _u64, C.POINTER(_u64), C.c_void_p, C.c_void_p,
                              _u64, C.POINTER(_u64)]),
    "cmpmc_gpu_create": (_i32, [C.c_void_p, C.POINTER(DetectorC), _i32, C.POINTER(C.c_void_p)]),
    "cmpmc_gpu_destroy": (None, [C.c_void_p]),
    "cmpmc_gpu_run_events": (_i32, [C.c_void_p, C.POINTER(RunDescC), C.POINTER(RunOutC)]),
    "cmpmc_gpu_adjoint": (_i32, [C.c_void_p, C.POINTER(AdjointDescC), C.POINTER(AdjointOutC)]),
    "cmpmc_gpu_last_error": (_i32, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "cmpmc_gpu_configure": (_i32, [C.c_void_p, _i32, _i32, _u64, _u64]),
    "cmpmc_gpu_device_count": (_i32, [C.POINTER(_i32)]),
    "cmpmc_cr_log": (_f64, [_f64]),
    "cmpmc_cr_sin": (_f64, [_f64]),
    "cmpmc_cr_cos": (_f64, [_f64]),
    "cmpmc_gpu_math_check": (_i32, [_i32, _u64, C.c_void_p, C.c_void_p]),
    "cmpmc_mesh_create": (_i32, [C.c_void_p, C.c_void_p, _u64, C.c_void_p, _u64, _f64, _f64,
                                 C.POINTER(C.c_void_p)]),
    "cmpmc_mesh_build_cartesian": (_i32, [_f64, _f64, _f64, _i32, _i32, _i32, C.c_void_p, C.c_void_p,
                                          C.POINTER(C.c_void_p)]),
    "cmpmc_mesh_load_files": (_i32, [C.c_char_p, C.c_char_p, _f64, _f64, C.POINTER(C.c_void_p)]),
    "cmpmc_recoil_potential": (_f64, [C.POINTER(_f64), C.c_void_p]),
    "cmpmc_recoil_mesh": (_i32, [C.POINTER(DetectorC), C.POINTER(C.c_void_p)]),
    "cmpmc_mesh_destroy": (None, [C.c_void_p]),
    "cmpmc_mesh_info": (_i32, [C.c_void_p, C.POINTER(_u64), C.POINTER(_u64)]),
    "cmpmc_mesh_field_at": (_i32, [C.c_void_p, C.POINTER(_f64), C.POINTER(_i32), C.POINTER(_f64)]),
    "cmpmc_mesh_potential_at": (_i32, [C.c_void_p, C.POINTER(_f64), C.POINTER(_i32), C.POINTER(_f64)]),
    "cmpmc_gpu_set_mesh": (_i32, [C.c_void_p, C.c_void_p]),
    "cmpmc_partition_options_default": (None, [C.POINTER(PartitionOptionsC)]),
    "cmpmc_ionization_yield": (_f64, [C.POINTER(CrystalConfigC), _i32, _f64, C.POINTER(PartitionOptionsC)]),
    "cmpmc_lindhard_yield": (_f64, [C.POINTER(CrystalConfigC), _f64, _f64, _f64]),
    "cmpmc_sample_fano_binomial": (_u64, [_f64, _f64, _U64x4]),
    "cmpmc_partition_deposit": (_i32, [C.c_void_p, C.POINTER(_f64), _f64, _f64, _i32, C.POINTER(PartitionOptionsC),
                                       _U64x4, C.c_void_p, _u64, C.POINTER(_u64), C.c_void_p, _u64,
                                       C.POINTER(_u64), C.POINTER(PartitionResultC)]),
    "cmpmc_gpu_partition_deposits": (_i32, [C.c_void_p, C.c_void_p, _u64, C.POINTER(PartitionOptionsC), C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, _u64, C.c_void_p, _u64, C.POINTER(_u64),
                                            C.POINTER(_u64)]),
    "cmpmc_hit_merger_create": (_i32, [C.c_void_p, _f64, C.POINTER(PartitionOptionsC), C.POINTER(C.c_void_p)]),
    "cmpmc_hit_merger_destroy": (None, [C.c_void_p]),
    "cmpmc_hit_merger_process_steps": (_i32, [C.c_void_p, C.POINTER(PrimaryStepC), _u64, _U64x4, C.POINTER(_u64)]),
    "cmpmc_hit_merger_flush": (_i32, [C.c_void_p, _U64x4, C.POINTER(PartitionResultC)]),
    "cmpmc_hit_merger_take": (_i32, [C.c_void_p, C.c_void_p, _u64, C.POINTER(_u64), C.c_void_p, _u64,
                                     C.POINTER(_u64)]),
    "cmpmc_mesh2d_create": (_i32, [C.c_void_p, C.c_void_p, _u64, C.c_void_p, _u64, _i32, C.POINTER(C.c_void_p)]),
    "cmpmc_mesh2d_build_grid": (_i32, [_f64, _f64, _f64, _f64, _i32, _i32, C.c_void_p, C.c_void_p, _i32,
                                       C.POINTER(C.c_void_p)]),
    "cmpmc_mesh2d_destroy": (None, [C.c_void_p]),
    "cmpmc_mesh2d_info": (_i32, [C.c_void_p, C.POINTER(_u64), C.POINTER(_u64)]),
    "cmpmc_mesh2d_field_at": (_i32, [C.c_void_p, C.POINTER(_f64), C.POINTER(_i32), C.POINTER(_f64)]),
    "cmpmc_mesh2d_potential_at": (_i32, [C.c_void_p, C.POINTER(_f64), C.POINTER(_i32), C.POINTER(_f64)]),
    "cmpmc_gpu_set_mesh2d": (_i32, [C.c_void_p, C.c_void_p]),
    "cmpmc_gpu_configure_queue": (_i32, [C.c_void_p, _u64]),
    "cmpmc_gpu_configure_graph": (_i32, [C.c_void_p, _i32]),
    "cmpmc_gpu_configure_phases": (_i32, [C.c_void_p, _u32]),
    "cmpmc_gpu_configure_pool": (_i32, [C.c_void_p, _i32, _u32]),
    "cmpmc_gpu_configure_staging": (_i32, [C.c_void_p, _i32]),
    "cmpmc_gpu_memcpy": (_i32, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "cmpmc_gpu_autotune": (_i32, [C.c_void_p, C.POINTER(RunDescC), _i32, C.POINTER(TuneResultC)]),
    "cmpmc_kaplan_surrogate_create": (_i32, [C.POINTER(FilmConfigC), _u64, C.POINTER(C.c_void_p)]),
    "cmpmc_kaplan_surrogate_destroy": (None, [C.c_void_p]),
    "cmpmc_kaplan_surrogate_info": (_i32, [C.c_void_p, C.POINTER(_u64), C.POINTER(_u64)]),
    "cmpmc_kaplan_surrogate_absorb": (_i32, [C.c_void_p, _f64, C.POINTER(_u64), C.c_void_p, _u64, C.POINTER(_u64),
                                             C.POINTER(_f64)]),
    "cmpmc_amm_transmission": (_f64, [C.POINTER(_f64), C.POINTER(_f64), _i32, _f64]),
    "cmpmc_gpu_set_electrode_mask": (_i32, [C.c_void_p, _i32, C.c_void_p, _u64]),
    "cmpmc_mask_supercdms_qet": (_i32, [_f64, _f64, C.c_void_p]),
    "cmpmc_mask_rectangular_grid": (_i32, [_i32, _i32, _f64, _f64, _f64, _f64, _f64, C.c_void_p, _u64,
                                           C.POINTER(_u64)]),
    "cmpmc_mask_find_channel": (_i32, [C.c_void_p, _u64, C.POINTER(_f64), C.POINTER(_u64), C.POINTER(_i32)]),
    "cmpmc_gpu_run_events_noalloc": (_i32, [C.c_void_p, C.POINTER(DetectorC), _i32, _u64, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _u64,
                                            C.c_void_p, C.POINTER(SimStatsC), C.POINTER(_u64)]),
}

EXPORTED = sorted(_SIG)

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree library once and checks the ABI layout against this binding."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cmpmc_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIG.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    sizes = (C.c_size_t * 12)()
    ver = lib.cmpmc_abi_sizes(sizes, 12)
    want = [128, 128, 56, 208, C.sizeof(CrystalConfigC), C.sizeof(FilmConfigC), C.sizeof(SurfaceC),
            C.sizeof(DetectorC), C.sizeof(RunDescC), C.sizeof(RunOutC), C.sizeof(AdjointDescC),
            C.sizeof(AdjointOutC)]
    if ver != ABI_VERSION or list(sizes) != want:
        raise ImportError(f"ABI mismatch: library v{ver} sizes {list(sizes)} vs binding {want}")
    assert PHONON_DTYPE.itemsize == 128 and CHARGE_DTYPE.itemsize == 128 and HIT_DTYPE.itemsize == 56
    assert STATS_DTYPE.itemsize == 208
    _lib = lib
    return lib


def ptr(a) -> int | None:
    """Address of a numpy array's data (None for None)."""
    if a is None:
        return None
    return a.ctypes.data
