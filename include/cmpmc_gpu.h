/*
 * cmpmc_gpu.h -- C ABI of the B200 (sm_100a) transport path for CMPMC.
 *
 * This is the drop-in boundary behind CMPMC's run_events / SimulationEngine API.
 * Every entry point takes plain pointers and sizes; no C++ or torch type crosses it.
 * Status codes are int (0 = OK, see CMPMC_* below); no exception crosses the ABI.
 *
 * Reference interfaces replaced (paths within the CMPMC project):
 *   run_events(engine, n, generate, options)   include/cmpmc/transport/parallel.hpp:76-148
 *   SimulationEngine::transport                include/cmpmc/transport/engine.hpp:403-582
 *   SimulationEngine::transport_charges        include/cmpmc/transport/engine.hpp:192-380
 *   SimulationEngine::make_track               include/cmpmc/transport/engine.hpp:171-187
 *   CrystalLattice(cfg) (host table build)     include/cmpmc/lattice/crystal_lattice.hpp:45-55
 *   Rng::for_stream                            include/cmpmc/core/rng.hpp:34-36
 *
 * Records (cmpmc_phonon_track, cmpmc_charge_track, cmpmc_sensor_hit, cmpmc_sim_stats)
 * are byte-compatible with the reference's PhononTrack, ChargeTrack, SensorHit and
 * SimStats (include/cmpmc/core/track.hpp:62-108, transport/engine.hpp:29-93), so a
 * caller can pass std::vector<PhononTrack>::data() directly.
 *
 * Threading: a context is bound to one device and one stream; calls on one context
 * must be serialized by the caller. Different contexts may run concurrently.
 */
#ifndef CMPMC_GPU_H
#define CMPMC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMPMC_GPU_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------------- */
#define CMPMC_OK                 0
#define CMPMC_ERR_INVALID        1  /* bad argument / unsupported configuration        */
#define CMPMC_ERR_CUDA           2  /* a CUDA runtime call failed                       */
#define CMPMC_ERR_UNVALIDATED    3  /* guarded module used without allow_unvalidated
                                       (reference: UnvalidatedModuleError,
                                       core/validation.hpp:20-29)                      */
#define CMPMC_ERR_CAPACITY       4  /* a device buffer (stack, hits) overflowed         */
#define CMPMC_ERR_DEVICE         5  /* a kernel reported an error status word           */
#define CMPMC_ERR_NO_DEVICE      6  /* no CUDA device / extension cannot run            */

/* ---- records (byte layout of the reference types) ------------------------------ */
enum { CMPMC_MODE_L = 0, CMPMC_MODE_FT = 1, CMPMC_MODE_ST = 2 };
enum { CMPMC_SURF_TOP = 0, CMPMC_SURF_BOTTOM = 1, CMPMC_SURF_SIDE = 2 };
enum { CMPMC_EXC_PHONON = 0, CMPMC_EXC_ELECTRON = 1, CMPMC_EXC_HOLE = 2 };

/* PhononTrack (track.hpp:62-72): 128 B, 64-byte aligned */
typedef struct cmpmc_phonon_track {
    double pos[3];
    double k_dir[3];
    double vg_dir[3];
    double energy;
    double vg_mag;
    double time;
    double weight;
    uint32_t bounces;
    uint8_t mode;
    uint8_t _pad[19];
} cmpmc_phonon_track;

/* ChargeTrack (track.hpp:75-84): 128 B, 64-byte aligned */
typedef struct cmpmc_charge_track {
    double pos[3];
    double p_eV[3];
    double ekin;
    double time;
    double weight;
    uint16_t valley;
    uint8_t type;
    uint8_t alive;
    uint8_t _pad[52];
} cmpmc_charge_track;

/* SensorHit (track.hpp:99-108): 56 B */
typedef struct cmpmc_sensor_hit {
    double pos[3];
    double time;
    double edep;
    double incident_energy;
    uint8_t surface_id;
    uint8_t excitation;
    uint8_t mode;
    uint8_t _pad;
    int32_t channel_id;
} cmpmc_sensor_hit;

/* SimStats (engine.hpp:29-93): 208 B, same field order */
typedef struct cmpmc_sim_stats {
    uint64_t total_steps, isotope_scatters, polycrystal_scatters, decays_L_to_TT, decays_L_to_LT,
             surface_refls, surface_downconversions, sensor_hits, killed_tracks;
    uint64_t charge_steps, luke_phonons_emitted, intervalley_scatters, charges_trapped,
             trap_ionizations, charge_surface_refls, charges_collected;
    double total_luke_phonon_eV, charge_recomb_edep_eV;
    uint64_t sc_pair_breakings, qp_diffusion_steps, qp_phonons_radiated, qp_recombinations,
             qp_local_traps;
    double total_injected_eV, total_deposited_eV, escaped_or_killed_eV;
} cmpmc_sim_stats;

/* ---- configuration (plain data mirrors of the reference structs) ---------------- */
#define CMPMC_MAX_VALLEYS 8
#define CMPMC_MAX_IV 4
#define CMPMC_MAX_POLY 8

/* CrystalConfig (materials/crystal_config.hpp:43-226); fields in SI / eV as there. */
typedef struct cmpmc_crystal_config {
    int32_t group;                 /* BravaisGroup */
    int32_t has_custom_C;
    double density;
    double C11, C12, C13, C14, C16, C33, C44, C66;
    double C_custom[6][6];
    double beta, gamma, lambda, mu;
    double B_iso, A_anh, fTT_frac, polycrystal_mfp_m;
    double fLDOS, fSTDOS, fFTDOS;
    double debye_freq, v_sound, v_trans;
    double bandgap, pair_energy, fano_factor, epsilon_rel, neutral_impurity_cm3, alpha_nonparabolic;
    double h_mass_ratio;
    double e_mass_tensor[3];
    int32_t n_valleys;
    int32_t iv_model;              /* IVRateModel: 0 Quadratic, 1 Linear, 2 Matrix */
    double valley_dirs[CMPMC_MAX_VALLEYS][3];
    double ac_deform_e, ac_deform_h;
    int32_t n_iv;
    int32_t _pad0;
    double iv_deform_eV_m[CMPMC_MAX_IV], iv_energy_eV[CMPMC_MAX_IV];
    double iv_min_energy, iv_quad_rate, iv_quad_field, iv_quad_power, iv_lin_rate0, iv_lin_rate1, iv_lin_power;
    double e_trapping_mfp_m, h_trapping_mfp_m, e_trap_ion_d0_mfp_m, e_trap_ion_a_mfp_m,
           h_trap_ion_d_mfp_m, h_trap_ion_a0_mfp_m;
    double orient[3][3];           /* crystal -> detector rotation */
    double atomic_Z, atomic_A;     /* for NIEL and the charge-cloud radius (crystal_config.hpp:46-47) */
} cmpmc_crystal_config;

/* SuperconductorFilmConfig (crystal_config.hpp:240-257) */
typedef struct cmpmc_film_config {
    double film_absorption, film_thickness, v_sound, gap_energy, phonon_lifetime,
           phonon_lifetime_slope, low_qp_limit, high_qp_limit, subgap_absorption, absorber_gap,
           absorber_eff, absorber_eff_slope, temperature;
    int32_t keep_all_phonons;
    int32_t loss_model;            /* FilmLossModel: 0 MeanFreePath, 1 KaplanRateCompetition */
    double phonon_loss_time;
} cmpmc_film_config;

/* SurfaceProperty (geometry/surface_property.hpp:23-45) */
typedef struct cmpmc_surface {
    double prob_abs, prob_refl, refl_cutoff, anh_cutoff;
    double prob_charge_abs, prob_charge_spec, min_k_elec, min_k_hole;
    double spec_prob_const;
    int32_t n_spec, n_diff, n_anh;
    int32_t demo_values;
    double spec_coeffs[CMPMC_MAX_POLY], diff_coeffs[CMPMC_MAX_POLY], anh_coeffs[CMPMC_MAX_POLY];
    int32_t has_film;
    int32_t has_amm;               /* IsotropicAMMInterface (phonon/interface_transmission.hpp:123-140):
                                      the substrate -> film transmission replaces film_absorption */
    int32_t has_mask;              /* must be 0: masks are attached with cmpmc_gpu_set_electrode_mask */
    int32_t _pad0;
    cmpmc_film_config film;
    double amm_substrate[3];       /* IsotropicMedium {rho (kg/m^3), vL, vT (m/s)} of the crystal */
    double amm_film[3];            /* and of the film                                           */
} cmpmc_surface;

/* DetectorModel (transport/engine.hpp:96-156) with a CylinderSolid */
typedef struct cmpmc_detector {
    double radius, half_z;
    double e_field[3];             /* UniformElectricField::field_Vm */
    cmpmc_surface surfaces[3];     /* TopFace, BottomFace, SideWall */
    uint32_t max_bounces;
    uint32_t russian_roulette_bounces;
    double russian_roulette_survival;
    double min_phonon_eV;
    double luke_sample_fraction;
    double charge_max_dk_frac, charge_dt_cap_s, charge_sampling_dk_frac;
    int32_t charge_stepping;       /* 0 FirstOrderDkCap, 1 LemanSecondOrder */
    int32_t charge_release;        /* DetectorModel::ChargeRelease: 0 RecordOnly, 1 BulkDebye,
                                      2 ElectrodeFilm (batched: a release phase per round) */
    double fermi_level_above_Ev_eV;
    double electrode_seed_max_gap;
    int32_t allow_unvalidated;
    int32_t jump_to_ballistic;     /* experimental; must be 0 */
    int32_t kinematics_mode;       /* must be 0: the mode is the lattice's (cmpmc_lattice_set_kinematics_mode) */
    int32_t _pad0;
} cmpmc_detector;

/* Germanium preset (materials/presets.hpp:18-25) and the default detector
 * (engine.hpp:96-156: Al Kaplan films on both faces, bare diffuse side wall). */
void cmpmc_crystal_config_germanium(cmpmc_crystal_config* cfg);
void cmpmc_detector_default(cmpmc_detector* det);
void cmpmc_film_aluminum(cmpmc_film_config* film);

/* ---- electrode masks (replaces ElectrodePatternMask, geometry/electrode_pattern.hpp) -- */
enum { CMPMC_PAD_DISK = 0, CMPMC_PAD_ANNULAR_SECTOR = 1, CMPMC_PAD_RECTANGLE = 2 };
/* ElectrodePad (electrode_pattern.hpp:23-35): 64 B */
typedef struct cmpmc_electrode_pad {
    int32_t shape;                 /* CMPMC_PAD_*                                          */
    int32_t channel_id;
    double cx, cy;                 /* centre (m) of a disk or rectangle                    */
    double r_min;                  /* inner radius, or half-width hx of a rectangle (m)    */
    double r_max;                  /* outer radius, or half-height hy of a rectangle (m)   */
    double phi_min, phi_max;       /* azimuth range in [0, 2 pi] of an annular sector      */
    double fill_fraction;          /* active metal fraction in (0, 1]                      */
} cmpmc_electrode_pad;
/* ElectrodePatternMask::supercdms_qet_mask (electrode_pattern.hpp:99-148): inner disk,
 * three 120-degree sectors and a guard ring; writes 5 pads. */
int cmpmc_mask_supercdms_qet(double crystal_radius_m, double fill_fraction, cmpmc_electrode_pad out[5]);
/* ElectrodePatternMask::rectangular_grid_mask (electrode_pattern.hpp:151-178): nx * ny
 * rectangles; *n receives nx * ny (CMPMC_ERR_CAPACITY when cap is smaller). */
int cmpmc_mask_rectangular_grid(int nx, int ny, double pitch_x, double pitch_y, double pad_half_w,
                                double pad_half_h, double fill_fraction, cmpmc_electrode_pad* out, uint64_t cap,
                                uint64_t* n);
/* ElectrodePatternMask::find_channel (electrode_pattern.hpp:82-92) on the host: the first
 * pad containing (pos[0], pos[1]); one draw from rng_state when its fill fraction is below
 * 1; -1 for bare crystal. */
int cmpmc_mask_find_channel(const cmpmc_electrode_pad* pads, uint64_t n, const double pos[3], uint64_t rng_state[4],
                            int32_t* channel);

/* IsotropicAMMInterface::transmission (phonon/interface_transmission.hpp:125-130) on the host:
 * substrate and film are {rho, vL, vT}; the transmitted energy flux of an L (longitudinal = 1)
 * or transverse phonon incident at cos_theta. */
double cmpmc_amm_transmission(const double substrate[3], const double film[3], int longitudinal, double cos_theta);

/* ---- Kaplan-cascade surrogate (replaces KaplanSurrogateLUT, kaplan_film.hpp:336-383) ---- */
typedef struct cmpmc_kaplan_lut cmpmc_kaplan_lut;
/* KaplanSurrogateLUT(film, seed) (kaplan_film.hpp:344-358): 128 energy nodes on
 * [2 Delta, 40 Delta] x 512 cascade outcomes drawn from Rng(seed) (the reference's
 * default seed is 1337). */
int cmpmc_kaplan_surrogate_create(const cmpmc_film_config* film, uint64_t seed, cmpmc_kaplan_lut** out);
void cmpmc_kaplan_surrogate_destroy(cmpmc_kaplan_lut* lut);
int cmpmc_kaplan_surrogate_info(const cmpmc_kaplan_lut* lut, uint64_t* n_outcomes, uint64_t* n_reflected);
/* KaplanSurrogateLUT::absorb_phonon_fast (kaplan_film.hpp:361-374) on the host: returns the
 * absorbed energy in *edep and the re-emitted energies in refl[0 .. *n_refl); draws from
 * rng_state. */
int cmpmc_kaplan_surrogate_absorb(const cmpmc_kaplan_lut* lut, double energy, uint64_t rng_state[4], double* refl,
                                  uint64_t cap, uint64_t* n_refl, double* edep);

/* ---- host lattice (replaces the CrystalLattice constructor) -------------------- */
typedef struct cmpmc_lattice cmpmc_lattice;

/* Builds the octahedral FP32 group-velocity table (3x256x256 {vx,vy,vz,|v|}), the
 * decay inverse-CDF tables (2x1024 FP64) and the Herring-Vogt valley tensors on the
 * host, with the reference's arithmetic (crystal_lattice.hpp:340-477). */
int cmpmc_lattice_create(const cmpmc_crystal_config* cfg, cmpmc_lattice** out);
void cmpmc_lattice_destroy(cmpmc_lattice* lat);
/* Read-only views of the tables (owned by the lattice). hv: 16 + 9*n_valleys doubles
 * in the order e_cond_mass, h_mass, mass_ratio[3], hv_sqrt[3], hv_sqrt_inv[3], l0_e,
 * l0_h, k_sound_e, k_sound_h, n_valleys, valley_rot[n][3][3]. */
int cmpmc_lattice_tables(const cmpmc_lattice* lat, const float** oct_lut, const double** cdf_lt,
                         const double** cdf_tt, const double** hv, size_t* n_hv);
/* CrystalLattice::set_kinematics_mode (crystal_lattice.hpp:63-74): 0 Octahedral (default),
 * 1 Exact (Cardano solve per call), 2 Bilinear (181 x 361 (cos theta, phi) table, built here
 * on first request). It applies to make_track, the generators and every device context
 * created afterwards from this lattice. The plain FP64 form evaluates them as the reference
 * does; the batched FP32 forms call the same FP64 maps out of line and round the group
 * velocity to FP32 (not with the Kaplan surrogate, and not in the adjoint). */
int cmpmc_lattice_set_kinematics_mode(cmpmc_lattice* lat, int mode);
int cmpmc_lattice_kinematics_mode(const cmpmc_lattice* lat);
/* CrystalLattice::map_k_to_vg (crystal_lattice.hpp:76-176, the lattice's mode), on the host. */
int cmpmc_lattice_map_k_to_vg(const cmpmc_lattice* lat, int mode, const double k_det[3],
                              double vg_dir[3], double* vg_mag);
/* SimulationEngine::make_track (engine.hpp:171-187), on the host. */
int cmpmc_make_track(const cmpmc_lattice* lat, const double pos[3], const double k_dir[3], int mode,
                     double energy_eV, double time_s, double weight, cmpmc_phonon_track* out);
/* ChargePhysics::make_charge (charge/charge_transport.hpp:49-70), on the host. */
int cmpmc_make_charge(const cmpmc_lattice* lat, int type, const double pos[3], const double dir[3],
                      double ekin_eV, int valley, double time_s, cmpmc_charge_track* out);

/* ---- tetrahedral field mesh (replaces TriLinearMesh3D, geometry/mesh_field.hpp:40-345) -- */
typedef struct cmpmc_mesh cmpmc_mesh;
/* TriLinearMesh3D(vertices, potentials, tetrahedra, V_min_clamp, V_max_clamp)
 * (mesh_field.hpp:47-58): vertices [n][3] (m), potentials [n] (V), tets [m][4] (0-based
 * node indices). Face neighbours, inverse edge matrices and the per-tetrahedron field
 * are computed on the host with the reference's arithmetic. */
int cmpmc_mesh_create(const double* vertices, const double* potentials, uint64_t n_vertices, const int32_t* tets,
                      uint64_t n_tets, double v_min_clamp, double v_max_clamp, cmpmc_mesh** out);
/* TriLinearMesh3D::build_cartesian_grid (mesh_field.hpp:131-189): a Kuhn-triangulated
 * box (6 tetrahedra per cell) over [-hx,hx] x [-hy,hy] x [-hz,hz]; potential(p, user)
 * gives the node potentials. */
typedef double (*cmpmc_potential_fn)(const double p[3], void* user);
int cmpmc_mesh_build_cartesian(double half_x, double half_y, double half_z, int nx, int ny, int nz,
                               cmpmc_potential_fn potential, void* user, cmpmc_mesh** out);
/* TriLinearMesh3D::load_from_files (mesh_field.hpp:190-231): whitespace-separated ASCII,
 * one node "x y z V" per line in coords_file and one tetrahedron "i0 i1 i2 i3" (0-based)
 * per line in tets_file; lines starting with '#' or '%' and lines that do not parse are
 * skipped; coordinates and potentials are multiplied by the units. A file that cannot be
 * opened gives no lines (an empty mesh, as in the reference); a node index out of range
 * returns CMPMC_ERR_INVALID (the reference reads past its node table there). */
int cmpmc_mesh_load_files(const char* coords_file, const char* tets_file, double coord_unit_m,
                          double potential_unit_V, cmpmc_mesh** out);
/* The node potential of the recoil workloads (user = const cmpmc_detector*):
 * V = 4 V (z + h) / 2h + 0.2 V (r / R)^2 sin(pi z / 2h). */
double cmpmc_recoil_potential(const double p[3], void* detector);
void cmpmc_mesh_destroy(cmpmc_mesh* mesh);
int cmpmc_mesh_info(const cmpmc_mesh* mesh, uint64_t* n_vertices, uint64_t* n_tets);
/* field_at / potential_at with a caller-held walk hint (mesh_field.hpp:66-116); zero
 * outside the mesh. */
int cmpmc_mesh_field_at(const cmpmc_mesh* mesh, const double p[3], int32_t* hint, double E[3]);
int cmpmc_mesh_potential_at(const cmpmc_mesh* mesh, const double p[3], int32_t* hint, double* V);

/* ---- 2D triangle field mesh (replaces BiLinearMesh2D, geometry/mesh_field.hpp:347-582) ---- */
typedef struct cmpmc_mesh2d cmpmc_mesh2d;
/* BiLinearMesh2D(vertices, potentials, triangles, axisymmetric_rz) (mesh_field.hpp:356-366):
 * uv [n][2] = (r, z) when axisymmetric (the field is rotated back into x, y, z), else (x, y). */
int cmpmc_mesh2d_create(const double* uv, const double* potentials, uint64_t n_vertices, const int32_t* tris,
                        uint64_t n_tris, int axisymmetric, cmpmc_mesh2d** out);
/* BiLinearMesh2D::build_grid (mesh_field.hpp:438-479): nu x nv cells of two triangles;
 * potential(u, v, user) gives the node potentials. */
typedef double (*cmpmc_potential2d_fn)(double u, double v, void* user);
int cmpmc_mesh2d_build_grid(double u_min, double u_max, double v_min, double v_max, int nu, int nv,
                            cmpmc_potential2d_fn potential, void* user, int axisymmetric, cmpmc_mesh2d** out);
void cmpmc_mesh2d_destroy(cmpmc_mesh2d* mesh);
int cmpmc_mesh2d_info(const cmpmc_mesh2d* mesh, uint64_t* n_vertices, uint64_t* n_tris);
/* field_at / potential_at with a caller-held walk hint (mesh_field.hpp:376-430); zero outside. */
int cmpmc_mesh2d_field_at(const cmpmc_mesh2d* mesh, const double p[3], int32_t* hint, double E[3]);
int cmpmc_mesh2d_potential_at(const cmpmc_mesh2d* mesh, const double p[3], int32_t* hint, double* V);

/* ---- energy partition and primary-step merging (charge/energy_partition.hpp, ----------
 * ---- charge/niel_models.hpp): the input side of the transport, on the host -------- */
enum {
    CMPMC_NIEL_LINDHARD    = 0,  /* NIELModel (niel_models.hpp:28-34) */
    CMPMC_NIEL_LEWIN_SMITH = 1,
    CMPMC_NIEL_SARKIS      = 2,
    CMPMC_NIEL_IMPACT_TUNL = 3,
    CMPMC_NIEL_EMPIRICAL   = 4
};
/* PartitionOptions with EmpiricalNIELParams (energy_partition.hpp:22-29, niel_models.hpp:36-43) */
typedef struct cmpmc_partition_options {
    int32_t niel_model;
    int32_t use_fano_fluctuations;
    int32_t use_charge_cloud;
    uint32_t max_sampled_pairs;
    uint32_t max_sampled_phonons;
    int32_t emp_energy_dependent_k;
    double emp_k_fixed, emp_k_low, emp_k_high, emp_e_low_eV, emp_e_high_eV;
} cmpmc_partition_options;
/* EnergyPartition::Result (energy_partition.hpp:36-48) */
typedef struct cmpmc_partition_result {
    double total_edep_eV, ionizing_eV, niel_eV, lindhard_yield;
    uint64_t n_pairs_true, n_pairs_sampled, n_phonons_true, n_phonons_sampled;
    double charge_weight, phonon_weight, prompt_phonon_eV;
} cmpmc_partition_result;
void cmpmc_partition_options_default(cmpmc_partition_options* opts);
/* physics::compute_ionization_yield (niel_models.hpp:161-176); opts supplies the empirical
 * parameters (NULL: defaults). */
double cmpmc_ionization_yield(const cmpmc_crystal_config* cfg, int niel_model, double energy_eV,
                              const cmpmc_partition_options* opts);
/* EnergyPartition::lindhard_ionization_yield(E, z1, a1) (energy_partition.hpp:53-73) */
double cmpmc_lindhard_yield(const cmpmc_crystal_config* cfg, double energy_eV, double z1, double a1);
/* physics::sample_fano_binomial (niel_models.hpp:202-263), drawing from rng_state */
uint64_t cmpmc_sample_fano_binomial(double mean, double fano, uint64_t rng_state[4]);
/* EnergyPartition::partition_deposit (energy_partition.hpp:78-167): writes 2 n_pairs_sampled
 * carriers (e-, h+ interleaved) and n_phonons_sampled prompt phonons, drawing from
 * rng_state. *n_charges / *n_phonons receive the counts; if a capacity is short the call
 * returns CMPMC_ERR_CAPACITY and leaves rng_state unchanged (retry with the counts). */
int cmpmc_partition_deposit(const cmpmc_lattice* lat, const double pos[3], double time_s, double total_edep_eV,
                            int is_nuclear_recoil, const cmpmc_partition_options* opts, uint64_t rng_state[4],
                            cmpmc_charge_track* charges, uint64_t charge_cap, uint64_t* n_charges,
                            cmpmc_phonon_track* phonons, uint64_t phonon_cap, uint64_t* n_phonons,
                            cmpmc_partition_result* result);
/* One energy deposit for the device partition: partition_deposit(pos, time_s, edep_eV,
 * is_nuclear_recoil, ...) (energy_partition.hpp:78-86) */
typedef struct cmpmc_deposit {
    double pos[3];
    double time_s;
    double edep_eV;
    int32_t is_nuclear_recoil;
    int32_t _pad;
} cmpmc_deposit;

/* PrimaryStepInput (energy_partition.hpp:182-192) */
typedef struct cmpmc_primary_step {
    int32_t track_id;
    int32_t is_charged;
    double start_pos[3];
    double end_pos[3];
    double time_s, edep_eV, eniel_eV;
    int32_t hit_boundary, track_stopped;
} cmpmc_primary_step;
/* HitMerger (energy_partition.hpp:229-323). The merged secondaries accumulate in the
 * merger (the reference appends them to the caller's vectors); cmpmc_hit_merger_take
 * moves them out. The lattice must outlive the merger. */
typedef struct cmpmc_hit_merger cmpmc_hit_merger;
int cmpmc_hit_merger_create(const cmpmc_lattice* lat, double combining_step_length_m,
                            const cmpmc_partition_options* opts, cmpmc_hit_merger** out);
void cmpmc_hit_merger_destroy(cmpmc_hit_merger* merger);
/* HitMerger::process_step for each step in order (energy_partition.hpp:236-266);
 * *n_flushes receives how many of them flushed. */
int cmpmc_hit_merger_process_steps(cmpmc_hit_merger* merger, const cmpmc_primary_step* steps, uint64_t n_steps,
                                   uint64_t rng_state[4], uint64_t* n_flushes);
/* HitMerger::flush (energy_partition.hpp:268-316) */
int cmpmc_hit_merger_flush(cmpmc_hit_merger* merger, uint64_t rng_state[4], cmpmc_partition_result* result);
/* Copies the accumulated carriers and phonons out and clears them (CMPMC_ERR_CAPACITY with
 * the counts set, and nothing cleared, if a capacity is short). */
int cmpmc_hit_merger_take(cmpmc_hit_merger* merger, cmpmc_charge_track* charges, uint64_t charge_cap,
                          uint64_t* n_charges, cmpmc_phonon_track* phonons, uint64_t phonon_cap,
                          uint64_t* n_phonons);

/* ---- random streams (core/rng.hpp) --------------------------------------------- */
void cmpmc_rng_for_stream(uint64_t seed, uint64_t stream, uint64_t state[4]);
uint64_t cmpmc_rng_next_u64(uint64_t state[4]);
double cmpmc_rng_uniform(uint64_t state[4]);

/* ---- canonical workload generators (host) --------------------------------------- */
enum {
    CMPMC_WL_SINGLE_L_ORIGIN = 0,  /* one L phonon, 7.5 meV, at the origin, isotropic          */
    CMPMC_WL_MIXED_ENERGY    = 1,  /* 100 phonons/event, log-uniform 1-30 meV, L/ST/FT mix      */
    CMPMC_WL_PAIR_DRIFT      = 2,  /* one e-/h+ pair per event, uniform origin                  */
    CMPMC_WL_RECOIL          = 3,  /* electron recoil 10 eV-10 keV (log-uniform), uniform origin,
                                      split by EnergyPartition::partition_deposit (pairs capped
                                      at 4096); all Luke phonons tracked; mesh field          */
    CMPMC_WL_SINGLE_L_VOLUME = 4,  /* one L phonon, 7.5 meV, uniform origin, isotropic          */
    CMPMC_WL_TEST_PARALLEL   = 5,  /* reference tests/test_parallel.cpp:110-125 generator        */
    CMPMC_WL_RECOIL_LIGHT    = 6,  /* as RECOIL with deposits 10-100 eV (log-uniform), at most 20
                                      prompt phonons (weighted) and 5 % of the Luke phonons
                                      tracked (weight 20): the parity case                   */
    CMPMC_WL_PUBLISHED_PHONON = 7, /* the reference's published phonon benchmark generator
                                      (benchmarks/cmpmc_bench.cpp:63-67): one 7.5 meV phonon at
                                      the origin, mode ST / FT / L by the DOS split, isotropic */
    CMPMC_WL_PUBLISHED_PAIR  = 8   /* its `charge` mode (cmpmc_bench.cpp:68-71): one e-/h+ pair
                                      at the origin, electron valley uniform                  */
};
/* Runs the workload's generator for events [first_event, first_event + n_events) from
 * Rng::for_stream(seed, ev) and writes, per event, the RNG state after the generator
 * (4 u64), the injected energy and the CSR-packed initial tracks. Capacities are in
 * records; *n_phonons / *n_charges receive the totals (CMPMC_ERR_CAPACITY if short; the
 * offsets are written either way, so a call with zero capacities sizes the buffers).
 * The recoil workloads expect det->luke_sample_fraction as they define it (1 or 0.05);
 * their field mesh is built by cmpmc_recoil_mesh. */
int cmpmc_generate(const cmpmc_lattice* lat, const cmpmc_detector* det, int workload, uint64_t seed,
                   uint64_t first_event, uint64_t n_events, int n_threads,
                   uint64_t* rng_state, double* injected_eV,
                   uint64_t* phonon_offsets, cmpmc_phonon_track* phonons, uint64_t phonon_cap,
                   uint64_t* n_phonons,
                   uint64_t* charge_offsets, cmpmc_charge_track* charges, uint64_t charge_cap,
                   uint64_t* n_charges);

/* The field mesh of the recoil workloads: build_cartesian_grid(R, R, h, 58, 58, 57) of the
 * detector's cylinder (59 x 59 x 58 = 201,898 nodes, 1,150,488 tetrahedra) with node
 * potentials cmpmc_recoil_potential. */
int cmpmc_recoil_mesh(const cmpmc_detector* det, cmpmc_mesh** out);

/* ---- device context and run ---------------------------------------------------- */
typedef struct cmpmc_gpu_ctx cmpmc_gpu_ctx;

enum {
    CMPMC_FORM_PLAIN_FP64          = 0,  /* bit-exact event streams, one event per device thread */
    CMPMC_FORM_BATCHED_FP32        = 1,  /* own substreams per primary, FP32 geometry, FP64
                                            ledger and time of flight; film cascades run apart
                                            from the transport steps and their re-emitted
                                            phonons re-enter through device queues (the warp
                                            pool, cmpmc_gpu_configure_pool; hits of an event in
                                            no fixed order, FP64 event sums by atomics); with
                                            charges: per-carrier substreams, FP32 drift, Luke
                                            phonons through the queue                         */
    CMPMC_FORM_BATCHED_FP32_INLINE = 2   /* the batched form with each primary's whole lineage on
                                            one thread (film cascades inline): hits in a fixed
                                            order, the forward of cmpmc_gpu_adjoint           */
};

typedef struct cmpmc_run_desc {
    uint64_t n_events;
    uint64_t first_event;          /* event id of record 0 (event ids feed the substreams)  */
    const uint64_t* rng_state;     /* [n_events][4] post-generator state                    */
    const double* injected_eV;     /* [n_events]                                            */
    const uint64_t* phonon_offsets;/* [n_events + 1]                                        */
    const cmpmc_phonon_track* phonons;
    const uint64_t* charge_offsets;/* [n_events + 1], or NULL when there are no charges     */
    const cmpmc_charge_track* charges;
    int32_t keep_hits;             /* RunOptions::keep_hits                                  */
    int32_t form;                  /* CMPMC_FORM_*                                           */
    int32_t inputs_on_device;      /* 1: the pointers above are device pointers             */
    int32_t outputs_on_device;     /* 1: leave hits / offsets / event stats on the device   */
    uint64_t seed;                 /* batched form: substream seed                          */
    int32_t want_event_stats;      /* 1: also return per-event SimStats                     */
    int32_t kaplan_surrogate;      /* batched form: 1 = film cascades from the surrogate
                                      table (KaplanSurrogateLUT, seed 1337) inside its
                                      energy range, the full cascade outside it            */
} cmpmc_run_desc;

typedef struct cmpmc_run_out {
    cmpmc_sim_stats stats;         /* summed over all events                                 */
    uint64_t n_hits;
    const cmpmc_sensor_hit* hits;  /* [n_hits], event order; owned by the context            */
    const uint64_t* hit_offsets;   /* [n_events + 1]; owned by the context                   */
    const cmpmc_sim_stats* event_stats; /* [n_events] if requested; owned by the context     */
    double kernel_ms;              /* device time of the transport kernel(s)                 */
    double total_ms;               /* device time of the whole call incl. copies            */
    uint32_t device_error;         /* error word written by the kernels (0 = none)           */
    uint32_t kernel_launches;      /* kernels this call launched                             */
} cmpmc_run_out;

int cmpmc_gpu_create(const cmpmc_lattice* lat, const cmpmc_detector* det, int device,
                     cmpmc_gpu_ctx** out);
void cmpmc_gpu_destroy(cmpmc_gpu_ctx* ctx);
/* run_events on the device for pre-generated events (the generator ran on the host). */
int cmpmc_gpu_run_events(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* desc, cmpmc_run_out* out);
/* Copies the message of the last failed call on ctx (or of a failed create when ctx is
 * NULL) into buf. Returns the status of that call. */
int cmpmc_gpu_last_error(const cmpmc_gpu_ctx* ctx, char* buf, size_t size);
/* Device-side tuning: threads per block and blocks per SM of the transport kernels,
 * stack capacity (tracks per device thread), hit staging capacity (records). 0 keeps
 * the current value. */
int cmpmc_gpu_configure(cmpmc_gpu_ctx* ctx, int threads_per_block, int blocks_per_sm,
                        uint64_t stack_capacity, uint64_t hit_capacity);
int cmpmc_gpu_device_count(int* count);
/* Synchronous copy between any two pointers (host or device, unified addressing): reads
 * outputs left on the device (outputs_on_device = 1) without a CUDA binding of your own. */
int cmpmc_gpu_memcpy(void* dst, const void* src, size_t bytes);
/* Batched FP32 form with charges: capacity of the device Luke-phonon queue in entries
 * (64 B each, default 2^24). Carriers queue their tracked Luke phonons there; when it is
 * full they are parked and resumed after the queued phonons have been transported, so a
 * small queue only adds phases. 0 keeps the current value. */
int cmpmc_gpu_configure_queue(cmpmc_gpu_ctx* ctx, uint64_t queue_capacity);
/* CUDA-graph replay (no counterpart in the reference): with enable = 1, a batched-form call
 * of phonon events whose inputs and outputs stay on the device (SM-phase pool, warp pool or
 * inline form) is captured after it ran cleanly (counter resets, unit map, the transport
 * launch, merge and the copies of the counters as one graph) and replayed by later calls
 * with the same descriptor pointers, sizes and configuration: one graph launch per call. A
 * replay whose buffers overflow falls back to the eager call, which grows them and
 * recaptures; any configure / set call on the context drops the captured graph. */
int cmpmc_gpu_configure_graph(cmpmc_gpu_ctx* ctx, int enable);

/* Wavefront split of the batched form (no counterpart in the reference): a track that has
 * taken `phase_steps` steps in one transport phase is parked for the next phase, on a
 * substream drawn from its own, so long tracks do not hold a phase open (default 0: no
 * limit). A limit changes which substream a long track continues on: the results are then
 * statistically, not bitwise, those of the unlimited run; the autotuner leaves it alone. */
int cmpmc_gpu_configure_phases(cmpmc_gpu_ctx* ctx, uint32_t phase_steps);

/* Launch form of the batched FP32 phonon transport (no counterpart in the reference).
 * form = 1 (the default): the SM-phase pool, one persistent launch per call with one
 *   512-thread block per SM that alternates a transport phase (every warp steps its lanes,
 *   refilled from the block's ring of pending phonons and the batch's primaries; film
 *   entries and daughters appended to block buffers) and a film phase (every thread runs
 *   the waiting film cascades, their re-emissions appended to the ring), so an SM runs one
 *   code path at a time; ring_capacity: pending phonons per block (default 2^17).
 * form = 2: the warp pool, one persistent launch in which every warp runs its own film
 *   cascades between its transport steps; ring_capacity: pending phonons per warp (default
 *   1024).
 * form = 0: the host-driven form, alternating transport and film launches until both device
 *   queues are empty (one host round trip per round; configure_phases applies to it only).
 * form = 3: the SM-phase pool computed in FP64 throughout (geometry, directions, rates and
 *   samplers of the plain form, 53-bit uniforms, the reference's 1e-11 m inward nudge) on
 *   the same substreams as form 1: the comparison point that shows what the FP32 form
 *   gains. Phonon-only batches with full film cascades (CMPMC_ERR_INVALID with charges or
 *   the Kaplan surrogate); ring entries 128 B, film records 80 B.
 * Rings are 80 B per entry; a ring (a power of two >= 64; 0 keeps the current value) that
 * overflows is grown 4x and the call rerun. All forms sample the same process; a daughter
 * runs on a substream drawn from its parent's in the pool forms, on the parent's own stream
 * in the host-driven form, so their hits agree in distribution, not bit for bit. */
int cmpmc_gpu_configure_pool(cmpmc_gpu_ctx* ctx, int form, uint32_t ring_capacity);

/* Shared-memory staging of the small tables (no counterpart in the reference): with
 * enable = 1 (the default) every block of the warp-pool kernel copies the two decay CDF
 * tables (CrystalLattice::sample_lt/tt_energy_fraction's, crystal_lattice.hpp:200-212; 8 KiB
 * as FP32) into shared memory with one TMA bulk copy and samples from there; 0 reads them
 * from global memory. The results are identical either way. */
int cmpmc_gpu_configure_staging(cmpmc_gpu_ctx* ctx, int enable);

/* Autotuner of the launch configuration (no counterpart in the reference): runs `sample`
 * (a representative call, outputs discarded) `repeats` times for each candidate, keeps the
 * fastest transport-kernel time and applies it to the context. Candidates: the current
 * configuration; 64 and 128 threads per block at the occupancy limit and at 3/4 and 1/2 of
 * it; for the batched charge form also Luke-phonon queues of 2^20, 2^22 and 2^24 entries.
 * The batched results do not depend on the configuration (every unit owns its substream). */
#define CMPMC_TUNE_MAX 16
typedef struct cmpmc_tune_result {
    int32_t threads_per_block, blocks_per_sm;   /* chosen */
    uint64_t queue_capacity;                    /* chosen (charge runs) */
    uint32_t phase_steps;                       /* in place (not tuned) */
    uint32_t _pad1;
    double best_ms;                             /* its transport-kernel time */
    double first_ms;                            /* the configuration in place before tuning */
    int32_t n_tried, _pad0;
    int32_t tried_tpb[CMPMC_TUNE_MAX], tried_bps[CMPMC_TUNE_MAX];
    uint64_t tried_queue[CMPMC_TUNE_MAX];
    double tried_ms[CMPMC_TUNE_MAX];
} cmpmc_tune_result;
int cmpmc_gpu_autotune(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* sample, int repeats, cmpmc_tune_result* out);

/* SurfaceProperty::electrode_mask (surface_property.hpp:45, evaluated at engine.hpp:284-289
 * and 483-488): attaches n pads to surface `surface` (CMPMC_SURF_*) of the context's
 * detector and copies them to the device; n = 0 removes the mask. A phonon or carrier
 * reaching bare crystal between pads reflects; a hit on a pad records its channel_id. */
int cmpmc_gpu_set_electrode_mask(cmpmc_gpu_ctx* ctx, int surface, const cmpmc_electrode_pad* pads, uint64_t n);
/* DetectorModel::mesh_field_3d (engine.hpp:99, looked up by electric_field_at,
 * engine.hpp:151-155): copies the mesh to the context's device; the charge transport then
 * takes its field from the mesh instead of the uniform e_field. NULL detaches it. Each
 * device thread keeps its own walk hint across carriers and events, like the reference's
 * thread_local hint (mesh_field.hpp:119-122). */
int cmpmc_gpu_set_mesh(cmpmc_gpu_ctx* ctx, const cmpmc_mesh* mesh);
/* DetectorModel::mesh_field_2d (engine.hpp:100, used when there is no 3D mesh,
 * engine.hpp:151-155): copies the 2D mesh to the context's device; NULL detaches it. */
int cmpmc_gpu_set_mesh2d(cmpmc_gpu_ctx* ctx, const cmpmc_mesh2d* mesh);

/* EnergyPartition::partition_deposit (energy_partition.hpp:78-167) for n deposits on the
 * context's device: deposit i draws from rng_state[i] (4 u64, advanced in place, e.g. an
 * event's state after its generator drew the deposit) with the reference's draw order, and
 * its 2 n_pairs_sampled carriers (e-, h+ interleaved) and n_phonons_sampled prompt phonons
 * go to charges[charge_offsets[i] .. charge_offsets[i+1]) and
 * phonons[phonon_offsets[i] .. phonon_offsets[i+1]): the initial stacks of
 * cmpmc_gpu_run_events with inputs_on_device. deposits, rng_state, the offsets ([n + 1])
 * and the records are device memory; *n_charges / *n_phonons (host) receive the totals.
 * A deposit whose energy, position or time is not finite makes the call return
 * CMPMC_ERR_INVALID before any record is written (rng_state unchanged); so does the host
 * cmpmc_partition_deposit.
 * A capacity that is too small returns CMPMC_ERR_CAPACITY with the totals and the offsets
 * written and rng_state unchanged. The device's transcendentals are correctly rounded, so
 * a record can differ from the host partition's (cmpmc_partition_deposit, which uses the
 * platform libm like the reference) in the last bits where the platform libm is not. */
int cmpmc_gpu_partition_deposits(cmpmc_gpu_ctx* ctx, const cmpmc_deposit* deposits, uint64_t n,
                                 const cmpmc_partition_options* opts, uint64_t* rng_state, uint64_t* charge_offsets,
                                 uint64_t* phonon_offsets, cmpmc_charge_track* charges, uint64_t charge_cap,
                                 cmpmc_phonon_track* phonons, uint64_t phonon_cap, uint64_t* n_charges,
                                 uint64_t* n_phonons);

/* Allocation-free run of the plain FP64 form (phonon-only events). No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc -- code running inside a
 * framework whose caching allocator owns the device memory, code with a fixed memory
 * budget, or latency-critical loops where an allocation may block or fail. It allocates
 * no device memory: every input and output below is caller-owned device memory, and the
 * per-thread stacks and counters live in a fixed array of the library (about 29 MiB, plus
 * 3 MiB of lattice tables), which every GPU that loads the library holds until exit.
 *   inputs : rng_state [n][4], injected_eV [n], phonon_offsets [n+1], phonons
 *   outputs: event_stats [n], hit_offsets [n+1], hits [hit_capacity] (event order)
 *   host   : *total (run SimStats), *n_hits (hits the run produced, also when they do not fit)
 * At most 64 tracks may sit on one event's stack at a time (CMPMC_ERR_CAPACITY otherwise);
 * CMPMC_ERR_CAPACITY is also returned when *n_hits > hit_capacity (nothing is written).
 * The lattice must use the octahedral kinematics mode (the default); a lattice switched to
 * Exact or Bilinear returns CMPMC_ERR_INVALID before any device work.
 * The transport runs twice (count, then write), so a call costs about two plain runs.
 * The first call on a device resolves the array's device address, and the first call with
 * a given lattice uploads its tables: make these calls before any stream capture. Every
 * call waits for `stream` to finish before it returns (it reads the run totals and the hit
 * count back to the host). Calls share the array and clear what they use, so calls whose
 * work overlaps on the GPU race: serialize them. `stream` is a cudaStream_t (NULL: the
 * default stream). */
int cmpmc_gpu_run_events_noalloc(const cmpmc_lattice* lat, const cmpmc_detector* det, int device,
                                 uint64_t n_events, const uint64_t* rng_state, const double* injected_eV,
                                 const uint64_t* phonon_offsets, const cmpmc_phonon_track* phonons,
                                 cmpmc_sim_stats* event_stats, uint64_t* hit_offsets,
                                 cmpmc_sensor_hit* hits, uint64_t hit_capacity, void* stream,
                                 cmpmc_sim_stats* total, uint64_t* n_hits);

/* ---- adjoint of the sensor-arrival histogram ---------------------------------------------
 * No function of the reference computes it; the forward quantity is the reference's own
 * transport (engine.hpp:403-582) observed through a binned histogram of SensorHit::time.
 * Parameters theta (absolute values):
 *   theta[0] isotope coefficient B_iso (CrystalConfig::B_iso, s^3)
 *   theta[1] anharmonic coefficient A_anh (CrystalConfig::A_anh, s^4)
 *   theta[2] diffuse fraction p_d of every surface: reflection_split gives p_spec = 1 - p_d,
 *            p_diff = p_d, p_anh = 0 at every frequency (spec_coeffs {1-p_d}, diff_coeffs {p_d},
 *            anh_coeffs {}, spec_prob_const 1-p_d in the reference's SurfaceProperty)
 *   theta[3] film absorption (SuperconductorFilmConfig::film_absorption of every film)
 * The transport is the batched FP32 form (each primary its own substream of `seed`); the
 * call returns the weighted hit counts per time bin h_b(theta) and, given bin weights
 * w_b = dLoss/dh_b, value = sum_b w_b h_b and its gradient d value / d theta estimated by
 * the score function: every theta-dependent random decision (the exponential free flights
 * with their isotope and anharmonic channels, the specular/diffuse choice, film entry)
 * adds d log p / d theta to the score of its track, daughters inherit their parent's score,
 * and every binned hit adds w_b * score. Tracks are recomputed from their RNG substreams
 * (nothing is stored between the forward and the backward call). */
#define CMPMC_ADJ_MAX_BINS 256
typedef struct cmpmc_adjoint_desc {
    uint64_t n_events;
    uint64_t first_event;
    uint64_t seed;
    const uint64_t* phonon_offsets;     /* [n_events + 1]                                    */
    const cmpmc_phonon_track* phonons;  /* initial phonons                                   */
    int inputs_on_device;
    int n_bins;                         /* 1 .. CMPMC_ADJ_MAX_BINS                            */
    double t_min, t_max;                /* histogram range of hit times (s)                  */
    double theta[4];
    const double* bin_weight;           /* host [n_bins]; NULL: histogram only               */
    double* per_primary;                /* optional [n_primaries][5]: value and d value /
                                           d theta_k of each primary's lineage               */
    int per_primary_on_device;          /* per_primary is device memory                      */
} cmpmc_adjoint_desc;

typedef struct cmpmc_adjoint_out {
    double hist[CMPMC_ADJ_MAX_BINS];    /* weighted hit counts per bin (FP64 sums)           */
    double value;                       /* sum_b bin_weight_b hist_b                          */
    double grad[4];                     /* d value / d theta_k                               */
    double value_var;                   /* variance estimates of value and grad from the      */
    double grad_var[4];                 /* spread over primaries (independent substreams)   */
    cmpmc_sim_stats stats;              /* summed over all primaries (no hit records kept)   */
    uint64_t n_primaries;
    double kernel_ms, total_ms;
    uint32_t device_error;
    uint32_t kernel_launches;
} cmpmc_adjoint_out;

int cmpmc_gpu_adjoint(cmpmc_gpu_ctx* ctx, const cmpmc_adjoint_desc* desc, cmpmc_adjoint_out* out);

/* Correctly rounded log / sin / cos of the device transport (crmath), evaluated on the
 * host; the device computes bit-identical values. */
double cmpmc_cr_log(double x);
double cmpmc_cr_sin(double x);
double cmpmc_cr_cos(double x);
/* Evaluates the device's log, sin and cos on n host inputs and writes out[3*i+{0,1,2}]
 * (for checking that device and host agree bit for bit). */
int cmpmc_gpu_math_check(int device, uint64_t n, const double* x, double* out);

/* Layout self-check for bindings: writes sizeof of the ABI structs in the order
 * phonon_track, charge_track, sensor_hit, sim_stats, crystal_config, film_config,
 * surface, detector, run_desc, run_out, adjoint_desc, adjoint_out (at most n values).
 * Returns the ABI version. */
int cmpmc_abi_sizes(size_t* out, int n);

#ifdef __cplusplus
}
#endif
#endif /* CMPMC_GPU_H */
