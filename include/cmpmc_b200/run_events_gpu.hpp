// run_events_gpu.hpp -- header-only C++ adapter from CMPMC's API to the B200 C ABI.
//
// Include this next to the reference's own headers ("cmpmc/cmpmc.hpp"). A call site of
// the reference's run_events (include/cmpmc/transport/parallel.hpp:76-148)
//
//     cmpmc::RunResult r = cmpmc::run_events(engine, n_events, generate, options);
//
// moves to the device by changing its namespace only:
//
//     cmpmc::RunResult r = cmpmc_b200::run_events(engine, n_events, generate, options);
//
// (an optional fifth argument, GpuRunOptions, picks the device and the form). The engine's
// lattice and detector are turned into a device context once and cached per (lattice,
// detector, device); a detector whose content changes gets a new context. The generator is
// the same user callback: it runs on the host, once per event, from
// Rng::for_stream(options.seed, i), with the reference's EventInput, Rng and
// SimulationEngine::make_track, so the initial stacks and the post-generator random state
// are exactly the reference's. Transport runs on the device; the RunResult is rebuilt from
// the device output (SensorHit and SimStats records are byte-identical, include/cmpmc_gpu.h).
//
// The reference's SimulationEngine keeps its lattice and detector as references in its
// first two data members (engine.hpp:871-872) and has no accessor for them; the adapter
// reads the two references from the engine's storage. That relies on the Itanium C++ ABI
// (GCC and Clang on Linux: a reference member is stored as a pointer, members in
// declaration order) and is checked at compile time against the engine's size.
//
// The explicit form is a cmpmc_b200::GpuEngine(lattice, detector) with
// gpu.run_events(n_events, generate, options); gpu_engine_for(engine) returns the cached
// one of an engine. Electrode masks are copied from the surfaces' ElectrodePatternMask
// pads. A TriLinearMesh3D field keeps its nodes private in the reference, so a detector
// with mesh_field_3d needs the same mesh handed over once with GpuEngine::set_mesh (its
// node coordinates, potentials and tetrahedra) or set_cartesian_mesh (the
// build_cartesian_grid arguments and the potential function); a detector with only
// mesh_field_2d needs its BiLinearMesh2D handed over the same way with set_mesh2d or
// set_grid_mesh2d (on gpu_engine_for(engine) for the drop-in form).
// Guarded modules raise the reference's UnvalidatedModuleError; configurations the device
// does not support (in the batched forms, the Kaplan surrogate with Exact / Bilinear
// kinematics) raise std::invalid_argument.
#pragma once

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <exception>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../cmpmc_gpu.h"

namespace cmpmc_b200 {

enum class Form { PlainFP64 = CMPMC_FORM_PLAIN_FP64, BatchedFP32 = CMPMC_FORM_BATCHED_FP32 };

struct GpuRunOptions {
    int device = 0;
    Form form = Form::PlainFP64;
    bool kaplan_surrogate = false;  // batched form: film cascades from the KaplanSurrogateLUT table
};

namespace detail {

inline void check(int status, const cmpmc_gpu_ctx* ctx, const char* what) {
    if (status == CMPMC_OK) return;
    char buf[1024];
    cmpmc_gpu_last_error(ctx, buf, sizeof(buf));
    const std::string msg = std::string(what) + ": " + buf;
    if (status == CMPMC_ERR_UNVALIDATED) throw cmpmc::UnvalidatedModuleError(msg);
    if (status == CMPMC_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

inline cmpmc_crystal_config to_c(const cmpmc::CrystalConfig& c) {
    cmpmc_crystal_config o;
    std::memset(&o, 0, sizeof(o));
    o.group = static_cast<int32_t>(c.group);
    o.has_custom_C = c.has_custom_C ? 1 : 0;
    o.density = c.density;
    o.C11 = c.C11; o.C12 = c.C12; o.C13 = c.C13; o.C14 = c.C14; o.C16 = c.C16; o.C33 = c.C33;
    o.C44 = c.C44; o.C66 = c.C66;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) o.C_custom[i][j] = c.C_custom[i][j];
    o.beta = c.beta; o.gamma = c.gamma; o.lambda = c.lambda; o.mu = c.mu;
    o.B_iso = c.B_iso; o.A_anh = c.A_anh; o.fTT_frac = c.fTT_frac; o.polycrystal_mfp_m = c.polycrystal_mfp_m;
    o.fLDOS = c.fLDOS; o.fSTDOS = c.fSTDOS; o.fFTDOS = c.fFTDOS;
    o.debye_freq = c.debye_freq; o.v_sound = c.v_sound; o.v_trans = c.v_trans;
    o.bandgap = c.bandgap; o.pair_energy = c.pair_energy; o.fano_factor = c.fano_factor;
    o.epsilon_rel = c.epsilon_rel; o.neutral_impurity_cm3 = c.neutral_impurity_cm3;
    o.alpha_nonparabolic = c.alpha_nonparabolic; o.h_mass_ratio = c.h_mass_ratio;
    o.e_mass_tensor[0] = c.e_mass_tensor.x; o.e_mass_tensor[1] = c.e_mass_tensor.y;
    o.e_mass_tensor[2] = c.e_mass_tensor.z;
    if (c.valley_dirs.size() > CMPMC_MAX_VALLEYS) throw std::invalid_argument("too many valleys");
    o.n_valleys = static_cast<int32_t>(c.valley_dirs.size());
    for (size_t k = 0; k < c.valley_dirs.size(); ++k) {
        o.valley_dirs[k][0] = c.valley_dirs[k].x;
        o.valley_dirs[k][1] = c.valley_dirs[k].y;
        o.valley_dirs[k][2] = c.valley_dirs[k].z;
    }
    o.ac_deform_e = c.ac_deform_e; o.ac_deform_h = c.ac_deform_h;
    const size_t n_iv = std::min<size_t>({c.iv_deform_eV_m.size(), c.iv_energy_eV.size(), CMPMC_MAX_IV});
    o.n_iv = static_cast<int32_t>(n_iv);
    for (size_t i = 0; i < n_iv; ++i) {
        o.iv_deform_eV_m[i] = c.iv_deform_eV_m[i];
        o.iv_energy_eV[i] = c.iv_energy_eV[i];
    }
    o.iv_min_energy = c.iv_min_energy;
    o.iv_model = static_cast<int32_t>(c.iv_model);
    o.iv_quad_rate = c.iv_quad_rate; o.iv_quad_field = c.iv_quad_field; o.iv_quad_power = c.iv_quad_power;
    o.iv_lin_rate0 = c.iv_lin_rate0; o.iv_lin_rate1 = c.iv_lin_rate1; o.iv_lin_power = c.iv_lin_power;
    o.e_trapping_mfp_m = c.e_trapping_mfp_m; o.h_trapping_mfp_m = c.h_trapping_mfp_m;
    o.e_trap_ion_d0_mfp_m = c.e_trap_ion_d0_mfp_m; o.e_trap_ion_a_mfp_m = c.e_trap_ion_a_mfp_m;
    o.h_trap_ion_d_mfp_m = c.h_trap_ion_d_mfp_m; o.h_trap_ion_a0_mfp_m = c.h_trap_ion_a0_mfp_m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o.orient[i][j] = c.orient.m[i][j];
    o.atomic_Z = c.atomic_Z;
    o.atomic_A = c.atomic_A;
    return o;
}

inline void poly(const std::vector<double>& v, double* dst, int32_t& n) {
    if (v.size() > CMPMC_MAX_POLY) throw std::invalid_argument("surface polynomial longer than CMPMC_MAX_POLY");
    n = static_cast<int32_t>(v.size());
    for (size_t i = 0; i < v.size(); ++i) dst[i] = v[i];
}

inline std::vector<cmpmc_electrode_pad> pads_of(const cmpmc::geometry::ElectrodePatternMask& m) {
    std::vector<cmpmc_electrode_pad> out;
    for (const auto& p : m.pads()) {
        cmpmc_electrode_pad q;
        std::memset(&q, 0, sizeof(q));
        q.shape = static_cast<int32_t>(p.shape);
        q.channel_id = p.channel_id;
        q.cx = p.cx; q.cy = p.cy; q.r_min = p.r_min; q.r_max = p.r_max;
        q.phi_min = p.phi_min; q.phi_max = p.phi_max; q.fill_fraction = p.fill_fraction;
        out.push_back(q);
    }
    return out;
}

inline cmpmc_detector to_c(const cmpmc::DetectorModel& d) {
    cmpmc_detector o;
    std::memset(&o, 0, sizeof(o));
    o.radius = d.solid.radius;
    o.half_z = d.solid.half_z;
    o.e_field[0] = d.e_field.field_Vm.x;
    o.e_field[1] = d.e_field.field_Vm.y;
    o.e_field[2] = d.e_field.field_Vm.z;
    for (int i = 0; i < 3; ++i) {
        const cmpmc::SurfaceProperty& s = d.surfaces[i];
        cmpmc_surface& t = o.surfaces[i];
        t.prob_abs = s.prob_abs; t.prob_refl = s.prob_refl; t.refl_cutoff = s.refl_cutoff; t.anh_cutoff = s.anh_cutoff;
        t.prob_charge_abs = s.prob_charge_abs; t.prob_charge_spec = s.prob_charge_spec;
        t.min_k_elec = s.min_k_elec; t.min_k_hole = s.min_k_hole; t.spec_prob_const = s.spec_prob_const;
        poly(s.spec_coeffs, t.spec_coeffs, t.n_spec);
        poly(s.diff_coeffs, t.diff_coeffs, t.n_diff);
        poly(s.anh_coeffs, t.anh_coeffs, t.n_anh);
        t.demo_values = s.demo_values ? 1 : 0;
        t.has_amm = s.amm_interface.has_value() ? 1 : 0;
        if (s.amm_interface.has_value()) {
            const auto& a = *s.amm_interface;
            t.amm_substrate[0] = a.substrate.rho; t.amm_substrate[1] = a.substrate.vL; t.amm_substrate[2] = a.substrate.vT;
            t.amm_film[0] = a.film.rho; t.amm_film[1] = a.film.vL; t.amm_film[2] = a.film.vT;
        }
        t.has_mask = 0;  // the pads are attached to the context (GpuEngine constructor)
        if (s.kaplan_sensor.has_value()) {
            const cmpmc::KaplanFilm& f = *s.kaplan_sensor;
            t.has_film = 1;
            t.film.film_absorption = f.film_absorption; t.film.film_thickness = f.film_thickness;
            t.film.v_sound = f.v_sound; t.film.gap_energy = f.gap_energy; t.film.phonon_lifetime = f.phonon_lifetime;
            t.film.phonon_lifetime_slope = f.phonon_lifetime_slope; t.film.low_qp_limit = f.low_qp_limit;
            t.film.high_qp_limit = f.high_qp_limit; t.film.subgap_absorption = f.subgap_absorption;
            t.film.absorber_gap = f.absorber_gap; t.film.absorber_eff = f.absorber_eff;
            t.film.absorber_eff_slope = f.absorber_eff_slope; t.film.temperature = f.temperature;
            t.film.keep_all_phonons = f.keep_all_phonons ? 1 : 0;
            t.film.loss_model = static_cast<int32_t>(f.loss_model);
            t.film.phonon_loss_time = f.phonon_loss_time;
        }
    }
    o.max_bounces = d.max_bounces;
    o.russian_roulette_bounces = d.russian_roulette_bounces;
    o.russian_roulette_survival = d.russian_roulette_survival;
    o.min_phonon_eV = d.min_phonon_eV;
    o.luke_sample_fraction = d.luke_sample_fraction;
    o.charge_max_dk_frac = d.charge_max_dk_frac;
    o.charge_dt_cap_s = d.charge_dt_cap_s;
    o.charge_sampling_dk_frac = d.charge_sampling_dk_frac;
    o.charge_stepping = static_cast<int32_t>(d.charge_stepping);
    o.charge_release = static_cast<int32_t>(d.charge_release);
    o.fermi_level_above_Ev_eV = d.fermi_level_above_Ev_eV;
    o.electrode_seed_max_gap = d.electrode_seed_max_gap;
    o.allow_unvalidated = d.allow_unvalidated ? 1 : 0;
    o.jump_to_ballistic = d.jump_to_ballistic.enabled ? 1 : 0;
    return o;
}

}  // namespace detail

// A device context for one crystal and detector (create once, run many times).
class GpuEngine {
public:
    GpuEngine(const cmpmc::CrystalConfig& cfg, const cmpmc::DetectorModel& det, int device = 0)
        : GpuEngine(cfg, 0, det, device) {}
    // The same with the lattice's kinematics mode (CrystalLattice::set_kinematics_mode).
    GpuEngine(const cmpmc::CrystalLattice& lattice, const cmpmc::DetectorModel& det, int device = 0)
        : GpuEngine(lattice.config(), static_cast<int>(lattice.kinematics_mode()), det, device) {}

    GpuEngine(const cmpmc::CrystalConfig& cfg, int kinematics_mode, const cmpmc::DetectorModel& det, int device)
        : ccfg_(detail::to_c(cfg)), cdet_(detail::to_c(det)), needs_mesh_(det.mesh_field_3d.has_value()),
          needs_mesh2_(!det.mesh_field_3d.has_value() && det.mesh_field_2d.has_value()) {
        detail::check(cmpmc_lattice_create(&ccfg_, &lat_), nullptr, "lattice");
        if (kinematics_mode != 0) detail::check(cmpmc_lattice_set_kinematics_mode(lat_, kinematics_mode), nullptr,
                                                "kinematics mode");
        const int st = cmpmc_gpu_create(lat_, &cdet_, device, &ctx_);
        if (st != CMPMC_OK) {
            cmpmc_lattice_destroy(lat_);
            detail::check(st, nullptr, "device context");
        }
        for (int i = 0; i < 3; ++i) {
            if (!det.surfaces[i].electrode_mask.has_value()) continue;
            const auto pads = detail::pads_of(*det.surfaces[i].electrode_mask);
            detail::check(cmpmc_gpu_set_electrode_mask(ctx_, i, pads.data(), pads.size()), ctx_, "electrode mask");
        }
    }
    ~GpuEngine() {
        cmpmc_gpu_destroy(ctx_);
        cmpmc_lattice_destroy(lat_);
        cmpmc_mesh_destroy(mesh_);
        cmpmc_mesh2d_destroy(mesh2_);
    }

    // DetectorModel::mesh_field_3d: the TriLinearMesh3D(vertices, potentials, tetrahedra)
    // the detector was built with (mesh_field.hpp:47-58).
    void set_mesh(const std::vector<cmpmc::Vec3>& vertices, const std::vector<double>& potentials,
                  const std::vector<std::array<int, 4>>& tets, double v_min_clamp = -1e30, double v_max_clamp = 1e30) {
        static_assert(sizeof(cmpmc::Vec3) == 3 * sizeof(double), "Vec3 layout");
        std::vector<int32_t> t(4 * tets.size());
        for (size_t i = 0; i < tets.size(); ++i)
            for (int j = 0; j < 4; ++j) t[4 * i + j] = tets[i][j];
        cmpmc_mesh* m = nullptr;
        detail::check(cmpmc_mesh_create(reinterpret_cast<const double*>(vertices.data()), potentials.data(),
                                        potentials.size(), t.data(), tets.size(), v_min_clamp, v_max_clamp, &m),
                      nullptr, "mesh");
        attach(m);
    }
    // The same for a mesh made by TriLinearMesh3D::build_cartesian_grid (mesh_field.hpp:131-189).
    template <class PotentialFn>
    void set_cartesian_mesh(double half_x, double half_y, double half_z, int nx, int ny, int nz, PotentialFn&& fn) {
        using Fn = std::remove_reference_t<PotentialFn>;
        auto thunk = [](const double p[3], void* user) -> double {
            return (*static_cast<Fn*>(user))(cmpmc::Vec3{p[0], p[1], p[2]});
        };
        cmpmc_mesh* m = nullptr;
        detail::check(cmpmc_mesh_build_cartesian(half_x, half_y, half_z, nx, ny, nz, thunk,
                                                 const_cast<void*>(static_cast<const void*>(&fn)), &m),
                      nullptr, "mesh");
        attach(m);
    }
    // DetectorModel::mesh_field_2d (used when there is no 3D mesh, engine.hpp:151-155): the
    // BiLinearMesh2D(vertices, potentials, triangles, axisymmetric_rz) (mesh_field.hpp:356-366).
    void set_mesh2d(const std::vector<cmpmc::geometry::BiLinearMesh2D::Point2D>& vertices,
                    const std::vector<double>& potentials, const std::vector<std::array<int, 3>>& triangles,
                    bool axisymmetric_rz = true) {
        static_assert(sizeof(cmpmc::geometry::BiLinearMesh2D::Point2D) == 2 * sizeof(double), "Point2D layout");
        std::vector<int32_t> t(3 * triangles.size());
        for (size_t i = 0; i < triangles.size(); ++i)
            for (int j = 0; j < 3; ++j) t[3 * i + j] = triangles[i][j];
        cmpmc_mesh2d* m = nullptr;
        detail::check(cmpmc_mesh2d_create(reinterpret_cast<const double*>(vertices.data()), potentials.data(),
                                          potentials.size(), t.data(), triangles.size(), axisymmetric_rz ? 1 : 0, &m),
                      nullptr, "2D mesh");
        attach2(m);
    }
    // The same for a mesh made by BiLinearMesh2D::build_grid (mesh_field.hpp:438-479).
    template <class PotentialFn2D>
    void set_grid_mesh2d(double u_min, double u_max, double v_min, double v_max, int nu, int nv, PotentialFn2D&& fn,
                         bool axisymmetric_rz = true) {
        using Fn = std::remove_reference_t<PotentialFn2D>;
        auto thunk = [](double u, double v, void* user) -> double { return (*static_cast<Fn*>(user))(u, v); };
        cmpmc_mesh2d* m = nullptr;
        detail::check(cmpmc_mesh2d_build_grid(u_min, u_max, v_min, v_max, nu, nv, thunk,
                                              const_cast<void*>(static_cast<const void*>(&fn)),
                                              axisymmetric_rz ? 1 : 0, &m),
                      nullptr, "2D mesh");
        attach2(m);
    }
    GpuEngine(const GpuEngine&) = delete;
    GpuEngine& operator=(const GpuEngine&) = delete;

    // run_events on the device; `engine` is the reference engine built from the same
    // lattice and detector (the generator calls its make_track).
    template <class Generator>
    cmpmc::RunResult run_events(uint64_t n_events, Generator&& generate, const cmpmc::RunOptions& options = {},
                                const GpuRunOptions& gpu = {}) {
        if (needs_mesh_ && !mesh_)
            throw std::invalid_argument("the detector has a mesh field: hand it over with set_mesh or set_cartesian_mesh");
        if (needs_mesh2_ && !mesh2_)
            throw std::invalid_argument("the detector has a 2D mesh field: hand it over with set_mesh2d or set_grid_mesh2d");
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<uint64_t> rng(4 * n_events), ph_off(n_events + 1, 0), ch_off(n_events + 1, 0);
        std::vector<double> injected(n_events, 0.0);
        std::vector<std::vector<cmpmc::PhononTrack>> ph(n_events);
        std::vector<std::vector<cmpmc::ChargeTrack>> ch(n_events);
        // generator on the host thread pool, one stream per event (parallel.hpp:102-109)
        const unsigned nt = options.threads ? options.threads : std::max(1u, std::thread::hardware_concurrency());
        std::atomic<uint64_t> next{0};
        std::exception_ptr error;
        std::mutex error_mutex;
        auto worker = [&]() {
            try {
                for (;;) {
                    const uint64_t ev = next.fetch_add(1);
                    if (ev >= n_events) return;
                    cmpmc::Rng r = cmpmc::Rng::for_stream(options.seed, ev);
                    cmpmc::EventInput in{ev, r, ph[ev], ch[ev], 0.0};
                    generate(in);
                    injected[ev] = in.injected_eV;
                    std::memcpy(&rng[4 * ev], r.s, 32);
                }
            } catch (...) {
                std::lock_guard<std::mutex> lock(error_mutex);
                if (!error) error = std::current_exception();
            }
        };
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
        if (error) std::rethrow_exception(error);
        std::vector<cmpmc::PhononTrack> phonons;
        std::vector<cmpmc::ChargeTrack> charges;
        for (uint64_t ev = 0; ev < n_events; ++ev) {
            phonons.insert(phonons.end(), ph[ev].begin(), ph[ev].end());
            charges.insert(charges.end(), ch[ev].begin(), ch[ev].end());
            ph_off[ev + 1] = phonons.size();
            ch_off[ev + 1] = charges.size();
        }
        static_assert(sizeof(cmpmc::PhononTrack) == sizeof(cmpmc_phonon_track), "PhononTrack layout");
        static_assert(sizeof(cmpmc::ChargeTrack) == sizeof(cmpmc_charge_track), "ChargeTrack layout");
        static_assert(sizeof(cmpmc::SensorHit) == sizeof(cmpmc_sensor_hit), "SensorHit layout");
        static_assert(sizeof(cmpmc::SimStats) == sizeof(cmpmc_sim_stats), "SimStats layout");
        cmpmc_run_desc d;
        std::memset(&d, 0, sizeof(d));
        d.n_events = n_events;
        d.rng_state = rng.data();
        d.injected_eV = injected.data();
        d.phonon_offsets = ph_off.data();
        d.phonons = reinterpret_cast<const cmpmc_phonon_track*>(phonons.data());
        if (!charges.empty()) {
            d.charge_offsets = ch_off.data();
            d.charges = reinterpret_cast<const cmpmc_charge_track*>(charges.data());
        }
        d.keep_hits = options.keep_hits ? 1 : 0;
        d.form = static_cast<int32_t>(gpu.form);
        d.kaplan_surrogate = gpu.kaplan_surrogate ? 1 : 0;
        d.seed = options.seed;
        cmpmc_run_out out;
        detail::check(cmpmc_gpu_run_events(ctx_, &d, &out), ctx_, "run_events");
        cmpmc::RunResult r;
        std::memcpy(&r.stats, &out.stats, sizeof(r.stats));
        r.hits.resize(out.n_hits);
        if (out.n_hits) std::memcpy(r.hits.data(), out.hits, out.n_hits * sizeof(cmpmc_sensor_hit));
        r.hit_offsets.assign(out.hit_offsets, out.hit_offsets + n_events + 1);
        r.threads_used = nt;
        r.wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return r;
    }

private:
    void attach(cmpmc_mesh* m) {
        const int st = cmpmc_gpu_set_mesh(ctx_, m);
        if (st != CMPMC_OK) {
            cmpmc_mesh_destroy(m);
            detail::check(st, ctx_, "mesh");
        }
        cmpmc_mesh_destroy(mesh_);
        mesh_ = m;
    }

    void attach2(cmpmc_mesh2d* m) {
        const int st = cmpmc_gpu_set_mesh2d(ctx_, m);
        if (st != CMPMC_OK) {
            cmpmc_mesh2d_destroy(m);
            detail::check(st, ctx_, "2D mesh");
        }
        cmpmc_mesh2d_destroy(mesh2_);
        mesh2_ = m;
    }

    cmpmc_crystal_config ccfg_;
    cmpmc_detector cdet_;
    bool needs_mesh_ = false;
    bool needs_mesh2_ = false;
    cmpmc_lattice* lat_ = nullptr;
    cmpmc_gpu_ctx* ctx_ = nullptr;
    cmpmc_mesh* mesh_ = nullptr;
    cmpmc_mesh2d* mesh2_ = nullptr;
};

namespace detail {

// The lattice and detector an engine was built with (see the file comment).
struct EngineRefs {
    const cmpmc::CrystalLattice* lattice;
    const cmpmc::DetectorModel* detector;
};
inline EngineRefs refs_of(const cmpmc::SimulationEngine& engine) {
    static_assert(sizeof(cmpmc::ChargePhysics) == sizeof(void*), "ChargePhysics holds one lattice reference");
    static_assert(sizeof(cmpmc::SimulationEngine) == 3 * sizeof(void*) &&
                      alignof(cmpmc::SimulationEngine) == alignof(void*),
                  "SimulationEngine is {const CrystalLattice&, const DetectorModel&, ChargePhysics}");
    EngineRefs r;
    std::memcpy(&r, static_cast<const void*>(&engine), sizeof(r));
    return r;
}

inline void append_bytes(std::vector<unsigned char>& k, const void* p, size_t n) {
    const auto* b = static_cast<const unsigned char*>(p);
    k.insert(k.end(), b, b + n);
}

// Everything a device context is built from: the crystal configuration, the kinematics
// mode, the detector image and the electrode pads (mesh nodes are handed over separately).
inline std::vector<unsigned char> context_key(const cmpmc::CrystalLattice& lat, const cmpmc::DetectorModel& det,
                                              int device) {
    std::vector<unsigned char> k;
    const cmpmc_crystal_config c = to_c(lat.config());
    const cmpmc_detector d = to_c(det);
    const int mode = static_cast<int>(lat.kinematics_mode());
    append_bytes(k, &device, sizeof(device));
    append_bytes(k, &mode, sizeof(mode));
    append_bytes(k, &c, sizeof(c));
    append_bytes(k, &d, sizeof(d));
    for (int i = 0; i < 3; ++i) {
        if (!det.surfaces[i].electrode_mask.has_value()) continue;
        const auto pads = pads_of(*det.surfaces[i].electrode_mask);
        append_bytes(k, &i, sizeof(i));
        if (!pads.empty()) append_bytes(k, pads.data(), pads.size() * sizeof(pads[0]));
    }
    return k;
}

struct CachedContext {
    const void* lattice;
    const void* detector;
    int device;
    std::vector<unsigned char> key;
    std::unique_ptr<GpuEngine> gpu;
    std::unique_ptr<std::mutex> busy;  // a device context serves one call at a time
};

struct ContextCache {
    std::mutex m;
    std::deque<CachedContext> entries;  // appends keep earlier entries in place
};
inline ContextCache& context_cache() {
    static ContextCache cache;
    return cache;
}

inline CachedContext& cached_context(const cmpmc::SimulationEngine& engine, int device) {
    const EngineRefs r = refs_of(engine);
    std::vector<unsigned char> key = context_key(*r.lattice, *r.detector, device);
    ContextCache& cache = context_cache();
    std::lock_guard<std::mutex> lock(cache.m);
    for (CachedContext& e : cache.entries) {
        if (e.lattice != r.lattice || e.detector != r.detector || e.device != device) continue;
        if (e.key != key) {  // the detector or lattice changed since: rebuild the context
            std::lock_guard<std::mutex> wait_idle(*e.busy);
            e.gpu.reset(new GpuEngine(*r.lattice, *r.detector, device));
            e.key = std::move(key);
        }
        return e;
    }
    CachedContext e{r.lattice, r.detector, device, std::move(key),
                    std::unique_ptr<GpuEngine>(new GpuEngine(*r.lattice, *r.detector, device)),
                    std::unique_ptr<std::mutex>(new std::mutex)};
    cache.entries.push_back(std::move(e));
    return cache.entries.back();
}

}  // namespace detail

// The cached device context of a reference engine (built on first use): hand a mesh field
// over with its set_mesh / set_cartesian_mesh / set_mesh2d / set_grid_mesh2d.
inline GpuEngine& gpu_engine_for(const cmpmc::SimulationEngine& engine, int device = 0) {
    return *detail::cached_context(engine, device).gpu;
}

// Drop-in for cmpmc::run_events(engine, n_events, generate, options) (parallel.hpp:76-78):
// the same arguments, the same RunResult; gpu selects the device and the form. Calls on
// the same engine and device are serialized; different engines run independently.
template <class Generator>
cmpmc::RunResult run_events(const cmpmc::SimulationEngine& engine, uint64_t n_events, Generator&& generate,
                            const cmpmc::RunOptions& options = {}, const GpuRunOptions& gpu = {}) {
    detail::CachedContext& c = detail::cached_context(engine, gpu.device);
    std::lock_guard<std::mutex> lock(*c.busy);
    return c.gpu->run_events(n_events, std::forward<Generator>(generate), options, gpu);
}

}  // namespace cmpmc_b200
