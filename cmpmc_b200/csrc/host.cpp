// host.cpp -- configuration defaults, validation, record conversion and the canonical
// workload generators (host side of run_events, transport/parallel.hpp:76-148: the
// generator is user code that runs on the host and leaves each event's Rng state,
// initial stacks and injected energy for the device).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.hpp"

using namespace cmpmc_gpu;

namespace cmpmc_gpu {

Track track_from_record(const cmpmc_phonon_track& r) {
    Track t;
    t.pos = v3(r.pos[0], r.pos[1], r.pos[2]);
    t.k = v3(r.k_dir[0], r.k_dir[1], r.k_dir[2]);
    t.vg = v3(r.vg_dir[0], r.vg_dir[1], r.vg_dir[2]);
    t.E = r.energy;
    t.vmag = r.vg_mag;
    t.t = r.time;
    t.w = r.weight;
    t.bounces = r.bounces;
    t.mode = r.mode;
    return t;
}

void track_to_record(const Track& t, cmpmc_phonon_track& r) {
    std::memset(&r, 0, sizeof(r));
    r.pos[0] = t.pos.x; r.pos[1] = t.pos.y; r.pos[2] = t.pos.z;
    r.k_dir[0] = t.k.x; r.k_dir[1] = t.k.y; r.k_dir[2] = t.k.z;
    r.vg_dir[0] = t.vg.x; r.vg_dir[1] = t.vg.y; r.vg_dir[2] = t.vg.z;
    r.energy = t.E;
    r.vg_mag = t.vmag;
    r.time = t.t;
    r.weight = t.w;
    r.bounces = t.bounces;
    r.mode = static_cast<uint8_t>(t.mode);
}

Charge charge_from_record(const cmpmc_charge_track& r) {
    Charge c;
    c.pos = v3(r.pos[0], r.pos[1], r.pos[2]);
    c.p = v3(r.p_eV[0], r.p_eV[1], r.p_eV[2]);
    c.ekin = r.ekin;
    c.t = r.time;
    c.w = r.weight;
    c.valley = r.valley;
    c.type = r.type;
    return c;
}

void charge_to_record(const Charge& c, cmpmc_charge_track& r) {
    std::memset(&r, 0, sizeof(r));
    r.pos[0] = c.pos.x; r.pos[1] = c.pos.y; r.pos[2] = c.pos.z;
    r.p_eV[0] = c.p.x; r.p_eV[1] = c.p.y; r.p_eV[2] = c.p.z;
    r.ekin = c.ekin;
    r.time = c.t;
    r.weight = c.w;
    r.valley = static_cast<uint16_t>(c.valley);
    r.type = static_cast<uint8_t>(c.type);
    r.alive = 1;
}

Film film_view(const cmpmc_film_config& f) {
    Film o;
    o.film_absorption = f.film_absorption;
    o.film_thickness = f.film_thickness;
    o.v_sound = f.v_sound;
    o.gap_energy = f.gap_energy;
    o.phonon_lifetime = f.phonon_lifetime;
    o.phonon_lifetime_slope = f.phonon_lifetime_slope;
    o.low_qp_limit = f.low_qp_limit;
    o.high_qp_limit = f.high_qp_limit;
    o.subgap_absorption = f.subgap_absorption;
    o.absorber_gap = f.absorber_gap;
    o.absorber_eff = f.absorber_eff;
    o.absorber_eff_slope = f.absorber_eff_slope;
    o.temperature = f.temperature;
    o.keep_all_phonons = f.keep_all_phonons;
    o.loss_model = f.loss_model;
    o.phonon_loss_time = f.phonon_loss_time;
    return o;
}

Pad pad_view(const cmpmc_electrode_pad& p) {
    Pad o;
    o.shape = p.shape;
    o.channel = p.channel_id;
    o.cx = p.cx;
    o.cy = p.cy;
    o.r_min = p.r_min;
    o.r_max = p.r_max;
    o.phi_min = p.phi_min;
    o.phi_max = p.phi_max;
    o.fill = p.fill_fraction;
    return o;
}

Detector detector_view(const cmpmc_detector& d) {
    Detector D;
    std::memset(&D, 0, sizeof(D));
    D.radius = d.radius;
    D.half_z = d.half_z;
    D.e_field = v3(d.e_field[0], d.e_field[1], d.e_field[2]);
    for (int i = 0; i < 3; ++i) {
        const cmpmc_surface& s = d.surfaces[i];
        Surface& o = D.surf[i];
        o.prob_abs = s.prob_abs;
        o.prob_refl = s.prob_refl;
        o.refl_cutoff = s.refl_cutoff;
        o.anh_cutoff = s.anh_cutoff;
        o.prob_charge_abs = s.prob_charge_abs;
        o.prob_charge_spec = s.prob_charge_spec;
        o.min_k_elec = s.min_k_elec;
        o.min_k_hole = s.min_k_hole;
        o.spec_prob_const = s.spec_prob_const;
        o.n_spec = s.n_spec;
        o.n_diff = s.n_diff;
        o.n_anh = s.n_anh;
        o.has_film = s.has_film;
        o.has_amm = s.has_amm;
        o.amm_sub = Medium{s.amm_substrate[0], s.amm_substrate[1], s.amm_substrate[2]};
        o.amm_film = Medium{s.amm_film[0], s.amm_film[1], s.amm_film[2]};
        for (int k = 0; k < CMPMC_MAX_POLY; ++k) {
            o.spec[k] = s.spec_coeffs[k];
            o.diff[k] = s.diff_coeffs[k];
            o.anh[k] = s.anh_coeffs[k];
        }
        o.film = film_view(s.film);
    }
    D.max_bounces = d.max_bounces;
    D.rr_bounces = d.russian_roulette_bounces;
    D.rr_survival = d.russian_roulette_survival;
    D.min_phonon_eV = d.min_phonon_eV;
    D.luke_sample_fraction = d.luke_sample_fraction;
    D.charge_max_dk_frac = d.charge_max_dk_frac;
    D.charge_dt_cap_s = d.charge_dt_cap_s;
    D.charge_sampling_dk_frac = d.charge_sampling_dk_frac;
    D.charge_stepping = d.charge_stepping;
    D.fermi_level_above_Ev_eV = d.fermi_level_above_Ev_eV;
    D.charge_release = d.charge_release;
    D.electrode_seed_max_gap = d.electrode_seed_max_gap;
    return D;
}

int validate_config(const cmpmc_crystal_config& cfg, const cmpmc_detector& det, bool has_charges,
                    std::string& err) {
    // Guards of the reference (engine.hpp:165-168, 197-199, 407-409).
    for (int i = 0; i < 3; ++i)
        if (det.surfaces[i].demo_values && !det.allow_unvalidated) {
            err = "CMPMC: 'SurfaceProperty::demo_polynomial_*' is not validated (demonstration "
                  "reflection/down-conversion polynomials, not physically motivated). Set allow_unvalidated "
                  "= true to run it anyway.";
            return CMPMC_ERR_UNVALIDATED;
        }
    if (det.jump_to_ballistic) {
        if (!det.allow_unvalidated) {
            err = "CMPMC: 'jump_to_ballistic' is not validated. Set allow_unvalidated = true to run it anyway.";
            return CMPMC_ERR_UNVALIDATED;
        }
        err = "jump_to_ballistic (experimental) is not available on the device";
        return CMPMC_ERR_INVALID;
    }
    if (has_charges && cfg.iv_model == 2) {
        if (!det.allow_unvalidated) {
            err = "CMPMC: 'IVRateModel::Matrix' is not validated (Z_f = 2N-1 for every phonon (x4 vs "
                  "Jacoboni-Reggiani in Si) and Erginsoy impurity term changes valley). Set allow_unvalidated "
                  "= true to run it anyway.";
            return CMPMC_ERR_UNVALIDATED;
        }
        err = "IVRateModel::Matrix is not available on the device";
        return CMPMC_ERR_INVALID;
    }
    for (int i = 0; i < 3; ++i) {
        const cmpmc_surface& s = det.surfaces[i];
        if (s.has_mask) {
            err = "electrode masks are attached with cmpmc_gpu_set_electrode_mask (has_mask must be 0)";
            return CMPMC_ERR_INVALID;
        }
        if (s.has_amm && !(s.amm_substrate[0] > 0.0 && s.amm_substrate[1] > 0.0 && s.amm_substrate[2] > 0.0 &&
                           s.amm_film[0] > 0.0 && s.amm_film[1] > 0.0 && s.amm_film[2] > 0.0)) {
            err = "AMM interface: densities and sound speeds must be positive";
            return CMPMC_ERR_INVALID;
        }
        if (s.n_spec < 0 || s.n_spec > CMPMC_MAX_POLY || s.n_diff < 0 || s.n_diff > CMPMC_MAX_POLY ||
            s.n_anh < 0 || s.n_anh > CMPMC_MAX_POLY) {
            err = "surface polynomial has too many coefficients";
            return CMPMC_ERR_INVALID;
        }
    }
    if (det.charge_release < 0 || det.charge_release > 2) {
        err = "charge_release must be RecordOnly, BulkDebye or ElectrodeFilm";
        return CMPMC_ERR_INVALID;
    }
    if (det.kinematics_mode != 0) {
        err = "only KinematicsMode::Octahedral is available on the device";
        return CMPMC_ERR_INVALID;
    }
    if (!(det.radius > 0.0) || !(det.half_z > 0.0)) {
        err = "cylinder radius and half height must be positive";
        return CMPMC_ERR_INVALID;
    }
    return CMPMC_OK;
}

}  // namespace cmpmc_gpu

namespace {

// origin uniform in the cylinder: rejection in (x, y), then z
V3 uniform_origin(double R, double h, Rng& rng) {
    double x, y;
    do {
        x = (2.0 * rng.uniform() - 1.0) * R;
        y = (2.0 * rng.uniform() - 1.0) * R;
    } while (x * x + y * y > R * R);
    const double z = (2.0 * rng.uniform() - 1.0) * h;
    return v3(x, y, z);
}

struct Counts {
    uint64_t phonons, charges;
};

// ---- recoil workloads: EnergyPartition::partition_deposit (partition_host.cpp) with the
// electron-recoil defaults and the pair cap of the recoil batch ----

bool is_recoil(int wl) { return wl == CMPMC_WL_RECOIL || wl == CMPMC_WL_RECOIL_LIGHT; }

constexpr uint32_t kRecoilMaxPairs = 4096;
constexpr uint32_t kRecoilMaxPhonons = 5000;      // PartitionOptions::max_sampled_phonons default
constexpr uint32_t kRecoilLightMaxPhonons = 20;

cmpmc_partition_options recoil_options(int wl) {
    cmpmc_partition_options o = default_partition_options();
    o.max_sampled_pairs = kRecoilMaxPairs;
    o.max_sampled_phonons = (wl == CMPMC_WL_RECOIL) ? kRecoilMaxPhonons : kRecoilLightMaxPhonons;
    return o;
}

// First draws of a recoil event: deposit energy, origin, then the pair count.
PartitionPlan recoil_plan(int wl, const cmpmc_crystal_config& cfg, const cmpmc_detector& det, Rng& rng, V3& pos) {
    const double u = rng.uniform();
    const double edep = (wl == CMPMC_WL_RECOIL) ? 10.0 * std::pow(10.0, 3.0 * u) : 10.0 * std::pow(10.0, u);
    pos = uniform_origin(det.radius, det.half_z, rng);
    return plan_partition(cfg, edep, false, recoil_options(wl), rng);
}

Counts counts_of(int wl, uint64_t ev) {
    switch (wl) {
        case CMPMC_WL_SINGLE_L_ORIGIN: return {1, 0};
        case CMPMC_WL_MIXED_ENERGY: return {100, 0};
        case CMPMC_WL_PAIR_DRIFT: return {0, 2};
        case CMPMC_WL_SINGLE_L_VOLUME: return {1, 0};
        case CMPMC_WL_TEST_PARALLEL: return (ev % 2 == 0) ? Counts{1, 0} : Counts{0, 2};
        case CMPMC_WL_PUBLISHED_PHONON: return {1, 0};
        case CMPMC_WL_PUBLISHED_PAIR: return {0, 2};
        default: return {0, 0};
    }
}

void gen_event(int wl, const Lattice& L, const cmpmc_crystal_config& cfg, const cmpmc_detector& det, uint64_t ev,
               Rng& rng, cmpmc_phonon_track* ph, cmpmc_charge_track* ch, double& injected) {
    injected = 0.0;
    const V3 origin = v3(0.0, 0.0, 0.0);
    switch (wl) {
        case CMPMC_WL_RECOIL:
        case CMPMC_WL_RECOIL_LIGHT: {
            V3 pos;
            const PartitionPlan d = recoil_plan(wl, cfg, det, rng, pos);
            fill_partition(L, cfg, d, recoil_options(wl), pos, 0.0, rng, ch, ph);
            injected += d.edep;
            break;
        }
        case CMPMC_WL_SINGLE_L_ORIGIN: {
            const V3 d = rng.isotropic_dir();
            track_to_record(make_track(L, origin, d, 0, 7.5e-3, 0.0, 1.0), ph[0]);
            injected += 7.5e-3;
            break;
        }
        case CMPMC_WL_MIXED_ENERGY: {
            for (int j = 0; j < 100; ++j) {
                const double E = 1e-3 * std::exp(std::log(30.0) * rng.uniform());
                const double um = rng.uniform();
                const int m = um < 0.10 ? 0 : (um < 0.46 ? 2 : 1);
                const V3 p = uniform_origin(det.radius, det.half_z, rng);
                const V3 d = rng.isotropic_dir();
                track_to_record(make_track(L, p, d, m, E, 0.0, 1.0), ph[j]);
                injected += E;
            }
            break;
        }
        case CMPMC_WL_PAIR_DRIFT: {
            const V3 p = uniform_origin(det.radius, det.half_z, rng);
            const int v = static_cast<int>(static_cast<uint16_t>(rng.next_u64() % 4));
            const V3 de = rng.isotropic_dir();
            charge_to_record(make_charge(L, 1, p, de, 1e-6, v, 0.0), ch[0]);
            const V3 dh = rng.isotropic_dir();
            charge_to_record(make_charge(L, 2, p, dh, 1e-6, 0, 0.0), ch[1]);
            break;
        }
        case CMPMC_WL_SINGLE_L_VOLUME: {
            const V3 p = uniform_origin(det.radius, det.half_z, rng);
            const V3 d = rng.isotropic_dir();
            track_to_record(make_track(L, p, d, 0, 7.5e-3, 0.0, 1.0), ph[0]);
            injected += 7.5e-3;
            break;
        }
        case CMPMC_WL_PUBLISHED_PHONON: {  // benchmarks/cmpmc_bench.cpp:63-67
            const double u = rng.uniform();
            const int m = u < 0.53539 ? 2 : (u < 0.90217 ? 1 : 0);
            const V3 d = rng.isotropic_dir();
            track_to_record(make_track(L, origin, d, m, 7.5e-3, 0.0, 1.0), ph[0]);
            injected += 7.5e-3;
            break;
        }
        case CMPMC_WL_PUBLISHED_PAIR:
        case CMPMC_WL_TEST_PARALLEL: {
            if (wl == CMPMC_WL_TEST_PARALLEL && ev % 2 == 0) {
                const V3 d = rng.isotropic_dir();
                track_to_record(make_track(L, origin, d, 1, 7.5e-3, 0.0, 1.0), ph[0]);
                injected += 7.5e-3;
            } else {
                const uint64_t nv = static_cast<uint64_t>(L.n_valleys);
                const int v = static_cast<int>(static_cast<uint16_t>(rng.uniform() * static_cast<double>(nv)) % nv);
                const V3 de = rng.isotropic_dir();
                charge_to_record(make_charge(L, 1, origin, de, 1e-6, v, 0.0), ch[0]);
                const V3 dh = rng.isotropic_dir();
                charge_to_record(make_charge(L, 2, origin, dh, 1e-6, 0, 0.0), ch[1]);
            }
            break;
        }
        default: break;
    }
}

}  // namespace

extern "C" {

double cmpmc_cr_log(double x) { return crmath::log(x); }

double cmpmc_amm_transmission(const double sub[3], const double film[3], int longitudinal, double cos_theta) {
    if (!sub || !film) return 0.0;
    return amm_transmission(Medium{sub[0], sub[1], sub[2]}, Medium{film[0], film[1], film[2]}, longitudinal != 0,
                            cos_theta);
}
double cmpmc_cr_sin(double x) { return crmath::sin(x); }
double cmpmc_cr_cos(double x) { return crmath::cos(x); }

int cmpmc_abi_sizes(size_t* out, int n) {
    const size_t sz[] = {sizeof(cmpmc_phonon_track), sizeof(cmpmc_charge_track), sizeof(cmpmc_sensor_hit),
                         sizeof(cmpmc_sim_stats),    sizeof(cmpmc_crystal_config), sizeof(cmpmc_film_config),
                         sizeof(cmpmc_surface),      sizeof(cmpmc_detector),      sizeof(cmpmc_run_desc),
                         sizeof(cmpmc_run_out),      sizeof(cmpmc_adjoint_desc), sizeof(cmpmc_adjoint_out)};
    for (int i = 0; i < n && i < static_cast<int>(sizeof(sz) / sizeof(sz[0])); ++i) out[i] = sz[i];
    return CMPMC_GPU_ABI_VERSION;
}

// DetectorModel defaults (engine.hpp:96-150): Al Kaplan films on both faces
// (SurfaceProperty::diffuse_al_sensor_surface, surface_property.hpp:98-103) and a bare
// diffuse side wall (surface_property.hpp:104-114).
void cmpmc_film_aluminum(cmpmc_film_config* f) {
    std::memset(f, 0, sizeof(*f));
    f->film_absorption = 0.20;
    f->film_thickness = 600.0 * 1e-9;
    f->v_sound = 3260.0;
    f->gap_energy = 173.715 * 1e-6;
    f->phonon_lifetime = 242.0 * 1e-12;
    f->phonon_lifetime_slope = 0.29;
    f->low_qp_limit = 3.0;
    f->high_qp_limit = 0.0;
    f->subgap_absorption = 0.10;
    f->absorber_gap = 0.0;
    f->absorber_eff = 1.0;
    f->absorber_eff_slope = 0.0;
    f->temperature = 0.05e-3;
    f->keep_all_phonons = 1;
    f->loss_model = 0;
    f->phonon_loss_time = 0.0;
}

void cmpmc_detector_default(cmpmc_detector* d) {
    std::memset(d, 0, sizeof(*d));
    d->radius = 3.81 * 1e-2;
    d->half_z = 1.27 * 1e-2;
    d->e_field[2] = -0.0 / (2.54 * 1e-2);
    for (int i = 0; i < 3; ++i) {
        cmpmc_surface& s = d->surfaces[i];
        s.prob_abs = 0.0;
        s.prob_refl = 1.0;
        s.refl_cutoff = 350.0;
        s.anh_cutoff = 520.0;
        s.prob_charge_abs = 1.0;
        s.prob_charge_spec = 0.0;
        s.n_spec = 1;
        s.spec_coeffs[0] = 0.0;
        s.n_diff = 1;
        s.diff_coeffs[0] = 1.0;
        s.n_anh = 0;
        s.spec_prob_const = 0.0;
        if (i < 2) {
            s.prob_abs = 1.0;
            s.has_film = 1;
            cmpmc_film_aluminum(&s.film);
        }
    }
    d->max_bounces = 5000;
    d->min_phonon_eV = 10.0 * 1e-6;
    d->luke_sample_fraction = 1.0;
    d->charge_max_dk_frac = 0.05;
    d->charge_dt_cap_s = 100.0 * 1e-12;
    d->charge_stepping = 0;
    d->charge_sampling_dk_frac = 0.25;
    d->charge_release = 0;
    d->fermi_level_above_Ev_eV = -1.0;
    d->electrode_seed_max_gap = 80.0;
    d->russian_roulette_bounces = 0;
    d->russian_roulette_survival = 0.5;
}

int cmpmc_generate(const cmpmc_lattice* lat, const cmpmc_detector* det, int workload, uint64_t seed,
                   uint64_t first_event, uint64_t n_events, int n_threads, uint64_t* rng_state,
                   double* injected_eV, uint64_t* phonon_offsets, cmpmc_phonon_track* phonons,
                   uint64_t phonon_cap, uint64_t* n_phonons, uint64_t* charge_offsets,
                   cmpmc_charge_track* charges, uint64_t charge_cap, uint64_t* n_charges) {
    if (!lat || !det || !rng_state || !injected_eV || !phonon_offsets || !charge_offsets) return CMPMC_ERR_INVALID;
    if (workload != CMPMC_WL_SINGLE_L_ORIGIN && workload != CMPMC_WL_MIXED_ENERGY &&
        workload != CMPMC_WL_PAIR_DRIFT && workload != CMPMC_WL_SINGLE_L_VOLUME &&
        workload != CMPMC_WL_TEST_PARALLEL && workload != CMPMC_WL_PUBLISHED_PHONON &&
        workload != CMPMC_WL_PUBLISHED_PAIR && !is_recoil(workload))
        return CMPMC_ERR_INVALID;
    const Lattice& L = lat->view;
    int nt = n_threads > 0 ? n_threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    if (static_cast<uint64_t>(nt) > n_events) nt = static_cast<int>(std::max<uint64_t>(1, n_events));
    auto parallel = [&](auto&& body) {
        if (nt <= 1) {
            body(uint64_t{0}, n_events);
            return;
        }
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) pool.emplace_back(body, n_events * t / nt, n_events * (t + 1) / nt);
        for (auto& th : pool) th.join();
    };
    // counts per event (recoil events: from the draws up to the pair count)
    std::vector<Counts> cnt(n_events);
    parallel([&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            if (is_recoil(workload)) {
                Rng rng = Rng::for_stream(seed, first_event + i);
                V3 pos;
                const PartitionPlan d = recoil_plan(workload, lat->cfg, *det, rng, pos);
                cnt[i] = {d.phonons_sampled, 2 * d.pairs_sampled};
            } else {
                cnt[i] = counts_of(workload, first_event + i);
            }
        }
    });
    uint64_t np = 0, nc = 0;
    phonon_offsets[0] = 0;
    charge_offsets[0] = 0;
    for (uint64_t i = 0; i < n_events; ++i) {
        np += cnt[i].phonons;
        nc += cnt[i].charges;
        phonon_offsets[i + 1] = np;
        charge_offsets[i + 1] = nc;
    }
    if (n_phonons) *n_phonons = np;
    if (n_charges) *n_charges = nc;
    if (np > phonon_cap || nc > charge_cap) return CMPMC_ERR_CAPACITY;
    if ((np && !phonons) || (nc && !charges)) return CMPMC_ERR_INVALID;
    parallel([&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            Rng rng = Rng::for_stream(seed, first_event + i);
            gen_event(workload, L, lat->cfg, *det, first_event + i, rng,
                      phonons ? phonons + phonon_offsets[i] : nullptr, charges ? charges + charge_offsets[i] : nullptr,
                      injected_eV[i]);
            for (int k = 0; k < 4; ++k) rng_state[4 * i + k] = rng.s[k];
        }
    });
    return CMPMC_OK;
}

int cmpmc_mask_supercdms_qet(double R, double fill, cmpmc_electrode_pad out[5]) {
    if (!out) return CMPMC_ERR_INVALID;
    std::memset(out, 0, 5 * sizeof(cmpmc_electrode_pad));
    out[0] = {CMPMC_PAD_DISK, 0, 0.0, 0.0, 0.0, 0.55 * R, 0.0, kTwoPi, fill};
    const double gap = 2.0 * (kPi / 180.0);
    const double span = kTwoPi / 3.0;
    for (int s = 0; s < 3; ++s)
        out[1 + s] = {CMPMC_PAD_ANNULAR_SECTOR, s + 1, 0.0, 0.0, 0.57 * R, 0.90 * R, s * span + 0.5 * gap,
                      (s + 1) * span - 0.5 * gap, fill};
    out[4] = {CMPMC_PAD_ANNULAR_SECTOR, 4, 0.0, 0.0, 0.92 * R, 0.98 * R, 0.0, kTwoPi, fill};
    return CMPMC_OK;
}

int cmpmc_mask_rectangular_grid(int nx, int ny, double pitch_x, double pitch_y, double hw, double hh, double fill,
                                cmpmc_electrode_pad* out, uint64_t cap, uint64_t* n) {
    if (nx < 0 || ny < 0) return CMPMC_ERR_INVALID;
    const uint64_t total = static_cast<uint64_t>(nx) * static_cast<uint64_t>(ny);
    if (n) *n = total;
    if (total > cap) return CMPMC_ERR_CAPACITY;
    if (total && !out) return CMPMC_ERR_INVALID;
    int32_t ch = 0;
    for (int ix = 0; ix < nx; ++ix) {
        const double cx = (ix - 0.5 * (nx - 1)) * pitch_x;
        for (int iy = 0; iy < ny; ++iy) {
            const double cy = (iy - 0.5 * (ny - 1)) * pitch_y;
            out[ch] = {CMPMC_PAD_RECTANGLE, ch, cx, cy, hw, hh, 0.0, 0.0, fill};
            ++ch;
        }
    }
    return CMPMC_OK;
}

int cmpmc_mask_find_channel(const cmpmc_electrode_pad* pads, uint64_t n, const double pos[3], uint64_t rng_state[4],
                            int32_t* channel) {
    if ((n && !pads) || !pos || !rng_state || !channel) return CMPMC_ERR_INVALID;
    std::vector<Pad> p(n);
    for (uint64_t i = 0; i < n; ++i) p[i] = pad_view(pads[i]);
    Rng rng;
    for (int k = 0; k < 4; ++k) rng.s[k] = rng_state[k];
    *channel = find_channel(p.data(), static_cast<int>(n), pos[0], pos[1], rng);
    for (int k = 0; k < 4; ++k) rng_state[k] = rng.s[k];
    return CMPMC_OK;
}

int cmpmc_recoil_mesh(const cmpmc_detector* det, cmpmc_mesh** out) {
    if (!det || !out) return CMPMC_ERR_INVALID;
    return cmpmc_mesh_build_cartesian(det->radius, det->radius, det->half_z, 58, 58, 57, cmpmc_recoil_potential,
                                      const_cast<cmpmc_detector*>(det), out);
}

}  // extern "C"
