// partition_host.cpp -- the input side of the transport on the host: the C ABI of the
// ionisation-yield models and of EnergyPartition::partition_deposit (partition.cuh, shared
// with the device), and StepAccumulator / HitMerger (energy_partition.hpp:182-323), which
// turns primary-particle steps into initial stacks. The outputs are compared bit for bit
// with the reference's; the host runs with the platform libm, as the reference does.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace cmpmc_gpu;

namespace cmpmc_gpu {

cmpmc_partition_options default_partition_options() {
    cmpmc_partition_options o;
    std::memset(&o, 0, sizeof(o));
    o.niel_model = CMPMC_NIEL_LINDHARD;
    o.use_fano_fluctuations = 1;
    o.use_charge_cloud = 1;
    o.max_sampled_pairs = 1000;
    o.max_sampled_phonons = 5000;
    o.emp_energy_dependent_k = 1;
    o.emp_k_fixed = 0.157;
    o.emp_k_low = 0.080;
    o.emp_k_high = 0.157;
    o.emp_e_low_eV = 100.0;
    o.emp_e_high_eV = 2000.0;
    return o;
}

}  // namespace cmpmc_gpu

// StepAccumulator + HitMerger (energy_partition.hpp:194-323). The merged secondaries go to
// the merger's own output lists, which cmpmc_hit_merger_take hands to the caller.
struct cmpmc_hit_merger {
    const cmpmc_lattice* lat;
    double combining_step_length;
    cmpmc_partition_options opts;
    // StepAccumulator
    int32_t track_id = -1;
    uint32_t n_steps = 0;
    V3 start_pos{0.0, 0.0, 0.0}, end_pos{0.0, 0.0, 0.0};
    double time_s = 0.0, edep_eV = 0.0, eniel_eV = 0.0;
    bool is_charged = true;
    std::vector<cmpmc_charge_track> charges;
    std::vector<cmpmc_phonon_track> phonons;

    void clear() {
        n_steps = 0;
        start_pos = end_pos = v3(0.0, 0.0, 0.0);
        time_s = edep_eV = eniel_eV = 0.0;
        is_charged = true;
    }
    void add(const cmpmc_primary_step& s) {
        if (n_steps == 0) {
            track_id = s.track_id;
            start_pos = v3(s.start_pos[0], s.start_pos[1], s.start_pos[2]);
            is_charged = s.is_charged != 0;
        }
        end_pos = v3(s.end_pos[0], s.end_pos[1], s.end_pos[2]);
        time_s = std::max(time_s, s.time_s);
        edep_eV += s.edep_eV;
        eniel_eV += s.eniel_eV;
        ++n_steps;
    }
    // HitMerger::flush (energy_partition.hpp:268-316)
    cmpmc_partition_result flush(Rng& rng) {
        cmpmc_partition_result res;
        std::memset(&res, 0, sizeof(res));
        res.lindhard_yield = 1.0;
        res.charge_weight = 1.0;
        res.phonon_weight = 1.0;
        if (n_steps == 0 || (edep_eV <= 0.0 && eniel_eV <= 0.0)) {
            clear();
            return res;
        }
        const size_t c0 = charges.size(), p0 = phonons.size();
        const double total_e = edep_eV + eniel_eV;
        const bool is_nr = eniel_eV > 0.5 * total_e;
        const V3 mid = (start_pos + end_pos) * 0.5;
        const PartitionPlan d = plan_partition(lat->cfg, total_e, is_nr, opts, rng);
        charges.resize(c0 + 2 * d.pairs_sampled);
        phonons.resize(p0 + d.phonons_sampled);
        fill_partition(lat->view, lat->cfg, d, opts, mid, time_s, rng, charges.data() + c0, phonons.data() + p0);
        res = result_of(d);
        // charged tracks with a chord: secondaries spread along it, steps dl +- dl/6
        const V3 traj = end_pos - start_pos;
        const double len = norm(traj);
        const size_t nsec = (charges.size() - c0) + (phonons.size() - p0);
        if (is_charged && len > 1e-7 && nsec > 1) {
            const V3 tdir = vdiv(traj, len);
            const double dl = len / static_cast<double>(nsec);
            const double sigl = dl / 6.0;
            V3 cur = start_pos;
            for (size_t i = c0; i < charges.size(); ++i) {
                cur = cur + tdir * std::max(0.0, dl + sigl * rng_normal(rng));
                std::memcpy(charges[i].pos, &cur, sizeof(double) * 3);
            }
            for (size_t i = p0; i < phonons.size(); ++i) {
                cur = cur + tdir * std::max(0.0, dl + sigl * rng_normal(rng));
                std::memcpy(phonons[i].pos, &cur, sizeof(double) * 3);
            }
        }
        clear();
        return res;
    }
    static cmpmc_partition_result result_of(const PartitionPlan& d) {
        cmpmc_partition_result r;
        std::memset(&r, 0, sizeof(r));
        r.total_edep_eV = d.edep;
        r.ionizing_eV = d.ionizing;
        r.niel_eV = d.niel;
        r.lindhard_yield = d.yield;
        r.n_pairs_true = d.pairs_true;
        r.n_pairs_sampled = d.pairs_sampled;
        r.n_phonons_true = d.phonons_true;
        r.n_phonons_sampled = d.phonons_sampled;
        r.charge_weight = d.charge_weight;
        r.phonon_weight = d.phonon_weight;
        r.prompt_phonon_eV = d.prompt_eV;
        return r;
    }
};

namespace {

bool options_ok(const cmpmc_partition_options& o) {
    return o.niel_model >= CMPMC_NIEL_LINDHARD && o.niel_model <= CMPMC_NIEL_EMPIRICAL && o.max_sampled_pairs > 0 &&
           o.max_sampled_phonons > 0;
}

Rng rng_of(const uint64_t s[4]) {
    Rng r;
    for (int i = 0; i < 4; ++i) r.s[i] = s[i];
    return r;
}

void store_rng(const Rng& r, uint64_t s[4]) {
    for (int i = 0; i < 4; ++i) s[i] = r.s[i];
}

}  // namespace

extern "C" {

void cmpmc_partition_options_default(cmpmc_partition_options* o) {
    if (o) *o = default_partition_options();
}

double cmpmc_ionization_yield(const cmpmc_crystal_config* cfg, int niel_model, double energy_eV,
                              const cmpmc_partition_options* opts) {
    if (!cfg) return 0.0;
    const cmpmc_partition_options o = opts ? *opts : default_partition_options();
    return ionization_yield(niel_model, energy_eV, *cfg, o);
}

double cmpmc_lindhard_yield(const cmpmc_crystal_config* cfg, double energy_eV, double z1, double a1) {
    if (!cfg) return 0.0;
    return lindhard_yield(energy_eV, *cfg, z1, a1);
}

uint64_t cmpmc_sample_fano_binomial(double mean, double fano, uint64_t rng_state[4]) {
    if (!rng_state) return 0;
    Rng r = rng_of(rng_state);
    const uint64_t n = sample_fano_binomial(mean, fano, r);
    store_rng(r, rng_state);
    return n;
}

int cmpmc_partition_deposit(const cmpmc_lattice* lat, const double pos[3], double time_s, double total_edep_eV,
                            int is_nuclear_recoil, const cmpmc_partition_options* opts, uint64_t rng_state[4],
                            cmpmc_charge_track* charges, uint64_t charge_cap, uint64_t* n_charges,
                            cmpmc_phonon_track* phonons, uint64_t phonon_cap, uint64_t* n_phonons,
                            cmpmc_partition_result* result) {
    if (!lat || !pos || !rng_state || !n_charges || !n_phonons) return CMPMC_ERR_INVALID;
    const cmpmc_partition_options o = opts ? *opts : default_partition_options();
    if (!options_ok(o)) return CMPMC_ERR_INVALID;
    // the NIEL yields and pair counts are undefined for a non-finite deposit: refuse it
    if (!std::isfinite(total_edep_eV) || !std::isfinite(time_s) || !std::isfinite(pos[0]) || !std::isfinite(pos[1]) ||
        !std::isfinite(pos[2]))
        return CMPMC_ERR_INVALID;
    Rng r = rng_of(rng_state);
    const PartitionPlan d = plan_partition(lat->cfg, total_edep_eV, is_nuclear_recoil != 0, o, r);
    *n_charges = 2 * d.pairs_sampled;
    *n_phonons = d.phonons_sampled;
    if (*n_charges > charge_cap || *n_phonons > phonon_cap || (*n_charges && !charges) || (*n_phonons && !phonons))
        return CMPMC_ERR_CAPACITY;  // no draw is kept: the caller retries with the sizes above
    fill_partition(lat->view, lat->cfg, d, o, v3(pos[0], pos[1], pos[2]), time_s, r, charges, phonons);
    store_rng(r, rng_state);
    if (result) *result = cmpmc_hit_merger::result_of(d);
    return CMPMC_OK;
}

int cmpmc_hit_merger_create(const cmpmc_lattice* lat, double combining_step_length_m,
                            const cmpmc_partition_options* opts, cmpmc_hit_merger** out) {
    if (!lat || !out) return CMPMC_ERR_INVALID;
    *out = nullptr;
    const cmpmc_partition_options o = opts ? *opts : default_partition_options();
    if (!options_ok(o)) return CMPMC_ERR_INVALID;
    cmpmc_hit_merger* m = new (std::nothrow) cmpmc_hit_merger();
    if (!m) return CMPMC_ERR_INVALID;
    m->lat = lat;
    m->combining_step_length = combining_step_length_m;
    m->opts = o;
    *out = m;
    return CMPMC_OK;
}

void cmpmc_hit_merger_destroy(cmpmc_hit_merger* m) { delete m; }

// HitMerger::process_step (energy_partition.hpp:236-266)
int cmpmc_hit_merger_process_steps(cmpmc_hit_merger* m, const cmpmc_primary_step* steps, uint64_t n_steps,
                                   uint64_t rng_state[4], uint64_t* n_flushes) {
    if (!m || (n_steps && !steps) || !rng_state) return CMPMC_ERR_INVALID;
    Rng r = rng_of(rng_state);
    uint64_t flushes = 0;
    for (uint64_t i = 0; i < n_steps; ++i) {
        const cmpmc_primary_step& s = steps[i];
        const V3 end = v3(s.end_pos[0], s.end_pos[1], s.end_pos[2]);
        const double dist = norm(end - m->end_pos);
        const bool do_add = m->n_steps == 0 || dist < m->combining_step_length || s.hit_boundary || s.track_stopped;
        const bool has_energy = s.edep_eV > 0.0 || s.eniel_eV > 0.0;
        if (do_add && has_energy) m->add(s);
        const bool ready = m->n_steps > 0 && (norm(end - m->end_pos) >= m->combining_step_length || !do_add ||
                                              s.hit_boundary || s.track_stopped);
        if (ready) {
            m->flush(r);
            ++flushes;
        }
        if (!do_add && has_energy) m->add(s);
    }
    store_rng(r, rng_state);
    if (n_flushes) *n_flushes = flushes;
    return CMPMC_OK;
}

int cmpmc_hit_merger_flush(cmpmc_hit_merger* m, uint64_t rng_state[4], cmpmc_partition_result* result) {
    if (!m || !rng_state) return CMPMC_ERR_INVALID;
    Rng r = rng_of(rng_state);
    const cmpmc_partition_result res = m->flush(r);
    store_rng(r, rng_state);
    if (result) *result = res;
    return CMPMC_OK;
}

int cmpmc_hit_merger_take(cmpmc_hit_merger* m, cmpmc_charge_track* charges, uint64_t charge_cap,
                          uint64_t* n_charges, cmpmc_phonon_track* phonons, uint64_t phonon_cap,
                          uint64_t* n_phonons) {
    if (!m || !n_charges || !n_phonons) return CMPMC_ERR_INVALID;
    *n_charges = m->charges.size();
    *n_phonons = m->phonons.size();
    if (*n_charges > charge_cap || *n_phonons > phonon_cap || (*n_charges && !charges) || (*n_phonons && !phonons))
        return CMPMC_ERR_CAPACITY;
    if (*n_charges) std::memcpy(charges, m->charges.data(), *n_charges * sizeof(cmpmc_charge_track));
    if (*n_phonons) std::memcpy(phonons, m->phonons.data(), *n_phonons * sizeof(cmpmc_phonon_track));
    m->charges.clear();
    m->phonons.clear();
    return CMPMC_OK;
}

}  // extern "C"
