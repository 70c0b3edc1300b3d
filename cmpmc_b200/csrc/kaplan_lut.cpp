// kaplan_lut.cpp -- the Kaplan-cascade surrogate table (KaplanSurrogateLUT,
// superconductor/kaplan_film.hpp:336-383), built on the host.
//
// For each of 128 incident energies evenly spaced on [2 Delta, 40 Delta] the table keeps
// 512 complete outcomes of the film cascade (KaplanFilm::absorb_phonon): the absorbed
// fraction and every re-emitted phonon energy, both as fractions of the incident energy.
// The outcomes are drawn with the reference's generator (Rng(seed), default seed 1337) and
// the reference's cascade arithmetic (phys.cuh, host libm), so the table equals the
// reference's bit for bit. A lookup picks one of the two bracketing nodes with linear
// interpolation probabilities and one stored outcome of it, and rescales it to the incident
// energy; sub-gap energies and energies outside the table take the full cascade.
#include <algorithm>
#include <cstring>
#include <new>

#include "internal.hpp"

using namespace cmpmc_gpu;

namespace {

double node_energy(int ie, double two_delta) {
    return two_delta * (1.0 + (kLutEMaxDiv2Gap - 1.0) * (static_cast<double>(ie) / (kLutNE - 1)));
}

}  // namespace

extern "C" {

int cmpmc_kaplan_surrogate_create(const cmpmc_film_config* film, uint64_t seed, cmpmc_kaplan_lut** out) {
    if (!film || !out) return CMPMC_ERR_INVALID;
    *out = nullptr;
    cmpmc_kaplan_lut* t = new (std::nothrow) cmpmc_kaplan_lut();
    if (!t) return CMPMC_ERR_INVALID;
    t->film = film_view(*film);
    t->abs.resize(static_cast<size_t>(kLutNE) * kLutNS);
    t->off.assign(static_cast<size_t>(kLutNE) * kLutNS + 1, 0);
    t->refl.reserve(static_cast<size_t>(kLutNE) * kLutNS * 4);
    Rng rng;
    rng.seed(seed);
    const double two_delta = 2.0 * std::max(t->film.gap_energy, 1e-12);
    double refl_d[kKaplanCap];
    std::vector<double> work(4 * kKaplanCap);
    for (int ie = 0; ie < kLutNE; ++ie) {
        const double E = node_energy(ie, two_delta);
        for (int s = 0; s < kLutNS; ++s) {
            const int k = ie * kLutNS + s;
            KBuf r{refl_d, 0};
            t->abs[k] = static_cast<float>(film_absorb_phonon(t->film, E, r, work.data(), rng) / E);
            for (int i = 0; i < r.n; ++i) t->refl.push_back(static_cast<float>(r.d[i] / E));
            t->off[k + 1] = static_cast<uint32_t>(t->refl.size());
        }
    }
    *out = t;
    return CMPMC_OK;
}

void cmpmc_kaplan_surrogate_destroy(cmpmc_kaplan_lut* t) { delete t; }

int cmpmc_kaplan_surrogate_info(const cmpmc_kaplan_lut* t, uint64_t* n_outcomes, uint64_t* n_reflected) {
    if (!t) return CMPMC_ERR_INVALID;
    if (n_outcomes) *n_outcomes = t->abs.size();
    if (n_reflected) *n_reflected = t->refl.size();
    return CMPMC_OK;
}

int cmpmc_kaplan_surrogate_absorb(const cmpmc_kaplan_lut* t, double energy, uint64_t rng_state[4], double* refl,
                                  uint64_t cap, uint64_t* n_refl, double* edep) {
    if (!t || !rng_state || !n_refl || !edep || (cap && !refl)) return CMPMC_ERR_INVALID;
    Rng rng;
    for (int k = 0; k < 4; ++k) rng.s[k] = rng_state[k];
    const double two_delta = 2.0 * std::max(t->film.gap_energy, 1e-12);
    const double u = (energy / two_delta - 1.0) / (kLutEMaxDiv2Gap - 1.0) * (kLutNE - 1);
    int st = CMPMC_OK;
    if (film_is_subgap(t->film, energy) || u < 0.0 || u > kLutNE - 1) {
        double refl_d[kKaplanCap];
        std::vector<double> work(4 * kKaplanCap);
        KBuf r{refl_d, 0};
        *edep = film_absorb_phonon(t->film, energy, r, work.data(), rng);
        *n_refl = static_cast<uint64_t>(r.n);
        for (int i = 0; i < r.n && static_cast<uint64_t>(i) < cap; ++i) refl[i] = r.d[i];
        if (static_cast<uint64_t>(r.n) > cap) st = CMPMC_ERR_CAPACITY;
    } else {
        int ie = std::min(static_cast<int>(u), kLutNE - 2);
        if (rng.uniform() < (u - ie)) ++ie;
        const int k = ie * kLutNS + std::min(kLutNS - 1, static_cast<int>(rng.uniform() * kLutNS));
        const uint32_t r0 = t->off[k], r1 = t->off[k + 1];
        *n_refl = r1 - r0;
        for (uint32_t r = r0; r < r1 && r - r0 < cap; ++r) refl[r - r0] = energy * t->refl[r];
        if (r1 - r0 > cap) st = CMPMC_ERR_CAPACITY;
        *edep = energy * static_cast<double>(t->abs[k]);
    }
    for (int k = 0; k < 4; ++k) rng_state[k] = rng.s[k];
    return st;
}

}  // extern "C"
