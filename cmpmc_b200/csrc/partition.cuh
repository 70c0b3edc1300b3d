// partition.cuh -- EnergyPartition::partition_deposit and its helpers, shared by the host
// (partition_host.cpp, the generators in host.cpp) and the device (partition_gpu.cu).
//
// Restates, with the reference's draw order and operation order:
//   * niel_models.hpp:43-176: Lindhard (Lewin-Smith form), Lewin-Smith, IMPACT@TUNL,
//     Sarkis and the CDMSlite empirical k(E) yields, and their dispatcher;
//   * niel_models.hpp:178-263: the interpolated Fano-binomial pair-number sampler;
//   * charge_kernels.hpp:131-150: the charge-cloud radius and offsets;
//   * energy_partition.hpp:78-167: partition_deposit, split into the draws up to the pair
//     count (plan_partition, which fixes the output sizes) and the rest (fill_partition).
// The transcendentals are phys.cuh's m_*: the platform libm on the host (so the host
// generators reproduce the reference bit for bit) and the correctly rounded functions on
// the device (which differ from the host's only where the platform libm is not correctly
// rounded, e.g. the last bit of cbrt in the charge-cloud radius).
#pragma once

#include <stdint.h>
#include <string.h>

#include "../../include/cmpmc_gpu.h"
#include "transport.cuh"

namespace cmpmc_gpu {

// partition_deposit in two parts: the draws up to the pair count, which fix the sizes
struct PartitionPlan {
    double edep, yield, ionizing, niel;
    uint64_t pairs_true, pairs_sampled, phonons_true, phonons_sampled;
    double charge_weight, phonon_weight, prompt_eV;
};


// the initial-stack records (zero padding, as the host's record conversion)
CMPMC_HD void part_track_record(const Track& t, cmpmc_phonon_track& r) {
    memset(&r, 0, sizeof(r));
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
CMPMC_HD void part_charge_record(const Charge& c, cmpmc_charge_track& r) {
    memset(&r, 0, sizeof(r));
    r.pos[0] = c.pos.x; r.pos[1] = c.pos.y; r.pos[2] = c.pos.z;
    r.p_eV[0] = c.p.x; r.p_eV[1] = c.p.y; r.p_eV[2] = c.p.z;
    r.ekin = c.ekin;
    r.time = c.t;
    r.weight = c.w;
    r.valley = static_cast<uint16_t>(c.valley);
    r.type = static_cast<uint8_t>(c.type);
    r.alive = 1;
}

// Rng::normal (core/rng.hpp:71-75): Box-Muller, one value per call
CMPMC_HD double rng_normal(Rng& rng) {
    const double u1 = rng.uniform();
    const double u2 = rng.uniform();
    return sqrt(-2.0 * m_log(u1)) * m_cos(kTwoPi * u2);
}

// detail::choose_binom / pdf_binomial (charge/niel_models.hpp:178-198)
CMPMC_HD double choose_binom(int64_t n, int64_t x) {
    if (x > n / 2) x = n - x;
    if (x < 0) return 0.0;
    if (x == 0) return 1.0;
    if (x == 1) return static_cast<double>(n);
    double c = 1.0;
    for (int64_t k = 1; k <= x; ++k) c *= static_cast<double>(n - k + 1) / static_cast<double>(k);
    return c;
}

CMPMC_HD double pdf_binomial(int64_t x, int64_t n, double p) {
    if (x > n || x < 0 || p <= 0.0 || p > 1.0) return 0.0;
    if (p == 1.0) return (x == n) ? 1.0 : 0.0;
    const double lnbin = m_log(p) * static_cast<double>(x) + m_log(1.0 - p) * static_cast<double>(n - x);
    if (lnbin < -708.3) return 0.0;
    if (lnbin > 709.7) return 1e300;
    return choose_binom(n, x) * m_exp(lnbin);
}

// ChargeCloudGenerator::compute_cloud_radius (charge/charge_kernels.hpp:132-143)
CMPMC_HD double cloud_radius(uint64_t n_pairs, const cmpmc_crystal_config& cfg) {
    const double n_avogadro = 6.02214076e23;
    const double vol_cell = (cfg.density > 0.0 && cfg.atomic_A > 0.0)
                                ? (8.0 * (cfg.atomic_A * 1e-3) / (n_avogadro * cfg.density))
                                : m_pow(0.55 * 1e-9, 3.0);
    const double a0 = m_cbrt(vol_cell);
    const double r_scale = 0.25 * a0;
    return dmax(a0, r_scale * m_cbrt(static_cast<double>(n_pairs)));
}

// ChargeCloudGenerator::sample_offset (charge_kernels.hpp:145-150)
CMPMC_HD V3 cloud_offset(double r_max, Rng& rng) {
    if (r_max <= 0.0) return v3(0.0, 0.0, 0.0);
    const double u = rng.uniform();
    const double r = r_max * (1.0 - sqrt(dmax(0.0, 1.0 - u * u)));
    return rng.isotropic_dir() * r;
}

// The reduced energy of Lewin & Smith, epsilon = 11.5 keV^-1 E Z^-7/3, and their h(eps)
CMPMC_HD double lewin_smith_h(double energy_eV, double Z) {
    const double z23 = m_cbrt(Z * Z);
    const double epsilon = (11.5 / 1e3) * energy_eV / (Z * z23 * z23);
    return 0.7 * m_pow(epsilon, 0.6) + 3.0 * m_pow(epsilon, 0.15) + epsilon;
}

// Sarkis et al., Phys. Rev. A 107, 062811 (2023): measured silicon yield at 64 energies
// (eV), interpolated linearly (niel_models.hpp:100-140). Published data: the knots must
// equal the reference's for the yields to agree.
struct YieldKnot {
    double e_eV, yield;
};
#define CMPMC_SARKIS_KNOTS {47.83270, 0.000000}, {52.76735, 0.009114}, {58.75143, 0.016981}, {65.97224, 0.023622}, {74.67257, 0.029413}, {85.16158, 0.034885}, {97.80973, 0.040365}, {113.05138, 0.045962}, {131.41991, 0.051702}, {153.56956, 0.057597}, {180.26945, 0.063652}, {212.44431, 0.069870}, {251.21921, 0.076252}, {297.95152, 0.082797}, {354.26532, 0.089510}, {422.11910, 0.096396}, {503.86504, 0.103464}, {602.35199, 0.110722}, {720.98828, 0.118187}, {863.90755, 0.125872}, {1036.03980, 0.133800}, {1243.36450, 0.141991}, {1493.04550, 0.150478}, {1793.74340, 0.159282}, {2155.85770, 0.168439}, {2591.89340, 0.177980}, {3116.95740, 0.187961}, {3749.18370, 0.198399}, {4510.42640, 0.209326}, {5427.00620, 0.220779}, {6530.63220, 0.232847}, {7859.32390, 0.245567}, {9445.41000, 0.258878}, {11368.94900, 0.273042}, {13685.03100, 0.288012}, {16473.85900, 0.303838}, {19832.02600, 0.320553}, {23876.07900, 0.338204}, {28746.29200, 0.356826}, {34611.68400, 0.376451}, {41676.09800, 0.397077}, {50184.87400, 0.418697}, {60434.10300, 0.441291}, {72780.28500, 0.464810}, {87653.00800, 0.489194}, {105570.14000, 0.514350}, {127155.61000, 0.540142}, {153161.31000, 0.566445}, {184493.27000, 0.593129}, {222243.38000, 0.620053}, {267727.15000, 0.647094}, {322529.80000, 0.674139}, {388561.59000, 0.701059}, {468124.30000, 0.727705}, {563991.37000, 0.753920}, {679504.88000, 0.779502}, {818691.76000, 0.804197}, {986404.40000, 0.827705}, {1188489.80000, 0.849716}, {1431993.30000, 0.869965}, {1725404.10000, 0.888262}, {2078951.70000, 0.904513}, {2504962.10000, 0.918716}, {3018287.70000, 0.930944}
#ifdef __CUDACC__
static __constant__ YieldKnot kSarkisDev[64] = {CMPMC_SARKIS_KNOTS};
#endif
static constexpr YieldKnot kSarkisHost[64] = {CMPMC_SARKIS_KNOTS};
CMPMC_HD YieldKnot sarkis_knot(int i) {
#ifdef __CUDA_ARCH__
    return kSarkisDev[i];
#else
    return kSarkisHost[i];
#endif
}

// physics::sample_fano_binomial (charge/niel_models.hpp:202-263)
CMPMC_HD uint64_t sample_fano_binomial(double mean, double fano, Rng& rng) {
    if (mean <= 0.0) return 0;
    if (mean <= 1.0) return 1;
    if (fabs(fano - 1.0) < 1e-9) {
        if (mean > 30.0)
            return static_cast<uint64_t>(dmax(0.0, round(mean + sqrt(mean) * rng_normal(rng))));
        const double lim = m_exp(-mean);
        uint64_t k = 0;
        double p = 1.0;
        do {
            ++k;
            p *= rng.uniform();
        } while (p > lim);
        return k - 1;
    }
    const double prob = dclamp(1.0 - fano, 1e-6, 1.0 - 1e-6);
    const double ntry = mean / prob;
    if (mean > 9.0 * (fano / prob) && mean > 9.0 * (prob / fano)) {
        const double sampled = round(mean + sqrt(mean * fano) * rng_normal(rng));
        return static_cast<uint64_t>(dmax(1.0, sampled));
    }
    const int64_t nlo = static_cast<int64_t>(floor(ntry));
    const int64_t nhi = static_cast<int64_t>(ceil(ntry));
    if (nlo == nhi) {
        uint64_t hits = 0;
        for (int64_t i = 0; i < nlo; ++i)
            if (rng.uniform() < prob) ++hits;
        return hits;
    }
    const double p_lo = dmin(mean / static_cast<double>(nlo), 1.0);
    const double p_hi = dmin(mean / static_cast<double>(nhi), 1.0);
    const double dp = (fabs(p_hi - p_lo) > 1e-15) ? ((prob - p_lo) / (p_hi - p_lo)) : 0.0;
    const double pdf_max = dmax(pdf_binomial(static_cast<int64_t>(floor(mean)), nlo, p_lo),
                                pdf_binomial(static_cast<int64_t>(ceil(mean)), nlo, p_lo));
    if (pdf_max <= 0.0) return static_cast<uint64_t>(round(mean));
    for (int iter = 0; iter < 1000; ++iter) {
        const int64_t pick = static_cast<int64_t>(rng.uniform() * static_cast<double>(nhi + 1));
        const double pick_p =
            (pdf_binomial(pick, nlo, p_lo) * (1.0 - dp) + pdf_binomial(pick, nhi, p_hi) * dp) / pdf_max;
        if (rng.uniform() <= pick_p) return static_cast<uint64_t>(pick > 0 ? pick : 0);
    }
    return static_cast<uint64_t>(round(mean));
}

// lindhard_ionization_yield (niel_models.hpp:43-66; EnergyPartition's copy,
// energy_partition.hpp:53-73): projectile (z1, a1) on the crystal's nucleus, self-recoil
// when z1 / a1 <= 0
CMPMC_HD double lindhard_yield(double energy_eV, const cmpmc_crystal_config& cfg, double z1, double a1) {
    if (energy_eV <= 0.0) return 0.0;
    const double z2 = cfg.atomic_Z;
    const double a2 = cfg.atomic_A;
    if (z1 <= 0.0) z1 = z2;
    if (a1 <= 0.0) a1 = a2;
    const double z1_23 = m_cbrt(z1 * z1);
    const double z2_23 = m_cbrt(z2 * z2);
    const double zpow = z1_23 + z2_23;
    const double asum = a1 + a2;
    const double el = 30.724 * 1.0 * z1 * z2 * sqrt(zpow) * asum / a2;
    const double fl = (0.0793 * z1_23 * sqrt(z2 * asum * asum * asum / (a1 * a1 * a1 * a2))) / m_pow(zpow, 0.75);
    const double eps = energy_eV / el;
    const double numer = fl * (eps + 3.4008 * m_pow(eps, 0.16667) + 0.40244 * m_pow(eps, 0.75));
    return numer / (1.0 + numer);
}

// lewin_smith_ionization_yield (niel_models.hpp:69-79)
CMPMC_HD double lewin_smith_yield(double energy_eV, const cmpmc_crystal_config& cfg) {
    if (energy_eV <= 0.0) return 0.0;
    const double Z = cfg.atomic_Z;
    const double k = 0.133 * m_cbrt(Z * Z) / sqrt(cfg.atomic_A);
    const double h = lewin_smith_h(energy_eV, Z);
    return (k * h) / (1.0 + k * h);
}

// compute_ionization_yield (niel_models.hpp:83-176)
CMPMC_HD double ionization_yield(int model, double energy_eV, const cmpmc_crystal_config& cfg,
                        const cmpmc_partition_options& o) {
    switch (model) {
        case CMPMC_NIEL_LEWIN_SMITH: return lewin_smith_yield(energy_eV, cfg);
        case CMPMC_NIEL_IMPACT_TUNL: {  // PRL 131, 091801 (2023): Y10 (E / 10 keV)^B for Si <= 10 keV
            if (energy_eV <= 0.0) return 0.0;
            const bool si = (fabs(cfg.atomic_Z - 14.0) < 0.5) || (fabs(cfg.atomic_A - 28.09) < 0.5);
            if (si && energy_eV <= 10.0 * 1e3) return 0.302 * m_pow(energy_eV / (10.0 * 1e3), 0.261);
            return lewin_smith_yield(energy_eV, cfg);
        }
        case CMPMC_NIEL_SARKIS: {
            if (energy_eV <= 0.0) return 0.0;
            const bool si = (fabs(cfg.atomic_Z - 14.0) < 0.5) && (fabs(cfg.atomic_A - 28.09) < 1.0);
            if (!si || energy_eV > 3.0 * 1e6) return lewin_smith_yield(energy_eV, cfg);
            if (energy_eV <= sarkis_knot(0).e_eV) return 0.0;
            if (energy_eV >= sarkis_knot(63).e_eV) return sarkis_knot(63).yield;
            int hi = 1;  // first knot above the energy (bounded: a NaN energy stops at the last knot)
            while (hi < 63 && !(energy_eV < sarkis_knot(hi).e_eV)) ++hi;
            const YieldKnot k0 = sarkis_knot(hi - 1);
            const YieldKnot k1 = sarkis_knot(hi);
            const double t = (energy_eV - k0.e_eV) / (k1.e_eV - k0.e_eV);
            return k0.yield + t * (k1.yield - k0.yield);
        }
        case CMPMC_NIEL_EMPIRICAL: {
            if (energy_eV <= 0.0) return 0.0;
            if (o.emp_energy_dependent_k && (energy_eV > o.emp_e_high_eV || o.emp_e_low_eV == o.emp_e_high_eV))
                return lewin_smith_yield(energy_eV, cfg);
            double k = o.emp_k_fixed;
            if (o.emp_energy_dependent_k) {
                const double dk = o.emp_k_high - o.emp_k_low;
                const double dE = o.emp_e_high_eV - o.emp_e_low_eV;
                k = dmax(0.0, o.emp_k_low + (energy_eV - o.emp_e_low_eV) * (dk / dE));
            }
            const double h = lewin_smith_h(energy_eV, cfg.atomic_Z);
            return (k * h) / (1.0 + k * h);
        }
        default: return lindhard_yield(energy_eV, cfg, 0.0, 0.0);
    }
}

// EnergyPartition::partition_deposit (energy_partition.hpp:78-118): the yield, then the
// draws of the pair count; everything that fixes the output sizes.
CMPMC_HD PartitionPlan plan_partition(const cmpmc_crystal_config& cfg, double edep, bool is_nr,
                             const cmpmc_partition_options& o, Rng& rng) {
    PartitionPlan d{};
    d.edep = edep;
    d.yield = is_nr ? ionization_yield(o.niel_model, edep, cfg, o) : 1.0;
    d.ionizing = edep * d.yield;
    d.niel = edep - d.ionizing;
    const double e_gap = cfg.bandgap, e_pair = cfg.pair_energy;
    if (d.ionizing >= e_gap && e_pair > 0.0) {
        const double mean_pairs = d.ionizing / e_pair;
        if (!o.use_fano_fluctuations || mean_pairs < 1.0) {
            d.pairs_true = static_cast<uint64_t>(floor(mean_pairs + rng.uniform()));
        } else {
            const uint64_t cap = static_cast<uint64_t>(floor(d.ionizing / e_gap));
            const uint64_t sampled = sample_fano_binomial(mean_pairs, cfg.fano_factor, rng);
            d.pairs_true = (cap < sampled) ? cap : sampled;
        }
    }
    const double init_ekin = 5.0 * 1e-3;
    const double pair_energy = static_cast<double>(d.pairs_true) * (e_gap + 2.0 * init_ekin);
    d.prompt_eV = dmax(0.0, edep - pair_energy);
    if (d.pairs_true > 0) {
        d.pairs_sampled = (d.pairs_true < o.max_sampled_pairs) ? d.pairs_true : o.max_sampled_pairs;
        d.charge_weight = static_cast<double>(d.pairs_true) / static_cast<double>(d.pairs_sampled);
    } else {
        d.charge_weight = 1.0;
    }
    d.phonon_weight = 1.0;
    const double e_debye = cfg.debye_freq * kHPlanck;
    if (d.prompt_eV > 0.0 && e_debye > 0.0) {
        const uint64_t n_ph = static_cast<uint64_t>(round(d.prompt_eV / e_debye));
        d.phonons_true = (n_ph > 1) ? n_ph : 1;
        d.phonons_sampled = (d.phonons_true < o.max_sampled_phonons) ? d.phonons_true : o.max_sampled_phonons;
        d.phonon_weight = static_cast<double>(d.phonons_true) / static_cast<double>(d.phonons_sampled);
    }
    return d;
}

// The rest of partition_deposit (energy_partition.hpp:120-164): the sampled pairs (cloud
// offset, valley, directions) and the prompt Debye phonons, in the reference's order.
CMPMC_HD void fill_partition(const Lattice& L, const cmpmc_crystal_config& cfg, const PartitionPlan& d,
                    const cmpmc_partition_options& o, V3 pos, double time_s, Rng& rng, cmpmc_charge_track* ch,
                    cmpmc_phonon_track* ph) {
    const double init_ekin = 5.0 * 1e-3;
    if (d.pairs_true > 0) {
        const uint64_t nv = static_cast<uint64_t>(L.n_valleys > 1 ? L.n_valleys : 1);
        const double r_cloud = o.use_charge_cloud ? cloud_radius(d.pairs_true, cfg) : 0.0;
        for (uint64_t i = 0; i < d.pairs_sampled; ++i) {
            const V3 pp = pos + cloud_offset(r_cloud, rng);
            const int valley = static_cast<int>(static_cast<uint16_t>(rng.next_u64() % nv));
            const V3 de = rng.isotropic_dir();
            Charge e = make_charge(L, 1, pp, de, init_ekin, valley, time_s);
            e.w = d.charge_weight;
            const V3 dh = rng.isotropic_dir();
            Charge h = make_charge(L, 2, pp, dh, init_ekin, 0, time_s);
            h.w = d.charge_weight;
            part_charge_record(e, ch[2 * i]);
            part_charge_record(h, ch[2 * i + 1]);
        }
    }
    if (d.phonons_sampled > 0) {
        const double e_single = d.prompt_eV / static_cast<double>(d.phonons_true);
        for (uint64_t i = 0; i < d.phonons_sampled; ++i) {
            const int mode = sample_dos_mode(L, rng);
            const V3 k = rng.isotropic_dir();
            const Kin kin = map_k_to_vg(L, mode, k);
            Track t;
            t.pos = pos;
            t.k = k;  // the drawn direction is stored as is (no unit())
            t.vg = kin.vg_dir;
            t.E = e_single;
            t.vmag = kin.vg_mag;
            t.t = time_s;
            t.w = d.phonon_weight;
            t.bounces = 0;
            t.mode = mode;
            part_track_record(t, ph[i]);
        }
    }
}

}  // namespace cmpmc_gpu
