// partition_host.cpp -- the input side of the transport on the host: ionisation-yield
// models, the energy partition of a deposit into carriers and prompt phonons, and the
// hit merger that turns primary-particle steps into initial stacks.
//
// Restates, with the reference's draw order and operation order (the outputs are compared
// bit for bit with the reference's):
//   * niel_models.hpp:43-176: Lindhard (Lewin-Smith form), Lewin-Smith, IMPACT@TUNL,
//     Sarkis and the CDMSlite empirical k(E) yields, and their dispatcher;
//   * niel_models.hpp:178-263: the interpolated Fano-binomial pair-number sampler;
//   * charge_kernels.hpp:131-150: the charge-cloud radius and offsets;
//   * energy_partition.hpp:78-167: EnergyPartition::partition_deposit, split here into the
//     draws up to the pair count (plan_partition, which fixes the output sizes) and the
//     rest (fill_partition);
//   * energy_partition.hpp:182-323: StepAccumulator and HitMerger.
// The generators run on the host with the platform libm, as in the reference.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace cmpmc_gpu;

namespace cmpmc_gpu {

// Rng::normal (core/rng.hpp:71-75): Box-Muller, one value per call
double rng_normal(Rng& rng) {
    const double u1 = rng.uniform();
    const double u2 = rng.uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(kTwoPi * u2);
}

namespace {

// detail::choose_binom / pdf_binomial (charge/niel_models.hpp:178-198)
double choose_binom(int64_t n, int64_t x) {
    if (x > n / 2) x = n - x;
    if (x < 0) return 0.0;
    if (x == 0) return 1.0;
    if (x == 1) return static_cast<double>(n);
    double c = 1.0;
    for (int64_t k = 1; k <= x; ++k) c *= static_cast<double>(n - k + 1) / static_cast<double>(k);
    return c;
}

double pdf_binomial(int64_t x, int64_t n, double p) {
    if (x > n || x < 0 || p <= 0.0 || p > 1.0) return 0.0;
    if (p == 1.0) return (x == n) ? 1.0 : 0.0;
    const double lnbin = std::log(p) * static_cast<double>(x) + std::log(1.0 - p) * static_cast<double>(n - x);
    if (lnbin < -708.3) return 0.0;
    if (lnbin > 709.7) return 1e300;
    return choose_binom(n, x) * std::exp(lnbin);
}

// ChargeCloudGenerator::compute_cloud_radius (charge/charge_kernels.hpp:132-143)
double cloud_radius(uint64_t n_pairs, const cmpmc_crystal_config& cfg) {
    const double n_avogadro = 6.02214076e23;
    const double vol_cell = (cfg.density > 0.0 && cfg.atomic_A > 0.0)
                                ? (8.0 * (cfg.atomic_A * 1e-3) / (n_avogadro * cfg.density))
                                : std::pow(0.55 * 1e-9, 3.0);
    const double a0 = std::cbrt(vol_cell);
    const double r_scale = 0.25 * a0;
    return std::max(a0, r_scale * std::cbrt(static_cast<double>(n_pairs)));
}

// ChargeCloudGenerator::sample_offset (charge_kernels.hpp:145-150)
V3 cloud_offset(double r_max, Rng& rng) {
    if (r_max <= 0.0) return v3(0.0, 0.0, 0.0);
    const double u = rng.uniform();
    const double r = r_max * (1.0 - std::sqrt(std::max(0.0, 1.0 - u * u)));
    return rng.isotropic_dir() * r;
}

// The reduced energy of Lewin & Smith, epsilon = 11.5 keV^-1 E Z^-7/3, and their h(eps)
double lewin_smith_h(double energy_eV, double Z) {
    const double z23 = std::cbrt(Z * Z);
    const double epsilon = (11.5 / 1e3) * energy_eV / (Z * z23 * z23);
    return 0.7 * std::pow(epsilon, 0.6) + 3.0 * std::pow(epsilon, 0.15) + epsilon;
}

// Sarkis et al., Phys. Rev. A 107, 062811 (2023): measured silicon yield at 64 energies
// (eV), interpolated linearly (niel_models.hpp:100-140). Published data: the knots must
// equal the reference's for the yields to agree.
struct YieldKnot {
    double e_eV, yield;
};
constexpr YieldKnot kSarkis[64] = {
    {47.83270, 0.000000},      {52.76735, 0.009114},      {58.75143, 0.016981},      {65.97224, 0.023622},
    {74.67257, 0.029413},      {85.16158, 0.034885},      {97.80973, 0.040365},      {113.05138, 0.045962},
    {131.41991, 0.051702},     {153.56956, 0.057597},     {180.26945, 0.063652},     {212.44431, 0.069870},
    {251.21921, 0.076252},     {297.95152, 0.082797},     {354.26532, 0.089510},     {422.11910, 0.096396},
    {503.86504, 0.103464},     {602.35199, 0.110722},     {720.98828, 0.118187},     {863.90755, 0.125872},
    {1036.03980, 0.133800},    {1243.36450, 0.141991},    {1493.04550, 0.150478},    {1793.74340, 0.159282},
    {2155.85770, 0.168439},    {2591.89340, 0.177980},    {3116.95740, 0.187961},    {3749.18370, 0.198399},
    {4510.42640, 0.209326},    {5427.00620, 0.220779},    {6530.63220, 0.232847},    {7859.32390, 0.245567},
    {9445.41000, 0.258878},    {11368.94900, 0.273042},   {13685.03100, 0.288012},   {16473.85900, 0.303838},
    {19832.02600, 0.320553},   {23876.07900, 0.338204},   {28746.29200, 0.356826},   {34611.68400, 0.376451},
    {41676.09800, 0.397077},   {50184.87400, 0.418697},   {60434.10300, 0.441291},   {72780.28500, 0.464810},
    {87653.00800, 0.489194},   {105570.14000, 0.514350},  {127155.61000, 0.540142},  {153161.31000, 0.566445},
    {184493.27000, 0.593129},  {222243.38000, 0.620053},  {267727.15000, 0.647094},  {322529.80000, 0.674139},
    {388561.59000, 0.701059},  {468124.30000, 0.727705},  {563991.37000, 0.753920},  {679504.88000, 0.779502},
    {818691.76000, 0.804197},  {986404.40000, 0.827705},  {1188489.80000, 0.849716}, {1431993.30000, 0.869965},
    {1725404.10000, 0.888262}, {2078951.70000, 0.904513}, {2504962.10000, 0.918716}, {3018287.70000, 0.930944}};

}  // namespace

// physics::sample_fano_binomial (charge/niel_models.hpp:202-263)
uint64_t sample_fano_binomial(double mean, double fano, Rng& rng) {
    if (mean <= 0.0) return 0;
    if (mean <= 1.0) return 1;
    if (std::fabs(fano - 1.0) < 1e-9) {
        if (mean > 30.0)
            return static_cast<uint64_t>(std::max(0.0, std::round(mean + std::sqrt(mean) * rng_normal(rng))));
        const double lim = std::exp(-mean);
        uint64_t k = 0;
        double p = 1.0;
        do {
            ++k;
            p *= rng.uniform();
        } while (p > lim);
        return k - 1;
    }
    const double prob = std::clamp(1.0 - fano, 1e-6, 1.0 - 1e-6);
    const double ntry = mean / prob;
    if (mean > 9.0 * (fano / prob) && mean > 9.0 * (prob / fano)) {
        const double sampled = std::round(mean + std::sqrt(mean * fano) * rng_normal(rng));
        return static_cast<uint64_t>(std::max(1.0, sampled));
    }
    const int64_t nlo = static_cast<int64_t>(std::floor(ntry));
    const int64_t nhi = static_cast<int64_t>(std::ceil(ntry));
    if (nlo == nhi) {
        uint64_t hits = 0;
        for (int64_t i = 0; i < nlo; ++i)
            if (rng.uniform() < prob) ++hits;
        return hits;
    }
    const double p_lo = std::min(mean / static_cast<double>(nlo), 1.0);
    const double p_hi = std::min(mean / static_cast<double>(nhi), 1.0);
    const double dp = (std::fabs(p_hi - p_lo) > 1e-15) ? ((prob - p_lo) / (p_hi - p_lo)) : 0.0;
    const double pdf_max = std::max(pdf_binomial(static_cast<int64_t>(std::floor(mean)), nlo, p_lo),
                                    pdf_binomial(static_cast<int64_t>(std::ceil(mean)), nlo, p_lo));
    if (pdf_max <= 0.0) return static_cast<uint64_t>(std::round(mean));
    for (int iter = 0; iter < 1000; ++iter) {
        const int64_t pick = static_cast<int64_t>(rng.uniform() * static_cast<double>(nhi + 1));
        const double pick_p =
            (pdf_binomial(pick, nlo, p_lo) * (1.0 - dp) + pdf_binomial(pick, nhi, p_hi) * dp) / pdf_max;
        if (rng.uniform() <= pick_p) return static_cast<uint64_t>(std::max<int64_t>(0, pick));
    }
    return static_cast<uint64_t>(std::round(mean));
}

// lindhard_ionization_yield (niel_models.hpp:43-66; EnergyPartition's copy,
// energy_partition.hpp:53-73): projectile (z1, a1) on the crystal's nucleus, self-recoil
// when z1 / a1 <= 0
double lindhard_yield(double energy_eV, const cmpmc_crystal_config& cfg, double z1, double a1) {
    if (energy_eV <= 0.0) return 0.0;
    const double z2 = cfg.atomic_Z;
    const double a2 = cfg.atomic_A;
    if (z1 <= 0.0) z1 = z2;
    if (a1 <= 0.0) a1 = a2;
    const double z1_23 = std::cbrt(z1 * z1);
    const double z2_23 = std::cbrt(z2 * z2);
    const double zpow = z1_23 + z2_23;
    const double asum = a1 + a2;
    const double el = 30.724 * 1.0 * z1 * z2 * std::sqrt(zpow) * asum / a2;
    const double fl = (0.0793 * z1_23 * std::sqrt(z2 * asum * asum * asum / (a1 * a1 * a1 * a2))) / std::pow(zpow, 0.75);
    const double eps = energy_eV / el;
    const double numer = fl * (eps + 3.4008 * std::pow(eps, 0.16667) + 0.40244 * std::pow(eps, 0.75));
    return numer / (1.0 + numer);
}

// lewin_smith_ionization_yield (niel_models.hpp:69-79)
double lewin_smith_yield(double energy_eV, const cmpmc_crystal_config& cfg) {
    if (energy_eV <= 0.0) return 0.0;
    const double Z = cfg.atomic_Z;
    const double k = 0.133 * std::cbrt(Z * Z) / std::sqrt(cfg.atomic_A);
    const double h = lewin_smith_h(energy_eV, Z);
    return (k * h) / (1.0 + k * h);
}

// compute_ionization_yield (niel_models.hpp:83-176)
double ionization_yield(int model, double energy_eV, const cmpmc_crystal_config& cfg,
                        const cmpmc_partition_options& o) {
    switch (model) {
        case CMPMC_NIEL_LEWIN_SMITH: return lewin_smith_yield(energy_eV, cfg);
        case CMPMC_NIEL_IMPACT_TUNL: {  // PRL 131, 091801 (2023): Y10 (E / 10 keV)^B for Si <= 10 keV
            if (energy_eV <= 0.0) return 0.0;
            const bool si = (std::fabs(cfg.atomic_Z - 14.0) < 0.5) || (std::fabs(cfg.atomic_A - 28.09) < 0.5);
            if (si && energy_eV <= 10.0 * 1e3) return 0.302 * std::pow(energy_eV / (10.0 * 1e3), 0.261);
            return lewin_smith_yield(energy_eV, cfg);
        }
        case CMPMC_NIEL_SARKIS: {
            if (energy_eV <= 0.0) return 0.0;
            const bool si = (std::fabs(cfg.atomic_Z - 14.0) < 0.5) && (std::fabs(cfg.atomic_A - 28.09) < 1.0);
            if (!si || energy_eV > 3.0 * 1e6) return lewin_smith_yield(energy_eV, cfg);
            if (energy_eV <= kSarkis[0].e_eV) return 0.0;
            if (energy_eV >= kSarkis[63].e_eV) return kSarkis[63].yield;
            int hi = 1;  // first knot above the energy
            while (!(energy_eV < kSarkis[hi].e_eV)) ++hi;
            const YieldKnot& k0 = kSarkis[hi - 1];
            const YieldKnot& k1 = kSarkis[hi];
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
                k = std::max(0.0, o.emp_k_low + (energy_eV - o.emp_e_low_eV) * (dk / dE));
            }
            const double h = lewin_smith_h(energy_eV, cfg.atomic_Z);
            return (k * h) / (1.0 + k * h);
        }
        default: return lindhard_yield(energy_eV, cfg, 0.0, 0.0);
    }
}

// EnergyPartition::partition_deposit (energy_partition.hpp:78-118): the yield, then the
// draws of the pair count; everything that fixes the output sizes.
PartitionPlan plan_partition(const cmpmc_crystal_config& cfg, double edep, bool is_nr,
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
            d.pairs_true = static_cast<uint64_t>(std::floor(mean_pairs + rng.uniform()));
        } else {
            const uint64_t cap = static_cast<uint64_t>(std::floor(d.ionizing / e_gap));
            d.pairs_true = std::min(cap, sample_fano_binomial(mean_pairs, cfg.fano_factor, rng));
        }
    }
    const double init_ekin = 5.0 * 1e-3;
    const double pair_energy = static_cast<double>(d.pairs_true) * (e_gap + 2.0 * init_ekin);
    d.prompt_eV = std::max(0.0, edep - pair_energy);
    if (d.pairs_true > 0) {
        d.pairs_sampled = std::min<uint64_t>(d.pairs_true, o.max_sampled_pairs);
        d.charge_weight = static_cast<double>(d.pairs_true) / static_cast<double>(d.pairs_sampled);
    } else {
        d.charge_weight = 1.0;
    }
    d.phonon_weight = 1.0;
    const double e_debye = cfg.debye_freq * kHPlanck;
    if (d.prompt_eV > 0.0 && e_debye > 0.0) {
        d.phonons_true = std::max<uint64_t>(1, static_cast<uint64_t>(std::round(d.prompt_eV / e_debye)));
        d.phonons_sampled = std::min<uint64_t>(d.phonons_true, o.max_sampled_phonons);
        d.phonon_weight = static_cast<double>(d.phonons_true) / static_cast<double>(d.phonons_sampled);
    }
    return d;
}

// The rest of partition_deposit (energy_partition.hpp:120-164): the sampled pairs (cloud
// offset, valley, directions) and the prompt Debye phonons, in the reference's order.
void fill_partition(const Lattice& L, const cmpmc_crystal_config& cfg, const PartitionPlan& d,
                    const cmpmc_partition_options& o, V3 pos, double time_s, Rng& rng, cmpmc_charge_track* ch,
                    cmpmc_phonon_track* ph) {
    const double init_ekin = 5.0 * 1e-3;
    if (d.pairs_true > 0) {
        const uint64_t nv = static_cast<uint64_t>(std::max(1, L.n_valleys));
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
            charge_to_record(e, ch[2 * i]);
            charge_to_record(h, ch[2 * i + 1]);
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
            track_to_record(t, ph[i]);
        }
    }
}

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
