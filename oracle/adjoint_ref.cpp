// Test infrastructure only (the checker): the CPU side of the adjoint checks.
//
// The reference has no adjoint. This program provides its two stand-ins on the reference's
// own transport, for events of the single-L-phonon volume workload (one L phonon of
// 7.5 meV per event, origin uniform in the cylinder, isotropic; seed 17):
//
//   1. central finite differences with common random numbers on the unmodified reference:
//      SimulationEngine::transport (transport/engine.hpp:403-582) run per event from
//      Rng::for_stream(seed, ev), at theta_k (1 +- step), with every other parameter fixed;
//   2. the score-function estimator on a CPU restatement of the same transport loop: the
//      loop of engine.hpp:403-582, written out here with the reference's own building blocks
//      (CrystalLattice rates / samplers / map_k_to_vg, CylinderSolid::intersect_exit,
//      SurfaceProperty::reflection_split, KaplanFilm::absorb_phonon, Rng), plus the score
//      of every theta-dependent decision. `check` pins the restatement: with the same
//      streams it must reproduce the reference's hits bit for bit.
//
// theta = (B_iso, A_anh, p_d, f_abs): CrystalConfig::B_iso and ::A_anh
// (materials/crystal_config.hpp:71-72); p_d the diffuse fraction of every surface
// (spec_coeffs {1-p_d}, diff_coeffs {p_d}, anh_coeffs {}, spec_prob_const 1-p_d, so that
// reflection_split, geometry/surface_property.hpp:72-86, gives p_diff = p_d at every
// frequency); f_abs the film_absorption of every Kaplan film (crystal_config.hpp:241, used at
// engine.hpp:495). The histogram has n_bins bins of hit time over [0, t_max).
//
// Usage (values in decimal; weights: a file of n_bins raw doubles, or "-" for zeros):
//   adjoint_ref check    B A pd f first n threads
//   adjoint_ref estimate B A pd f first n threads n_bins t_max weights out
//       out: hist[n_bins] f64, then per event f64[5] = value, d value / d theta_0..3
//   adjoint_ref values   B A pd f first n threads n_bins t_max weights out
//       the reference's own transport: hist[n_bins] f64, then per event f64 value
#include "cmpmc/cmpmc.hpp"

#include <atomic>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using namespace cmpmc;

namespace {

constexpr uint64_t kSeed = 17;

struct Theta {
    double B, A, pd, f;
};

struct Setup {
    CrystalLattice lattice;
    DetectorModel det;
    Setup(const Theta& th) : lattice(make_cfg(th)), det(make_det(th)) {}
    static CrystalConfig make_cfg(const Theta& th) {
        CrystalConfig c = materials::Germanium();
        c.B_iso = th.B;
        c.A_anh = th.A;
        return c;
    }
    static DetectorModel make_det(const Theta& th) {
        DetectorModel d;
        for (auto& s : d.surfaces) {
            s.spec_coeffs = {1.0 - th.pd};
            s.diff_coeffs = {th.pd};
            s.anh_coeffs = {};
            s.spec_prob_const = 1.0 - th.pd;
            if (s.kaplan_sensor.has_value()) s.kaplan_sensor->film_absorption = th.f;
        }
        return d;
    }
};

// the single-L-phonon volume generator (one L phonon of 7.5 meV, origin uniform in the
// cylinder by rejection in x, y then z, isotropic direction)
PhononTrack generate(const SimulationEngine& eng, const DetectorModel& det, Rng& rng) {
    double x, y;
    const double R = det.solid.radius;
    do {
        x = (2.0 * rng.uniform() - 1.0) * R;
        y = (2.0 * rng.uniform() - 1.0) * R;
    } while (x * x + y * y > R * R);
    const double z = (2.0 * rng.uniform() - 1.0) * det.solid.half_z;
    const Vec3 d = rng.isotropic_dir();
    return eng.make_track({x, y, z}, d, PhononMode::L, 7.5e-3);
}

struct Hist {
    int n_bins;
    double t_max;
    int bin(double t) const {
        if (!(t >= 0.0) || !(t < t_max)) return -1;
        const int b = static_cast<int>(t * (n_bins / t_max));
        return b < n_bins ? b : -1;
    }
};

// ---- restated transport with scores ------------------------------------------------------
struct STrack {
    PhononTrack t;
    double s[4];  // d log p / d log theta_k of the lineage's decisions so far
};

class Restated {
  public:
    Restated(const CrystalLattice& L, const DetectorModel& D, const Theta& th) : L_(L), D_(D), eng_(L, D), th_(th) {}

    // engine.hpp:927-936
    Vec3 sample_inward(PhononMode m, const Vec3& n, Rng& rng) const {
        for (int trial = 0; trial < 16; ++trial) {
            const Vec3 kd = rng.lambertian_dir(n);
            const auto kin = L_.map_k_to_vg(m, kd);
            if (kin.vg_dir.dot(n) > 1e-6) return kd;
        }
        return n;
    }

    // engine.hpp:403-582 with scores; hits are appended with the score of their track
    void transport(std::vector<STrack>& stack, std::vector<SensorHit>& hits, std::vector<std::array<double, 4>>& hs,
                   SimStats& st, Rng& rng) const {
        KaplanBuffer refl;
        while (!stack.empty()) {
            STrack tr = stack.back();
            stack.pop_back();
            PhononTrack& trk = tr.t;
            for (;;) {
                if (trk.energy < D_.min_phonon_eV || trk.bounces >= D_.max_bounces) {
                    st.killed_tracks++;
                    st.escaped_or_killed_eV += trk.energy * trk.weight;
                    break;
                }
                if (!apply_russian_roulette(trk.weight, trk.bounces, D_.russian_roulette_bounces,
                                            D_.russian_roulette_survival, rng)) {
                    st.killed_tracks++;
                    break;
                }
                st.total_steps++;
                const double r_iso = L_.isotope_rate(trk.energy);
                const double r_poly = L_.polycrystal_rate(trk.vg_mag);
                const double r_down = L_.downconversion_rate(trk.mode, trk.energy);
                const double r_tot = r_iso + r_poly + r_down;
                const double d_phys = (r_tot > 1e-12) ? (-std::log(rng.uniform()) * (trk.vg_mag / r_tot))
                                                      : std::numeric_limits<double>::infinity();
                const BoundaryHit bh = D_.solid.intersect_exit(trk.pos, trk.vg_dir);
                if (d_phys < bh.distance) {
                    trk.pos += trk.vg_dir * d_phys;
                    trk.time += d_phys / trk.vg_mag;
                    tr.s[0] -= r_iso * (d_phys / trk.vg_mag);
                    tr.s[1] -= r_down * (d_phys / trk.vg_mag);
                    const double u_proc = rng.uniform() * r_tot;
                    if (r_down > 0.0 && u_proc < r_down) {
                        tr.s[1] += 1.0;
                        decay_tt(tr, stack, st, rng);
                    } else {
                        if (u_proc < r_down + r_iso) {
                            st.isotope_scatters++;
                            tr.s[0] += 1.0;
                        } else {
                            st.polycrystal_scatters++;
                        }
                        trk.mode = L_.sample_dos_mode(rng);
                        trk.k_dir = rng.isotropic_dir();
                        const auto kin = L_.map_k_to_vg(trk.mode, trk.k_dir);
                        trk.vg_dir = kin.vg_dir;
                        trk.vg_mag = kin.vg_mag;
                    }
                    continue;
                }
                trk.pos += trk.vg_dir * bh.distance;
                trk.time += bh.distance / trk.vg_mag;
                tr.s[0] -= r_iso * (bh.distance / trk.vg_mag);
                tr.s[1] -= r_down * (bh.distance / trk.vg_mag);
                trk.bounces++;
                const SurfaceProperty& surf = D_.surfaces[static_cast<size_t>(bh.surface_id)];
                if (surf.kaplan_sensor.has_value() && rng.uniform() < surf.prob_abs) {
                    const KaplanFilm& film = *surf.kaplan_sensor;
                    const bool enter = rng.uniform() < film.film_absorption;
                    tr.s[3] += enter ? 1.0 : -film.film_absorption / (1.0 - film.film_absorption);
                    if (enter) {
                        const double edep = film.absorb_phonon(trk.energy, refl, rng);
                        if (edep > 0.0) {
                            st.sensor_hits++;
                            st.total_deposited_eV += edep * trk.weight;
                            hits.push_back(SensorHit{.pos = trk.pos, .time = trk.time, .edep = edep * trk.weight,
                                                     .incident_energy = trk.energy, .surface_id = bh.surface_id,
                                                     .excitation = ExcitationType::Phonon, .mode = trk.mode,
                                                     .channel_id = -1});
                            hs.push_back({tr.s[0], tr.s[1], tr.s[2], tr.s[3]});
                        }
                        double sum_refl = 0.0;
                        for (double re : refl) sum_refl += re;
                        st.escaped_or_killed_eV += std::max(0.0, trk.energy - edep - sum_refl) * trk.weight;
                        if (refl.empty()) break;
                        const Vec3 rp = trk.pos + bh.inward_normal * 1e-11;
                        for (size_t i = 1; i < refl.size(); ++i) {
                            const PhononMode m = L_.sample_dos_mode(rng);
                            const Vec3 kd = sample_inward(m, bh.inward_normal, rng);
                            STrack d;
                            d.t = eng_.make_track(rp, kd, m, refl[i], trk.time, trk.weight);
                            std::memcpy(d.s, tr.s, sizeof(d.s));
                            stack.push_back(d);
                        }
                        trk.pos = rp;
                        trk.energy = refl[0];
                        trk.mode = L_.sample_dos_mode(rng);
                        trk.k_dir = sample_inward(trk.mode, bh.inward_normal, rng);
                        const auto kin = L_.map_k_to_vg(trk.mode, trk.k_dir);
                        trk.vg_dir = kin.vg_dir;
                        trk.vg_mag = kin.vg_mag;
                        continue;
                    }
                }
                if (rng.uniform() > surf.prob_refl) {
                    st.killed_tracks++;
                    st.escaped_or_killed_eV += trk.energy * trk.weight;
                    break;
                }
                st.surface_refls++;
                trk.pos += bh.inward_normal * 1e-11;
                const auto split = surf.reflection_split(trk.energy);
                const double u_refl = rng.uniform();
                if (u_refl < split.p_anh) {
                    // p_anh is 0 under the theta surfaces; kept for the loop's shape
                    st.surface_downconversions++;
                    const bool tt = rng.uniform() < L_.config().fTT_frac;
                    const double x = tt ? L_.sample_tt_energy_fraction(rng) : L_.sample_lt_energy_fraction(rng);
                    const PhononMode m1 = tt ? L_.sample_transverse_mode(rng) : PhononMode::L;
                    const PhononMode m2 = L_.sample_transverse_mode(rng);
                    const Vec3 k2 = sample_inward(m2, bh.inward_normal, rng);
                    STrack d;
                    d.t = eng_.make_track(trk.pos, k2, m2, (1.0 - x) * trk.energy, trk.time, trk.weight);
                    std::memcpy(d.s, tr.s, sizeof(d.s));
                    stack.push_back(d);
                    trk.energy = x * trk.energy;
                    trk.mode = m1;
                    trk.k_dir = sample_inward(m1, bh.inward_normal, rng);
                    const auto kin = L_.map_k_to_vg(m1, trk.k_dir);
                    trk.vg_dir = kin.vg_dir;
                    trk.vg_mag = kin.vg_mag;
                } else if (u_refl < split.p_anh + split.p_spec) {
                    tr.s[2] += -th_.pd / (1.0 - th_.pd);
                    Vec3 kr = trk.k_dir - bh.inward_normal * (2.0 * trk.k_dir.dot(bh.inward_normal));
                    auto kin = L_.map_k_to_vg(trk.mode, kr);
                    if (kin.vg_dir.dot(bh.inward_normal) <= 1e-6) {
                        kr = sample_inward(trk.mode, bh.inward_normal, rng);
                        kin = L_.map_k_to_vg(trk.mode, kr);
                    }
                    trk.k_dir = kr;
                    trk.vg_dir = kin.vg_dir;
                    trk.vg_mag = kin.vg_mag;
                } else {
                    tr.s[2] += 1.0;
                    trk.k_dir = sample_inward(trk.mode, bh.inward_normal, rng);
                    const auto kin = L_.map_k_to_vg(trk.mode, trk.k_dir);
                    trk.vg_dir = kin.vg_dir;
                    trk.vg_mag = kin.vg_mag;
                }
            }
        }
    }

  private:
    // engine.hpp:938-988 (draw order: phi, TT/LT choice, x, then the modes); the daughter
    // starts with the parent's score
    void decay_tt(STrack& tr, std::vector<STrack>& stack, SimStats& st, Rng& rng) const {
        PhononTrack& trk = tr.t;
        const Vec3 d1 = trk.k_dir;
        const Vec3 perp = d1.orthogonal_unit();
        const double phi = units::two_pi * rng.uniform();
        const double cp = std::cos(phi), sp = std::sin(phi);
        double x;
        Vec3 k1, k2;
        PhononMode m1, m2;
        if (rng.uniform() < L_.config().fTT_frac) {
            st.decays_L_to_TT++;
            x = L_.sample_tt_energy_fraction(rng);
            const double a1 = L_.theta_TT(x), a2 = L_.theta_TT(1.0 - x);
            k1 = d1.rotate_around(perp, std::cos(a1), std::sin(a1)).rotate_around(d1, cp, sp).unit();
            k2 = d1.rotate_around(perp, std::cos(-a2), std::sin(-a2)).rotate_around(d1, cp, sp).unit();
            m1 = L_.sample_transverse_mode(rng);
            m2 = L_.sample_transverse_mode(rng);
        } else {
            st.decays_L_to_LT++;
            x = L_.sample_lt_energy_fraction(rng);
            const double a1 = L_.theta_L_to_LT(x), a2 = L_.theta_T_from_LT(x);
            k1 = d1.rotate_around(perp, std::cos(a1), std::sin(a1)).rotate_around(d1, cp, sp).unit();
            k2 = d1.rotate_around(perp, std::cos(-a2), std::sin(-a2)).rotate_around(d1, cp, sp).unit();
            m1 = PhononMode::L;
            m2 = L_.sample_transverse_mode(rng);
        }
        STrack d;
        d.t = eng_.make_track(trk.pos, k2, m2, (1.0 - x) * trk.energy, trk.time, trk.weight);
        std::memcpy(d.s, tr.s, sizeof(d.s));
        stack.push_back(d);
        trk.energy = x * trk.energy;
        trk.mode = m1;
        trk.k_dir = k1;
        const auto kin = L_.map_k_to_vg(m1, k1);
        trk.vg_dir = kin.vg_dir;
        trk.vg_mag = kin.vg_mag;
    }
    const CrystalLattice& L_;
    const DetectorModel& D_;
    const SimulationEngine eng_;
    Theta th_;
};

template <class F>
void parallel_for(uint64_t n, unsigned threads, F&& f) {
    std::atomic<uint64_t> next{0};
    const unsigned nt = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                const uint64_t i = next.fetch_add(1);
                if (i >= n) return;
                f(i);
            }
        });
    for (auto& t : pool) t.join();
}

std::vector<double> read_weights(const std::string& path, int n_bins) {
    std::vector<double> w(n_bins, 0.0);
    if (path == "-") return w;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(w.data(), 8, n_bins, f) != static_cast<size_t>(n_bins)) {
        std::fprintf(stderr, "cannot read %d weights from %s\n", n_bins, path.c_str());
        std::exit(1);
    }
    std::fclose(f);
    return w;
}

bool same_hit(const SensorHit& a, const SensorHit& b) {
    return std::memcmp(&a.pos, &b.pos, sizeof(a.pos)) == 0 && a.time == b.time && a.edep == b.edep &&
           a.incident_energy == b.incident_energy && a.surface_id == b.surface_id && a.mode == b.mode &&
           a.channel_id == b.channel_id;
}

int cmd_check(const Theta& th, uint64_t first, uint64_t n, unsigned threads) {
    const Setup S(th);
    const SimulationEngine eng(S.lattice, S.det);
    const Restated R(S.lattice, S.det, th);
    std::atomic<uint64_t> bad{0}, hits{0};
    parallel_for(n, threads, [&](uint64_t i) {
        Rng rng = Rng::for_stream(kSeed, first + i);
        const PhononTrack p = generate(eng, S.det, rng);
        Rng rng2 = rng;
        std::vector<PhononTrack> st1{p};
        std::vector<SensorHit> h1, h2;
        SimStats s1, s2;
        eng.transport(st1, h1, s1, rng);
        std::vector<STrack> st2{STrack{p, {0, 0, 0, 0}}};
        std::vector<std::array<double, 4>> hs;
        R.transport(st2, h2, hs, s2, rng2);
        bool ok = h1.size() == h2.size() && s1.total_steps == s2.total_steps &&
                  s1.isotope_scatters == s2.isotope_scatters && s1.surface_refls == s2.surface_refls &&
                  s1.decays_L_to_TT == s2.decays_L_to_TT && s1.decays_L_to_LT == s2.decays_L_to_LT &&
                  s1.killed_tracks == s2.killed_tracks && s1.total_deposited_eV == s2.total_deposited_eV &&
                  s1.escaped_or_killed_eV == s2.escaped_or_killed_eV;
        for (size_t k = 0; ok && k < h1.size(); ++k) ok = same_hit(h1[k], h2[k]);
        if (!ok) bad++;
        hits += h1.size();
    });
    std::printf("{\"events\": %" PRIu64 ", \"mismatched_events\": %" PRIu64 ", \"hits\": %" PRIu64 "}\n", n,
                bad.load(), hits.load());
    return bad.load() == 0 ? 0 : 1;
}

int cmd_estimate(const Theta& th, uint64_t first, uint64_t n, unsigned threads, const Hist& H,
                 const std::vector<double>& w, const std::string& out, bool restated) {
    const Setup S(th);
    const SimulationEngine eng(S.lattice, S.det);
    const Restated R(S.lattice, S.det, th);
    const int cols = restated ? 5 : 1;
    std::vector<double> rows(n * cols, 0.0);
    std::vector<std::vector<double>> hist_ev(n);
    const double inv_th[4] = {1.0 / th.B, 1.0 / th.A, 1.0 / th.pd, 1.0 / th.f};
    parallel_for(n, threads, [&](uint64_t i) {
        Rng rng = Rng::for_stream(kSeed, first + i);
        const PhononTrack p = generate(eng, S.det, rng);
        std::vector<SensorHit> hits;
        std::vector<std::array<double, 4>> hs;
        SimStats st;
        if (restated) {
            std::vector<STrack> stack{STrack{p, {0, 0, 0, 0}}};
            R.transport(stack, hits, hs, st, rng);
        } else {
            std::vector<PhononTrack> stack{p};
            eng.transport(stack, hits, st, rng);
        }
        std::vector<double>& he = hist_ev[i];
        he.assign(H.n_bins, 0.0);
        double* row = rows.data() + i * cols;
        for (size_t k = 0; k < hits.size(); ++k) {
            const int b = H.bin(hits[k].time);
            if (b < 0) continue;
            he[b] += 1.0;  // weight 1 (no roulette)
            row[0] += w[b];
            if (restated)
                for (int c = 0; c < 4; ++c) row[1 + c] += w[b] * hs[k][c] * inv_th[c];
        }
    });
    std::vector<double> hist(H.n_bins, 0.0);
    for (uint64_t i = 0; i < n; ++i)
        for (int b = 0; b < H.n_bins; ++b) hist[b] += hist_ev[i][b];
    FILE* f = std::fopen(out.c_str(), "wb");
    if (!f) { std::perror(out.c_str()); return 1; }
    std::fwrite(hist.data(), 8, hist.size(), f);
    std::fwrite(rows.data(), 8, rows.size(), f);
    std::fclose(f);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 9) {
        std::fprintf(stderr, "usage: %s check|estimate|values B A pd f first n threads [n_bins t_max weights out]\n",
                     argv[0]);
        return 2;
    }
    const std::string cmd = argv[1];
    const Theta th{std::strtod(argv[2], nullptr), std::strtod(argv[3], nullptr), std::strtod(argv[4], nullptr),
                   std::strtod(argv[5], nullptr)};
    const uint64_t first = std::strtoull(argv[6], nullptr, 10), n = std::strtoull(argv[7], nullptr, 10);
    const unsigned threads = static_cast<unsigned>(std::atoi(argv[8]));
    if (cmd == "check") return cmd_check(th, first, n, threads);
    if ((cmd == "estimate" || cmd == "values") && argc == 13) {
        const Hist H{std::atoi(argv[9]), std::strtod(argv[10], nullptr)};
        const std::vector<double> w = read_weights(argv[11], H.n_bins);
        return cmd_estimate(th, first, n, threads, H, w, argv[12], cmd == "estimate");
    }
    std::fprintf(stderr, "bad arguments\n");
    return 2;
}
