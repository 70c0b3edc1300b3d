// Test of the C++ drop-in (include/cmpmc_b200/run_events_gpu.hpp). Built by oracle/Makefile
// (target _ref/shim_example) against the reference's own headers and linked with the
// correctly rounded libm of oracle/crlibm_libm.cpp for the reference's CPU transport; run by
// tests/test_shim.py.
//
// Every call site below is the reference's `run_events(engine, n, generate, options)` with
// its namespace changed to cmpmc_b200. Checks:
//   1. plain FP64 form on the mixed workload of the reference's tests/test_parallel.cpp:110-125
//      (203 events, phonons and e-/h+ pairs, Luke phonons sampled): every event identical to
//      the reference's CPU run_events (hit count, discrete hit fields, integer counters; hit
//      time, energy, incident energy and position within 1e-9 relative; FP64 totals 1e-12);
//   2. the same detector with SuperCDMS QET masks and a Cartesian mesh field (at least 97 % of
//      the events identical: facet ties of the mesh walk, see compare_exact), and with an
//      axisymmetric 2D mesh field (identical); meshes handed over with gpu_engine_for(engine);
//   3. batched FP32 form on 2,000 single-L events: hits per event and the deposited fraction
//      within 5 standard errors of the CPU run, and the ledger closed to 1e-6;
//   4. the cached context is reused for the same engine and rebuilt after a detector change.
// Exit status: 0 all checks pass, 1 a check failed (the reason is printed), 3 no device.
#include "cmpmc/cmpmc.hpp"
#include "cmpmc_b200/run_events_gpu.hpp"

#include <cmath>
#include <cstdio>
#include <functional>
#include <string>

// oracle/crlibm_libm.cpp (linked in): the reference's transport runs against a correctly
// rounded libm while the calling thread's flag is on
extern "C" void cmpmc_oracle_set_crlibm(int on);

namespace {

int g_failures = 0;

void check(bool ok, const std::string& what) {
    if (!ok) {
        std::printf("FAIL: %s\n", what.c_str());
        ++g_failures;
    }
}

bool rel_close(double a, double b, double rel) { return std::fabs(a - b) <= rel * std::max(std::fabs(b), 1e-300); }

// The reference's CPU run with the correctly rounded libm in the transport; the generator
// keeps the platform libm, as it does on the host side of the device path.
template <class Gen>
cmpmc::RunResult cpu_run(const cmpmc::SimulationEngine& engine, uint64_t n, Gen&& gen, const cmpmc::RunOptions& opt) {
    auto wrapped = [&](cmpmc::EventInput& in) {
        cmpmc_oracle_set_crlibm(0);
        gen(in);
        cmpmc_oracle_set_crlibm(1);
    };
    cmpmc::RunResult r = cmpmc::run_events(engine, n, wrapped, opt);
    cmpmc_oracle_set_crlibm(0);
    return r;
}

bool same_hit(const cmpmc::SensorHit& a, const cmpmc::SensorHit& b) {
    return a.surface_id == b.surface_id && a.excitation == b.excitation && a.mode == b.mode &&
           a.channel_id == b.channel_id && rel_close(a.time, b.time, 1e-9) && rel_close(a.edep, b.edep, 1e-9) &&
           rel_close(a.incident_energy, b.incident_energy, 1e-9) && rel_close(a.pos.x, b.pos.x, 1e-9) &&
           rel_close(a.pos.y, b.pos.y, 1e-9) && rel_close(a.pos.z, b.pos.z, 1e-9);
}

// min_frac < 1: a 3D mesh field, whose walk starts from a per-thread hint kept across events
// (mesh_field.hpp:119-122); a point within rounding of a facet can then resolve to the
// neighbouring tetrahedron, whose field differs in the last bits, depending on the thread's
// history, on the CPU as on the device. Such events and the totals they enter may differ.
void compare_exact(const char* name, const cmpmc::RunResult& dev, const cmpmc::RunResult& cpu, uint64_t n,
                   double min_frac = 1.0) {
    size_t agree = 0;
    for (uint64_t ev = 0; ev < n; ++ev) {
        const uint64_t d0 = dev.hit_offsets[ev], d1 = dev.hit_offsets[ev + 1];
        const uint64_t c0 = cpu.hit_offsets[ev], c1 = cpu.hit_offsets[ev + 1];
        bool ok = (d1 - d0) == (c1 - c0);
        for (uint64_t i = 0; ok && i < d1 - d0; ++i) ok = same_hit(dev.hits[d0 + i], cpu.hits[c0 + i]);
        agree += ok;
    }
    const cmpmc::SimStats& a = dev.stats;
    const cmpmc::SimStats& b = cpu.stats;
    const bool counters = a.total_steps == b.total_steps && a.isotope_scatters == b.isotope_scatters &&
                          a.decays_L_to_TT == b.decays_L_to_TT && a.decays_L_to_LT == b.decays_L_to_LT &&
                          a.surface_refls == b.surface_refls && a.sensor_hits == b.sensor_hits &&
                          a.killed_tracks == b.killed_tracks && a.charge_steps == b.charge_steps &&
                          a.luke_phonons_emitted == b.luke_phonons_emitted &&
                          a.intervalley_scatters == b.intervalley_scatters &&
                          a.charge_surface_refls == b.charge_surface_refls &&
                          a.charges_collected == b.charges_collected;
    const bool sums = rel_close(a.total_injected_eV, b.total_injected_eV, 1e-12) &&
                      rel_close(a.total_deposited_eV, b.total_deposited_eV, 1e-12) &&
                      rel_close(a.escaped_or_killed_eV, b.escaped_or_killed_eV, 1e-12) &&
                      rel_close(a.total_luke_phonon_eV, b.total_luke_phonon_eV, 1e-12) &&
                      rel_close(a.charge_recomb_edep_eV, b.charge_recomb_edep_eV, 1e-12);
    std::printf("%s: %zu of %llu events identical, %zu device hits, %zu CPU hits, steps %llu / %llu\n", name, agree,
                (unsigned long long)n, dev.hits.size(), cpu.hits.size(), (unsigned long long)a.total_steps,
                (unsigned long long)b.total_steps);
    if (min_frac >= 1.0) {
        check(agree == n, std::string(name) + ": every event identical");
        check(counters, std::string(name) + ": integer counters equal");
        check(sums, std::string(name) + ": energy totals within 1e-12");
    } else {
        check(static_cast<double>(agree) >= min_frac * static_cast<double>(n),
              std::string(name) + ": events identical up to facet ties of the mesh walk");
    }
}

}  // namespace

int main() {
    using namespace cmpmc;
    int n_dev = 0;
    if (cmpmc_gpu_device_count(&n_dev) != CMPMC_OK || n_dev < 1) {
        std::printf("no CUDA device\n");
        return 3;
    }
    const CrystalLattice lattice(materials::Germanium());
    DetectorModel det;
    det.e_field = UniformElectricField::from_bias(2.0, 2.54 * units::cm);
    det.luke_sample_fraction = 0.02;
    const SimulationEngine engine(lattice, det);
    const ChargePhysics charges(lattice);
    const size_t n_valleys = lattice.config().valley_dirs.size();
    // the reference's own generator (tests/test_parallel.cpp:110-125)
    auto gen = [&](EventInput& in) {
        if (in.event_id % 2 == 0) {
            in.phonons.push_back(engine.make_track({0, 0, 0}, in.rng.isotropic_dir(), PhononMode::FT, 7.5e-3));
            in.injected_eV += 7.5e-3;
        } else {
            const auto v = static_cast<uint16_t>(in.rng.uniform() * n_valleys) % n_valleys;
            in.charges.push_back(charges.make_charge(ExcitationType::Electron, {0, 0, 0}, in.rng.isotropic_dir(), 1e-6, v));
            in.charges.push_back(charges.make_charge(ExcitationType::Hole, {0, 0, 0}, in.rng.isotropic_dir(), 1e-6, 0));
        }
    };
    RunOptions opt;
    opt.seed = 77;

    // 1. plain FP64 through the drop-in
    const RunResult r = cmpmc_b200::run_events(engine, 203, gen, opt);
    const RunResult c = cpu_run(engine, 203, gen, opt);
    compare_exact("mixed pairs/phonons", r, c, 203);
    check(r.hit_offsets.size() == 204 && r.hit_offsets.back() == r.hits.size(), "hit_offsets shape");

    // 4a. the same engine reuses its cached context
    cmpmc_b200::GpuEngine* first = &cmpmc_b200::gpu_engine_for(engine);
    check(first == &cmpmc_b200::gpu_engine_for(engine), "cached context reused");

    // 2. masks + Cartesian mesh field; axisymmetric 2D mesh field
    const double R = det.solid.radius, h = det.solid.half_z;
    {
        DetectorModel det2 = det;
        auto pot = [h](const Vec3& p) { return 2.0 * (p.z + h) / (2.0 * h); };
        for (int f = 0; f < 2; ++f)
            det2.surfaces[f].electrode_mask = geometry::ElectrodePatternMask::supercdms_qet_mask(R, 0.8);
        det2.mesh_field_3d = geometry::TriLinearMesh3D::build_cartesian_grid(R, R, h, 8, 8, 8, pot);
        const SimulationEngine engine2(lattice, det2);
        cmpmc_b200::gpu_engine_for(engine2).set_cartesian_mesh(R, R, h, 8, 8, 8, pot);
        const RunResult m = cmpmc_b200::run_events(engine2, 203, gen, opt);
        const RunResult mc = cpu_run(engine2, 203, gen, opt);
        compare_exact("masks + 3D mesh", m, mc, 203, 0.97);
        size_t on_pad = 0;
        for (const SensorHit& x : m.hits) on_pad += (x.channel_id >= 0);
        check(on_pad > 0, "masked hits carry channels");
    }
    {
        DetectorModel det3 = det;
        auto pot2 = [h](double r, double z) { return 2.0 * (z + h) / (2.0 * h) + 0.1 * r / h; };
        det3.mesh_field_2d = geometry::BiLinearMesh2D::build_grid(0.0, R, -h, h, 16, 16, pot2, true);
        const SimulationEngine engine3(lattice, det3);
        cmpmc_b200::gpu_engine_for(engine3).set_grid_mesh2d(0.0, R, -h, h, 16, 16, pot2, true);
        const RunResult a = cmpmc_b200::run_events(engine3, 203, gen, opt);
        const RunResult ac = cpu_run(engine3, 203, gen, opt);
        compare_exact("2D mesh", a, ac, 203);
    }

    // 3. batched FP32 form: statistics against the CPU
    {
        const DetectorModel det0;
        const SimulationEngine engine0(lattice, det0);
        auto gen0 = [&](EventInput& in) {
            in.phonons.push_back(engine0.make_track({0, 0, 0}, in.rng.isotropic_dir(), PhononMode::L, 7.5e-3));
            in.injected_eV += 7.5e-3;
        };
        RunOptions o0;
        o0.seed = 42;
        const uint64_t n = 2000;
        cmpmc_b200::GpuRunOptions batched;
        batched.form = cmpmc_b200::Form::BatchedFP32;
        const RunResult b = cmpmc_b200::run_events(engine0, n, gen0, o0, batched);
        const RunResult bc = cpu_run(engine0, n, gen0, o0);
        auto per_event = [n](const RunResult& x, double& mean_hits, double& se_hits, double& mean_dep, double& se_dep) {
            double s1 = 0, s2 = 0, d1 = 0, d2 = 0;
            for (uint64_t ev = 0; ev < n; ++ev) {
                const double k = static_cast<double>(x.hit_offsets[ev + 1] - x.hit_offsets[ev]);
                double dep = 0;
                for (uint64_t i = x.hit_offsets[ev]; i < x.hit_offsets[ev + 1]; ++i) dep += x.hits[i].edep;
                s1 += k; s2 += k * k; d1 += dep; d2 += dep * dep;
            }
            mean_hits = s1 / n;
            se_hits = std::sqrt(std::max(0.0, s2 / n - mean_hits * mean_hits) / n);
            mean_dep = d1 / n;
            se_dep = std::sqrt(std::max(0.0, d2 / n - mean_dep * mean_dep) / n);
        };
        double mh, sh, md, sd, mhc, shc, mdc, sdc;
        per_event(b, mh, sh, md, sd);
        per_event(bc, mhc, shc, mdc, sdc);
        const double zh = std::fabs(mh - mhc) / std::sqrt(sh * sh + shc * shc);
        const double zd = std::fabs(md - mdc) / std::sqrt(sd * sd + sdc * sdc);
        const double closure =
            std::fabs(b.stats.total_injected_eV - b.stats.total_deposited_eV - b.stats.escaped_or_killed_eV) /
            b.stats.total_injected_eV;
        std::printf("batched FP32 single L: hits/event %.3f vs %.3f (z %.2f), deposited/event %.4e vs %.4e eV (z %.2f), "
                    "closure %.2e\n", mh, mhc, zh, md, mdc, zd, closure);
        check(zh < 5.0 && zd < 5.0, "batched hits and deposits within 5 standard errors");
        check(closure < 1e-6, "batched ledger closes");
    }

    // 4b. a detector changed after the first call gets a new context
    {
        DetectorModel det4 = det;
        const SimulationEngine engine4(lattice, det4);
        const RunResult x = cmpmc_b200::run_events(engine4, 8, gen, opt);
        det4.max_bounces = 10;  // the engine holds a reference: it sees the change
        const RunResult y = cmpmc_b200::run_events(engine4, 8, gen, opt);
        const RunResult yc = cpu_run(engine4, 8, gen, opt);
        compare_exact("detector changed after a call", y, yc, 8);
        check(x.stats.total_steps != y.stats.total_steps, "the changed detector is used");
    }
    std::printf("%s\n", g_failures ? "shim checks FAILED" : "shim checks passed");
    return g_failures ? 1 : 0;
}
