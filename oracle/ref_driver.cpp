// Test infrastructure only (the checker): drives the unmodified reference CMPMC
// library, compiled from its own headers, on the canonical workloads and writes
// its per-event results as raw binary records. Nothing in the product links or
// runs this program; tests/golden/make_golden.py and bench.py's CPU-baseline leg
// call it.
//
// Usage:
//   cmpmc_ref dump <workload> <first_event> <n_events> <threads> <out_prefix>
//       Runs events [first, first+n) one by one (each from Rng::for_stream(seed, ev),
//       as run_events does, parallel.hpp:102-114) and writes
//         <prefix>.init   per event: u64 rng_state[4] after the generator, f64 injected,
//                         u64 n_phonons, u64 n_charges, then the PhononTrack /
//                         ChargeTrack records (128 B each)
//         <prefix>.events per event: u64 n_hits, SimStats (208 B)
//         <prefix>.hits   SensorHit records (56 B each), in event order
//   cmpmc_ref time <workload> <first_event> <n_events> <threads>
//       Times the reference's own run_events (parallel.hpp:76-148) on the workload
//       and prints one JSON line (wall seconds from RunResult::wall_seconds).
//   cmpmc_ref rng <seed> <stream> <count>
//       Prints next_u64 / uniform / isotropic_dir / lambertian_dir vectors.
//   cmpmc_ref mask <n_points> <out>
//       For n points uniform in [-R, R]^2 (Rng::for_stream(9, 0)): the channel of the
//       SuperCDMS QET mask (fill 0.8, find_channel drawing from the same stream after each
//       point) and of a 4 x 4 rectangular grid (find_geometric_channel); x, y as doubles,
//       then the two channels as int32.
//   cmpmc_ref kin <n> <out>
//       map_k_to_vg of the Ge lattice in the Exact and the Bilinear modes for n directions
//       (Rng::for_stream(21, 0) isotropic) and the three modes: per direction and mode
//       (vg_dir[3], vg_mag) for Exact, then for Bilinear (8 doubles)
//   cmpmc_ref amm <n> <out>
//       IsotropicAMMInterface (the c0a media): transmission of L and transverse phonons at
//       cos theta = (i + 0.5) / n, i < n; 2n doubles (L then T)
//   cmpmc_ref kaplan <n> <out>
//       KaplanSurrogateLUT of the default Al film (seed 1337): for n energies
//       E = Delta (1 + 45 u) (Rng::for_stream(3, 0), sub-gap, in-table and above-table),
//       absorb_phonon_fast(E) with the same stream; per record E, edep (f64), the count
//       (u32) and the re-emitted energies (f64).
//   cmpmc_ref yield <out>
//       Ionisation yields at 400 energies 10^(7 i / 399) eV for Germanium() and Silicon():
//       the five NIEL models (default empirical parameters), Empirical with a fixed k, and
//       EnergyPartition::lindhard_ionization_yield(E, 2, 4); [2][7][400] doubles.
//   cmpmc_ref partition <out>
//       EnergyPartition::partition_deposit on the Germanium lattice for 48 deposits (case i:
//       E = 10^(1 + 4 i / 47) eV, nuclear recoil when i is odd, pos (i, -2, 3) mm, time
//       i ns, Rng::for_stream(8, i), at most 100 sampled pairs and 150 sampled phonons,
//       options by i % 4: defaults / no Fano fluctuations / no charge cloud and 16 sampled
//       pairs / Empirical yield and 7 sampled phonons);
//       per case the Result, the record counts, the records and the final Rng state.
//   cmpmc_ref merge <out>
//       HitMerger(lattice, 1 mm, 64 pairs / 64 phonons) over three synthetic primary
//       tracks of 12 steps (charged; neutral; nuclear-recoil-like), Rng::for_stream(9, 0),
//       then a final flush: per step the process_step flag, then the records, the final
//       Rng state.
//   cmpmc_ref mesh2 <n_points> <out>
//       Builds the tp2 axisymmetric (r, z) mesh and a planar (x, y) mesh
//       (build_grid(-R, R, -R, R, 32, 32) of V = 3 (x + R) / 2R + 0.5 (y / R)^2) and writes,
//       for n points (the first 16 on the axis, x = y = 0, the rest drawn in the cylinder,
//       Rng::for_stream(6, 0)), the point, then field_at and potential_at of each mesh
//       (one walk hint per mesh and query kind): 11 doubles per point.
//   cmpmc_ref meshfile <coords> <tets> <coord_unit_m> <potential_unit_V> <n_points> <out>
//       TriLinearMesh3D::load_from_files of the two ASCII files, then as `mesh` for n points
//       drawn in the default cylinder from Rng::for_stream(7, 0): 7 doubles per point.
//   cmpmc_ref mesh <n_points> <out>
//       Builds the c3 field mesh and writes, for n points drawn in the cylinder
//       (Rng::for_stream(5, 0)), the point, field_at and potential_at (each with one
//       walk hint carried from point to point) as 7 doubles per point.
//
// Workloads (seeds and draw orders are the canonical generators of this project):
//   c0  default Ge detector; one L phonon, 7.5 meV, at the origin, isotropic; seed 42
//   c1  default detector; 100 phonons per event: E = 1 meV*exp(ln30*u), mode L/ST/FT
//       at u < 0.10 / < 0.46 / else, origin uniform in the cylinder (rejection in x,y
//       then z), direction isotropic; seed 7
//   c2  uniform field 4 V over 2.54 cm, luke_sample_fraction 0; one e-/h+ pair per
//       event: origin as c1, valley = next_u64() % 4, e- isotropic, h+ isotropic,
//       1 ueV each; seed 11; events_per_chunk 1
//   c4  default detector; one L phonon, 7.5 meV, origin as c1, isotropic; seed 17
//   tp  the mixed workload of the reference's own tests/test_parallel.cpp:110-125
//       (even events: FT 7.5 meV phonon at the origin; odd events: e-/h+ pair),
//       field 2 V over 2.54 cm, luke_sample_fraction 0.02; seed 77
//   tpl same as tp with luke_sample_fraction 1 (every Luke phonon tracked)
//   c3  electron recoils: E = 10 eV * 10^(3u), origin as c1, split by the reference's
//       EnergyPartition::partition_deposit (max_sampled_pairs 4096, other options at their
//       defaults); field from TriLinearMesh3D::build_cartesian_grid(R, R, h, 58, 58, 57)
//       with V = 4 (z + h) / 2h + 0.2 ((x^2 + y^2) / R^2) sin(pi z / 2h); all Luke phonons
//       tracked; seed 13; events_per_chunk 1
//   c0a c0 with an IsotropicAMMInterface (Ge substrate {5323, 5324.2077, 3258.7879}, Al film
//       {2700, 6420, 3040}) on both faces; seed 42
//   tpd tp with ChargeRelease::BulkDebye; tpe tp with ChargeRelease::ElectrodeFilm; seed 77
//   c0x c0 with KinematicsMode::Exact; c0b c0 with KinematicsMode::Bilinear; seed 42
//   tp2 tp with the field of an axisymmetric BiLinearMesh2D::build_grid(0, R, -h, h, 40, 40)
//       of V = 2 (z + h) / 2h + 0.3 (r / R)^2 (z / h) (mesh_field_2d; no 3D mesh); seed 77
//   c0m c0 with the SuperCDMS QET electrode mask (fill fraction 0.8) on both faces; seed 42
//   tpm tp with the same masks on both faces; seed 77
//   c3s the same with E = 10 eV * 10^u, max_sampled_phonons 20 (prompt phonons carry the
//       weight n_true / 20) and luke_sample_fraction 0.05
//   c0r c0 with Russian roulette (russian_roulette_bounces 64, survival 0.5); seed 42
//   tps tp with DetectorModel::ChargeStepping::LemanSecondOrder; seed 77
//   tpt tp in a crystal with every trapping and trap-ionisation mean free path set
//       (e 2 cm, h 3 cm; ionisation e 4 / 5 cm, h 4.5 / 6 cm); seed 77
//   pub the reference's published phonon benchmark (benchmarks/cmpmc_bench.cpp:45-67):
//       demo polynomial surfaces (sensor faces with prob_abs 1, bare side wall),
//       max_bounces 100, no field; one 7.5 meV phonon at the origin, mode ST / FT / L at
//       u < 0.53539 / < 0.90217 / else, isotropic; seed 12345 (the benchmark's default)
//   pubc the same detector at 4 V with luke_sample_fraction 0 and one e-/h+ pair per event at
//       the origin (the benchmark's `charge` mode); seed 12345
//
// Built with -DCMPMC_ORACLE_CRLIBM and linked with crlibm_libm.cpp (as cmpmc_ref_crlibm),
// the same program runs the reference against a correctly rounded libm in the transport;
// the generators and the lattice build keep the platform libm, as they do in the device
// path (they run on the host there). The reference's headers are compiled identically in
// both builds.
#ifdef CMPMC_ORACLE_CRLIBM
extern "C" void cmpmc_oracle_set_crlibm(int on);
#define CMPMC_SET_CRLIBM(v) cmpmc_oracle_set_crlibm((v) ? 1 : 0)
#else
#define CMPMC_SET_CRLIBM(v) ((void)0)
#endif
#include "cmpmc/cmpmc.hpp"

#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using namespace cmpmc;

namespace {

struct Workload {
    std::string name;
    uint64_t seed = 1;
    uint32_t events_per_chunk = 16;
};

Workload make_workload(const std::string& w) {
    Workload wl;
    wl.name = w;
    if (w == "c0" || w == "c0m" || w == "c0a" || w == "c0x" || w == "c0b" || w == "c0r") wl.seed = 42;
    else if (w == "pub") { wl.seed = 12345; wl.events_per_chunk = 64; }
    else if (w == "pubc") { wl.seed = 12345; wl.events_per_chunk = 1; }
    else if (w == "tps" || w == "tpt") wl.seed = 77;
    else if (w == "c1") wl.seed = 7;
    else if (w == "c2") { wl.seed = 11; wl.events_per_chunk = 1; }
    else if (w == "c4") wl.seed = 17;
    else if (w == "tp" || w == "tpl" || w == "tpm" || w == "tpd" || w == "tpe" || w == "tp2") wl.seed = 77;
    else if (w == "c3" || w == "c3s") { wl.seed = 13; wl.events_per_chunk = 1; }
    else { std::fprintf(stderr, "unknown workload %s\n", w.c_str()); std::exit(2); }
    return wl;
}

physics::IsotropicAMMInterface amm_ge_al() {
    physics::IsotropicAMMInterface a;
    a.substrate = {5323.0, 5324.2077, 3258.7879};
    a.film = {2700.0, 6420.0, 3040.0};
    return a;
}

double recoil_potential(const Vec3& p, double R, double h) {
    const double rr = (p.x * p.x + p.y * p.y) / (R * R);
    return 4.0 * (p.z + h) / (2.0 * h) + 0.2 * rr * std::sin(units::pi * p.z / (2.0 * h));
}

geometry::TriLinearMesh3D recoil_mesh(const CylinderSolid& s) {
    const double R = s.radius, h = s.half_z;
    return geometry::TriLinearMesh3D::build_cartesian_grid(
        R, R, h, 58, 58, 57, [R, h](const Vec3& p) { return recoil_potential(p, R, h); });
}

double axisym_potential(double r, double z, double R, double h) {
    return 2.0 * (z + h) / (2.0 * h) + 0.3 * (r / R) * (r / R) * (z / h);
}

geometry::BiLinearMesh2D axisym_mesh(const CylinderSolid& s) {
    const double R = s.radius, h = s.half_z;
    return geometry::BiLinearMesh2D::build_grid(
        0.0, R, -h, h, 40, 40, [R, h](double r, double z) { return axisym_potential(r, z, R, h); }, true);
}

geometry::BiLinearMesh2D planar_mesh(const CylinderSolid& s) {
    const double R = s.radius;
    return geometry::BiLinearMesh2D::build_grid(
        -R, R, -R, R, 32, 32, [R](double x, double y) { return 3.0 * (x + R) / (2.0 * R) + 0.5 * (y / R) * (y / R); },
        false);
}

// tpt: every trapping and trap-ionisation channel on (charge_kernels.hpp:103-126), mean
// free paths of a few cm so that a fair share of the carriers trap or ionise a trap
CrystalConfig config_for(const std::string& w) {
    CrystalConfig c = materials::Germanium();
    if (w == "tpt") {
        c.e_trapping_mfp_m = 0.02;
        c.h_trapping_mfp_m = 0.03;
        c.e_trap_ion_d0_mfp_m = 0.04;
        c.e_trap_ion_a_mfp_m = 0.05;
        c.h_trap_ion_d_mfp_m = 0.045;
        c.h_trap_ion_a0_mfp_m = 0.06;
    }
    return c;
}

void setup_lattice(const std::string& w, CrystalLattice& lattice) {
    if (w == "c0x") lattice.set_kinematics_mode(CrystalLattice::KinematicsMode::Exact);
    if (w == "c0b") lattice.set_kinematics_mode(CrystalLattice::KinematicsMode::Bilinear);
}

void setup_detector(const std::string& w, DetectorModel& det) {
    if (w == "c3" || w == "c3s") {
        det.mesh_field_3d = recoil_mesh(det.solid);
        det.luke_sample_fraction = (w == "c3") ? 1.0 : 0.05;
    } else if (w == "c2") {
        det.e_field = UniformElectricField::from_bias(4.0, 2.54 * units::cm);
        det.luke_sample_fraction = 0.0;
    } else if (w == "pub" || w == "pubc") {
        // the published benchmark's detector (benchmarks/cmpmc_bench.cpp:45-57)
        det.allow_unvalidated = true;
        SurfaceProperty sensor = SurfaceProperty::demo_polynomial_sensor_surface();
        sensor.prob_abs = 1.0;
        const SurfaceProperty wall = SurfaceProperty::demo_polynomial_bare_surface();
        det.surfaces = {sensor, sensor, wall};
        det.max_bounces = 100;
        det.e_field = UniformElectricField::from_bias(w == "pub" ? 0.0 : 4.0, 2.54 * units::cm);
        det.luke_sample_fraction = (w == "pubc") ? 0.0 : 1.0;
    } else if (w == "tp" || w == "tpl" || w == "tpm" || w == "tpd" || w == "tpe" || w == "tp2" || w == "tps" ||
               w == "tpt") {
        det.e_field = UniformElectricField::from_bias(2.0, 2.54 * units::cm);
        if (w == "tps") det.charge_stepping = DetectorModel::ChargeStepping::LemanSecondOrder;
        if (w == "tp2") det.mesh_field_2d = axisym_mesh(det.solid);
        det.luke_sample_fraction = (w == "tpl") ? 1.0 : 0.02;
        if (w == "tpd") det.charge_release = DetectorModel::ChargeRelease::BulkDebye;
        if (w == "tpe") det.charge_release = DetectorModel::ChargeRelease::ElectrodeFilm;
    }
    if (w == "c0r") det.russian_roulette_bounces = 64;  // survival 0.5 (the default)
    if (w == "c0a")
        for (int f = 0; f < 2; ++f) det.surfaces[f].amm_interface = amm_ge_al();
    if (w == "c0m" || w == "tpm")
        for (int f = 0; f < 2; ++f)
            det.surfaces[f].electrode_mask =
                geometry::ElectrodePatternMask::supercdms_qet_mask(det.solid.radius, 0.8);
}

Vec3 uniform_origin(const CylinderSolid& s, Rng& rng) {
    double x, y;
    do {
        x = (2.0 * rng.uniform() - 1.0) * s.radius;
        y = (2.0 * rng.uniform() - 1.0) * s.radius;
    } while (x * x + y * y > s.radius * s.radius);
    const double z = (2.0 * rng.uniform() - 1.0) * s.half_z;
    return {x, y, z};
}

struct Generator {
    std::string w;
    const SimulationEngine* engine;
    const ChargePhysics* charges;
    const DetectorModel* det;
    size_t n_valleys;
    const EnergyPartition* partition;

    // the generator runs on the host with the platform libm in every build
    void operator()(EventInput& in) const {
        CMPMC_SET_CRLIBM(false);
        generate(in);
        CMPMC_SET_CRLIBM(true);
    }

    void generate(EventInput& in) const {
        if (w == "c0" || w == "c0m" || w == "c0a" || w == "c0x" || w == "c0b" || w == "c0r") {
            in.phonons.push_back(engine->make_track({0, 0, 0}, in.rng.isotropic_dir(), PhononMode::L, 7.5e-3));
            in.injected_eV += 7.5e-3;
        } else if (w == "pub") {  // benchmarks/cmpmc_bench.cpp:63-67
            const double u = in.rng.uniform();
            const PhononMode m = u < 0.53539 ? PhononMode::ST : u < 0.90217 ? PhononMode::FT : PhononMode::L;
            in.phonons.push_back(engine->make_track({0, 0, 0}, in.rng.isotropic_dir(), m, 7.5e-3));
            in.injected_eV += 7.5e-3;
        } else if (w == "pubc") {  // benchmarks/cmpmc_bench.cpp:68-71
            const auto v = static_cast<uint16_t>(in.rng.uniform() * n_valleys) % n_valleys;
            in.charges.push_back(charges->make_charge(ExcitationType::Electron, {0, 0, 0}, in.rng.isotropic_dir(), 1e-6, v));
            in.charges.push_back(charges->make_charge(ExcitationType::Hole, {0, 0, 0}, in.rng.isotropic_dir(), 1e-6, 0));
        } else if (w == "c1") {
            for (int j = 0; j < 100; ++j) {
                const double E = 1e-3 * std::exp(std::log(30.0) * in.rng.uniform());
                const double um = in.rng.uniform();
                const PhononMode m = um < 0.10 ? PhononMode::L : (um < 0.46 ? PhononMode::ST : PhononMode::FT);
                const Vec3 p = uniform_origin(det->solid, in.rng);
                const Vec3 d = in.rng.isotropic_dir();
                in.phonons.push_back(engine->make_track(p, d, m, E));
                in.injected_eV += E;
            }
        } else if (w == "c2") {
            const Vec3 p = uniform_origin(det->solid, in.rng);
            const uint16_t v = static_cast<uint16_t>(in.rng.next_u64() % 4);
            const Vec3 de = in.rng.isotropic_dir();
            in.charges.push_back(charges->make_charge(ExcitationType::Electron, p, de, 1e-6, v));
            const Vec3 dh = in.rng.isotropic_dir();
            in.charges.push_back(charges->make_charge(ExcitationType::Hole, p, dh, 1e-6, 0));
        } else if (w == "c3" || w == "c3s") {
            const double u = in.rng.uniform();
            const double E = (w == "c3") ? 10.0 * std::pow(10.0, 3.0 * u) : 10.0 * std::pow(10.0, u);
            const Vec3 p = uniform_origin(det->solid, in.rng);
            PartitionOptions opts;
            opts.max_sampled_pairs = 4096;
            if (w == "c3s") opts.max_sampled_phonons = 20;
            partition->partition_deposit(p, 0.0, E, false, in.charges, in.phonons, in.rng, opts);
            in.injected_eV += E;
        } else if (w == "c4") {
            const Vec3 p = uniform_origin(det->solid, in.rng);
            const Vec3 d = in.rng.isotropic_dir();
            in.phonons.push_back(engine->make_track(p, d, PhononMode::L, 7.5e-3));
            in.injected_eV += 7.5e-3;
        } else {  // tp, tpl: tests/test_parallel.cpp:110-125
            if (in.event_id % 2 == 0) {
                in.phonons.push_back(engine->make_track({0, 0, 0}, in.rng.isotropic_dir(), PhononMode::FT, 7.5e-3));
                in.injected_eV += 7.5e-3;
            } else {
                const auto v = static_cast<uint16_t>(in.rng.uniform() * n_valleys) % n_valleys;
                in.charges.push_back(charges->make_charge(ExcitationType::Electron, {0, 0, 0}, in.rng.isotropic_dir(), 1e-6, v));
                in.charges.push_back(charges->make_charge(ExcitationType::Hole, {0, 0, 0}, in.rng.isotropic_dir(), 1e-6, 0));
            }
        }
    }
};

struct EventRecord {
    uint64_t rng_after_gen[4];
    double injected;
    std::vector<PhononTrack> phonons;
    std::vector<ChargeTrack> charges;
    SimStats stats;
    std::vector<SensorHit> hits;
};

FILE* open_or_die(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(1); }
    return f;
}

int cmd_dump(const std::string& w, uint64_t first, uint64_t n, unsigned threads, const std::string& prefix) {
    const Workload wl = make_workload(w);
    CrystalLattice lattice(config_for(w));
    setup_lattice(w, lattice);
    DetectorModel det;
    setup_detector(w, det);
    const SimulationEngine engine(lattice, det);
    const ChargePhysics cp(lattice);
    const EnergyPartition part(lattice);
    const Generator gen{w, &engine, &cp, &det, lattice.config().valley_dirs.size(), &part};

    std::vector<EventRecord> rec(n);
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        std::vector<PhononTrack> ph;
        std::vector<ChargeTrack> ch;
        for (;;) {
            const uint64_t i = next.fetch_add(1);
            if (i >= n) return;
            const uint64_t ev = first + i;
            EventRecord& r = rec[i];
            Rng rng = Rng::for_stream(wl.seed, ev);
            ph.clear();
            ch.clear();
            EventInput in{ev, rng, ph, ch, 0.0};
            gen(in);
            std::memcpy(r.rng_after_gen, rng.s, sizeof(r.rng_after_gen));
            r.injected = in.injected_eV;
            r.phonons = ph;
            r.charges = ch;
            r.stats.total_injected_eV += in.injected_eV;
            if (!ch.empty()) engine.transport_charges(ch, ph, r.hits, r.stats, rng);
            if (!ph.empty()) engine.transport(ph, r.hits, r.stats, rng);
        }
    };
    const unsigned nt = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();

    FILE* fi = open_or_die(prefix + ".init");
    FILE* fe = open_or_die(prefix + ".events");
    FILE* fh = open_or_die(prefix + ".hits");
    static_assert(sizeof(PhononTrack) == 128 && sizeof(ChargeTrack) == 128 && sizeof(SensorHit) == 56 &&
                  sizeof(SimStats) == 208, "record layout");
    for (const EventRecord& r : rec) {
        const uint64_t np = r.phonons.size(), nc = r.charges.size(), nh = r.hits.size();
        std::fwrite(r.rng_after_gen, 8, 4, fi);
        std::fwrite(&r.injected, 8, 1, fi);
        std::fwrite(&np, 8, 1, fi);
        std::fwrite(&nc, 8, 1, fi);
        if (np) std::fwrite(r.phonons.data(), sizeof(PhononTrack), np, fi);
        if (nc) std::fwrite(r.charges.data(), sizeof(ChargeTrack), nc, fi);
        std::fwrite(&nh, 8, 1, fe);
        std::fwrite(&r.stats, sizeof(SimStats), 1, fe);
        if (nh) std::fwrite(r.hits.data(), sizeof(SensorHit), nh, fh);
    }
    std::fclose(fi);
    std::fclose(fe);
    std::fclose(fh);
    return 0;
}

int cmd_time(const std::string& w, uint64_t first, uint64_t n, unsigned threads) {
    const Workload wl = make_workload(w);
    const auto t0 = std::chrono::steady_clock::now();
    CrystalLattice lattice(config_for(w));
    setup_lattice(w, lattice);
    DetectorModel det;
    setup_detector(w, det);
    const SimulationEngine engine(lattice, det);
    const ChargePhysics cp(lattice);
    const EnergyPartition part(lattice);
    const Generator gen{w, &engine, &cp, &det, lattice.config().valley_dirs.size(), &part};
    const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    // run_events numbers events from 0; an offset range runs through a shifted generator
    // whose streams are Rng::for_stream(seed, first + i), exactly as in the full run.
    RunOptions opt;
    opt.threads = threads;
    opt.seed = wl.seed;
    opt.events_per_chunk = wl.events_per_chunk;
    opt.keep_hits = true;
    RunResult r;
    if (first == 0) {
        r = run_events(engine, n, gen, opt);
    } else {
        auto shifted = [&](EventInput& in) {
            in.rng = Rng::for_stream(wl.seed, first + in.event_id);
            EventInput sh{first + in.event_id, in.rng, in.phonons, in.charges, 0.0};
            gen(sh);
            in.injected_eV = sh.injected_eV;
        };
        r = run_events(engine, n, shifted, opt);
    }
    uint64_t n_primary = 0;
    if (w == "c1") n_primary = 100 * n; else n_primary = n;
    std::printf("{\"workload\": \"%s\", \"first_event\": %" PRIu64 ", \"n_events\": %" PRIu64
                ", \"threads\": %u, \"wall_seconds\": %.6f, \"init_seconds\": %.6f, \"primaries\": %" PRIu64
                ", \"total_steps\": %" PRIu64 ", \"charge_steps\": %" PRIu64 ", \"sensor_hits\": %" PRIu64
                ", \"n_hits\": %zu, \"injected_eV\": %.17g, \"deposited_eV\": %.17g, \"escaped_eV\": %.17g}\n",
                w.c_str(), first, n, r.threads_used, r.wall_seconds, init_s, n_primary,
                r.stats.total_steps, r.stats.charge_steps, r.stats.sensor_hits, r.hits.size(),
                r.stats.total_injected_eV, r.stats.total_deposited_eV, r.stats.escaped_or_killed_eV);
    return 0;
}

int cmd_rng(uint64_t seed, uint64_t stream, int count) {
    Rng a = Rng::for_stream(seed, stream);
    std::printf("state %" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 "\n", a.s[0], a.s[1], a.s[2], a.s[3]);
    for (int i = 0; i < count; ++i) std::printf("u64 %" PRIu64 "\n", a.next_u64());
    for (int i = 0; i < count; ++i) std::printf("uniform %.17g\n", a.uniform());
    for (int i = 0; i < count; ++i) {
        const Vec3 d = a.isotropic_dir();
        std::printf("iso %.17g %.17g %.17g\n", d.x, d.y, d.z);
    }
    const Vec3 normals[3] = {{0, 0, -1}, {0, 0, 1}, {-0.6, -0.8, 0}};
    for (int i = 0; i < count; ++i) {
        const Vec3 d = a.lambertian_dir(normals[i % 3]);
        std::printf("lamb %.17g %.17g %.17g\n", d.x, d.y, d.z);
    }
    Rng b(12345);
    std::printf("seeded %" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 "\n", b.s[0], b.s[1], b.s[2], b.s[3]);
    return 0;
}

int cmd_mask(uint64_t n, const std::string& out) {
    const DetectorModel det;
    const double R = det.solid.radius;
    const auto qet = geometry::ElectrodePatternMask::supercdms_qet_mask(R, 0.8);
    const auto grid = geometry::ElectrodePatternMask::rectangular_grid_mask(4, 4, 1.5e-2, 1.5e-2, 0.6e-2, 0.5e-2);
    Rng rng = Rng::for_stream(9, 0);
    FILE* f = open_or_die(out);
    for (uint64_t i = 0; i < n; ++i) {
        const double x = (2.0 * rng.uniform() - 1.0) * R;
        const double y = (2.0 * rng.uniform() - 1.0) * R;
        const int32_t cq = qet.find_channel({x, y, 0.0}, rng);
        const int32_t cg = grid.find_geometric_channel(x, y);
        std::fwrite(&x, 8, 1, f);
        std::fwrite(&y, 8, 1, f);
        std::fwrite(&cq, 4, 1, f);
        std::fwrite(&cg, 4, 1, f);
    }
    std::fclose(f);
    return 0;
}

int cmd_kin(uint64_t n, const std::string& out) {
    CrystalLattice lat(materials::Germanium());
    Rng rng = Rng::for_stream(21, 0);
    std::vector<Vec3> ks(n);
    for (auto& k : ks) k = rng.isotropic_dir();
    FILE* f = open_or_die(out);
    for (auto mode : {CrystalLattice::KinematicsMode::Exact, CrystalLattice::KinematicsMode::Bilinear}) {
        lat.set_kinematics_mode(mode);
        for (const Vec3& k : ks)
            for (int m = 0; m < 3; ++m) {
                const auto kin = lat.map_k_to_vg(static_cast<PhononMode>(m), k);
                const double rec[4] = {kin.vg_dir.x, kin.vg_dir.y, kin.vg_dir.z, kin.vg_mag};
                std::fwrite(rec, 8, 4, f);
            }
    }
    std::fclose(f);
    return 0;
}

int cmd_amm(uint64_t n, const std::string& out) {
    const physics::IsotropicAMMInterface a = amm_ge_al();
    FILE* f = open_or_die(out);
    for (int lon = 1; lon >= 0; --lon)
        for (uint64_t i = 0; i < n; ++i) {
            const double t = a.transmission(lon == 1, (static_cast<double>(i) + 0.5) / static_cast<double>(n));
            std::fwrite(&t, 8, 1, f);
        }
    std::fclose(f);
    return 0;
}

int cmd_kaplan(uint64_t n, const std::string& out) {
    const DetectorModel det;
    const KaplanFilm& film = *det.surfaces[0].kaplan_sensor;
    const KaplanSurrogateLUT lut(film);
    Rng rng = Rng::for_stream(3, 0);
    KaplanBuffer refl;
    FILE* f = open_or_die(out);
    for (uint64_t i = 0; i < n; ++i) {
        const double E = film.gap_energy * (1.0 + 45.0 * rng.uniform());
        const double edep = lut.absorb_phonon_fast(E, refl, rng);
        const uint32_t cnt = static_cast<uint32_t>(refl.size());
        std::fwrite(&E, 8, 1, f);
        std::fwrite(&edep, 8, 1, f);
        std::fwrite(&cnt, 4, 1, f);
        for (double r : refl) std::fwrite(&r, 8, 1, f);
    }
    std::fclose(f);
    return 0;
}

int cmd_mesh2(uint64_t n, const std::string& out) {
    const DetectorModel det;
    const geometry::BiLinearMesh2D ax = axisym_mesh(det.solid), pl = planar_mesh(det.solid);
    Rng rng = Rng::for_stream(6, 0);
    int he_a = 0, hv_a = 0, he_p = 0, hv_p = 0;
    FILE* f = open_or_die(out);
    for (uint64_t i = 0; i < n; ++i) {
        Vec3 p = uniform_origin(det.solid, rng);
        if (i < 16) p.x = p.y = 0.0;
        const Vec3 Ea = ax.field_at(p, he_a);
        const double Va = ax.potential_at(p, hv_a);
        const Vec3 Ep = pl.field_at(p, he_p);
        const double Vp = pl.potential_at(p, hv_p);
        const double rec[11] = {p.x, p.y, p.z, Ea.x, Ea.y, Ea.z, Va, Ep.x, Ep.y, Ep.z, Vp};
        std::fwrite(rec, 8, 11, f);
    }
    std::fclose(f);
    std::printf("{\"axisym_vertices\": %zu, \"axisym_triangles\": %zu, \"planar_vertices\": %zu, "
                "\"planar_triangles\": %zu}\n",
                ax.num_vertices(), ax.num_triangles(), pl.num_vertices(), pl.num_triangles());
    return 0;
}

int cmd_meshfile(const char* coords, const char* tets, double cu, double vu, uint64_t n, const std::string& out) {
    const DetectorModel det;
    const geometry::TriLinearMesh3D mesh = geometry::TriLinearMesh3D::load_from_files(coords, tets, cu, vu);
    Rng rng = Rng::for_stream(7, 0);
    int hint_e = 0, hint_v = 0;
    FILE* f = open_or_die(out);
    for (uint64_t i = 0; i < n; ++i) {
        const Vec3 p = uniform_origin(det.solid, rng);
        const Vec3 E = mesh.field_at(p, hint_e);
        const double V = mesh.potential_at(p, hint_v);
        const double rec[7] = {p.x, p.y, p.z, E.x, E.y, E.z, V};
        std::fwrite(rec, 8, 7, f);
    }
    std::fclose(f);
    std::printf("{\"vertices\": %zu, \"tetrahedra\": %zu}\n", mesh.num_vertices(), mesh.num_tetrahedra());
    return 0;
}

int cmd_yield(const std::string& out) {
    FILE* f = open_or_die(out);
    const CrystalConfig cfgs[2] = {materials::Germanium(), materials::Silicon()};
    for (const CrystalConfig& cfg : cfgs) {
        const CrystalLattice lat(cfg);
        const EnergyPartition part(lat);
        physics::EmpiricalNIELParams fixed;
        fixed.energy_dependent_k = false;
        for (int col = 0; col < 7; ++col)
            for (int i = 0; i < 400; ++i) {
                const double E = std::pow(10.0, 7.0 * i / 399.0);
                double y;
                if (col < 5) y = physics::compute_ionization_yield(static_cast<physics::NIELModel>(col), E, cfg);
                else if (col == 5) y = physics::compute_ionization_yield(physics::NIELModel::Empirical, E, cfg, fixed);
                else y = part.lindhard_ionization_yield(E, 2.0, 4.0);
                std::fwrite(&y, 8, 1, f);
            }
    }
    std::fclose(f);
    return 0;
}

void write_result(FILE* f, const EnergyPartition::Result& r) {
    const double d[4] = {r.total_edep_eV, r.ionizing_eV, r.niel_eV, r.lindhard_yield};
    const uint64_t n[4] = {r.n_pairs_true, r.n_pairs_sampled, r.n_phonons_true, r.n_phonons_sampled};
    const double w[3] = {r.charge_weight, r.phonon_weight, r.prompt_phonon_eV};
    std::fwrite(d, 8, 4, f);
    std::fwrite(n, 8, 4, f);
    std::fwrite(w, 8, 3, f);
}

void write_records(FILE* f, const std::vector<ChargeTrack>& ch, const std::vector<PhononTrack>& ph, const Rng& rng) {
    const uint64_t n[2] = {ch.size(), ph.size()};
    std::fwrite(n, 8, 2, f);
    static_assert(sizeof(ChargeTrack) == 128 && sizeof(PhononTrack) == 128, "record layout");
    if (!ch.empty()) std::fwrite(ch.data(), sizeof(ChargeTrack), ch.size(), f);
    if (!ph.empty()) std::fwrite(ph.data(), sizeof(PhononTrack), ph.size(), f);
    Rng copy = rng;
    const uint64_t next = copy.next_u64();  // the stream position after the call
    std::fwrite(&next, 8, 1, f);
}

int cmd_partition(const std::string& out) {
    const CrystalLattice lattice(materials::Germanium());
    const EnergyPartition part(lattice);
    FILE* f = open_or_die(out);
    for (int i = 0; i < 48; ++i) {
        PartitionOptions o;
        o.max_sampled_pairs = 100;
        o.max_sampled_phonons = 150;
        if (i % 4 == 1) o.use_fano_fluctuations = false;
        if (i % 4 == 2) {
            o.use_charge_cloud = false;
            o.max_sampled_pairs = 16;
        }
        if (i % 4 == 3) {
            o.niel_model = physics::NIELModel::Empirical;
            o.max_sampled_phonons = 7;
        }
        const double E = std::pow(10.0, 1.0 + 4.0 * i / 47.0);
        Rng rng = Rng::for_stream(8, static_cast<uint64_t>(i));
        std::vector<ChargeTrack> ch;
        std::vector<PhononTrack> ph;
        const Vec3 pos{1e-3 * i, -2e-3, 3e-3};
        const EnergyPartition::Result r = part.partition_deposit(pos, 1e-9 * i, E, (i % 2) == 1, ch, ph, rng, o);
        write_result(f, r);
        write_records(f, ch, ph, rng);
    }
    std::fclose(f);
    return 0;
}

// The synthetic primary tracks of `merge` (also restated by the tests)
std::vector<PrimaryStepInput> merge_steps() {
    std::vector<PrimaryStepInput> steps;
    for (int t = 0; t < 3; ++t) {
        Vec3 p{-5e-3 + 4e-3 * t, 1e-3 * t, -4e-3};
        for (int k = 0; k < 12; ++k) {
            PrimaryStepInput s;
            s.track_id = t + 1;
            s.start_pos = p;
            const double len = 1e-4 * (2 + (k * 7 + t * 3) % 6);
            p = p + Vec3{0.6 * len, 0.3 * len, 0.74161984870956632 * len};
            s.end_pos = p;
            s.time_s = 1e-12 * (10 * t + k);
            s.edep_eV = (t == 2) ? 20.0 * (k % 3) : 40.0 + 15.0 * ((k * 5 + t) % 7);
            s.eniel_eV = (t == 2) ? 300.0 + 50.0 * (k % 4) : 0.0;
            s.is_charged = (t != 1);
            s.hit_boundary = (k == 7 && t == 0);
            s.track_stopped = (k == 11);
            steps.push_back(s);
        }
    }
    return steps;
}

int cmd_merge(const std::string& out) {
    const CrystalLattice lattice(materials::Germanium());
    PartitionOptions o;
    o.max_sampled_pairs = 64;
    o.max_sampled_phonons = 64;
    HitMerger merger(lattice, 1.0 * units::mm, o);
    Rng rng = Rng::for_stream(9, 0);
    std::vector<ChargeTrack> ch;
    std::vector<PhononTrack> ph;
    FILE* f = open_or_die(out);
    const std::vector<PrimaryStepInput> steps = merge_steps();
    for (const PrimaryStepInput& s : steps) {
        const uint8_t ready = merger.process_step(s, ch, ph, rng) ? 1 : 0;
        std::fwrite(&ready, 1, 1, f);
    }
    const EnergyPartition::Result r = merger.flush(ch, ph, rng);
    write_result(f, r);
    write_records(f, ch, ph, rng);
    std::fclose(f);
    return 0;
}

int cmd_mesh(uint64_t n, const std::string& out) {
    const DetectorModel det;
    const geometry::TriLinearMesh3D mesh = recoil_mesh(det.solid);
    Rng rng = Rng::for_stream(5, 0);
    int hint_e = 0, hint_v = 0;
    FILE* f = open_or_die(out);
    for (uint64_t i = 0; i < n; ++i) {
        const Vec3 p = uniform_origin(det.solid, rng);
        const Vec3 E = mesh.field_at(p, hint_e);
        const double V = mesh.potential_at(p, hint_v);
        const double rec[7] = {p.x, p.y, p.z, E.x, E.y, E.z, V};
        std::fwrite(rec, 8, 7, f);
    }
    std::fclose(f);
    std::printf("{\"vertices\": %zu, \"tetrahedra\": %zu}\n", mesh.num_vertices(), mesh.num_tetrahedra());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s dump|time|rng ...\n", argv[0]);
        return 2;
    }
    const std::string cmd = argv[1];
    if (cmd == "dump" && argc == 7)
        return cmd_dump(argv[2], std::strtoull(argv[3], nullptr, 10), std::strtoull(argv[4], nullptr, 10),
                        static_cast<unsigned>(std::atoi(argv[5])), argv[6]);
    if (cmd == "time" && argc == 6)
        return cmd_time(argv[2], std::strtoull(argv[3], nullptr, 10), std::strtoull(argv[4], nullptr, 10),
                        static_cast<unsigned>(std::atoi(argv[5])));
    if (cmd == "kin" && argc == 4) return cmd_kin(std::strtoull(argv[2], nullptr, 10), argv[3]);
    if (cmd == "amm" && argc == 4) return cmd_amm(std::strtoull(argv[2], nullptr, 10), argv[3]);
    if (cmd == "kaplan" && argc == 4) return cmd_kaplan(std::strtoull(argv[2], nullptr, 10), argv[3]);
    if (cmd == "mask" && argc == 4) return cmd_mask(std::strtoull(argv[2], nullptr, 10), argv[3]);
    if (cmd == "meshfile" && argc == 8)
        return cmd_meshfile(argv[2], argv[3], std::strtod(argv[4], nullptr), std::strtod(argv[5], nullptr),
                            std::strtoull(argv[6], nullptr, 10), argv[7]);
    if (cmd == "yield" && argc == 3) return cmd_yield(argv[2]);
    if (cmd == "partition" && argc == 3) return cmd_partition(argv[2]);
    if (cmd == "merge" && argc == 3) return cmd_merge(argv[2]);
    if (cmd == "mesh2" && argc == 4) return cmd_mesh2(std::strtoull(argv[2], nullptr, 10), argv[3]);
    if (cmd == "mesh" && argc == 4) return cmd_mesh(std::strtoull(argv[2], nullptr, 10), argv[3]);
    if (cmd == "rng" && argc == 5)
        return cmd_rng(std::strtoull(argv[2], nullptr, 10), std::strtoull(argv[3], nullptr, 10), std::atoi(argv[4]));
    std::fprintf(stderr, "bad arguments\n");
    return 2;
}
