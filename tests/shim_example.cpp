// Compiled by tests/test_shim.py against the reference's headers: the reference's own
// generator code (tests/test_parallel.cpp:110-125) unchanged, run through the device adapter.
#include "cmpmc/cmpmc.hpp"
#include "cmpmc_b200/run_events_gpu.hpp"

#include <cstdio>

int main() {
    using namespace cmpmc;
    const CrystalLattice lattice(materials::Germanium());
    DetectorModel det;
    det.e_field = UniformElectricField::from_bias(2.0, 2.54 * units::cm);
    det.luke_sample_fraction = 0.02;
    const SimulationEngine engine(lattice, det);
    const ChargePhysics charges(lattice);
    const size_t n_valleys = lattice.config().valley_dirs.size();
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
    try {
        cmpmc_b200::GpuEngine gpu(lattice.config(), det);
        const RunResult r = gpu.run_events(203, gen, opt);
        const RunResult c = run_events(engine, 203, gen, opt);
        std::printf("device hits %zu cpu hits %zu steps %llu vs %llu\n", r.hits.size(), c.hits.size(),
                    (unsigned long long)r.stats.total_steps, (unsigned long long)c.stats.total_steps);
        // electrode masks (copied from the surfaces) and a mesh field (handed over once)
        DetectorModel det2 = det;
        const double R = det.solid.radius, h = det.solid.half_z;
        auto pot = [h](const Vec3& p) { return 2.0 * (p.z + h) / (2.0 * h); };
        for (int f = 0; f < 2; ++f)
            det2.surfaces[f].electrode_mask = geometry::ElectrodePatternMask::supercdms_qet_mask(R, 0.8);
        det2.mesh_field_3d = geometry::TriLinearMesh3D::build_cartesian_grid(R, R, h, 8, 8, 8, pot);
        const SimulationEngine engine2(lattice, det2);
        cmpmc_b200::GpuEngine gpu2(lattice.config(), det2);
        gpu2.set_cartesian_mesh(R, R, h, 8, 8, 8, pot);
        const RunResult m = gpu2.run_events(203, gen, opt);
        const RunResult mc = run_events(engine2, 203, gen, opt);
        size_t on_pad = 0;
        for (const SensorHit& x : m.hits) on_pad += (x.channel_id >= 0);
        std::printf("masked + mesh: device hits %zu (%zu on pads) cpu hits %zu\n", m.hits.size(), on_pad,
                    mc.hits.size());
        // an axisymmetric 2D mesh field (mesh_field_2d, handed over once)
        DetectorModel det3 = det;
        auto pot2 = [h](double r, double z) { return 2.0 * (z + h) / (2.0 * h) + 0.1 * r / h; };
        det3.mesh_field_2d = geometry::BiLinearMesh2D::build_grid(0.0, R, -h, h, 16, 16, pot2, true);
        const SimulationEngine engine3(lattice, det3);
        cmpmc_b200::GpuEngine gpu3(lattice.config(), det3);
        gpu3.set_grid_mesh2d(0.0, R, -h, h, 16, 16, pot2, true);
        const RunResult a = gpu3.run_events(203, gen, opt);
        const RunResult ac = run_events(engine3, 203, gen, opt);
        std::printf("2D mesh: device hits %zu cpu hits %zu charge steps %llu vs %llu\n", a.hits.size(), ac.hits.size(),
                    (unsigned long long)a.stats.charge_steps, (unsigned long long)ac.stats.charge_steps);
        return 0;
    } catch (const std::runtime_error& e) {
        std::printf("device unavailable: %s\n", e.what());
        return 3;
    }
}
