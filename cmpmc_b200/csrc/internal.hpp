// internal.hpp -- host-side types shared by the library's translation units.
#pragma once

#include <array>
#include <string>
#include <vector>

#include "../../include/cmpmc_gpu.h"
#include "mesh.cuh"
#include "partition.cuh"
#include "transport.cuh"

struct cmpmc_lattice {
    cmpmc_crystal_config cfg;
    std::vector<cmpmc_gpu::OctEntry> oct;  // [3][256][256]
    std::vector<double> cdf_lt, cdf_tt;    // [1024] each
    std::vector<double> hv;                // flattened HV tensors (see cmpmc_lattice_tables)
    cmpmc_gpu::Stiffness stiff;            // C_ijlm (exact kinematics)
    std::vector<double> bil;               // [3][181][361][3] (bilinear kinematics, built on request)
    cmpmc_gpu::Lattice view;               // host pointers into the members above
    uint64_t id = 0;                       // unique per created lattice (never reused in a process)
};

struct cmpmc_kaplan_lut {
    cmpmc_gpu::Film film;
    std::vector<float> abs;        // [kLutNE * kLutNS]
    std::vector<uint32_t> off;     // [kLutNE * kLutNS + 1]
    std::vector<float> refl;
};

// TriLinearMesh3D (geometry/mesh_field.hpp:40-345): node table, potentials, sorted
// tetrahedra and the per-tetrahedron records the device walks (mesh.cuh).
struct cmpmc_mesh {
    std::vector<double> X;                   // [n_vertices][3]
    std::vector<double> V;                   // [n_vertices], clamped
    std::vector<std::array<int32_t, 4>> tets;
    std::vector<cmpmc_gpu::MeshTet> rec;     // [n_tets]
};

// BiLinearMesh2D (geometry/mesh_field.hpp:347-582)
struct cmpmc_mesh2d {
    std::vector<double> X;                   // [n][2] (u, v)
    std::vector<double> V;
    std::vector<std::array<int32_t, 3>> tris;
    std::vector<cmpmc_gpu::MeshTri> rec;
    int axisym = 1;
};

namespace cmpmc_gpu {

// Checks a detector / crystal pair against what the device path supports and applies the
// reference's guards (engine.hpp:165-168, 197-199, 407-409). Returns a CMPMC_* status.
int validate_config(const cmpmc_crystal_config& cfg, const cmpmc_detector& det, bool has_charges,
                    std::string& err);
Detector detector_view(const cmpmc_detector& det);
Pad pad_view(const cmpmc_electrode_pad& p);
Film film_view(const cmpmc_film_config& f);

// KaplanSurrogateLUT (superconductor/kaplan_film.hpp:336-383) tables: 128 energy nodes on
// [2 Delta, 40 Delta] x 512 pre-sampled cascade outcomes (absorbed fraction and the
// re-emitted energies as fractions of the incident energy)
constexpr int kLutNE = 128;
constexpr int kLutNS = 512;
constexpr double kLutEMaxDiv2Gap = 20.0;

// Record conversion between the reference layouts and the register-state structs.
Track track_from_record(const cmpmc_phonon_track& r);
void track_to_record(const Track& t, cmpmc_phonon_track& r);
Charge charge_from_record(const cmpmc_charge_track& r);
void charge_to_record(const Charge& c, cmpmc_charge_track& r);

// EnergyPartition::partition_deposit (partition.cuh) with the reference's default options
cmpmc_partition_options default_partition_options();

}  // namespace cmpmc_gpu
