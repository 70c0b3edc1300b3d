// Test infrastructure only (the checker): builds the reference CrystalLattice for
// Germanium (crystal_lattice.hpp:45-55) and writes its precomputed tables so that
// the product's own host-side lattice builder can be compared with it bit for bit.
// The tables are private members of CrystalLattice, so this one translation unit
// opens them up with a preprocessor definition; every standard header is included
// first so that only the reference's own classes are affected.
//
// Usage: cmpmc_ref_tables <out_prefix>
//   <prefix>.oct   float32 [3][256][256][4]  (vg_oct_lut_, crystal_lattice.hpp:370-392)
//   <prefix>.bil   float64 [3][181][361][3]  (vg_lut_, crystal_lattice.hpp:350-368)
//   <prefix>.cdf   float64 [2][1024]         (cdf_lt_, cdf_tt_, crystal_lattice.hpp:440-477)
//   <prefix>.hv    float64: e_cond_mass, h_mass, mass_ratio[3], hv_sqrt[3], hv_sqrt_inv[3],
//                  l0_e, l0_h, k_sound_e, k_sound_h, n_valleys, valley_rot[n][3][3]
//                  (crystal_lattice.hpp:394-438)
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <fstream>
#include <functional>
#include <limits>
#include <mutex>
#include <numbers>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#define private public
#include "cmpmc/cmpmc.hpp"
#undef private

using namespace cmpmc;

static void write_or_die(const std::string& path, const void* p, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(p, 1, n, f) != n) { std::perror(path.c_str()); std::exit(1); }
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc != 2) { std::fprintf(stderr, "usage: %s <out_prefix>\n", argv[0]); return 2; }
    const std::string prefix = argv[1];
    const CrystalLattice lat(materials::Germanium());
    write_or_die(prefix + ".oct", lat.vg_oct_lut_.data(), lat.vg_oct_lut_.size() * sizeof(CrystalLattice::OctLutEntry));
    write_or_die(prefix + ".bil", lat.vg_lut_.data(), lat.vg_lut_.size() * sizeof(Vec3));
    std::vector<double> cdf(lat.cdf_lt_.begin(), lat.cdf_lt_.end());
    cdf.insert(cdf.end(), lat.cdf_tt_.begin(), lat.cdf_tt_.end());
    write_or_die(prefix + ".cdf", cdf.data(), cdf.size() * sizeof(double));
    std::vector<double> hv = {lat.e_cond_mass_eV_, lat.h_mass_eV_,
                              lat.mass_ratio_.x, lat.mass_ratio_.y, lat.mass_ratio_.z,
                              lat.hv_sqrt_.x, lat.hv_sqrt_.y, lat.hv_sqrt_.z,
                              lat.hv_sqrt_inv_.x, lat.hv_sqrt_inv_.y, lat.hv_sqrt_inv_.z,
                              lat.l0_e_, lat.l0_h_, lat.k_sound_e_, lat.k_sound_h_,
                              static_cast<double>(lat.valley_rot_.size())};
    for (const Mat3& m : lat.valley_rot_)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) hv.push_back(m.m[i][j]);
    write_or_die(prefix + ".hv", hv.data(), hv.size() * sizeof(double));
    return 0;
}
