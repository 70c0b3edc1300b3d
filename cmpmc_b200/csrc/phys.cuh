// phys.cuh -- FP64 physics of the CMPMC transport path, shared by the device kernels
// and the host-side helpers (make_track, generators) of this library.
//
// Every function restates the reference's arithmetic in the reference's operation
// order, because the plain FP64 form must reproduce the CPU's event streams: the
// translation units that use it for parity are compiled without FMA contraction, so
// + - * / and sqrt round exactly as on x86-64 SSE. Every transcendental is correctly
// rounded on the device (crmath.cuh, see m_log below).
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define CMPMC_HD __host__ __device__ __forceinline__
#else
#define CMPMC_HD inline
#endif

#include "crmath.cuh"

namespace cmpmc_gpu {

// Transcendentals of the transport. On the device, log, sin, cos, acos, exp, pow, hypot
// and cbrt are the correctly
// rounded functions of crmath.cuh (path lengths, energies and charge kinematics feed
// trajectories that are sensitive to the last bit); on the host they are the platform libm,
// so host-side generators and make_track reproduce the CPU reference. Defining
// CMPMC_HOST_CRMATH selects the correctly rounded functions on the host as well.
// CMPMC_DEVICE_FAST_MATH (the batched FP32 form) keeps CUDA's libm on the device.
#if (defined(__CUDA_ARCH__) && !defined(CMPMC_DEVICE_FAST_MATH)) || defined(CMPMC_HOST_CRMATH)
CMPMC_HD double m_log(double x) { return crmath::log(x); }
CMPMC_HD double m_sin(double x) { return crmath::sin(x); }
CMPMC_HD double m_cos(double x) { return crmath::cos(x); }
CMPMC_HD double m_exp(double x) { return crmath::exp(x); }
CMPMC_HD double m_pow(double x, double y) { return crmath::pow(x, y); }
CMPMC_HD double m_hypot(double x, double y) { return crmath::hypot(x, y); }
CMPMC_HD double m_cbrt(double x) { return crmath::cbrt(x); }
CMPMC_HD double m_acos(double x) { return crmath::acos(x); }
CMPMC_HD double m_atan2(double y, double x) { return crmath::atan2(y, x); }
#else
CMPMC_HD double m_log(double x) { return ::log(x); }
CMPMC_HD double m_sin(double x) { return ::sin(x); }
CMPMC_HD double m_cos(double x) { return ::cos(x); }
CMPMC_HD double m_exp(double x) { return ::exp(x); }
CMPMC_HD double m_pow(double x, double y) { return ::pow(x, y); }
CMPMC_HD double m_hypot(double x, double y) { return ::hypot(x, y); }
CMPMC_HD double m_cbrt(double x) { return ::cbrt(x); }
CMPMC_HD double m_acos(double x) { return ::acos(x); }
CMPMC_HD double m_atan2(double y, double x) { return ::atan2(y, x); }
#endif

// ---- constants (core/units.hpp:26-72) ---------------------------------------------
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kHalfPi = 0.5 * kPi;
constexpr double kCLight = 299792458.0;
constexpr double kHPlanck = 4.135667696e-15;
constexpr double kHbar = 6.582119569e-16;
constexpr double kHbarC = kHbar * kCLight;
constexpr double kBoltzmann = 8.617333262e-5;
constexpr double kGHz = 1e9;
constexpr double kInf = __builtin_huge_val();

// std::min / std::max / std::clamp semantics (NaN and signed-zero behaviour included)
CMPMC_HD double dmin(double a, double b) { return (b < a) ? b : a; }
CMPMC_HD double dmax(double a, double b) { return (a < b) ? b : a; }
CMPMC_HD double dclamp(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
CMPMC_HD int imin(int a, int b) { return (b < a) ? b : a; }
CMPMC_HD int iclamp(int v, int lo, int hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

// ---- Vec3 / Mat3 (core/math.hpp:15-99) ---------------------------------------------
struct V3 {
    double x, y, z;
};
CMPMC_HD V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
CMPMC_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
CMPMC_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
CMPMC_HD V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
// Vec3::operator/ multiplies by the reciprocal (math.hpp:30-33)
CMPMC_HD V3 vdiv(V3 a, double s) { const double inv = 1.0 / s; return v3(a.x * inv, a.y * inv, a.z * inv); }
CMPMC_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CMPMC_HD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
CMPMC_HD double norm2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
CMPMC_HD double norm(V3 a) { return sqrt(norm2(a)); }
// Vec3::unit: 1/sqrt then three multiplies; zero vector -> +z (math.hpp:47-52)
CMPMC_HD V3 unit(V3 a) {
    const double n2 = norm2(a);
    if (n2 <= 0.0) return v3(0.0, 0.0, 1.0);
    const double inv = 1.0 / sqrt(n2);
    return v3(a.x * inv, a.y * inv, a.z * inv);
}
// Rodrigues rotation (math.hpp:55-57)
CMPMC_HD V3 rotate_around(V3 v, V3 k, double c, double s) {
    return v * c + cross(k, v) * s + k * (dot(k, v) * (1.0 - c));
}
// math.hpp:60-63
CMPMC_HD V3 orthogonal_unit(V3 v) {
    const V3 a = (fabs(v.x) < 0.9) ? v3(1.0, 0.0, 0.0) : v3(0.0, 1.0, 0.0);
    return unit(cross(v, a));
}
struct M3 {
    double m[3][3];
};
CMPMC_HD V3 mul(const M3& M, V3 v) {
    return v3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z,
              M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z,
              M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z);
}
CMPMC_HD V3 mul_transpose(const M3& M, V3 v) {
    return v3(M.m[0][0] * v.x + M.m[1][0] * v.y + M.m[2][0] * v.z,
              M.m[0][1] * v.x + M.m[1][1] * v.y + M.m[2][1] * v.z,
              M.m[0][2] * v.x + M.m[1][2] * v.y + M.m[2][2] * v.z);
}

// ---- xoshiro256** stream (core/rng.hpp:17-97) --------------------------------------
CMPMC_HD uint64_t splitmix_step(uint64_t z) {
    uint64_t x = z;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
CMPMC_HD uint64_t mix64(uint64_t x) { return splitmix_step(x + 0x9e3779b97f4a7c15ULL); }
CMPMC_HD uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct Rng {
    uint64_t s[4];

    // Rng(seed): splitmix64 seeding (rng.hpp:20-29)
    CMPMC_HD void seed(uint64_t seed_value) {
        uint64_t z = seed_value;
        for (int i = 0; i < 4; ++i) {
            z += 0x9e3779b97f4a7c15ULL;
            s[i] = splitmix_step(z);
        }
    }
    // Rng::for_stream (rng.hpp:34-36)
    CMPMC_HD static Rng for_stream(uint64_t seed_value, uint64_t stream) {
        Rng r;
        r.seed(mix64(seed_value) ^ mix64(stream + 0x632be59bd9b4e019ULL));
        return r;
    }
    CMPMC_HD uint64_t next_u64() {
        const uint64_t result = rotl64(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl64(s[3], 45);
        return result;
    }
    // (0,1): ((x >> 11) | 1) * 2^-53 (rng.hpp:62-64)
    CMPMC_HD double uniform() {
        return static_cast<double>((next_u64() >> 11) | 1ULL) * (1.0 / 9007199254740992.0);
    }
    // rng.hpp:78-83
    CMPMC_HD V3 isotropic_dir() {
        const double cos_theta = 2.0 * uniform() - 1.0;
        const double sin_theta = sqrt(dmax(0.0, 1.0 - cos_theta * cos_theta));
        const double phi = kTwoPi * uniform();
        return v3(sin_theta * m_cos(phi), sin_theta * m_sin(phi), cos_theta);
    }
    // rng.hpp:86-96
    CMPMC_HD V3 lambertian_dir(V3 n) {
        const double phi = kTwoPi * uniform();
        const double sin_theta = sqrt(uniform());
        const double cos_theta = sqrt(dmax(0.0, 1.0 - sin_theta * sin_theta));
        const V3 u = orthogonal_unit(n);
        const V3 v = cross(n, u);
        return unit(u * (sin_theta * m_cos(phi)) + v * (sin_theta * m_sin(phi)) + n * cos_theta);
    }
};

// ---- lattice view (what CrystalLattice holds that the transport reads) ------------
constexpr int kNOct = 256;
constexpr int kNCdf = 1024;

struct OctEntry {
    float vx, vy, vz, vmag;
};

struct Stiffness;

// CrystalLattice::KinematicsMode (crystal_lattice.hpp:63-74)
enum { kKinOctahedral = 0, kKinExact = 1, kKinBilinear = 2 };
constexpr int kNCTheta = 181, kNPhi = 361;  // bilinear (cos theta, phi) table (crystal_lattice.hpp:28-29)

struct Lattice {
    const OctEntry* oct;   // [3][256][256]
    int kin_mode;          // kKin*
    double density;
    const Stiffness* stiff;  // C_ijlm (exact mode)
    const double* bil;       // [3][181][361][3] group velocities (bilinear mode)
    const double* cdf_lt;  // [1024]
    const double* cdf_tt;  // [1024]
    M3 orient;
    double B_iso, A_anh, fTT_frac, poly_mfp;
    double fLDOS, fSTDOS, fFTDOS;
    double v_sound, v_trans;
    double bandgap;
    double debye_energy;  // CrystalLattice::debye_energy (crystal_lattice.hpp:62)
    // Herring-Vogt (crystal_lattice.hpp:322-331, built 394-438)
    double e_cond_mass, h_mass;
    V3 mass_ratio, hv_sqrt, hv_sqrt_inv;
    double l0_e, l0_h, k_sound_e, k_sound_h;
    int n_valleys;
    M3 valley_rot[8];
    // charge rates (charge/charge_kernels.hpp:82-126)
    int iv_model;
    double iv_min_energy, iv_quad_rate, iv_quad_field, iv_quad_power, iv_lin_rate0, iv_lin_rate1,
        iv_lin_power;
    double e_trap_mfp, h_trap_mfp, e_ion_d0_mfp, e_ion_a_mfp, h_ion_d_mfp, h_ion_a0_mfp;
};

struct Kin {
    V3 vg_dir;
    double vg_mag;
};

// CrystalLattice::oct_encode (crystal_lattice.hpp:117-130)
CMPMC_HD void oct_encode(V3 k, double& u_out, double& v_out) {
    const double l1 = fabs(k.x) + fabs(k.y) + fabs(k.z);
    const double inv_l1 = (l1 > 1e-18) ? (1.0 / l1) : 1.0;
    double px = k.x * inv_l1;
    double py = k.y * inv_l1;
    if (k.z < 0.0) {
        const double ox = (1.0 - fabs(py)) * (px >= 0.0 ? 1.0 : -1.0);
        const double oy = (1.0 - fabs(px)) * (py >= 0.0 ? 1.0 : -1.0);
        px = ox;
        py = oy;
    }
    u_out = dclamp(px, -1.0, 1.0);
    v_out = dclamp(py, -1.0, 1.0);
}

// CrystalLattice::map_k_to_vg_oct (crystal_lattice.hpp:144-176): FP32 bilinear blend
// with the reference's float weights and summation order, then FP64 normalisation.
template <class LoadEntry>
CMPMC_HD Kin map_k_to_vg_oct_impl(const Lattice& L, int mode, V3 k_det, LoadEntry&& load) {
    const V3 k = mul_transpose(L.orient, k_det);
    double u_oct = 0.0, v_oct = 0.0;
    oct_encode(k, u_oct, v_oct);
    const double u = (u_oct + 1.0) * 0.5 * (kNOct - 1);
    const double v = (v_oct + 1.0) * 0.5 * (kNOct - 1);
    const int i0 = iclamp(static_cast<int>(u), 0, kNOct - 2);
    const int j0 = iclamp(static_cast<int>(v), 0, kNOct - 2);
    const float du = static_cast<float>(u - i0);
    const float dv = static_cast<float>(v - j0);
    const float w00 = (1.0f - du) * (1.0f - dv);
    const float w10 = du * (1.0f - dv);
    const float w01 = (1.0f - du) * dv;
    const float w11 = du * dv;
    const int base = (mode * kNOct + i0) * kNOct + j0;
    const OctEntry e00 = load(base);
    const OctEntry e10 = load(base + kNOct);
    const OctEntry e01 = load(base + 1);
    const OctEntry e11 = load(base + kNOct + 1);
    const V3 vg_cryst = v3(static_cast<double>(e00.vx * w00 + e10.vx * w10 + e01.vx * w01 + e11.vx * w11),
                           static_cast<double>(e00.vy * w00 + e10.vy * w10 + e01.vy * w01 + e11.vy * w11),
                           static_cast<double>(e00.vz * w00 + e10.vz * w10 + e01.vz * w01 + e11.vz * w11));
    const double mag = norm(vg_cryst);
    const V3 vg_det = mul(L.orient, vdiv(vg_cryst, dmax(mag, 1e-12)));
    Kin r;
    r.vg_dir = unit(vg_det);
    r.vg_mag = mag;
    return r;
}

#ifdef __CUDA_ARCH__
CMPMC_HD OctEntry load_oct(const OctEntry* t, int i) {
    const float4 f = __ldg(reinterpret_cast<const float4*>(t) + i);
    OctEntry e;
    e.vx = f.x; e.vy = f.y; e.vz = f.z; e.vmag = f.w;
    return e;
}
#else
CMPMC_HD OctEntry load_oct(const OctEntry* t, int i) { return t[i]; }
#endif

#ifdef __CUDACC__
#define CMPMC_HD_COLD static __host__ __device__ __noinline__
#else
#define CMPMC_HD_COLD static inline
#endif
}  // namespace cmpmc_gpu
#include "christoffel.cuh"
namespace cmpmc_gpu {

// CrystalLattice::map_k_to_vg_exact (crystal_lattice.hpp:76-84): the Cardano solve per call
CMPMC_HD_COLD Kin map_k_to_vg_exact(const Lattice& L, int mode, V3 k_det) {
    const V3 k = unit(mul_transpose(L.orient, k_det));
    V3 vg[3];
    solve_christoffel_cardano(*L.stiff, L.density, k, vg);
    const V3 v = vg[mode];
    const double mag = norm(v);
    Kin r;
    r.vg_dir = unit(mul(L.orient, vdiv(v, dmax(mag, 1e-12))));
    r.vg_mag = mag;
    return r;
}

// CrystalLattice::map_k_to_vg, bilinear (cos theta, phi) table (crystal_lattice.hpp:86-114)
CMPMC_HD_COLD Kin map_k_to_vg_bilinear(const Lattice& L, int mode, V3 k_det) {
    const V3 k = unit(mul_transpose(L.orient, k_det));
    const double ctheta = dclamp(k.z, -1.0, 1.0);
    double phi = m_atan2(k.y, k.x);
    if (phi < 0.0) phi += kTwoPi;
    const double u = (ctheta + 1.0) * 0.5 * (kNCTheta - 1);
    const double v = (phi / kTwoPi) * (kNPhi - 1);
    const int ui = static_cast<int>(u), vi = static_cast<int>(v);
    const int i0 = (ui < 0) ? 0 : ((ui > kNCTheta - 2) ? kNCTheta - 2 : ui);
    const int j0 = (vi < 0) ? 0 : ((vi > kNPhi - 2) ? kNPhi - 2 : vi);
    const double du = u - i0;
    const double dv = v - j0;
    auto at = [&](int i, int j) {
        const double* e = L.bil + 3 * ((static_cast<size_t>(mode) * kNCTheta + i) * kNPhi + j);
        return v3(e[0], e[1], e[2]);
    };
    const V3 vg = at(i0, j0) * ((1.0 - du) * (1.0 - dv)) + at(i0 + 1, j0) * (du * (1.0 - dv)) +
                  at(i0, j0 + 1) * ((1.0 - du) * dv) + at(i0 + 1, j0 + 1) * (du * dv);
    const double mag = norm(vg);
    const V3 vg_det = mul(L.orient, vdiv(vg, dmax(mag, 1e-12)));
    Kin r;
    r.vg_dir = unit(vg_det);
    r.vg_mag = mag;
    return r;
}

// CrystalLattice::map_k_to_vg (crystal_lattice.hpp:86-89): dispatch on the kinematics mode
CMPMC_HD Kin map_k_to_vg(const Lattice& L, int mode, V3 k_det) {
    if (L.kin_mode == kKinOctahedral)
        return map_k_to_vg_oct_impl(L, mode, k_det, [&](int i) { return load_oct(L.oct, i); });
    if (L.kin_mode == kKinExact) return map_k_to_vg_exact(L, mode, k_det);
    return map_k_to_vg_bilinear(L, mode, k_det);
}

// ---- phonon rates and samplers (phonon/phonon_kernels.hpp:29-92) --------------------
CMPMC_HD double isotope_rate(const Lattice& L, double e) {
    const double nu = e / kHPlanck;
    const double nu2 = nu * nu;
    return L.B_iso * (nu2 * nu2);
}
CMPMC_HD double downconversion_rate(const Lattice& L, int mode, double e) {
    if (mode != 0) return 0.0;
    const double nu = e / kHPlanck;
    const double nu2 = nu * nu;
    return L.A_anh * (nu2 * nu2 * nu);
}
CMPMC_HD double polycrystal_rate(const Lattice& L, double vg_mag) {
    if (L.poly_mfp <= 0.0) return 0.0;
    return vg_mag / L.poly_mfp;
}
// L = 0, FT = 1, ST = 2 (track.hpp:38-43)
CMPMC_HD int sample_dos_mode(const Lattice& L, Rng& rng) {
    const double u = rng.uniform();
    if (u < L.fLDOS) return 0;
    if (u < L.fLDOS + L.fSTDOS) return 2;
    return 1;
}
CMPMC_HD int sample_transverse_mode(const Lattice& L, Rng& rng) {
    const double p_st = L.fSTDOS / (L.fSTDOS + L.fFTDOS);
    return (rng.uniform() < p_st) ? 2 : 1;
}
CMPMC_HD double decay_angle_L_to_LT(double x, double vl, double vt) {
    const double m = vl / vt;
    const double cos_th = (1.0 + (x * x) * (1.0 - m * m) + 2.0 * x * m * m - m * m) / (2.0 * x);
    return m_acos(dclamp(cos_th, -1.0, 1.0));
}
CMPMC_HD double decay_angle_T_from_LT(double x, double vl, double vt) {
    const double m = vl / vt;
    const double cos_th = (1.0 - x * x + m * m * (1.0 - x) * (1.0 - x)) / (2.0 * m * (1.0 - x));
    return m_acos(dclamp(cos_th, -1.0, 1.0));
}
CMPMC_HD double decay_angle_TT(double x, double vl, double vt) {
    const double m = vl / vt;
    const double cos_th = (1.0 - m * m * (1.0 - x) * (1.0 - x) + m * m * x * x) / (2.0 * m * x);
    return m_acos(dclamp(cos_th, -1.0, 1.0));
}
// crystal_lattice.hpp:200-212
CMPMC_HD double sample_cdf(const double* cdf, Rng& rng) {
    const double u = rng.uniform() * (kNCdf - 1);
    const int i = imin(static_cast<int>(u), kNCdf - 2);
    const double frac = u - i;
    return cdf[i] * (1.0 - frac) + cdf[i + 1] * frac;
}

// ---- cylinder exit (geometry/solids.hpp:46-93) -------------------------------------
struct BHit {
    double distance;
    V3 n_in;
    int surf;
};
CMPMC_HD BHit intersect_exit(double radius, double half_z, V3 p, V3 v) {
    double t_min = kInf;
    int surf = 2;
    if (v.z > 1e-15) {
        const double tz = (half_z - p.z) / v.z;
        if (tz >= 0.0 && tz < t_min) { t_min = tz; surf = 0; }
    } else if (v.z < -1e-15) {
        const double tz = (-half_z - p.z) / v.z;
        if (tz >= 0.0 && tz < t_min) { t_min = tz; surf = 1; }
    }
    const double a = v.x * v.x + v.y * v.y;
    if (a > 1e-18) {
        const double b = p.x * v.x + p.y * v.y;
        const double c = p.x * p.x + p.y * p.y - radius * radius;
        const double disc = dmax(0.0, b * b - a * c);
        const double tr = (-b + sqrt(disc)) / a;
        if (tr >= 0.0 && tr < t_min) { t_min = tr; surf = 2; }
    }
    t_min = dmax(0.0, t_min);
    BHit h;
    h.distance = t_min;
    h.surf = surf;
    if (surf == 0) {
        h.n_in = v3(0.0, 0.0, -1.0);
    } else if (surf == 1) {
        h.n_in = v3(0.0, 0.0, 1.0);
    } else {
        const V3 hp = p + v * t_min;
        const double r_xy = m_hypot(hp.x, hp.y);
        h.n_in = (r_xy > 1e-15) ? v3(-hp.x / r_xy, -hp.y / r_xy, 0.0) : v3(-1.0, 0.0, 0.0);
    }
    return h;
}

// ---- surfaces and the Kaplan film ----------------------------------------------------
struct Film {
    double film_absorption, film_thickness, v_sound, gap_energy, phonon_lifetime,
        phonon_lifetime_slope, low_qp_limit, high_qp_limit, subgap_absorption, absorber_gap,
        absorber_eff, absorber_eff_slope, temperature;
    int keep_all_phonons;
    int loss_model;
    double phonon_loss_time;
};

// ElectrodePad (geometry/electrode_pattern.hpp:23-63): a readout pad on a face
struct Pad {
    int shape;  // 0 disk, 1 annular sector, 2 rectangle
    int channel;
    double cx, cy, r_min, r_max, phi_min, phi_max, fill;
};

// ElectrodePad::contains (electrode_pattern.hpp:37-62). The sector test takes atan2 of the
// offset: CUDA's atan2 on the device (a last-ulp difference to the host's only matters
// for a point within ~1e-16 rad of a sector edge).
CMPMC_HD bool pad_contains(const Pad& p, double x, double y) {
    if (p.shape == 0) {
        const double dx = x - p.cx, dy = y - p.cy;
        return (dx * dx + dy * dy) <= (p.r_max * p.r_max);
    }
    if (p.shape == 1) {
        const double dx = x - p.cx, dy = y - p.cy;
        const double r2 = dx * dx + dy * dy;
        if (r2 < p.r_min * p.r_min || r2 > p.r_max * p.r_max) return false;
        double phi = atan2(dy, dx);
        if (phi < 0.0) phi += kTwoPi;
        if (p.phi_min <= p.phi_max) return phi >= p.phi_min && phi <= p.phi_max;
        return phi >= p.phi_min || phi <= p.phi_max;
    }
    if (p.shape == 2) return (fabs(x - p.cx) <= p.r_min) && (fabs(y - p.cy) <= p.r_max);
    return false;
}

// IsotropicMedium (phonon/interface_transmission.hpp:36-49)
struct Medium {
    double rho, vL, vT;
};

struct Surface {
    double prob_abs, prob_refl, refl_cutoff, anh_cutoff;
    double prob_charge_abs, prob_charge_spec, min_k_elec, min_k_hole;
    double spec_prob_const;
    int n_spec, n_diff, n_anh;
    int has_film;
    double spec[8], diff[8], anh[8];
    Film film;
    // SurfaceProperty::electrode_mask (surface_property.hpp:45): n_pads > 0 when present
    const Pad* pads;
    int n_pads;
    // IsotropicAMMInterface (surface_property.hpp:44): substrate -> film transmission
    // replaces the film's film_absorption (engine.hpp:492-495)
    int has_amm;
    Medium amm_sub, amm_film;
    // KaplanSurrogateLUT tables of the film (batched form, when requested): absorbed
    // fractions [128 * 512], offsets into the re-emitted fractions [128 * 512 + 1]
    const float* lut_abs;
    const uint32_t* lut_off;
    const float* lut_refl;
};

// ---- acoustic mismatch transmission (phonon/interface_transmission.hpp:51-140) ----------
// Complex numbers for the P-SV boundary solve. Division by Smith's method and the principal
// square root; a last-ulp difference to the host's complex library only moves the
// transmission by ~1e-16, which decides a film entry only if the uniform draw lands within
// that distance of it.
struct Cx {
    double re, im;
};
CMPMC_HD Cx cx(double re, double im = 0.0) { return Cx{re, im}; }
CMPMC_HD Cx operator+(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
CMPMC_HD Cx operator-(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
CMPMC_HD Cx operator*(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
CMPMC_HD Cx operator*(double s, Cx a) { return cx(s * a.re, s * a.im); }
CMPMC_HD Cx cneg(Cx a) { return cx(-a.re, -a.im); }
CMPMC_HD Cx cdiv(Cx a, Cx b) {
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, den = b.re + b.im * r;
        return cx((a.re + a.im * r) / den, (a.im - a.re * r) / den);
    }
    const double r = b.re / b.im, den = b.re * r + b.im;
    return cx((a.re * r + a.im) / den, (a.im * r - a.re) / den);
}
CMPMC_HD double cabs_(Cx a) { return m_hypot(a.re, a.im); }
CMPMC_HD double cnorm(Cx a) { return a.re * a.re + a.im * a.im; }
// sqrt of a real number on the principal branch (the slownesses of amm_psv: Im >= 0)
CMPMC_HD Cx csqrt_real(double x) { return (x >= 0.0) ? cx(sqrt(x), 0.0) : cx(0.0, sqrt(-x)); }

CMPMC_HD double amm_sh(const Medium& m1, const Medium& m2, double theta1) {
    const double s2 = m2.vT / m1.vT * m_sin(theta1);
    if (s2 >= 1.0) return 0.0;
    const double c1 = m_cos(theta1), c2 = sqrt(1.0 - s2 * s2);
    const double a = m1.rho * m1.vT * c1, b = m2.rho * m2.vT * c2;
    return (a + b > 0.0) ? 4.0 * a * b / ((a + b) * (a + b)) : 0.0;
}

struct AmmWave {
    Cx dx, dz, txz, tzz;
};
CMPMC_HD AmmWave amm_wave(const Medium& m, bool P, Cx s, double p) {
    const double v = P ? m.vL : m.vT;
    const Cx dx = P ? cx(v * p) : v * s;
    const Cx dz = P ? v * s : cx(-v * p);
    const double mu = m.rho * m.vT * m.vT, la = m.rho * (m.vL * m.vL - 2.0 * m.vT * m.vT);
    AmmWave w;
    w.dx = dx;
    w.dz = dz;
    w.txz = mu * (s * dx + p * dz);
    w.tzz = la * (p * dx + s * dz) + ((2.0 * mu) * s) * dz;
    return w;
}

// transmitted energy flux T_P + T_S of a P or SV wave (amm_psv, interface_transmission.hpp:74-117)
CMPMC_HD double amm_psv_transmitted(const Medium& m1, const Medium& m2, bool incident_P, double theta1) {
    const double v_inc = incident_P ? m1.vL : m1.vT;
    const double p = m_sin(theta1) / v_inc;
    const Cx a1 = csqrt_real(1.0 / (m1.vL * m1.vL) - p * p), b1 = csqrt_real(1.0 / (m1.vT * m1.vT) - p * p);
    const Cx a2 = csqrt_real(1.0 / (m2.vL * m2.vL) - p * p), b2 = csqrt_real(1.0 / (m2.vT * m2.vT) - p * p);
    const AmmWave inc = amm_wave(m1, incident_P, incident_P ? a1 : b1, p);
    const AmmWave w[4] = {amm_wave(m1, true, cneg(a1), p), amm_wave(m1, false, cneg(b1), p),
                          amm_wave(m2, true, a2, p), amm_wave(m2, false, b2, p)};
    const double sgn[4] = {1.0, 1.0, -1.0, -1.0};
    Cx M[4][5];
    for (int j = 0; j < 4; ++j) {
        M[0][j] = sgn[j] * w[j].dx;
        M[1][j] = sgn[j] * w[j].dz;
        M[2][j] = sgn[j] * w[j].txz;
        M[3][j] = sgn[j] * w[j].tzz;
    }
    M[0][4] = cneg(inc.dx);
    M[1][4] = cneg(inc.dz);
    M[2][4] = cneg(inc.txz);
    M[3][4] = cneg(inc.tzz);
    for (int c = 0; c < 4; ++c) {  // Gauss-Jordan with partial pivoting
        int piv = c;
        for (int r = c + 1; r < 4; ++r)
            if (cabs_(M[r][c]) > cabs_(M[piv][c])) piv = r;
        if (piv != c)
            for (int k = 0; k < 5; ++k) {
                const Cx t = M[c][k];
                M[c][k] = M[piv][k];
                M[piv][k] = t;
            }
        const Cx d = M[c][c];
        if (cabs_(d) == 0.0) return 0.0;
        for (int k = c; k < 5; ++k) M[c][k] = cdiv(M[c][k], d);
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                const Cx f = M[r][c];
                for (int k = c; k < 5; ++k) M[r][k] = M[r][k] - f * M[c][k];
            }
    }
    const double flux_inc = m1.rho * v_inc * v_inc * (incident_P ? a1 : b1).re;
    const double tP = m2.rho * m2.vL * m2.vL * fabs(a2.re) * cnorm(M[2][4]) / flux_inc;
    const double tS = m2.rho * m2.vT * m2.vT * fabs(b2.re) * cnorm(M[3][4]) / flux_inc;
    return tP + tS;
}

// IsotropicAMMInterface::transmission (interface_transmission.hpp:125-130)
CMPMC_HD double amm_transmission(const Medium& sub, const Medium& film, bool longitudinal, double cos_theta) {
    const double th = m_acos(dclamp(fabs(cos_theta), 0.0, 1.0));
    if (longitudinal) return amm_psv_transmitted(sub, film, true, th);
    return 0.5 * (amm_psv_transmitted(sub, film, false, th) + amm_sh(sub, film, th));
}

// ElectrodePatternMask::find_channel (electrode_pattern.hpp:82-92): the first pad that
// contains (x, y) gives the channel, drawing once when its fill fraction is below 1;
// -1 for bare crystal. `U` is the generator (FP64 uniform()).
template <class U>
CMPMC_HD int find_channel(const Pad* pads, int n_pads, double x, double y, U& rng) {
    for (int i = 0; i < n_pads; ++i) {
        const Pad& p = pads[i];
        if (pad_contains(p, x, y)) {
            if (p.fill >= 1.0 || rng.uniform() < p.fill) return p.channel;
            return -1;
        }
    }
    return -1;
}

// SurfaceProperty::eval_poly (surface_property.hpp:48-55): Horner from the top
CMPMC_HD double eval_poly(const double* c, int n, double f) {
    if (n <= 0) return 0.0;
    double acc = 0.0;
    for (int i = n - 1; i >= 0; --i) acc = acc * f + c[i];
    return acc;
}
struct Split {
    double p_spec, p_diff, p_anh;
};
// SurfaceProperty::reflection_split (surface_property.hpp:72-86)
CMPMC_HD Split reflection_split(const Surface& s, double e) {
    const double f = (e / kHPlanck) / kGHz;
    const double anh = (s.n_anh == 0 || f > s.anh_cutoff) ? 0.0 : eval_poly(s.anh, s.n_anh, f);
    double diff;
    if (s.n_diff == 0 || f > s.anh_cutoff) diff = 1.0 - s.spec_prob_const;
    else diff = eval_poly(s.diff, s.n_diff, dmin(f, s.refl_cutoff));
    double spec;
    if (s.n_spec == 0 || f > s.refl_cutoff) spec = 1.0 - diff - anh;
    else spec = eval_poly(s.spec, s.n_spec, f);
    spec = dmax(0.0, spec);
    diff = dmax(0.0, diff);
    const double a = dmax(0.0, anh);
    const double nrm = spec + diff + a;
    Split r;
    if (nrm <= 0.0) { r.p_spec = 0.0; r.p_diff = 1.0; r.p_anh = 0.0; return r; }
    r.p_spec = spec / nrm;
    r.p_diff = diff / nrm;
    r.p_anh = a / nrm;
    return r;
}

// Fixed-capacity buffer with the reference's silent drop when full (math.hpp:101-131)
constexpr int kKaplanCap = 256;
struct KBuf {
    double* d;
    int n;
    CMPMC_HD void clear() { n = 0; }
    CMPMC_HD void push(double v) { if (n < kKaplanCap) d[n++] = v; }
};

// KaplanFilm (superconductor/kaplan_film.hpp:39-323)
CMPMC_HD bool film_is_subgap(const Film& f, double e) { return e < 2.0 * f.gap_energy; }
template <class G>
CMPMC_HD bool film_is_thermalized(const Film& f, double e, G& rng) {
    if (f.temperature <= 0.0) return false;
    const double kT = kBoltzmann * f.temperature;
    return e < kT * (-m_log(rng.uniform()));
}
CMPMC_HD double film_escape_probability(const Film& f, double e, double thickness_frac) {
    if (f.gap_energy <= 0.0) return 1.0;
    const double denom = 1.0 + f.phonon_lifetime_slope * (e / f.gap_energy - 2.0);
    if (denom <= 0.0) return 1.0;
    const double mfp = (f.v_sound * f.phonon_lifetime) / denom;
    const double path = thickness_frac * f.film_thickness;
    return m_exp(-path / mfp);
}
CMPMC_HD double film_pb_integral(const Film& f, double omega) {
    const double d = f.gap_energy;
    if (omega < 2.0 * d) return 0.0;
    const double s = omega - 2.0 * d;
    double acc = 0.0;
    for (int i = 0; i < 48; ++i) {
        const double t = kPi * (i + 0.5) / 48;
        const double E = d + 0.5 * s * (1.0 - m_cos(t));
        acc += (E * (omega - E) + d * d) / sqrt((E + d) * (omega - E + d));
    }
    return acc * kPi / 48;
}
CMPMC_HD double film_pb_rate(const Film& f, double omega) {
    if (f.gap_energy <= 0.0 || f.phonon_lifetime <= 0.0 || omega < 2.0 * f.gap_energy) return 0.0;
    return film_pb_integral(f, omega) / (kPi * f.gap_energy * f.phonon_lifetime);
}
CMPMC_HD double film_loss_probability(const Film& f, double e, double thickness_frac) {
    if (f.loss_model == 1) {
        if (f.phonon_loss_time <= 0.0) return 0.0;
        const double g = film_pb_rate(f, e);
        if (g <= 0.0) return 1.0;
        return 1.0 / (1.0 + g * f.phonon_loss_time);
    }
    return film_escape_probability(f, e, thickness_frac);
}
template <class G>
CMPMC_HD bool film_direct_absorption(const Film& f, double e, G& rng) {
    if (e < 2.0 * f.absorber_gap) return false;
    return rng.uniform() < f.subgap_absorption;
}
template <class G>
CMPMC_HD double film_calc_direct_absorption(const Film& f, double e, KBuf& keep, G& rng) {
    if (film_direct_absorption(f, e, rng)) return e;
    keep.push(e);
    return 0.0;
}
CMPMC_HD double film_qp_efficiency(const Film& f, double qpE) {
    const double eff = (f.gap_energy > 0.0) ? (f.absorber_eff + f.absorber_eff_slope * (qpE / f.gap_energy)) : 1.0;
    return dclamp(eff, 0.0, 1.0);
}
template <class G>
CMPMC_HD double film_calc_qp_absorption(const Film& f, double qpE, KBuf& phon, KBuf& qp, G& rng) {
    if (rng.uniform() > film_qp_efficiency(f, qpE)) return 0.0;
    if (qpE >= f.low_qp_limit * f.gap_energy) {
        qp.push(qpE);
        return 0.0;
    } else if (qpE > f.gap_energy) {
        const double edep = film_calc_direct_absorption(f, qpE - f.gap_energy, phon, rng);
        return edep + f.gap_energy;
    }
    return qpE;
}
CMPMC_HD double qp_weight(double E, double d, double x) {
    return (x * (E - x) + d * d) / sqrt((x + d) * (E - x + d));
}
// Case-II (photon) split weight (kaplan_film.hpp:229-245)
CMPMC_HD double qp_weight_case2(double E, double d, double x) {
    return dmax(0.0, x * (E - x) - d * d) / sqrt((x + d) * (E - x + d));
}
template <class G>
CMPMC_HD double film_sample_qp_energy_case2(const Film& f, double E, G& rng) {
    const double d = f.gap_energy;
    const double span = E - 2.0 * d;
    if (span <= 1e-16) return 0.5 * E;
    const double w_max = dmax(qp_weight_case2(E, d, d), qp_weight_case2(E, d, 0.5 * E)) * 1.0001;
    for (;;) {
        const double u = rng.uniform();
        const double s = m_sin(kHalfPi * u);
        const double x = d + span * (s * s);
        if (rng.uniform() * w_max <= qp_weight_case2(E, d, x)) return x;
    }
}
// kaplan_film.hpp:209-227
template <class G>
CMPMC_HD double film_sample_qp_energy(const Film& f, double E, G& rng) {
    const double d = f.gap_energy;
    const double span = E - 2.0 * d;
    if (span <= 1e-16) return 0.5 * E;
    const double w_max = dmax(qp_weight(E, d, d), qp_weight(E, d, 0.5 * E));
    for (;;) {
        const double u = rng.uniform();
        const double s = m_sin(kHalfPi * u);
        const double x = d + span * (s * s);
        if (rng.uniform() * w_max <= qp_weight(E, d, x)) return x;
    }
}
CMPMC_HD double ph_weight(double E, double d, double d2E, double x) {
    const double diff = E - x;
    return (diff * diff) * (x - d2E) / sqrt(x + d);
}
// kaplan_film.hpp:269-289
template <class G>
CMPMC_HD double film_sample_phonon_energy(const Film& f, double E, G& rng) {
    const double d = f.gap_energy;
    const double span = E - d;
    if (span <= 1e-16) return 0.0;
    const double d2E = (d * d) / E;
    const double x_peak = dclamp(0.25 * (E + 3.0 * d2E), d, E);
    const double w_max = dmax(ph_weight(E, d, d2E, d), ph_weight(E, d, d2E, x_peak)) * 1.02;
    for (;;) {
        const double u = rng.uniform();
        const double x = d + span * (u * u);
        if (rng.uniform() * w_max <= ph_weight(E, d, d2E, x)) return E - x;
    }
}

// KaplanFilm::absorb_quantum (kaplan_film.hpp:106-206): a phonon seed (photon = false) or a
// photon seed (an absorbed quantum split into two quasiparticles, no entry step). The four
// generation buffers of the reference are value-copied at the end of each stage; here
// the same buffers are swapped, which leaves identical contents. `work` must hold
// 4 * kKaplanCap doubles; `refl` receives the re-emitted phonon energies.
// entry_checked: a phonon seed whose entry step (direct absorption, loss at entry) the caller
// has already drawn and passed, so the cascade starts at once.
template <class G>
CMPMC_HD double film_absorb_quantum(const Film& f, double energy, KBuf& refl, double* work, G& rng, bool photon,
                                    bool entry_checked = false) {
    refl.clear();
    const bool entry = !photon && !entry_checked;
    if (entry && film_direct_absorption(f, energy, rng)) return energy;
    if (film_is_subgap(f, energy) || (entry && rng.uniform() <= film_loss_probability(f, energy, 4.0))) {
        refl.push(energy);
        return 0.0;
    }
    double edep = 0.0;
    const int n_pairs = (f.high_qp_limit > 0.0 && f.gap_energy > 0.0)
                            ? static_cast<int>(ceil(energy / (2.0 * f.high_qp_limit * f.gap_energy)))
                            : 1;
    KBuf qp{work, 0}, phon{work + kKaplanCap, 0}, next_phon{work + 2 * kKaplanCap, 0},
        next_qp{work + 3 * kKaplanCap, 0};
    const double init_e = energy / n_pairs;
    if (photon) {
        // case-II split of the absorbed quantum into two quasiparticles (kaplan_film.hpp:134-139)
        for (int i = 0; i < n_pairs; ++i) {
            const double qpE = film_sample_qp_energy_case2(f, init_e, rng);
            edep += film_calc_qp_absorption(f, qpE, phon, qp, rng);
            edep += film_calc_qp_absorption(f, init_e - qpE, phon, qp, rng);
        }
    } else {
        for (int i = 0; i < n_pairs; ++i) phon.push(init_e);
    }

    while (qp.n != 0 || phon.n != 0) {
        // A. phonons >= 2 Delta break pairs
        if (phon.n != 0) {
            next_phon.clear();
            for (int i = 0; i < phon.n; ++i) {
                const double E = phon.d[i];
                if (film_is_subgap(f, E)) {
                    next_phon.push(E);
                    continue;
                }
                const double qpE = film_sample_qp_energy(f, E, rng);
                edep += film_calc_qp_absorption(f, qpE, next_phon, qp, rng);
                edep += film_calc_qp_absorption(f, E - qpE, next_phon, qp, rng);
            }
            const KBuf t = phon; phon = next_phon; next_phon = t;
        }
        // B. quasiparticles >= low_qp_limit Delta radiate phonons
        if (qp.n != 0) {
            next_qp.clear();
            for (int i = 0; i < qp.n; ++i) {
                const double E = qp.d[i];
                const double phonE = film_sample_phonon_energy(f, E, rng);
                const double qpE = E - phonE;
                if (film_is_subgap(f, phonE)) {
                    edep += film_calc_direct_absorption(f, phonE, phon, rng);
                } else {
                    phon.push(phonE);
                }
                edep += film_calc_qp_absorption(f, qpE, phon, next_qp, rng);
            }
            const KBuf t = qp; qp = next_qp; next_qp = t;
        }
        // C. film phonons escape into the crystal or stay for the next generation
        if (phon.n != 0) {
            next_phon.clear();
            for (int i = 0; i < phon.n; ++i) {
                const double E = phon.d[i];
                if (film_is_thermalized(f, E, rng)) continue;
                if (f.loss_model == 1) {
                    if (film_is_subgap(f, E) || rng.uniform() < film_loss_probability(f, E, 1.0)) refl.push(E);
                    else next_phon.push(E);
                    continue;
                }
                // The reference writes both draws in one unsequenced expression
                // (kaplan_film.hpp:193-194); its GCC build takes the left one first.
                const double u_side = rng.uniform();
                const double u_angle = rng.uniform();
                const double frac = ((u_side < 0.5) ? 0.5 : 1.5) / m_cos(u_angle * 1.47);
                if (rng.uniform() < film_escape_probability(f, E, frac)) {
                    refl.push(E);
                } else if (f.keep_all_phonons || !film_is_subgap(f, E)) {
                    next_phon.push(E);
                }
            }
            const KBuf t = phon; phon = next_phon; next_phon = t;
        }
    }
    return edep;
}

// KaplanFilm::absorb_phonon (kaplan_film.hpp:106-108)
template <class G>
CMPMC_HD double film_absorb_phonon(const Film& f, double energy, KBuf& refl, double* work, G& rng) {
    return film_absorb_quantum(f, energy, refl, work, rng, false);
}

}  // namespace cmpmc_gpu
