// fp32.cuh -- FP32 primitives of the batched forms (phonon and charge kernels): vectors,
// the per-substream xoshiro128** generator, the FP32 crystal view with the octahedral
// group-velocity lookup, mode and decay samplers, the cylinder exit test and inward
// Lambertian sampling. Everything here is device code with internal linkage, so every
// translation unit that includes it gets its own copy.
#pragma once

#include "device.cuh"

namespace cmpmc_gpu {
namespace {

constexpr float kNudge = 1e-8f;  // inward displacement after a boundary event (m)
constexpr float kTwoPiF = 6.28318530717958648f;

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 fcross(F3 a, F3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ F3 funit(F3 a) {
    const float n2 = fdot(a, a);
    if (n2 <= 0.0f) return f3(0.0f, 0.0f, 1.0f);
    return a * rsqrtf(n2);
}
__device__ __forceinline__ F3 frotate(F3 v, F3 k, float c, float s) {
    return v * c + fcross(k, v) * s + k * (fdot(k, v) * (1.0f - c));
}
__device__ __forceinline__ F3 forth(F3 v) {
    const F3 a = (fabsf(v.x) < 0.9f) ? f3(1.0f, 0.0f, 0.0f) : f3(0.0f, 1.0f, 0.0f);
    return funit(fcross(v, a));
}

// xoshiro128** (Blackman and Vigna) per substream; FP32 uniforms in (0, 1) with 24 bits and
// FP64 uniforms with 53 bits for the Kaplan cascade
struct R128 {
    uint32_t s0, s1, s2, s3;
    __device__ __forceinline__ void seed(uint64_t key) {
        uint64_t z = key;
        const uint64_t a = splitmix_step(z += 0x9e3779b97f4a7c15ULL);
        const uint64_t b = splitmix_step(z += 0x9e3779b97f4a7c15ULL);
        s0 = static_cast<uint32_t>(a);
        s1 = static_cast<uint32_t>(a >> 32);
        s2 = static_cast<uint32_t>(b);
        s3 = static_cast<uint32_t>(b >> 32) | 1u;  // never all zero
    }
    __device__ __forceinline__ uint32_t next() {
        const uint32_t r = __funnelshift_l(s1 * 5u, s1 * 5u, 7) * 9u;
        const uint32_t t = s1 << 9;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = __funnelshift_l(s3, s3, 11);
        return r;
    }
    __device__ __forceinline__ float u() {
        return __uint2float_rn(((next() >> 9) << 1) | 1u) * 5.9604644775390625e-8f;  // (2m+1) / 2^24
    }
    __device__ __forceinline__ double uniform() {  // 53-bit, for the FP64 cascade
        const uint64_t x = (static_cast<uint64_t>(next()) << 21) ^ (next() >> 11);
        return static_cast<double>(x | 1ULL) * (1.0 / 9007199254740992.0);
    }
};

// FP32 view of the crystal (scaled so that rates stay in FP32 range)
struct FLat {
    const float4* oct;
    const float* cdf_lt;
    const float* cdf_tt;
    float o[9];
    float inv_h_thz;  // E[eV] -> nu[THz]
    float b4, a5;     // B_iso * 1e48, A_anh * 1e60 (nu in THz)
    float poly_inv;   // 1 / polycrystal mfp (0 disables)
    float fL, fLST, p_st_trans, fTT;
    float m_ratio;    // v_L / v_T
    // per surface: constant reflection split (1 when the polynomials do not depend on energy)
    int split_const[3];
    float p_anh[3], p_anh_spec[3];
    // KinematicsMode: Octahedral (the table above) or the lattice's Exact / Bilinear map
    int kin_mode;
    double density;
    const Stiffness* stiff;
    const double* bil;
    M3 orient64;
};

struct FKin {
    F3 dir;
    float mag;
};

// The Exact (Cardano per call) and Bilinear kinematics modes (crystal_lattice.hpp:76-114):
// the lattice's FP64 maps, out of line, rounded to FP32 at the end
__device__ __noinline__ FKin fmap_solve(const FLat* Lp, int mode, F3 k) {
    Lattice l{};
    l.kin_mode = Lp->kin_mode;
    l.density = Lp->density;
    l.stiff = Lp->stiff;
    l.bil = Lp->bil;
    l.orient = Lp->orient64;
    const Kin r = map_k_to_vg(l, mode, v3(k.x, k.y, k.z));
    FKin f;
    f.dir = F3{static_cast<float>(r.vg_dir.x), static_cast<float>(r.vg_dir.y), static_cast<float>(r.vg_dir.z)};
    f.mag = static_cast<float>(r.vg_mag);
    return f;
}

// kRot = false: the crystal frame is the detector frame (identity orientation, the default
// lattice), so both rotations are skipped
template <bool kRot = true>
__device__ __forceinline__ FKin fmap(const FLat& L, int mode, F3 k) {
    F3 kc = k;
    if constexpr (kRot)
        kc = f3(L.o[0] * k.x + L.o[3] * k.y + L.o[6] * k.z, L.o[1] * k.x + L.o[4] * k.y + L.o[7] * k.z,
                L.o[2] * k.x + L.o[5] * k.y + L.o[8] * k.z);
    const float l1 = fabsf(kc.x) + fabsf(kc.y) + fabsf(kc.z);
    const float inv = (l1 > 1e-18f) ? __frcp_rn(l1) : 1.0f;
    float px = kc.x * inv, py = kc.y * inv;
    if (kc.z < 0.0f) {
        const float ox = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
        const float oy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
        px = ox;
        py = oy;
    }
    const float u = (fminf(fmaxf(px, -1.0f), 1.0f) + 1.0f) * 127.5f;
    const float v = (fminf(fmaxf(py, -1.0f), 1.0f) + 1.0f) * 127.5f;
    const int i0 = min(max(static_cast<int>(u), 0), kNOct - 2);
    const int j0 = min(max(static_cast<int>(v), 0), kNOct - 2);
    const float du = u - i0, dv = v - j0;
    const int base = (mode * kNOct + i0) * kNOct + j0;
    const float4 e00 = __ldg(L.oct + base), e01 = __ldg(L.oct + base + 1);
    const float4 e10 = __ldg(L.oct + base + kNOct), e11 = __ldg(L.oct + base + kNOct + 1);
    const float w00 = (1.0f - du) * (1.0f - dv), w10 = du * (1.0f - dv), w01 = (1.0f - du) * dv, w11 = du * dv;
    const F3 vc = f3(e00.x * w00 + e10.x * w10 + e01.x * w01 + e11.x * w11,
                     e00.y * w00 + e10.y * w10 + e01.y * w01 + e11.y * w11,
                     e00.z * w00 + e10.z * w10 + e01.z * w01 + e11.z * w11);
    const float mag = sqrtf(fdot(vc, vc));
    const F3 vn = vc * __frcp_rn(fmaxf(mag, 1e-12f));
    FKin r;
    r.dir = vn;
    if constexpr (kRot)
        r.dir = f3(L.o[0] * vn.x + L.o[1] * vn.y + L.o[2] * vn.z, L.o[3] * vn.x + L.o[4] * vn.y + L.o[5] * vn.z,
                   L.o[6] * vn.x + L.o[7] * vn.y + L.o[8] * vn.z);
    r.mag = mag;
    return r;
}

// the orientation is the identity (the kernels' kKin = 2 variant may be used)
inline bool flat_identity_orientation(const FLat& f) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (f.o[3 * i + j] != (i == j ? 1.0f : 0.0f)) return false;
    return true;
}

// The group-velocity map of the kernel's kinematics: the octahedral table (kKin 0), the
// lattice's Exact / Bilinear map (kKin 1, out of line) or the octahedral table of a crystal
// with the identity orientation (kKin 2: no rotations). A compile-time choice: an
// out-of-line call in the octahedral kernels' step loop would cost them a third.
template <int kKin>
__device__ __forceinline__ FKin fmapk(const FLat& L, int mode, F3 k) {
    if constexpr (kKin == 1) return fmap_solve(&L, mode, k);
    else if constexpr (kKin == 2) return fmap<false>(L, mode, k);
    else return fmap(L, mode, k);
}

__device__ __forceinline__ int fdos(const FLat& L, float u) { return (u < L.fL) ? 0 : ((u < L.fLST) ? 2 : 1); }
__device__ __forceinline__ int ftrans(const FLat& L, R128& g) { return (g.u() < L.p_st_trans) ? 2 : 1; }
__device__ __forceinline__ float fcdf(const float* cdf, R128& g) {
    const float u = g.u() * (kNCdf - 1);
    const int i = min(static_cast<int>(u), kNCdf - 2);
    const float f = u - i;
    return __ldg(cdf + i) * (1.0f - f) + __ldg(cdf + i + 1) * f;
}
__device__ __forceinline__ float facos_clamped(float c) { return acosf(fminf(fmaxf(c, -1.0f), 1.0f)); }

// inward Lambertian wavevector whose group velocity points inward (engine.hpp:927-936)
template <int kKin = 0>
__device__ __forceinline__ F3 finward(const FLat& L, int mode, F3 n, R128& g, FKin& kin) {
    const F3 a = forth(n);
    const F3 b = fcross(n, a);
    for (int trial = 0; trial < 16; ++trial) {
        const float phi = kTwoPiF * g.u();
        const float st = sqrtf(g.u());
        const float ct = sqrtf(fmaxf(0.0f, 1.0f - st * st));
        float s, c;
        __sincosf(phi, &s, &c);
        const F3 kd = funit(a * (st * c) + b * (st * s) + n * ct);
        kin = fmapk<kKin>(L, mode, kd);
        if (fdot(kin.dir, n) > 1e-6f) return kd;
    }
    kin = fmapk<kKin>(L, mode, n);
    return n;
}

struct FBHit {
    float d;
    F3 n;
    int surf;
};

__device__ __forceinline__ FBHit fexit(float R, float H, F3 p, F3 v) {
    float t = __int_as_float(0x7f800000);
    int surf = 2;
    if (v.z > 1e-15f) {
        const float tz = (H - p.z) / v.z;
        if (tz >= 0.0f && tz < t) { t = tz; surf = 0; }
    } else if (v.z < -1e-15f) {
        const float tz = (-H - p.z) / v.z;
        if (tz >= 0.0f && tz < t) { t = tz; surf = 1; }
    }
    const float a = v.x * v.x + v.y * v.y;
    if (a > 1e-18f) {
        const float b = p.x * v.x + p.y * v.y;
        const float c = p.x * p.x + p.y * p.y - R * R;
        const float disc = fmaxf(0.0f, b * b - a * c);
        const float tr = (-b + sqrtf(disc)) / a;
        if (tr >= 0.0f && tr < t) { t = tr; surf = 2; }
    }
    FBHit h;
    h.d = fmaxf(0.0f, t);
    h.surf = surf;
    if (surf == 0) h.n = f3(0.0f, 0.0f, -1.0f);
    else if (surf == 1) h.n = f3(0.0f, 0.0f, 1.0f);
    else {
        const F3 hp = p + v * h.d;
        const float r = sqrtf(hp.x * hp.x + hp.y * hp.y);
        h.n = (r > 1e-15f) ? f3(-hp.x / r, -hp.y / r, 0.0f) : f3(-1.0f, 0.0f, 0.0f);
    }
    return h;
}

// The exit distance and surface only (the phonon step loop): the normal is needed only
// when the step ends on the boundary, so fnormal computes it there.
__device__ __forceinline__ FBHit fexit_d(float R, float H, F3 p, F3 v) {
    float t = __int_as_float(0x7f800000);
    int surf = 2;
    if (v.z > 1e-15f) {
        const float tz = (H - p.z) / v.z;
        if (tz >= 0.0f && tz < t) { t = tz; surf = 0; }
    } else if (v.z < -1e-15f) {
        const float tz = (-H - p.z) / v.z;
        if (tz >= 0.0f && tz < t) { t = tz; surf = 1; }
    }
    const float a = v.x * v.x + v.y * v.y;
    if (a > 1e-18f) {
        const float b = p.x * v.x + p.y * v.y;
        const float c = p.x * p.x + p.y * p.y - R * R;
        const float disc = fmaxf(0.0f, b * b - a * c);
        const float tr = (-b + sqrtf(disc)) / a;
        if (tr >= 0.0f && tr < t) { t = tr; surf = 2; }
    }
    FBHit h;
    h.d = fmaxf(0.0f, t);
    h.surf = surf;
    h.n = f3(0.0f, 0.0f, 1.0f);
    return h;
}

// inward normal of surface `surf` at the hit point hp (as fexit)
__device__ __forceinline__ F3 fnormal(int surf, F3 hp) {
    if (surf == 0) return f3(0.0f, 0.0f, -1.0f);
    if (surf == 1) return f3(0.0f, 0.0f, 1.0f);
    const float r = sqrtf(hp.x * hp.x + hp.y * hp.y);
    return (r > 1e-15f) ? f3(-hp.x / r, -hp.y / r, 0.0f) : f3(-1.0f, 0.0f, 0.0f);
}

// FP32 constants of the crystal derived from the FP64 lattice view
inline FLat make_flat(const Lattice& L, const float* cdf_f, const Detector& D) {
    FLat f;
    f.oct = reinterpret_cast<const float4*>(L.oct);
    f.cdf_lt = cdf_f;
    f.cdf_tt = cdf_f + kNCdf;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) f.o[3 * i + j] = static_cast<float>(L.orient.m[i][j]);
    f.inv_h_thz = static_cast<float>(1.0 / (kHPlanck * 1e12));
    f.b4 = static_cast<float>(L.B_iso * 1e48);
    f.a5 = static_cast<float>(L.A_anh * 1e60);
    f.poly_inv = (L.poly_mfp > 0.0) ? static_cast<float>(1.0 / L.poly_mfp) : 0.0f;
    f.fL = static_cast<float>(L.fLDOS);
    f.fLST = static_cast<float>(L.fLDOS + L.fSTDOS);
    f.p_st_trans = static_cast<float>(L.fSTDOS / (L.fSTDOS + L.fFTDOS));
    f.fTT = static_cast<float>(L.fTT_frac);
    f.m_ratio = static_cast<float>(L.v_sound / L.v_trans);
    for (int i = 0; i < 3; ++i) {
        const Surface& s = D.surf[i];
        // the split is energy independent when every polynomial is constant (or absent)
        const bool cst = s.n_spec <= 1 && s.n_diff <= 1 && s.n_anh <= 1;
        f.split_const[i] = cst ? 1 : 0;
        // constant polynomials still switch at the cut-offs; evaluate below and above them
        const Split lo = reflection_split(s, 1e-6), hi = reflection_split(s, 1.0);
        if (cst && (lo.p_anh != hi.p_anh || lo.p_spec != hi.p_spec)) f.split_const[i] = 0;
        f.p_anh[i] = static_cast<float>(lo.p_anh);
        f.p_anh_spec[i] = static_cast<float>(lo.p_anh + lo.p_spec);
    }
    f.kin_mode = L.kin_mode;
    f.density = L.density;
    f.stiff = L.stiff;
    f.bil = L.bil;
    f.orient64 = L.orient;
    return f;
}

}  // namespace
}  // namespace cmpmc_gpu
