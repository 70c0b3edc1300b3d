// transport_batched.cu -- the batched FP32 form: one device thread per primary track.
//
// The plain form keeps each event's single random stream, so an event's tracks run one
// after another on one thread. Here every primary phonon owns its own xoshiro256**
// substream, Rng::for_stream(seed, (event << 20) | index within the event), so all
// primaries of a batch run concurrently and the result does not depend on how the device
// schedules them. A thread transports its primary and every daughter of it (decay,
// film re-emission, surface down-conversion) from a per-thread LIFO in global memory.
//
// Precision: position, directions, group velocity, the octahedral table blend, rates and
// sampling are FP32 (fast CUDA intrinsics); the phonon energy, time of flight, weight and
// the energy ledger are FP64, as is the Kaplan film cascade (so the ledger closes to
// rounding). The physics and its random-draw structure follow SimulationEngine::transport
// (transport/engine.hpp:403-582); only the stream assignment and the precision differ.
// A reflected track is moved 10 nm inward (the reference moves it 1e-11 m, below FP32
// resolution at the cylinder wall).
#define CMPMC_DEVICE_FAST_MATH 1
#include "device.cuh"

namespace cmpmc_gpu {

namespace {

constexpr float kNudge = 1e-8f;  // inward displacement after a boundary event (m)

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

// per-primary stream: xoshiro256** with a 24-bit FP32 uniform in (0, 1)
struct FRng {
    Rng r;
    __device__ __forceinline__ float u() {
        const uint32_t m = static_cast<uint32_t>(r.next_u64() >> 41);  // 23 bits
        return __uint2float_rn(2u * m + 1u) * 5.9604644775390625e-8f;  // (2m+1) / 2^24
    }
    __device__ __forceinline__ F3 iso() {
        const float ct = 2.0f * u() - 1.0f;
        const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float s, c;
        __sincosf(6.28318530717958648f * u(), &s, &c);
        return f3(st * c, st * s, ct);
    }
    __device__ __forceinline__ F3 lambert(F3 n) {
        const float phi = 6.28318530717958648f * u();
        const float st = sqrtf(u());
        const float ct = sqrtf(fmaxf(0.0f, 1.0f - st * st));
        const F3 a = forth(n);
        const F3 b = fcross(n, a);
        float s, c;
        __sincosf(phi, &s, &c);
        return funit(a * (st * c) + b * (st * s) + n * ct);
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
};

struct FKin {
    F3 dir;
    float mag;
};

__device__ __forceinline__ FKin fmap(const FLat& L, int mode, F3 k) {
    const F3 kc = f3(L.o[0] * k.x + L.o[3] * k.y + L.o[6] * k.z, L.o[1] * k.x + L.o[4] * k.y + L.o[7] * k.z,
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
    r.dir = f3(L.o[0] * vn.x + L.o[1] * vn.y + L.o[2] * vn.z, L.o[3] * vn.x + L.o[4] * vn.y + L.o[5] * vn.z,
               L.o[6] * vn.x + L.o[7] * vn.y + L.o[8] * vn.z);
    r.mag = mag;
    return r;
}

__device__ __forceinline__ int fdos(const FLat& L, FRng& g) {
    const float u = g.u();
    return (u < L.fL) ? 0 : ((u < L.fLST) ? 2 : 1);
}
__device__ __forceinline__ int ftrans(const FLat& L, FRng& g) { return (g.u() < L.p_st_trans) ? 2 : 1; }
__device__ __forceinline__ float fcdf(const float* cdf, FRng& g) {
    const float u = g.u() * (kNCdf - 1);
    const int i = min(static_cast<int>(u), kNCdf - 2);
    const float f = u - i;
    return __ldg(cdf + i) * (1.0f - f) + __ldg(cdf + i + 1) * f;
}
__device__ __forceinline__ float facos_clamped(float c) { return acosf(fminf(fmaxf(c, -1.0f), 1.0f)); }

struct FTrack {
    F3 pos, k, vg;
    float vmag;
    double E, t, w;
    uint32_t bounces;
    int mode;
};

struct alignas(16) GFTrack {
    float px, py, pz, kx, ky, kz, vx, vy, vz, vmag;
    uint32_t bounces;
    int mode;
    double E, t, w;
};

// inward Lambertian wavevector whose group velocity points inward (engine.hpp:927-936)
__device__ __forceinline__ F3 finward(const FLat& L, int mode, F3 n, FRng& g, FKin& kin) {
    for (int trial = 0; trial < 16; ++trial) {
        const F3 kd = g.lambert(n);
        kin = fmap(L, mode, kd);
        if (fdot(kin.dir, n) > 1e-6f) return kd;
    }
    kin = fmap(L, mode, n);
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

struct BatchCtx {
    GFTrack* stk;
    uint32_t n_stk, cap;
    unsigned err;
    __device__ __forceinline__ void push(const FTrack& t) {
        if (n_stk >= cap) {
            err |= kErrPhononStack;
            return;
        }
        GFTrack g;
        g.px = t.pos.x; g.py = t.pos.y; g.pz = t.pos.z;
        g.kx = t.k.x; g.ky = t.k.y; g.kz = t.k.z;
        g.vx = t.vg.x; g.vy = t.vg.y; g.vz = t.vg.z;
        g.vmag = t.vmag;
        g.bounces = t.bounces;
        g.mode = t.mode;
        g.E = t.E; g.t = t.t; g.w = t.w;
        stk[n_stk++] = g;
    }
    __device__ __forceinline__ void pop(FTrack& t) {
        const GFTrack g = stk[--n_stk];
        t.pos = f3(g.px, g.py, g.pz);
        t.k = f3(g.kx, g.ky, g.kz);
        t.vg = f3(g.vx, g.vy, g.vz);
        t.vmag = g.vmag;
        t.bounces = g.bounces;
        t.mode = g.mode;
        t.E = g.E; t.t = g.t; t.w = g.w;
    }
};

__device__ __forceinline__ FTrack fmake(const FLat& L, F3 pos, F3 k, int mode, double E, double t, double w) {
    FTrack r;
    r.pos = pos;
    r.k = funit(k);
    const FKin kin = fmap(L, mode, r.k);
    r.vg = kin.dir;
    r.vmag = kin.mag;
    r.E = E;
    r.t = t;
    r.w = w;
    r.bounces = 0;
    r.mode = mode;
    return r;
}

__global__ void __launch_bounds__(128) k_unit_event(const uint64_t* __restrict__ ph_off, uint64_t n_events,
                                                    uint32_t* __restrict__ unit_event) {
    for (uint64_t ev = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; ev < n_events;
         ev += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        for (uint64_t j = ph_off[ev]; j < ph_off[ev + 1]; ++j) unit_event[j] = static_cast<uint32_t>(ev);
}

__global__ void __launch_bounds__(128) k_batched_fp32(const FLat L, const Detector D, const RunArgs a,
                                                      const uint32_t* __restrict__ unit_event) {
    const uint64_t slot = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    KBuf refl{refl_buf, 0};
    BatchCtx ctx;
    ctx.stk = reinterpret_cast<GFTrack*>(a.stack) + slot * a.stack_cap;
    ctx.cap = a.stack_cap;
    ctx.err = 0;
    const float R = static_cast<float>(D.radius), H = static_cast<float>(D.half_z);
    for (;;) {
        const unsigned long long unit = atomicAdd(a.next_work, 1ull);
        if (unit >= a.n_events) break;
        const uint32_t ev = unit_event[unit];
        const uint64_t j = unit - a.ph_off[ev];
        FRng g;
        g.r = Rng::for_stream(a.seed, ((a.first_event + ev) << 20) | j);
        const cmpmc_phonon_track& in = a.ph[unit];
        FTrack trk;
        trk.pos = f3(static_cast<float>(in.pos[0]), static_cast<float>(in.pos[1]), static_cast<float>(in.pos[2]));
        trk.k = f3(static_cast<float>(in.k_dir[0]), static_cast<float>(in.k_dir[1]), static_cast<float>(in.k_dir[2]));
        trk.vg = f3(static_cast<float>(in.vg_dir[0]), static_cast<float>(in.vg_dir[1]),
                    static_cast<float>(in.vg_dir[2]));
        trk.vmag = static_cast<float>(in.vg_mag);
        trk.E = in.energy;
        trk.t = in.time;
        trk.w = in.weight;
        trk.bounces = in.bounces;
        trk.mode = in.mode;
        ctx.n_stk = 0;
        EvStats st;
        memset(&st, 0, sizeof(st));
        uint32_t n_hits = 0;
        for (bool have = true; have; have = (ctx.n_stk > 0) ? (ctx.pop(trk), true) : false) {
            for (;;) {
                if (trk.E < D.min_phonon_eV || trk.bounces >= D.max_bounces) {
                    st.killed_tracks++;
                    st.escaped_eV += trk.E * trk.w;
                    break;
                }
                if (D.rr_bounces != 0 && trk.bounces > D.rr_bounces && (trk.bounces - D.rr_bounces) % 32 == 0) {
                    if (g.u() < static_cast<float>(D.rr_survival)) {
                        trk.w /= D.rr_survival;
                    } else {
                        st.killed_tracks++;
                        break;
                    }
                }
                st.total_steps++;
                const float nu = static_cast<float>(trk.E) * L.inv_h_thz;
                const float nu2 = nu * nu;
                const float r_iso = L.b4 * (nu2 * nu2);
                const float r_poly = trk.vmag * L.poly_inv;
                const float r_down = (trk.mode == 0) ? L.a5 * (nu2 * nu2 * nu) : 0.0f;
                const float r_tot = r_iso + r_poly + r_down;
                const float d_phys = (r_tot > 1e-12f) ? (-__logf(g.u()) * trk.vmag / r_tot)
                                                      : __int_as_float(0x7f800000);
                const FBHit bh = fexit(R, H, trk.pos, trk.vg);
                if (d_phys < bh.d) {
                    trk.pos = trk.pos + trk.vg * d_phys;
                    trk.t += static_cast<double>(d_phys / trk.vmag);
                    const float u_proc = g.u() * r_tot;
                    if (r_down > 0.0f && u_proc < r_down) {
                        // anharmonic decay (engine.hpp:938-988)
                        const F3 d1 = trk.k;
                        const F3 perp = forth(d1);
                        float sp, cp;
                        __sincosf(6.28318530717958648f * g.u(), &sp, &cp);
                        float x, th1, th2;
                        int m1, m2;
                        const float m = L.m_ratio, mm = m * m;
                        if (g.u() < L.fTT) {
                            st.decays_TT++;
                            x = fcdf(L.cdf_tt, g);
                            const float y = 1.0f - x;
                            th1 = facos_clamped((1.0f - mm * y * y + mm * x * x) / (2.0f * m * x));
                            th2 = facos_clamped((1.0f - mm * x * x + mm * y * y) / (2.0f * m * y));
                            m1 = ftrans(L, g);
                            m2 = ftrans(L, g);
                        } else {
                            st.decays_LT++;
                            x = fcdf(L.cdf_lt, g);
                            th1 = facos_clamped((1.0f + x * x * (1.0f - mm) + 2.0f * x * mm - mm) / (2.0f * x));
                            th2 = facos_clamped((1.0f - x * x + mm * (1.0f - x) * (1.0f - x)) / (2.0f * m * (1.0f - x)));
                            m1 = 0;
                            m2 = ftrans(L, g);
                        }
                        float s1, c1, s2, c2;
                        __sincosf(th1, &s1, &c1);
                        __sincosf(-th2, &s2, &c2);
                        const F3 k1 = funit(frotate(frotate(d1, perp, c1, s1), d1, cp, sp));
                        const F3 k2 = funit(frotate(frotate(d1, perp, c2, s2), d1, cp, sp));
                        const double xd = static_cast<double>(x);
                        ctx.push(fmake(L, trk.pos, k2, m2, (1.0 - xd) * trk.E, trk.t, trk.w));
                        trk.E = xd * trk.E;
                        trk.mode = m1;
                        trk.k = k1;
                        const FKin kin = fmap(L, m1, k1);
                        trk.vg = kin.dir;
                        trk.vmag = kin.mag;
                    } else {
                        if (u_proc < r_down + r_iso) st.isotope_scatters++;
                        else st.polycrystal_scatters++;
                        trk.mode = fdos(L, g);
                        trk.k = g.iso();
                        const FKin kin = fmap(L, trk.mode, trk.k);
                        trk.vg = kin.dir;
                        trk.vmag = kin.mag;
                    }
                    continue;
                }
                trk.pos = trk.pos + trk.vg * bh.d;
                trk.t += static_cast<double>(bh.d / trk.vmag);
                trk.bounces++;
                const Surface& s = D.surf[bh.surf];
                if (s.has_film && g.u() < static_cast<float>(s.prob_abs) &&
                    g.u() < static_cast<float>(s.film.film_absorption)) {
                    // Kaplan cascade in FP64 (CUDA libm); a substream-local Rng drives it
                    const double edep = film_absorb_phonon(s.film, trk.E, refl, kwork, g.r);
                    if (edep > 0.0) {
                        const double wedep = edep * trk.w;
                        st.sensor_hits++;
                        st.deposited_eV += wedep;
                        const uint32_t local = n_hits++;
                        if (a.keep_hits) {
                            const unsigned long long idx = atomicAdd(a.hit_count, 1ull);
                            if (idx < a.hit_cap) {
                                cmpmc_sensor_hit r;
                                r.pos[0] = trk.pos.x; r.pos[1] = trk.pos.y; r.pos[2] = trk.pos.z;
                                r.time = trk.t;
                                r.edep = wedep;
                                r.incident_energy = trk.E;
                                r.surface_id = static_cast<uint8_t>(bh.surf);
                                r.excitation = 0;
                                r.mode = static_cast<uint8_t>(trk.mode);
                                r._pad = 0;
                                r.channel_id = -1;
                                a.hit_stage[idx] = r;
                                a.hit_key[idx] = (static_cast<uint64_t>(unit) << 32) | local;
                            }
                        }
                    }
                    double sum_refl = 0.0;
                    for (int i = 0; i < refl.n; ++i) sum_refl += refl.d[i];
                    st.escaped_eV += dmax(0.0, trk.E - edep - sum_refl) * trk.w;
                    if (refl.n == 0) break;
                    const F3 re = trk.pos + bh.n * kNudge;
                    for (int i = 1; i < refl.n; ++i) {
                        const int m = fdos(L, g);
                        FKin kin;
                        const F3 kd = finward(L, m, bh.n, g, kin);
                        FTrack d;
                        d.pos = re; d.k = kd; d.vg = kin.dir; d.vmag = kin.mag;
                        d.E = refl.d[i]; d.t = trk.t; d.w = trk.w; d.bounces = 0; d.mode = m;
                        ctx.push(d);
                    }
                    trk.pos = re;
                    trk.E = refl.d[0];
                    trk.mode = fdos(L, g);
                    FKin kin;
                    trk.k = finward(L, trk.mode, bh.n, g, kin);
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                    continue;
                }
                if (g.u() > static_cast<float>(s.prob_refl)) {
                    st.killed_tracks++;
                    st.escaped_eV += trk.E * trk.w;
                    break;
                }
                st.surface_refls++;
                trk.pos = trk.pos + bh.n * kNudge;
                const Split sp = reflection_split(s, trk.E);
                const float u_refl = g.u();
                if (u_refl < static_cast<float>(sp.p_anh)) {
                    st.surface_downconversions++;
                    const bool tt = g.u() < L.fTT;
                    const float x = tt ? fcdf(L.cdf_tt, g) : fcdf(L.cdf_lt, g);
                    const int m1 = tt ? ftrans(L, g) : 0;
                    const int m2 = ftrans(L, g);
                    FKin k2kin;
                    const F3 k2 = finward(L, m2, bh.n, g, k2kin);
                    FTrack d;
                    d.pos = trk.pos; d.k = k2; d.vg = k2kin.dir; d.vmag = k2kin.mag;
                    d.E = (1.0 - static_cast<double>(x)) * trk.E; d.t = trk.t; d.w = trk.w; d.bounces = 0; d.mode = m2;
                    ctx.push(d);
                    trk.E = static_cast<double>(x) * trk.E;
                    trk.mode = m1;
                    FKin kin;
                    trk.k = finward(L, m1, bh.n, g, kin);
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                } else if (u_refl < static_cast<float>(sp.p_anh + sp.p_spec)) {
                    F3 kr = trk.k - bh.n * (2.0f * fdot(trk.k, bh.n));
                    FKin kin = fmap(L, trk.mode, kr);
                    if (fdot(kin.dir, bh.n) <= 1e-6f) kr = finward(L, trk.mode, bh.n, g, kin);
                    trk.k = kr;
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                } else {
                    FKin kin;
                    trk.k = finward(L, trk.mode, bh.n, g, kin);
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                }
            }
        }
        stats_from_event(st, 0.0, a.ev_stats[unit]);
        a.ev_nhits[unit] = a.keep_hits ? n_hits : 0;
    }
    if (ctx.err) atomicOr(a.err, ctx.err);
}

}  // namespace

// FP32 constants of the crystal derived from the FP64 lattice view
static FLat make_flat(const Lattice& L, const float* cdf_f) {
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
    return f;
}

cudaError_t launch_unit_event(const uint64_t* ph_off, uint64_t n_events, uint32_t* unit_event, cudaStream_t s) {
    k_unit_event<<<4 * 148, 128, 0, s>>>(ph_off, n_events, unit_event);
    return cudaGetLastError();
}

cudaError_t launch_batched_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const uint32_t* unit_event, int grid, int block, cudaStream_t s) {
    k_batched_fp32<<<grid, block, 0, s>>>(make_flat(L, cdf_f), D, a, unit_event);
    return cudaGetLastError();
}

cudaError_t batched_fp32_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_batched_fp32, block, 0);
}

size_t batched_stack_entry_bytes() { return sizeof(GFTrack); }

}  // namespace cmpmc_gpu
