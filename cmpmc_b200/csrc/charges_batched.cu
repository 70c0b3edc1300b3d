// charges_batched.cu -- the batched FP32 form of the charge transport
// (SimulationEngine::transport_charges, transport/engine.hpp:192-380): one device thread per
// carrier, drift steps in FP32, per-carrier time of flight and the energy ledger in FP64.
//
// Every carrier owns a random substream keyed by (run seed, event, index within the event),
// so carriers run concurrently in any order. A carrier that emits a tracked
// Neganov-Trofimov-Luke phonon appends it to a device queue instead of a per-event stack;
// the phonon kernel (k_queue_fp32) drains the queue between charge phases. Each queued
// phonon carries its own substream key (the carrier's lineage key mixed with the emission
// index), so a phonon's history does not depend on when or where it is transported.
//
// Queue room is reserved in blocks of kQBlock slots per thread, before the step that may
// need it. When the queue is full the carrier is parked with its generator state
// (QCharge) and the thread stops; the host drains the queue and resumes the parked
// carriers. Nothing waits on another thread, so no phase can stall.
//
// The field is the detector's uniform field or the tetrahedral mesh (DetectorModel::
// electric_field_at, engine.hpp:151-155), walked in FP32 from a per-carrier hint.
//
// FP32 care: kinetic energies are formed as p^2 / (sqrt(p^2 + m^2) + m), not
// sqrt(p^2 + m^2) - m (the rest energies are ~60 keV, the kinetic energies meV), and the
// second-order step solves its quadratic in the cancellation-free form.
#define CMPMC_DEVICE_FAST_MATH 1
#include "device.cuh"
#include "fp32.cuh"

namespace cmpmc_gpu {

namespace {

constexpr int kQBlock = 32;     // queue slots reserved per thread at a time
constexpr int kKnockCap = 8;    // knock-on carriers (trap ionization) pending per thread
constexpr float kHbarCF = static_cast<float>(kHbarC);
constexpr float kCLightF = static_cast<float>(kCLight);
constexpr float kInfF = __builtin_huge_valf();
constexpr float kMeshTol = -2e-6f;  // FP32 barycentric tolerance (rounding of p - x3 ~ 1e-6)
constexpr int kMeshMaxSteps = 4096;

// FP32 crystal constants of the charge transport (crystal_lattice.hpp:239-293, 322-331;
// charge_kernels.hpp:82-126)
struct FCLat {
    float rot[CMPMC_MAX_VALLEYS][9];
    F3 hv_sqrt, hv_sqrt_inv, inv_mass_ratio;
    float m_e, m_h;          // e_cond_mass, h_mass (eV)
    float ks_e, ks_h;        // k_sound (1/m)
    float tstep_e, tstep_h;  // 3 l0 / v_sound (s)
    float vs_hbar;           // v_sound * hbar (eV m)
    float hv_max;
    int n_valleys;
    int iv_model;
    float iv_min, iv_qrate, iv_qfield, iv_qpow_half, iv_lrate0, iv_lrate1, iv_lpow;
    float inv_trap_e, inv_trap_h, inv_ion_e_d0, inv_ion_e_a, inv_ion_h_d, inv_ion_h_a0;
    float fL, fLST;
    float bandgap;
    double bandgap_d;
};

struct FCSurf {
    float prob_abs, prob_spec, min_k_e, min_k_h;
    int n_pads;
    const Pad* pads;  // electrode mask
    int release;      // the collected energy goes to the release kernel (BulkDebye, or
                      // ElectrodeFilm on a surface with a film)
};

struct FCDet {
    float R, H;
    F3 e_field;
    FCSurf surf[3];
    float dt_cap, dk_frac;
    int second;              // Leman second-order stepping
    float luke_prob, luke_wt;
    double muF;
    MeshView32 mesh;
    MeshView2_32 mesh2;
};

struct FCharge {
    F3 pos, p;
    float ekin;
    double t;
    float w;
    int valley, type;  // type 1 electron, 2 hole
};

struct CStats {
    uint32_t steps, luke, iv, trapped, ion, crefl, collected;
    double luke_eV, recomb_eV, dep, esc;
};

__device__ __forceinline__ F3 mulr(const float* m, F3 v) {
    return f3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
__device__ __forceinline__ F3 mulrt(const float* m, F3 v) {
    return f3(m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
              m[2] * v.x + m[5] * v.y + m[8] * v.z);
}
__device__ __forceinline__ F3 hmul(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float fnorm(F3 a) { return sqrtf(fdot(a, a)); }

// Herring-Vogt maps (crystal_lattice.hpp:239-293)
__device__ __forceinline__ F3 e2s(const FCLat& L, int iv, F3 v) { return hmul(mulr(L.rot[iv], v), L.hv_sqrt_inv); }
__device__ __forceinline__ F3 s2e(const FCLat& L, int iv, F3 v) { return mulrt(L.rot[iv], hmul(v, L.hv_sqrt)); }
__device__ __forceinline__ float kin_from_p2(float p2, float m) { return p2 / (sqrtf(p2 + m * m) + m); }
__device__ __forceinline__ float ekin_e(const FCLat& L, int iv, F3 p) {
    const F3 ph = e2s(L, iv, p);
    return kin_from_p2(fdot(ph, ph), L.m_e);
}
__device__ __forceinline__ float ekin_h(const FCLat& L, F3 p) { return kin_from_p2(fdot(p, p), L.m_h); }
__device__ __forceinline__ float ekin_of(const FCLat& L, const FCharge& c) {
    return (c.type == 1) ? ekin_e(L, c.valley, c.p) : ekin_h(L, c.p);
}
__device__ __forceinline__ F3 vel_of(const FCLat& L, int type, int iv, F3 p) {
    if (type == 1) {
        const float ek = ekin_e(L, iv, p);
        return mulrt(L.rot[iv], hmul(mulr(L.rot[iv], p), L.inv_mass_ratio)) * (kCLightF / (ek + L.m_e));
    }
    return p * (kCLightF / (ekin_h(L, p) + L.m_h));
}
__device__ __forceinline__ F3 ekin_to_p_e(const FCLat& L, int iv, F3 dir, float ek) {
    const F3 u = funit(dir);
    const F3 uh = e2s(L, iv, u);
    const float band = fdot(uh, uh);
    if (band <= 0.0f || ek <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    return u * sqrtf((ek * ek + 2.0f * ek * L.m_e) / band);
}
__device__ __forceinline__ float kmag_of(const FCLat& L, const FCharge& c) {
    return (c.type == 1) ? fnorm(e2s(L, c.valley, c.p * (1.0f / kHbarCF))) : fnorm(c.p) * (1.0f / kHbarCF);
}

// ChargePhysics::make_charge (charge_transport.hpp:49-70)
__device__ FCharge make_charge_f(const FCLat& L, int type, F3 pos, F3 dir, float ek, int valley, double t, float w) {
    FCharge c;
    const F3 u = funit(dir);
    c.p = (type == 1) ? ekin_to_p_e(L, valley, u, ek) : u * sqrtf(fmaxf(0.0f, ek * ek + 2.0f * ek * L.m_h));
    c.pos = pos;
    c.ekin = ek;
    c.t = t;
    c.w = w;
    c.valley = valley;
    c.type = type;
    return c;
}

// electrode mask lookup out of line (keeps atan2 out of the step loop)
__device__ __noinline__ int mask_call(const Pad* pads, int n_pads, float x, float y, R128* g) {
    return find_channel(pads, n_pads, static_cast<double>(x), static_cast<double>(y), *g);
}

struct FRates {
    float luke, iv, trap, ion_e, ion_h, tot;
};

// SimulationEngine::charge_rates (engine.hpp:876-886) with luke_emission_rate
// (charge_transport.hpp:82-106) and the Quadratic / Linear intervalley rates
// (charge_kernels.hpp:82-99); `iv_field` is the field-dependent intervalley rate of E.
__device__ __forceinline__ FRates rates_of(const FCLat& L, const FCharge& c, float iv_field) {
    const bool e = (c.type == 1);
    const float v = fnorm(vel_of(L, c.type, c.valley, c.p));
    FRates r;
    const float k = kmag_of(L, c);
    const float ks = e ? L.ks_e : L.ks_h;
    if (k > ks) {
        const float mach = k / ks;
        const float dm = mach - 1.0f;
        r.luke = (dm * dm * dm) / ((e ? L.tstep_e : L.tstep_h) * mach);
    } else {
        r.luke = 0.0f;
    }
    r.iv = (e && L.n_valleys >= 2 && c.ekin >= L.iv_min) ? iv_field : 0.0f;
    r.trap = v * (e ? L.inv_trap_e : L.inv_trap_h);
    r.ion_e = v * (e ? L.inv_ion_e_d0 : L.inv_ion_h_d);
    r.ion_h = v * (e ? L.inv_ion_e_a : L.inv_ion_h_a0);
    r.tot = r.luke + r.iv + r.trap + r.ion_e + r.ion_h;
    return r;
}

__device__ __forceinline__ float iv_rate_of_field(const FCLat& L, F3 E) {
    if (L.iv_model == 0) return L.iv_qrate * __powf(L.iv_qfield * L.iv_qfield + fdot(E, E), L.iv_qpow_half);
    return L.iv_lrate0 + L.iv_lrate1 * __powf(fnorm(E) * 0.01f, L.iv_lpow);
}

// FP32 facet walk (TriLinearMesh3D::find_tetrahedron, mesh_field.hpp:66-100) with a
// tolerance above FP32 rounding; zero field outside the mesh
__device__ __forceinline__ F3 mesh_field_f(const MeshView32& m, F3 p, int32_t& hint) {
    if (hint < 0 || hint >= m.n_tets) hint = m.n_tets / 2;
    for (int step = 0; step < kMeshMaxSteps; ++step) {
        const MeshTet32& t = m.tet[hint];
        const float4 a = __ldg(reinterpret_cast<const float4*>(&t) + 0);  // tinv 0-3
        const float4 b = __ldg(reinterpret_cast<const float4*>(&t) + 1);  // tinv 4-7
        const float4 c = __ldg(reinterpret_cast<const float4*>(&t) + 2);  // tinv 8, x3
        const float dx = p.x - c.y, dy = p.y - c.z, dz = p.z - c.w;
        const float b0 = a.x * dx + a.y * dy + a.z * dz;
        const float b1 = a.w * dx + b.x * dy + b.y * dz;
        const float b2 = b.z * dx + b.w * dy + c.x * dz;
        const float b3 = 1.0f - b0 - b1 - b2;
        float mn = b0;
        int mi = 0;
        if (b1 < mn) { mn = b1; mi = 1; }
        if (b2 < mn) { mn = b2; mi = 2; }
        if (b3 < mn) { mn = b3; mi = 3; }
        if (mn >= kMeshTol) {
            const float4 e = __ldg(reinterpret_cast<const float4*>(&t) + 3);  // e, nb0
            return f3(e.x, e.y, e.z);
        }
        const int32_t next = __ldg(&t.nb[mi]);
        if (next < 0) break;
        hint = next;
    }
    return f3(0.0f, 0.0f, 0.0f);
}

// FP32 edge walk (BiLinearMesh2D::find_triangle / field_at, mesh_field.hpp:376-430) with
// the same FP32 tolerance; the axisymmetric field is rotated back around the z axis
__device__ __forceinline__ F3 mesh2_field_f(const MeshView2_32& m, F3 p, int32_t& hint) {
    float u = p.x, v = p.y;
    if (m.axisym) {
        u = sqrtf(p.x * p.x + p.y * p.y);
        v = p.z;
    }
    if (hint < 0 || hint >= m.n_tris) hint = m.n_tris / 2;
    for (int step = 0; step < kMeshMaxSteps; ++step) {
        const MeshTri32& t = m.tri[hint];
        const float4 a = __ldg(reinterpret_cast<const float4*>(&t) + 0);  // tinv
        const float4 b = __ldg(reinterpret_cast<const float4*>(&t) + 1);  // x2, e
        const float du = u - b.x, dv = v - b.y;
        const float b0 = a.x * du + a.y * dv;
        const float b1 = a.z * du + a.w * dv;
        const float b2 = 1.0f - b0 - b1;
        float mn = b0;
        int mi = 0;
        if (b1 < mn) { mn = b1; mi = 1; }
        if (b2 < mn) { mn = b2; mi = 2; }
        if (mn >= kMeshTol) {
            if (!m.axisym) return f3(b.z, b.w, 0.0f);
            if (u > 1e-15f) return f3(b.z * (p.x / u), b.z * (p.y / u), b.w);
            return f3(0.0f, 0.0f, b.w);
        }
        const int32_t next = __ldg(&t.nb[mi]);
        if (next < 0) break;
        hint = next;
    }
    return f3(0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ void sink_charge(const RunArgs& a, uint32_t ev, const CStats& st) {
    cmpmc_sim_stats& o = a.ev_stats[ev];
    auto add = [](uint64_t* p, uint32_t v) {
        if (v) atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
    };
    auto addd = [](double* p, double v) {
        if (v != 0.0) atomicAdd(p, v);
    };
    add(&o.charge_steps, st.steps);
    add(&o.luke_phonons_emitted, st.luke);
    add(&o.intervalley_scatters, st.iv);
    add(&o.charges_trapped, st.trapped);
    add(&o.trap_ionizations, st.ion);
    add(&o.charge_surface_refls, st.crefl);
    add(&o.charges_collected, st.collected);
    addd(&o.total_luke_phonon_eV, st.luke_eV);
    addd(&o.charge_recomb_edep_eV, st.recomb_eV);
    addd(&o.total_deposited_eV, st.dep);
    addd(&o.escaped_or_killed_eV, st.esc);
}

// a carrier and the bookkeeping that travels with it between phases
struct Carrier {
    FCharge c;
    R128 g;
    uint64_t ckey;
    uint32_t ev, luke_idx, n_knock, steps;
    int32_t hint;
};

__device__ __forceinline__ QCharge park(const Carrier& k) {
    QCharge q;
    q.px = k.c.pos.x; q.py = k.c.pos.y; q.pz = k.c.pos.z;
    q.qx = k.c.p.x; q.qy = k.c.p.y; q.qz = k.c.p.z;
    q.ekin = k.c.ekin;
    q.w = k.c.w;
    q.t = k.c.t;
    q.ckey = k.ckey;
    q.rng[0] = k.g.s0; q.rng[1] = k.g.s1; q.rng[2] = k.g.s2; q.rng[3] = k.g.s3;
    q.ev = k.ev;
    q.luke_idx = k.luke_idx;
    q.n_knock = k.n_knock;
    q.hint = k.hint;
    q.valley_type = static_cast<uint32_t>(k.c.valley) | (static_cast<uint32_t>(k.c.type) << 16);
    q.pad[0] = k.steps;
    q.pad[1] = q.pad[2] = 0;
    return q;
}
__device__ __forceinline__ Carrier unpark(const QCharge& q) {
    Carrier k;
    k.c.pos = f3(q.px, q.py, q.pz);
    k.c.p = f3(q.qx, q.qy, q.qz);
    k.c.ekin = q.ekin;
    k.c.w = q.w;
    k.c.t = q.t;
    k.c.valley = static_cast<int>(q.valley_type & 0xffffu);
    k.c.type = static_cast<int>(q.valley_type >> 16);
    k.ckey = q.ckey;
    k.g.s0 = q.rng[0]; k.g.s1 = q.rng[1]; k.g.s2 = q.rng[2]; k.g.s3 = q.rng[3];
    k.ev = q.ev;
    k.luke_idx = q.luke_idx;
    k.n_knock = q.n_knock;
    k.hint = q.hint;
    k.steps = q.pad[0];
    return k;
}

__device__ __forceinline__ uint64_t luke_key(uint64_t ckey, uint32_t idx) {
    return mix64(ckey ^ (0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(idx) + 1)));
}

// (128, 5): 96 registers, five blocks per SM (pair drift of 200,000 events 467 -> 431 ms
// against (128, 4) at 104 registers; (128, 6) at 80 registers 432 ms)
__global__ void __launch_bounds__(128, 5) k_charges_fp32(const __grid_constant__ FCLat Lp,
                                                         const __grid_constant__ FCDet D,
                                                         const __grid_constant__ RunArgs a,
                                                         const __grid_constant__ ChargeArgs ca) {
    // the crystal constants (the Herring-Vogt valley rotations and mass tensor among them) in
    // shared memory: the step reads the rotation of each carrier's own valley, an index that
    // differs between the lanes of a warp, which the constant bank of the kernel parameters
    // serves one distinct address at a time
    __shared__ alignas(16) FCLat sL;
    static_assert(sizeof(FCLat) % 4 == 0, "FCLat is copied in 4-byte words");
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(FCLat) / 4); i += blockDim.x)
        reinterpret_cast<uint32_t*>(&sL)[i] = reinterpret_cast<const uint32_t*>(&Lp)[i];
    __syncthreads();
    const FCLat& L = sL;
    Carrier k;
    CStats st{};
    QCharge knock[kKnockCap];
    int n_knock_stk = 0;
    uint64_t q_next = 0, q_end = 0;  // queue slots reserved by this thread
    unsigned err = 0;
    bool live = false, stop = false, dirty = false;
    const bool track_luke = D.luke_prob > 0.0f;
    const double e_gap = L.bandgap_d;
    F3 E_last = f3(kInfF, 0.0f, 0.0f);
    float iv_last = 0.0f;
    for (;;) {
        if (!live) {
            if (dirty) {
                sink_charge(a, k.ev, st);
                st = CStats{};
                dirty = false;
            }
            if (n_knock_stk > 0) {
                k = unpark(knock[--n_knock_stk]);
            } else if (stop) {
                break;
            } else {
                const unsigned long long r = (ca.n_resume_in > 0) ? atomicAdd(ca.resume_next, 1ull) : ~0ull;
                if (r < ca.n_resume_in) {
                    k = unpark(ca.resume_in[r]);
                } else {
                    const unsigned long long i = atomicAdd(ca.next_carrier, 1ull);
                    if (i >= ca.n_carriers) break;
                    const uint32_t ev = ca.carrier_event[i];
                    const uint64_t j = i - a.ch_off[ev];
                    const cmpmc_charge_track& in = a.ch[i];
                    k.c.pos = f3(static_cast<float>(in.pos[0]), static_cast<float>(in.pos[1]),
                                 static_cast<float>(in.pos[2]));
                    k.c.p = f3(static_cast<float>(in.p_eV[0]), static_cast<float>(in.p_eV[1]),
                               static_cast<float>(in.p_eV[2]));
                    k.c.ekin = static_cast<float>(in.ekin);
                    k.c.t = in.time;
                    k.c.w = static_cast<float>(in.weight);
                    k.c.valley = in.valley;
                    k.c.type = in.type;
                    k.ckey = mix64(ca.carrier_seed ^ mix64(((a.first_event + ev) << 20) | j));
                    k.g.seed(k.ckey);
                    k.ev = ev;
                    k.luke_idx = 0;
                    k.n_knock = 0;
                    k.steps = 0;
                    k.hint = -1;
                }
            }
            live = true;
        }
        // one step may queue one Luke phonon: hold a free slot before drawing anything
        if (track_luke && q_next == q_end) {
            const unsigned long long base = atomicAdd(ca.q_tail, static_cast<unsigned long long>(kQBlock));
            if (base + kQBlock > ca.q_cap) {
                // queue full: park this carrier and every pending knock-on, stop the thread
                const unsigned long long slot = atomicAdd(ca.n_resume_out, 1ull);
                if (slot < ca.resume_cap) ca.resume_out[slot] = park(k);
                else err |= kErrResume;
                while (n_knock_stk > 0) {
                    const unsigned long long s2 = atomicAdd(ca.n_resume_out, 1ull);
                    if (s2 < ca.resume_cap) ca.resume_out[s2] = knock[--n_knock_stk];
                    else { err |= kErrResume; --n_knock_stk; }
                }
                live = false;
                stop = true;
                continue;
            }
            q_next = base;
            q_end = base + kQBlock;
        }
        if (k.steps >= 20000000u) {  // the reference's step bound per carrier (engine.hpp:208)
            live = false;
            continue;
        }
        FCharge& c = k.c;
        ++k.steps;
        ++st.steps;
        dirty = true;
        const float q_sign = (c.type == 1) ? -1.0f : 1.0f;
        const F3 E = D.mesh.tet ? mesh_field_f(D.mesh, c.pos, k.hint)
                                : (D.mesh2.tri ? mesh2_field_f(D.mesh2, c.pos, k.hint) : D.e_field);
        if (E.x != E_last.x || E.y != E_last.y || E.z != E_last.z) {
            E_last = E;
            iv_last = iv_rate_of_field(L, E);
        }
        const FRates R0 = rates_of(L, c, iv_last);
        FRates R = R0;
        float dt_max = D.dt_cap;
        if (D.dk_frac > 0.0f) {
            const bool is_e = (c.type == 1);
            const float ks = is_e ? L.ks_e : L.ks_h;
            const float dk_rate = fnorm(E) * (kCLightF / kHbarCF) * (is_e ? L.hv_max : 1.0f);
            if (dk_rate > 0.0f) dt_max = fminf(dt_max, D.dk_frac * fmaxf(ks, kmag_of(L, c)) / dk_rate);
        }
        float dt_phys;
        if (D.second) {
            // Leman second-order stepping (engine.hpp:235-254): rate linear in time
            FCharge trial = c;
            trial.p = trial.p + E * (q_sign * kCLightF * dt_max);
            trial.ekin = ekin_of(L, trial);
            const float a0 = R0.tot;
            const float a1 = (rates_of(L, trial, iv_last).tot - a0) / dt_max;
            const float lnu = __logf(k.g.u());
            if (fabsf(a1) * dt_max <= 1e-6f * fmaxf(a0, 1e-30f)) {
                dt_phys = (a0 > 0.0f) ? (-lnu / a0) : kInfF;
            } else {
                const float disc = a0 * a0 - 2.0f * a1 * lnu;
                const float den = sqrtf(fmaxf(disc, 0.0f)) + a0;  // (sqrt(disc) - a0) / a1, cancellation-free
                dt_phys = (disc < 0.0f || !(den > 0.0f)) ? kInfF : (-2.0f * lnu / den);
                if (!(dt_phys >= 0.0f)) dt_phys = kInfF;
            }
        } else {
            dt_phys = (R0.tot > 1.0f) ? (-__logf(k.g.u()) / R0.tot) : kInfF;
        }
        const float dt = fminf(dt_phys, dt_max);
        const F3 dp = E * (q_sign * kCLightF * dt);
        const F3 p_mid = c.p + dp * 0.5f;
        const F3 v_mid = vel_of(L, c.type, c.valley, p_mid);
        const float v_mag = fnorm(v_mid);
        const float d_step = v_mag * dt;
        if (v_mag > 1e-6f) {
            const F3 v_dir = v_mid * (1.0f / v_mag);
            const FBHit bh = fexit(D.R, D.H, c.pos, v_dir);
            if (bh.d <= d_step) {
                const float dt_b = bh.d / v_mag;
                c.pos = c.pos + v_dir * bh.d;
                c.t += static_cast<double>(dt_b);
                c.p = c.p + E * (q_sign * kCLightF * dt_b);
                c.ekin = ekin_of(L, c);
                const FCSurf& s = D.surf[bh.surf];
                // electrode mask (engine.hpp:284-289), then ChargePhysics::should_absorb_boundary
                // (charge_transport.hpp:187-199)
                int ch_id = -1;
                bool absorb = true;
                if (s.n_pads > 0) {
                    // the out-of-line call gets a copy: only it has its address taken, so
                    // the carrier state stays in registers
                    R128 g_c = k.g;
                    ch_id = mask_call(s.pads, s.n_pads, c.pos.x, c.pos.y, &g_c);
                    k.g = g_c;
                    absorb = ch_id >= 0;
                }
                const float k_perp = -fdot(c.p * (1.0f / kHbarCF), bh.n);
                if (absorb) absorb = k_perp > ((c.type == 1) ? s.min_k_e : s.min_k_h) && k.g.u() < s.prob_abs;
                if (!absorb) {
                    ++st.crefl;
                    c.pos = c.pos + bh.n * kNudge;
                    // ChargePhysics::reflect_at_boundary (charge_transport.hpp:203-241)
                    bool done = false;
                    if (k.g.u() < s.prob_spec) {
                        const F3 kd = funit(c.p);
                        const F3 kr = funit(kd - bh.n * (2.0f * fdot(kd, bh.n)));
                        if (c.type == 2) {
                            c.p = kr * fnorm(c.p);
                            done = true;
                        } else {
                            const F3 pt = ekin_to_p_e(L, c.valley, kr, c.ekin);
                            if (fdot(vel_of(L, 1, c.valley, pt), bh.n) > 1e-6f) {
                                c.p = pt;
                                done = true;
                            }
                        }
                    }
                    if (!done) {
                        const F3 e1 = forth(bh.n);
                        const F3 e2 = fcross(bh.n, e1);
                        if (c.type == 2) {
                            const float phi = kTwoPiF * k.g.u();
                            const float st_ = sqrtf(k.g.u());
                            const float ct = sqrtf(fmaxf(0.0f, 1.0f - st_ * st_));
                            float sp, cp;
                            __sincosf(phi, &sp, &cp);
                            c.p = funit(e1 * (st_ * cp) + e2 * (st_ * sp) + bh.n * ct) * fnorm(c.p);
                        } else {
                            int trial = 0;
                            for (; trial < 16; ++trial) {
                                const float phi = kTwoPiF * k.g.u();
                                const float st_ = sqrtf(k.g.u());
                                const float ct = sqrtf(fmaxf(0.0f, 1.0f - st_ * st_));
                                float sp, cp;
                                __sincosf(phi, &sp, &cp);
                                const F3 dir = funit(e1 * (st_ * cp) + e2 * (st_ * sp) + bh.n * ct);
                                const F3 pt = ekin_to_p_e(L, c.valley, dir, c.ekin);
                                if (fdot(vel_of(L, 1, c.valley, pt), bh.n) > 1e-6f) {
                                    c.p = pt;
                                    break;
                                }
                            }
                            if (trial == 16) c.p = ekin_to_p_e(L, c.valley, bh.n, c.ekin);
                        }
                    }
                    continue;
                }
                // collection_release_energy (engine.hpp:889-893)
                const double e_rel = static_cast<double>(c.ekin) + ((c.type == 1) ? (e_gap - D.muF) : D.muF);
                ++st.collected;
                if (s.release) {
                    // BulkDebye / ElectrodeFilm (engine.hpp:302-313): the release kernel emits
                    // the phonons, runs the film cascades and records the hit
                    const unsigned long long slot = atomicAdd(ca.rel_tail, 1ull);
                    if (slot < ca.rel_cap) {
                        ReleaseRec r;
                        r.px = c.pos.x; r.py = c.pos.y; r.pz = c.pos.z;
                        r.w = c.w;
                        r.e_rel = e_rel;
                        r.t = c.t;
                        const uint64_t hi = k.g.next();
                        r.key = (hi << 32) | k.g.next();
                        r.ev = k.ev;
                        r.ch_id = ch_id;
                        r.surf = static_cast<uint8_t>(bh.surf);
                        r.type = static_cast<uint8_t>(c.type);
                        r.pad0 = r.pad1 = 0;
                        r.pad2 = 0;
                        ca.rel[slot] = r;
                    } else {
                        err |= kErrRelease;
                    }
                    live = false;
                    continue;
                }
                // ChargeRelease::RecordOnly
                const double recomb = e_rel * static_cast<double>(c.w);
                st.recomb_eV += recomb;
                st.dep += recomb;
                if (a.keep_hits) {
                    atomicAdd(reinterpret_cast<unsigned long long*>(a.ev_nhits + k.ev), 1ull);
                    const unsigned long long idx = atomicAdd(a.hit_count, 1ull);
                    if (idx < a.hit_cap) {
                        cmpmc_sensor_hit h;
                        h.pos[0] = c.pos.x; h.pos[1] = c.pos.y; h.pos[2] = c.pos.z;
                        h.time = c.t;
                        h.edep = recomb;
                        h.incident_energy = e_rel;
                        h.surface_id = static_cast<uint8_t>(bh.surf);
                        h.excitation = static_cast<uint8_t>(c.type);
                        h.mode = 0;
                        h._pad = 0;
                        h.channel_id = ch_id;
                        a.hit_stage[idx] = h;
                        a.hit_key[idx] = k.ev;
                    }
                }
                live = false;
                continue;
            }
        }
        c.pos = c.pos + v_mid * dt;
        c.t += static_cast<double>(dt);
        c.p = c.p + dp;
        c.ekin = ekin_of(L, c);
        if (dt_phys <= dt_max) {
            if (D.second) {
                R = rates_of(L, c, iv_last);
                if (R.tot <= 0.0f) continue;
            }
            const float u_proc = k.g.u() * R.tot;
            if (u_proc < R.trap) {
                ++st.trapped;
                st.esc += (static_cast<double>(c.ekin) + 0.5 * e_gap) * static_cast<double>(c.w);
                live = false;
                continue;
            } else if (u_proc < R.trap + R.ion_e + R.ion_h) {
                ++st.ion;
                const bool lib_e = (u_proc < R.trap + R.ion_e);
                const uint32_t nv = (L.n_valleys > 1) ? static_cast<uint32_t>(L.n_valleys) : 1u;
                const int kv = lib_e ? static_cast<int>(k.g.next() % nv) : 0;
                const float u1 = k.g.u(), u2 = k.g.u();
                const float ct = 2.0f * u1 - 1.0f, sn = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
                float sp, cp;
                __sincosf(kTwoPiF * u2, &sp, &cp);
                Carrier kn;
                kn.c = make_charge_f(L, lib_e ? 1 : 2, c.pos, f3(sn * cp, sn * sp, ct), 1.0e-6f, kv, c.t, c.w);
                kn.ckey = mix64(k.ckey ^ (0xd6e8feb86659fd93ULL * (static_cast<uint64_t>(++k.n_knock))));
                kn.g.seed(kn.ckey);
                kn.ev = k.ev;
                kn.luke_idx = 0;
                kn.n_knock = 0;
                kn.steps = 0;
                kn.hint = k.hint;
                if (n_knock_stk < kKnockCap) knock[n_knock_stk++] = park(kn);
                else err |= kErrChargeStack;
            } else if (u_proc < R.trap + R.ion_e + R.ion_h + R.iv) {
                // ChargePhysics::scatter_intervalley (charge_transport.hpp:169-184)
                const int nv = L.n_valleys;
                if (c.type == 1 && nv >= 2) {
                    const F3 kv = mulr(L.rot[c.valley], c.p * (1.0f / kHbarCF));
                    const int off = 1 + min(static_cast<int>(k.g.u() * static_cast<float>(nv - 1)), nv - 2);
                    const int nvl = (c.valley + off) % nv;
                    const F3 kn = mulrt(L.rot[nvl], kv);
                    c.valley = nvl;
                    c.p = ekin_to_p_e(L, nvl, kn * kHbarCF, c.ekin);
                }
                ++st.iv;
            } else if (R.luke > 0.0f) {
                // ChargePhysics::emit_luke_phonon (charge_transport.hpp:109-166)
                const bool is_e = (c.type == 1);
                const F3 kt = is_e ? e2s(L, c.valley, c.p * (1.0f / kHbarCF)) : c.p * (1.0f / kHbarCF);
                const float ks = is_e ? L.ks_e : L.ks_h;
                const float km = fnorm(kt);
                if (km > ks * 1.0001f) {
                    const F3 kdir = kt * (1.0f / km);
                    const float v = ks / km;
                    const float u = k.g.u();
                    const float cth = fminf(fmaxf(v + (1.0f - v) * cbrtf(1.0f - u), v), 1.0f);
                    const float sth = sqrtf(fmaxf(0.0f, 1.0f - cth * cth));
                    const float phi = kTwoPiF * k.g.u();
                    const float q = 2.0f * (km * cth - ks);
                    if (q > 0.0f) {
                        float sp, cp;
                        __sincosf(phi, &sp, &cp);
                        const F3 perp = forth(kdir);
                        const F3 qv = frotate(frotate(kdir * q, perp, cth, sth), kdir, cp, sp);
                        const F3 krec = kt - qv;
                        const float e_ph = fnorm(qv) * L.vs_hbar;
                        if (e_ph < c.ekin && e_ph > 0.0f) {
                            F3 qdir;
                            if (!is_e) {
                                c.p = krec * kHbarCF;
                                c.ekin = ekin_h(L, c.p);
                                qdir = funit(qv);
                            } else {
                                qdir = funit(s2e(L, c.valley, qv));
                                const float e_rec = c.ekin - e_ph;
                                c.p = ekin_to_p_e(L, c.valley, s2e(L, c.valley, krec) * kHbarCF, e_rec);
                                c.ekin = e_rec;
                            }
                            ++st.luke;
                            st.luke_eV += static_cast<double>(e_ph) * static_cast<double>(c.w);
                            if (track_luke && (D.luke_prob >= 1.0f || k.g.u() < D.luke_prob)) {
                                const float um = k.g.u();
                                QPhonon qp;
                                qp.px = c.pos.x; qp.py = c.pos.y; qp.pz = c.pos.z;
                                qp.kx = qdir.x; qp.ky = qdir.y; qp.kz = qdir.z;
                                qp.w = c.w * D.luke_wt;
                                qp.mode = static_cast<uint32_t>((um < L.fL) ? 0 : ((um < L.fLST) ? 2 : 1));
                                qp.E = static_cast<double>(e_ph);
                                qp.t = c.t;
                                qp.key = luke_key(k.ckey, k.luke_idx++);
                                qp.ev = k.ev;
                                qp.pad = 0;
                                ca.queue[q_next++] = qp;
                            }
                        }
                    }
                }
            }
        }
    }
    if (dirty) sink_charge(a, k.ev, st);
    if (err) atomicOr(a.err, err);
}

__global__ void k_carrier_event(const uint64_t* __restrict__ ch_off, uint64_t n_events,
                                uint32_t* __restrict__ carrier_event) {
    for (uint64_t ev = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; ev < n_events;
         ev += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        for (uint64_t j = ch_off[ev]; j < ch_off[ev + 1]; ++j) carrier_event[j] = static_cast<uint32_t>(ev);
}

// The release phase of the batched charge form (engine.hpp:302-313, 894-925): one collected
// carrier per thread, from its own substream. BulkDebye emits round(E_rel / E_Debye) (at
// least one) Debye phonons; ElectrodeFilm sends the energy into the electrode's film as
// quanta of at most max(4, electrode_seed_max_gap) Delta (photon seeds): the absorbed part
// is the hit, the escaping phonons re-enter the crystal, the rest is lost. The phonons go,
// inward Lambertian with a DOS mode and their own substreams, into the phonon queue of
// the round; the hit and the ledger go to the carrier's event.
template <int kKin>
__global__ void __launch_bounds__(128, 8) k_release_fp32(const __grid_constant__ FLat L,
                                                         const __grid_constant__ Detector D,
                                                         const __grid_constant__ RunArgs a,
                                                         const __grid_constant__ ChargeArgs ca,
                                                         const ReleaseRec* __restrict__ rel, uint64_t n_rel,
                                                         double debye_energy) {
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    unsigned err = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n_rel;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const ReleaseRec r = rel[i];
        R128 g;
        g.seed(r.key);
        const F3 hp = f3(r.px, r.py, r.pz);
        const F3 n_in = fnormal(r.surf, hp);
        const F3 p0 = hp + n_in * kNudge;
        uint32_t n_ph = 0;  // phonons queued so far (substream index)
        auto emit = [&](double e, unsigned long long slot) {
            const int mode = fdos(L, g.u());
            FKin kin;
            const F3 kd = finward<kKin>(L, mode, n_in, g, kin);
            QPhonon q;
            q.px = p0.x; q.py = p0.y; q.pz = p0.z;
            q.kx = kd.x; q.ky = kd.y; q.kz = kd.z;
            q.w = r.w;
            q.mode = static_cast<uint32_t>(mode);
            q.E = e;
            q.t = r.t;
            q.key = mix64(r.key ^ (0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(n_ph++) + 1)));
            q.ev = r.ev;
            q.pad = 0;
            ca.queue[slot] = q;
        };
        double hit_eV = 0.0, lost = 0.0;
        if (D.charge_release == 1) {
            const int k = static_cast<int>(round(r.e_rel / debye_energy));
            const int n = (k < 1) ? 1 : k;
            const unsigned long long base = atomicAdd(ca.q_tail, static_cast<unsigned long long>(n));
            if (base + n > ca.q_cap) {
                err |= kErrRelease;
            } else {
                for (int j = 0; j < n; ++j) emit(r.e_rel / n, base + j);
            }
        } else {
            const Film& film = D.surf[r.surf].film;
            const double qmax = dmax(4.0, D.electrode_seed_max_gap) * film.gap_energy;
            const int k = static_cast<int>(ceil(r.e_rel / qmax));
            const int n = (k < 1) ? 1 : k;
            const double q = r.e_rel / n;
            double absorbed = 0.0, emitted = 0.0;
            KBuf refl{refl_buf, 0};
            for (int j = 0; j < n; ++j) {
                absorbed += film_absorb_quantum(film, q, refl, kwork, g, true);
                if (refl.n == 0) continue;
                const unsigned long long base = atomicAdd(ca.q_tail, static_cast<unsigned long long>(refl.n));
                if (base + refl.n > ca.q_cap) {
                    err |= kErrRelease;
                    continue;
                }
                for (int m = 0; m < refl.n; ++m) {
                    emit(refl_buf[m], base + m);
                    emitted += refl_buf[m];
                }
            }
            lost = dmax(0.0, r.e_rel - absorbed - emitted);
            hit_eV = absorbed;
        }
        const double recomb = hit_eV * static_cast<double>(r.w);
        cmpmc_sim_stats& o = a.ev_stats[r.ev];
        if (recomb != 0.0) {
            atomicAdd(&o.charge_recomb_edep_eV, recomb);
            atomicAdd(&o.total_deposited_eV, recomb);
        }
        if (lost != 0.0) atomicAdd(&o.escaped_or_killed_eV, lost * static_cast<double>(r.w));
        if (a.keep_hits) {
            atomicAdd(reinterpret_cast<unsigned long long*>(a.ev_nhits + r.ev), 1ull);
            const unsigned long long idx = atomicAdd(a.hit_count, 1ull);
            if (idx < a.hit_cap) {
                cmpmc_sensor_hit h;
                h.pos[0] = r.px; h.pos[1] = r.py; h.pos[2] = r.pz;
                h.time = r.t;
                h.edep = recomb;
                h.incident_energy = r.e_rel;
                h.surface_id = r.surf;
                h.excitation = r.type;
                h.mode = 0;
                h._pad = 0;
                h.channel_id = r.ch_id;
                a.hit_stage[idx] = h;
                a.hit_key[idx] = r.ev;
            }
        }
    }
    if (err) atomicOr(a.err, err);
}

FCLat make_fclat(const Lattice& L, const float* cdf_f, const Detector& D) {
    FCLat f{};
    for (int v = 0; v < CMPMC_MAX_VALLEYS && v < L.n_valleys; ++v)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) f.rot[v][3 * i + j] = static_cast<float>(L.valley_rot[v].m[i][j]);
    f.hv_sqrt = F3{static_cast<float>(L.hv_sqrt.x), static_cast<float>(L.hv_sqrt.y), static_cast<float>(L.hv_sqrt.z)};
    f.hv_sqrt_inv = F3{static_cast<float>(L.hv_sqrt_inv.x), static_cast<float>(L.hv_sqrt_inv.y),
                       static_cast<float>(L.hv_sqrt_inv.z)};
    f.inv_mass_ratio = F3{static_cast<float>(1.0 / L.mass_ratio.x), static_cast<float>(1.0 / L.mass_ratio.y),
                          static_cast<float>(1.0 / L.mass_ratio.z)};
    f.m_e = static_cast<float>(L.e_cond_mass);
    f.m_h = static_cast<float>(L.h_mass);
    f.ks_e = static_cast<float>(L.k_sound_e);
    f.ks_h = static_cast<float>(L.k_sound_h);
    f.tstep_e = static_cast<float>((3.0 * L.l0_e) / L.v_sound);
    f.tstep_h = static_cast<float>((3.0 * L.l0_h) / L.v_sound);
    f.vs_hbar = static_cast<float>(L.v_sound * kHbar);
    f.hv_max = static_cast<float>(hv_max_scale(L));
    f.n_valleys = L.n_valleys;
    f.iv_model = L.iv_model;
    f.iv_min = static_cast<float>(L.iv_min_energy);
    f.iv_qrate = static_cast<float>(L.iv_quad_rate);
    f.iv_qfield = static_cast<float>(L.iv_quad_field);
    f.iv_qpow_half = static_cast<float>(0.5 * L.iv_quad_power);
    f.iv_lrate0 = static_cast<float>(L.iv_lin_rate0);
    f.iv_lrate1 = static_cast<float>(L.iv_lin_rate1);
    f.iv_lpow = static_cast<float>(L.iv_lin_power);
    auto inv = [](double mfp) { return (mfp > 0.0 && mfp < 1e20) ? static_cast<float>(1.0 / mfp) : 0.0f; };
    f.inv_trap_e = inv(L.e_trap_mfp);
    f.inv_trap_h = inv(L.h_trap_mfp);
    f.inv_ion_e_d0 = inv(L.e_ion_d0_mfp);
    f.inv_ion_e_a = inv(L.e_ion_a_mfp);
    f.inv_ion_h_d = inv(L.h_ion_d_mfp);
    f.inv_ion_h_a0 = inv(L.h_ion_a0_mfp);
    f.fL = static_cast<float>(L.fLDOS);
    f.fLST = static_cast<float>(L.fLDOS + L.fSTDOS);
    f.bandgap = static_cast<float>(L.bandgap);
    f.bandgap_d = L.bandgap;
    (void)cdf_f;
    (void)D;
    return f;
}

FCDet make_fcdet(const Detector& D, const MeshView32& mesh, const Lattice& L) {
    FCDet f{};
    f.R = static_cast<float>(D.radius);
    f.H = static_cast<float>(D.half_z);
    f.e_field = F3{static_cast<float>(D.e_field.x), static_cast<float>(D.e_field.y), static_cast<float>(D.e_field.z)};
    for (int i = 0; i < 3; ++i) {
        f.surf[i].prob_abs = static_cast<float>(D.surf[i].prob_charge_abs);
        f.surf[i].prob_spec = static_cast<float>(D.surf[i].prob_charge_spec);
        f.surf[i].min_k_e = static_cast<float>(D.surf[i].min_k_elec);
        f.surf[i].min_k_h = static_cast<float>(D.surf[i].min_k_hole);
        f.surf[i].n_pads = D.surf[i].n_pads;
        f.surf[i].pads = D.surf[i].pads;
        f.surf[i].release = (D.charge_release == 1 || (D.charge_release == 2 && D.surf[i].has_film)) ? 1 : 0;
    }
    f.dt_cap = static_cast<float>(D.charge_dt_cap_s);
    const bool second = (D.charge_stepping == 1);
    f.dk_frac = static_cast<float>(second ? D.charge_sampling_dk_frac : D.charge_max_dk_frac);
    f.second = second ? 1 : 0;
    const double lp = dclamp(D.luke_sample_fraction, 0.0, 1.0);
    f.luke_prob = static_cast<float>(lp);
    f.luke_wt = (lp > 0.0) ? static_cast<float>(1.0 / lp) : 0.0f;
    f.muF = (D.fermi_level_above_Ev_eV >= 0.0) ? D.fermi_level_above_Ev_eV : 0.5 * L.bandgap;
    f.mesh = mesh;
    f.mesh2 = D.mesh2_32;
    return f;
}

}  // namespace

cudaError_t launch_charges_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const ChargeArgs& c, int grid, int block, cudaStream_t s) {
    k_charges_fp32<<<grid, block, 0, s>>>(make_fclat(L, cdf_f, D), make_fcdet(D, D.mesh32, L), a, c);
    return cudaGetLastError();
}

cudaError_t charges_fp32_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_charges_fp32, block, 0);
}

cudaError_t launch_release_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const ChargeArgs& c, uint64_t n_rel, int grid, int block, cudaStream_t s) {
    const FLat f = make_flat(L, cdf_f, D);
    if (L.kin_mode != kKinOctahedral)
        k_release_fp32<1><<<grid, block, 0, s>>>(f, D, a, c, c.rel, n_rel, L.debye_energy);
    else
        k_release_fp32<0><<<grid, block, 0, s>>>(f, D, a, c, c.rel, n_rel, L.debye_energy);
    return cudaGetLastError();
}

cudaError_t launch_carrier_event(const uint64_t* ch_off, uint64_t n_events, uint32_t* carrier_event,
                                 cudaStream_t s) {
    k_carrier_event<<<4 * 148, 128, 0, s>>>(ch_off, n_events, carrier_event);
    return cudaGetLastError();
}

}  // namespace cmpmc_gpu
