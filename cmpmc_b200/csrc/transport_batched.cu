// transport_batched.cu -- the batched FP32 form: one device thread per primary track.
//
// The plain form keeps each event's single random stream, so an event's tracks run one
// after another on one thread. Here every primary phonon owns its own random substream
// (xoshiro128**, seeded from (run seed, event << 20 | index within the event)), so all
// primaries of a batch run concurrently and the result does not depend on how the device
// schedules them. A thread transports its primary and every daughter of it (decay, film
// re-emission, surface down-conversion) from a per-thread LIFO in global memory.
//
// The physics follows SimulationEngine::transport (transport/engine.hpp:403-582); the draw
// order differs (each substream is private, so any order of independent draws samples
// the same distributions). The step is arranged so the lanes of a warp stay converged:
// bulk scatter (isotropic) and diffuse reflection (Lambertian about the inward normal)
// share one direction-sampling and table-lookup path; decays, film entries, specular and
// down-converting reflections are the rare branches, and the Kaplan cascade is an
// out-of-line call so the step loop keeps few registers.
//
// Precision: position, directions, group velocity, the octahedral table blend, rates and
// sampling are FP32; the phonon energy, time of flight and the energy ledger are FP64, as
// is the Kaplan film cascade (so the ledger closes to rounding). A reflected track is
// moved 10 nm inward (the reference moves it 1e-11 m, below FP32 resolution at the wall).
#define CMPMC_DEVICE_FAST_MATH 1
#include <type_traits>

#include "device.cuh"
#include "fp32.cuh"

namespace cmpmc_gpu {

namespace {

struct FTrack {
    F3 pos, k, vg;
    float vmag;
    double E, t;
    float w;
    uint32_t bounces;
    int mode;
};

// A track of the adjoint kernel also carries its score: the derivative of the log density
// of every random decision of its lineage so far with respect to log theta_k (k = isotope
// coefficient, anharmonic coefficient, diffuse fraction, film absorption). It is summed in
// FP64: a long lineage adds thousands of free-flight terms.
struct FTrackA : FTrack {
    double s[4];
};

template <bool kAdj>
using TrackOf = typename std::conditional<kAdj, FTrackA, FTrack>::type;

struct alignas(16) GFTrack {
    float px, py, pz, kx, ky, kz, vx, vy, vz, vmag, w;
    uint32_t bounces_mode;  // bounces << 2 | mode
    double E, t;
};
struct alignas(16) GFTrackA {
    GFTrack g;
    double s[4];
};
template <bool kAdj>
using EntryOf = typename std::conditional<kAdj, GFTrackA, GFTrack>::type;

// a daughter starts with its parent's score (the decisions that made it)
template <bool kAdj>
__device__ __forceinline__ void inherit(TrackOf<kAdj>& d, const TrackOf<kAdj>& parent) {
    if constexpr (kAdj) {
#pragma unroll
        for (int i = 0; i < 4; ++i) d.s[i] = parent.s[i];
    }
}

template <bool kAdj>
__device__ __forceinline__ void push_track(EntryOf<kAdj>* stk, uint32_t& n, uint32_t cap, unsigned& err,
                                           const TrackOf<kAdj>& t) {
    if (n >= cap) {
        err |= kErrPhononStack;
        return;
    }
    GFTrack g;
    g.px = t.pos.x; g.py = t.pos.y; g.pz = t.pos.z;
    g.kx = t.k.x; g.ky = t.k.y; g.kz = t.k.z;
    g.vx = t.vg.x; g.vy = t.vg.y; g.vz = t.vg.z;
    g.vmag = t.vmag;
    g.w = t.w;
    g.bounces_mode = (t.bounces << 2) | static_cast<uint32_t>(t.mode);
    g.E = t.E;
    g.t = t.t;
    if constexpr (kAdj) {
        GFTrackA e;
        e.g = g;
        for (int i = 0; i < 4; ++i) e.s[i] = t.s[i];
        stk[n++] = e;
    } else {
        stk[n++] = g;
    }
}
template <bool kAdj>
__device__ __forceinline__ void pop_track(const EntryOf<kAdj>* stk, uint32_t& n, TrackOf<kAdj>& t) {
    --n;
    GFTrack g;
    if constexpr (kAdj) {
        const GFTrackA e = stk[n];
        g = e.g;
        for (int i = 0; i < 4; ++i) t.s[i] = e.s[i];
    } else {
        g = stk[n];
    }
    t.pos = f3(g.px, g.py, g.pz);
    t.k = f3(g.kx, g.ky, g.kz);
    t.vg = f3(g.vx, g.vy, g.vz);
    t.vmag = g.vmag;
    t.w = g.w;
    t.bounces = g.bounces_mode >> 2;
    t.mode = static_cast<int>(g.bounces_mode & 3u);
    t.E = g.E;
    t.t = g.t;
}

// Per-unit counters of a thread (a primary's lineage stays far below 2^32 steps). They
// live in shared memory, one structure of arrays per block (counter c of thread t at
// [c][t]: consecutive threads hit consecutive banks), so the step loop's registers hold
// the track state instead of spilling it.
constexpr int kMaxBlock = 128;  // every kernel running the step loop has __launch_bounds__(128)
enum { kCSteps = 0, kCIso, kCPoly, kCTT, kCLT, kCRefl, kCDown, kCHits, kCKilled, kNCnt };
template <int kStride>
struct UStatsT {
    uint32_t* c;  // &counters[0][thread]: counter i at c[i * kStride]
    double* f;    // &ledger[0][thread]: deposited, then escaped or killed
    __device__ __forceinline__ uint32_t& at(int i) const { return c[i * kStride]; }
    __device__ __forceinline__ uint32_t& steps() const { return at(kCSteps); }
    __device__ __forceinline__ uint32_t& iso() const { return at(kCIso); }
    __device__ __forceinline__ uint32_t& poly() const { return at(kCPoly); }
    __device__ __forceinline__ uint32_t& tt() const { return at(kCTT); }
    __device__ __forceinline__ uint32_t& lt() const { return at(kCLT); }
    __device__ __forceinline__ uint32_t& refl() const { return at(kCRefl); }
    __device__ __forceinline__ uint32_t& down() const { return at(kCDown); }
    __device__ __forceinline__ uint32_t& hits() const { return at(kCHits); }
    __device__ __forceinline__ uint32_t& killed() const { return at(kCKilled); }
    __device__ __forceinline__ double& dep() const { return f[0]; }
    __device__ __forceinline__ double& esc() const { return f[kStride]; }
    __device__ __forceinline__ void clear() const {
#pragma unroll
        for (int i = 0; i < kNCnt; ++i) at(i) = 0;
        dep() = 0.0;
        esc() = 0.0;
    }
};
using UStats = UStatsT<kMaxBlock>;

// Kaplan cascade out of line: its FP64 registers stay out of the step loop
__device__ __noinline__ double kaplan_call(const Film* f, double E, double* refl, int* n_refl, double* work,
                                           R128* g) {
    KBuf r{refl, 0};
    const double edep = film_absorb_phonon(*f, E, r, work, *g);
    *n_refl = r.n;
    return edep;
}

// the pair-breaking cascade of a film entry whose entry step was drawn in line (film_quick)
__device__ __noinline__ double kaplan_cascade_call(const Film* f, double E, double* refl, int* n_refl, double* work,
                                                   R128* g) {
    KBuf r{refl, 0};
    const double edep = film_absorb_quantum(*f, E, r, work, *g, false, true);
    *n_refl = r.n;
    return edep;
}

// The entry step of KaplanFilm::absorb_quantum for a phonon seed (kaplan_film.hpp:106-120),
// drawn in line by the transport step: direct absorption (the whole energy deposited), or the
// phonon comes back out unchanged (sub-gap, or lost on its way in); only the rest needs the
// pair-breaking cascade. With the surrogate table (whose stored outcomes include the entry
// step) only sub-gap phonons are decided here: the table does not cover them. Inlined: as an
// out-of-line call in the boundary branch (which ~3 lanes of a warp take) it cost 8 % of the
// batch (198 -> 181 ms).
enum { kFilmAbsorbed = 0, kFilmReemit = 1, kFilmCascade = 2 };
template <bool kSur>
__device__ __forceinline__ int film_quick(const Film* f, double E, R128* g) {
    if (kSur && !film_is_subgap(*f, E)) return kFilmCascade;
    if (film_direct_absorption(*f, E, *g)) return kFilmAbsorbed;
    if (film_is_subgap(*f, E) || g->uniform() <= film_loss_probability(*f, E, 4.0)) return kFilmReemit;
    return kFilmCascade;
}

// a hit of the transport step (film absorbed in line): staged with its event as key, the
// slots reserved once per group of lanes that hit together
__device__ __forceinline__ void stage_hit(const RunArgs& a, uint32_t ev, const cmpmc_sensor_hit& h) {
    if (!a.keep_hits) return;
    atomicAdd(reinterpret_cast<unsigned long long*>(a.ev_nhits + ev), 1ull);
    const unsigned grp = __activemask();
    const int leader = __ffs(grp) - 1;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(a.hit_count, static_cast<unsigned long long>(__popc(grp)));
    base = __shfl_sync(grp, base, leader);
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    const unsigned long long idx = base + __popc(grp & lt);
    if (idx < a.hit_cap) {
        a.hit_stage[idx] = h;
        a.hit_key[idx] = ev;
    }
}

// electrode mask lookup out of line: the sector test's atan2 stays out of the step loop's
// instruction stream
__device__ __noinline__ int mask_call(const Pad* pads, int n_pads, float x, float y, R128* g) {
    return find_channel(pads, n_pads, static_cast<double>(x), static_cast<double>(y), *g);
}

// IsotropicAMMInterface::transmission out of line (the complex boundary solve is rare)
__device__ __noinline__ float amm_call(const Surface* s, bool longitudinal, float cos_theta) {
    return static_cast<float>(amm_transmission(s->amm_sub, s->amm_film, longitudinal, static_cast<double>(cos_theta)));
}

// KaplanSurrogateLUT::absorb_phonon_fast (kaplan_film.hpp:361-374): one stored cascade
// outcome of a bracketing energy node, rescaled; the full cascade outside the table
__device__ __noinline__ double surrogate_call(const Surface* s, double E, double* refl, int* n_refl, double* work,
                                              R128* g) {
    const double two_delta = 2.0 * dmax(s->film.gap_energy, 1e-12);
    const double u = (E / two_delta - 1.0) / (20.0 - 1.0) * 127.0;
    if (film_is_subgap(s->film, E) || u < 0.0 || u > 127.0) return kaplan_call(&s->film, E, refl, n_refl, work, g);
    int ie = min(static_cast<int>(u), 126);
    if (g->uniform() < (u - ie)) ++ie;
    const int k = ie * 512 + min(511, static_cast<int>(g->uniform() * 512.0));
    const uint32_t r0 = __ldg(s->lut_off + k), r1 = __ldg(s->lut_off + k + 1);
    const int n = min(static_cast<int>(r1 - r0), kKaplanCap);
    for (int i = 0; i < n; ++i) refl[i] = E * static_cast<double>(__ldg(s->lut_refl + r0 + i));
    *n_refl = n;
    return E * static_cast<double>(__ldg(s->lut_abs + k));
}

// anharmonic decay of an L phonon (engine.hpp:938-988), FP32 angles
template <bool kAdj, int kKin = 0>
__device__ __noinline__ void decay_call(const FLat* Lp, TrackOf<kAdj>* tp, EntryOf<kAdj>* stk, uint32_t* n_stk,
                                        uint32_t cap, unsigned* err, const UStats* st, R128* gp) {
    const FLat& L = *Lp;
    TrackOf<kAdj>& trk = *tp;
    R128& g = *gp;
    const F3 d1 = trk.k;
    const F3 perp = forth(d1);
    float sp, cp;
    __sincosf(kTwoPiF * g.u(), &sp, &cp);
    float x, th1, th2;
    int m1, m2;
    const float m = L.m_ratio, mm = m * m;
    if (g.u() < L.fTT) {
        ++st->tt();
        x = fcdf(L.cdf_tt, g);
        const float y = 1.0f - x;
        th1 = facos_clamped((1.0f - mm * y * y + mm * x * x) / (2.0f * m * x));
        th2 = facos_clamped((1.0f - mm * x * x + mm * y * y) / (2.0f * m * y));
        m1 = ftrans(L, g);
        m2 = ftrans(L, g);
    } else {
        ++st->lt();
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
    TrackOf<kAdj> d;
    d.pos = trk.pos;
    d.k = k2;
    const FKin kin2 = fmapk<kKin>(L, m2, k2);
    d.vg = kin2.dir;
    d.vmag = kin2.mag;
    d.E = (1.0 - xd) * trk.E;
    d.t = trk.t;
    d.w = trk.w;
    d.bounces = 0;
    d.mode = m2;
    inherit<kAdj>(d, trk);
    push_track<kAdj>(stk, *n_stk, cap, *err, d);
    trk.E = xd * trk.E;
    trk.mode = m1;
    trk.k = k1;
    const FKin kin = fmapk<kKin>(L, m1, k1);
    trk.vg = kin.dir;
    trk.vmag = kin.mag;
}

__global__ void __launch_bounds__(128) k_unit_event(const uint64_t* __restrict__ ph_off, uint64_t n_events,
                                                    uint32_t* __restrict__ unit_event) {
    for (uint64_t ev = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; ev < n_events;
         ev += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        for (uint64_t j = ph_off[ev]; j < ph_off[ev + 1]; ++j) unit_event[j] = static_cast<uint32_t>(ev);
}

__device__ __forceinline__ void write_unit(const RunArgs& a, uint64_t unit, const UStats& st, uint32_t n_hits) {
    cmpmc_sim_stats& o = a.ev_stats[unit];
    o.total_steps = st.steps();
    o.isotope_scatters = st.iso();
    o.polycrystal_scatters = st.poly();
    o.decays_L_to_TT = st.tt();
    o.decays_L_to_LT = st.lt();
    o.surface_refls = st.refl();
    o.surface_downconversions = st.down();
    o.sensor_hits = st.hits();
    o.killed_tracks = st.killed();
    o.charge_steps = 0; o.luke_phonons_emitted = 0; o.intervalley_scatters = 0; o.charges_trapped = 0;
    o.trap_ionizations = 0; o.charge_surface_refls = 0; o.charges_collected = 0;
    o.total_luke_phonon_eV = 0.0; o.charge_recomb_edep_eV = 0.0;
    o.sc_pair_breakings = 0; o.qp_diffusion_steps = 0; o.qp_phonons_radiated = 0; o.qp_recombinations = 0;
    o.qp_local_traps = 0;
    o.total_injected_eV = 0.0;
    o.total_deposited_eV = st.dep();
    o.escaped_or_killed_eV = st.esc();
    a.ev_nhits[unit] = a.keep_hits ? n_hits : 0;
}

// event sink: a finished unit adds its counters to its event (units of one event run on
// many threads; the doubles are FP64 atomics, so their last bits depend on the order).
// Inlined: out of line it cost the SM-phase pool 5 % of the batch (181 -> 172 ms).
__device__ __forceinline__ void add_u64(unsigned long long* p, uint32_t v) {
    if (v) atomicAdd(p, static_cast<unsigned long long>(v));
}
__device__ __forceinline__ void add_f64(double* p, double v) {
    if (v != 0.0) atomicAdd(p, v);
}
template <class ST>
__device__ __forceinline__ void sink_unit(const RunArgs* a, uint32_t ev, const ST st) {
    cmpmc_sim_stats& o = a->ev_stats[ev];
    add_u64(reinterpret_cast<unsigned long long*>(&o.total_steps), st.steps());
    add_u64(reinterpret_cast<unsigned long long*>(&o.isotope_scatters), st.iso());
    add_u64(reinterpret_cast<unsigned long long*>(&o.polycrystal_scatters), st.poly());
    add_u64(reinterpret_cast<unsigned long long*>(&o.decays_L_to_TT), st.tt());
    add_u64(reinterpret_cast<unsigned long long*>(&o.decays_L_to_LT), st.lt());
    add_u64(reinterpret_cast<unsigned long long*>(&o.surface_refls), st.refl());
    add_u64(reinterpret_cast<unsigned long long*>(&o.surface_downconversions), st.down());
    add_u64(reinterpret_cast<unsigned long long*>(&o.sensor_hits), st.hits());
    add_u64(reinterpret_cast<unsigned long long*>(&o.killed_tracks), st.killed());
    add_f64(&o.total_deposited_eV, st.dep());
    add_f64(&o.escaped_or_killed_eV, st.esc());
}

enum { kSrcInput = 0, kSrcQueue = 1 };

// The step loop of both batched kernels. kAdj adds the score bookkeeping of the adjoint
// (every decision's d log p / d log theta, carried per track and inherited by daughters)
// and bins hits into the time histogram instead of writing hit records.
// kSrc selects where units come from: the caller's primary phonon records (kSrcInput,
// substream (event << 20 | index)) or the Luke-phonon queue of the charge form
// (kSrcQueue, the entry's own substream key; empty slots are skipped).
// kSink: units add to per-event sinks (runs with charges, wavefront split); kSur: film
// cascades from the surrogate tables; kSplit: a track that enters a film is queued for the
// film kernel and ends here (wavefront split). All are compile-time, so the default kernel
// carries none of their branches.
template <bool kAdj, int kSrc = kSrcInput, bool kSink = false, bool kSur = false, bool kSplit = false,
          int kKin = 0>
__device__ __forceinline__ void batched_loop(const FLat& L, const Detector& D, const RunArgs& a,
                                             const uint32_t* __restrict__ unit_event,
                                             const QPhonon* __restrict__ queue, const AdjArgs& adj,
                                             float* s_w, float* s_hist) {
    const uint64_t slot = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    EntryOf<kAdj>* stk = reinterpret_cast<EntryOf<kAdj>*>(a.stack) + slot * a.stack_cap;
    uint32_t n_stk = 0;
    unsigned err = 0;
    const float R = static_cast<float>(D.radius), H = static_cast<float>(D.half_z);
    const double min_E = D.min_phonon_eV;
    const uint64_t seed_key = mix64(a.seed ^ 0x5851f42d4c957f2dULL);

    TrackOf<kAdj> trk;
    R128 g;
    __shared__ uint32_t s_cnt[kNCnt][kMaxBlock];
    __shared__ double s_led[2][kMaxBlock];
    const UStats st{&s_cnt[0][threadIdx.x], &s_led[0][threadIdx.x]};
    uint32_t n_hits = 0;
    uint64_t unit = ~0ull;
    uint32_t ev_cur = 0;  // event of the unit in flight
    uint32_t n_phase = 0;  // steps of the track in flight in this phase (wavefront split)
    bool live = false;  // trk holds a track in flight
    for (;;) {
        if (!live) {
            n_phase = 0;
            if (n_stk > 0) {
                pop_track<kAdj>(stk, n_stk, trk);
                live = true;
            } else {
                if (unit != ~0ull) {
                    if constexpr (kSink) sink_unit(&a, ev_cur, st);
                    else write_unit(a, unit, st, n_hits);
                }
                unit = atomicAdd(a.next_work, 1ull);
                if (unit >= a.n_events) break;
                if constexpr (kSrc == kSrcQueue) {
                    const QPhonon q = queue[unit];
                    if (q.ev == kQEmpty) {
                        unit = ~0ull;
                        continue;
                    }
                    ev_cur = q.ev;
                    g.seed(q.key);
                    trk.pos = f3(q.px, q.py, q.pz);
                    trk.k = f3(q.kx, q.ky, q.kz);
                    trk.mode = static_cast<int>(q.mode);
                    const FKin kin = fmapk<kKin>(L, trk.mode, trk.k);
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                    trk.E = q.E;
                    trk.t = q.t;
                    trk.w = q.w;
                    trk.bounces = q.pad;
                    st.clear();
                    n_hits = 0;
                    live = true;
                    continue;
                }
                const uint32_t ev = unit_event[unit];
                ev_cur = ev;
                const uint64_t j = unit - a.ph_off[ev];
                g.seed(seed_key ^ mix64(((a.first_event + ev) << 20) | j));
                const cmpmc_phonon_track& in = a.ph[unit];
                trk.pos = f3(static_cast<float>(in.pos[0]), static_cast<float>(in.pos[1]),
                             static_cast<float>(in.pos[2]));
                trk.k = f3(static_cast<float>(in.k_dir[0]), static_cast<float>(in.k_dir[1]),
                           static_cast<float>(in.k_dir[2]));
                trk.vg = f3(static_cast<float>(in.vg_dir[0]), static_cast<float>(in.vg_dir[1]),
                            static_cast<float>(in.vg_dir[2]));
                trk.vmag = static_cast<float>(in.vg_mag);
                trk.E = in.energy;
                trk.t = in.time;
                trk.w = static_cast<float>(in.weight);
                trk.bounces = in.bounces;
                trk.mode = in.mode;
                if constexpr (kAdj) {
                    trk.s[0] = trk.s[1] = trk.s[2] = trk.s[3] = 0.0;
                    double* row = adj.prim + unit * kAdjCols;
#pragma unroll
                    for (int c = 0; c < kAdjCols; ++c) row[c] = 0.0;
                }
                st.clear();
                n_hits = 0;
                live = true;
            }
        }
        if (trk.E < min_E || trk.bounces >= D.max_bounces) {
            ++st.killed();
            st.esc() += trk.E * trk.w;
            live = false;
            continue;
        }
        if (D.rr_bounces != 0 && trk.bounces > D.rr_bounces && (trk.bounces - D.rr_bounces) % 32 == 0) {
            if (g.u() < static_cast<float>(D.rr_survival)) {
                trk.w /= static_cast<float>(D.rr_survival);
            } else {
                ++st.killed();
                live = false;
                continue;
            }
        }
        if constexpr (kSplit) {
            if (a.phase_steps && ++n_phase > a.phase_steps) {
                // park the track for the next phase on a substream derived from its own
                const unsigned long long slot = atomicAdd(a.reemit_tail, 1ull);
                if (slot < a.reemit_cap) {
                    QPhonon q;
                    q.px = trk.pos.x; q.py = trk.pos.y; q.pz = trk.pos.z;
                    q.kx = trk.k.x; q.ky = trk.k.y; q.kz = trk.k.z;
                    q.w = trk.w;
                    q.mode = static_cast<uint32_t>(trk.mode);
                    q.E = trk.E;
                    q.t = trk.t;
                    const uint64_t hi = g.next();
                    q.key = (hi << 32) | g.next();
                    q.ev = ev_cur;
                    q.pad = trk.bounces;
                    a.reemit[slot] = q;
                } else {
                    err |= kErrQueue;
                }
                live = false;
                continue;
            }
        }
        ++st.steps();
        const float nu = static_cast<float>(trk.E) * L.inv_h_thz;
        const float nu2 = nu * nu;
        const float r_iso = L.b4 * (nu2 * nu2);
        const float r_poly = trk.vmag * L.poly_inv;
        const float r_down = (trk.mode == 0) ? L.a5 * (nu2 * nu2 * nu) : 0.0f;
        const float r_tot = r_iso + r_poly + r_down;
        const float d_phys = (r_tot > 1e-12f) ? (-logf(g.u()) * trk.vmag / r_tot) : __int_as_float(0x7f800000);
        FBHit bh = fexit_d(R, H, trk.pos, trk.vg);
        const bool bulk = d_phys < bh.d;
        const float d = bulk ? d_phys : bh.d;
        trk.pos = trk.pos + trk.vg * d;
        trk.t += static_cast<double>(d / trk.vmag);
        if constexpr (kAdj) {
            // free flight: survival exp(-r t) of each theta-dependent channel over the segment
            const float seg = d / trk.vmag;
            trk.s[0] -= static_cast<double>(r_iso * seg);
            trk.s[1] -= static_cast<double>(r_down * seg);
        }
        // 0: new isotropic direction (bulk scatter), 1: Lambertian about bh.n, 2: nothing more
        int sample = 2;
        if (bulk) {
            const float u_proc = g.u() * r_tot;
            if (r_down > 0.0f && u_proc < r_down) {
                if constexpr (kAdj) trk.s[1] += 1.0f;  // density of a decay: r_down exp(-r_tot t)
                // the out-of-line call works on copies: only they have their address
                // taken, so the loop's own track and generator stay in registers
                TrackOf<kAdj> t_c = trk;
                R128 g_c = g;
                uint32_t n_c = n_stk;
                unsigned e_c = err;
                decay_call<kAdj, kKin>(&L, &t_c, stk, &n_c, a.stack_cap, &e_c, &st, &g_c);
                trk = t_c;
                g = g_c;
                n_stk = n_c;
                err = e_c;
            } else {
                if (u_proc < r_down + r_iso) {
                    ++st.iso();
                    if constexpr (kAdj) trk.s[0] += 1.0f;
                } else {
                    ++st.poly();
                }
                trk.mode = fdos(L, g.u());
                sample = 0;
            }
        } else {
            bh.n = fnormal(bh.surf, trk.pos);  // trk.pos is the hit point
            trk.bounces++;
            const Surface& s = D.surf[bh.surf];
            bool enter = false;
            int ch_id = -1;
            bool active_pad = true;
            if (s.n_pads > 0) {  // electrode mask (engine.hpp:483-488)
                R128 g_c = g;
                ch_id = mask_call(s.pads, s.n_pads, trk.pos.x, trk.pos.y, &g_c);
                g = g_c;
                active_pad = ch_id >= 0;
            }
            if (active_pad && s.has_film && g.u() < static_cast<float>(s.prob_abs)) {
                const float p_enter = s.has_amm ? amm_call(&s, trk.mode == 0, fdot(trk.k, bh.n))
                                                : static_cast<float>(s.film.film_absorption);
                enter = g.u() < p_enter;
                if constexpr (kAdj) trk.s[3] += enter ? 1.0f : adj.film_miss_score;
            }
            if constexpr (kSplit) {
                if (enter) {
                    // film entry: hand the phonon to the film kernel and end the track here
                    const unsigned long long slot = atomicAdd(a.film_tail, 1ull);
                    if (slot < a.film_cap) {
                        FilmRec r;
                        r.px = trk.pos.x; r.py = trk.pos.y; r.pz = trk.pos.z;
                        r.w = trk.w;
                        r.E = trk.E;
                        r.t = trk.t;
                        const uint64_t hi = g.next();
                        r.key = (hi << 32) | g.next();
                        r.ev = ev_cur;
                        r.ch_id = ch_id;
                        r.bounces = trk.bounces;
                        r.surf = static_cast<uint8_t>(bh.surf);
                        r.mode = static_cast<uint8_t>(trk.mode);
                        r.pad0 = r.pad1 = 0;
                        a.film[slot] = r;
                    } else {
                        err |= kErrFilmQueue;
                    }
                    live = false;
                    continue;
                }
            }
            if (enter) {
                int n_refl = 0;
                double edep;
                R128 g_c = g;
                if constexpr (kSur) {
                    edep = s.lut_abs ? surrogate_call(&s, trk.E, refl_buf, &n_refl, kwork, &g_c)
                                     : kaplan_call(&s.film, trk.E, refl_buf, &n_refl, kwork, &g_c);
                } else {
                    edep = kaplan_call(&s.film, trk.E, refl_buf, &n_refl, kwork, &g_c);
                }
                g = g_c;
                if (edep > 0.0) {
                    const double wedep = edep * trk.w;
                    ++st.hits();
                    st.dep() += wedep;
                    const uint32_t local = n_hits++;
                    if constexpr (kAdj) {
                        const double tb = (trk.t - adj.t0) * adj.inv_dt;
                        if (tb >= 0.0 && tb < static_cast<double>(adj.n_bins)) {
                            const int b = static_cast<int>(tb);
                            atomicAdd(s_hist + b, trk.w);
                            const double gw = static_cast<double>(s_w[b]) * trk.w;
                            if (gw != 0.0) {
                                double* row = adj.prim + unit * kAdjCols;
                                row[0] += gw;
#pragma unroll
                                for (int c = 0; c < 4; ++c) row[1 + c] += gw * trk.s[c] * adj.inv_theta[c];
                            }
                        }
                    } else if (a.keep_hits) {
                        if constexpr (kSink)
                            atomicAdd(reinterpret_cast<unsigned long long*>(a.ev_nhits + ev_cur), 1ull);
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
                            r.channel_id = ch_id;
                            a.hit_stage[idx] = r;
                            a.hit_key[idx] = kSink ? static_cast<uint64_t>(ev_cur) : ((unit << 32) | local);
                        }
                    }
                }
                double sum_refl = 0.0;
                for (int i = 0; i < n_refl; ++i) sum_refl += refl_buf[i];
                st.esc() += dmax(0.0, trk.E - edep - sum_refl) * trk.w;
                if (n_refl == 0) {
                    live = false;
                    continue;
                }
                const F3 re = trk.pos + bh.n * kNudge;
                for (int i = 1; i < n_refl; ++i) {
                    TrackOf<kAdj> dtr;
                    dtr.mode = fdos(L, g.u());
                    FKin kin;
                    dtr.k = finward<kKin>(L, dtr.mode, bh.n, g, kin);
                    dtr.pos = re;
                    dtr.vg = kin.dir;
                    dtr.vmag = kin.mag;
                    dtr.E = refl_buf[i];
                    dtr.t = trk.t;
                    dtr.w = trk.w;
                    dtr.bounces = 0;
                    inherit<kAdj>(dtr, trk);
                    push_track<kAdj>(stk, n_stk, a.stack_cap, err, dtr);
                }
                trk.pos = re;
                trk.E = refl_buf[0];
                trk.mode = fdos(L, g.u());
                sample = 1;
            } else if (g.u() > static_cast<float>(s.prob_refl)) {
                ++st.killed();
                st.esc() += trk.E * trk.w;
                live = false;
                continue;
            } else {
                ++st.refl();
                trk.pos = trk.pos + bh.n * kNudge;
                float p_anh, p_anh_spec;
                if (L.split_const[bh.surf]) {
                    p_anh = L.p_anh[bh.surf];
                    p_anh_spec = L.p_anh_spec[bh.surf];
                } else {
                    const Split sp = reflection_split(s, trk.E);
                    p_anh = static_cast<float>(sp.p_anh);
                    p_anh_spec = static_cast<float>(sp.p_anh + sp.p_spec);
                }
                const float u_refl = g.u();
                if (u_refl < p_anh) {
                    ++st.down();
                    const bool tt = g.u() < L.fTT;
                    const float x = tt ? fcdf(L.cdf_tt, g) : fcdf(L.cdf_lt, g);
                    const int m1 = tt ? ftrans(L, g) : 0;
                    const int m2 = ftrans(L, g);
                    TrackOf<kAdj> dtr;
                    FKin k2kin;
                    dtr.k = finward<kKin>(L, m2, bh.n, g, k2kin);
                    dtr.pos = trk.pos;
                    dtr.vg = k2kin.dir;
                    dtr.vmag = k2kin.mag;
                    dtr.E = (1.0 - static_cast<double>(x)) * trk.E;
                    dtr.t = trk.t;
                    dtr.w = trk.w;
                    dtr.bounces = 0;
                    dtr.mode = m2;
                    inherit<kAdj>(dtr, trk);
                    push_track<kAdj>(stk, n_stk, a.stack_cap, err, dtr);
                    trk.E = static_cast<double>(x) * trk.E;
                    trk.mode = m1;
                    sample = 1;
                } else if (u_refl < p_anh_spec) {
                    if constexpr (kAdj) trk.s[2] += adj.spec_score;  // d log(1 - p_d) / d log p_d
                    F3 kr = trk.k - bh.n * (2.0f * fdot(trk.k, bh.n));
                    FKin kin = fmapk<kKin>(L, trk.mode, kr);
                    if (fdot(kin.dir, bh.n) <= 1e-6f) kr = finward<kKin>(L, trk.mode, bh.n, g, kin);
                    trk.k = kr;
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                } else {
                    if constexpr (kAdj) trk.s[2] += 1.0f;  // d log p_d / d log p_d
                    sample = 1;
                }
            }
        }
        // shared new-direction path: isotropic (bulk scatter) or Lambertian about the
        // inward normal (diffuse reflection / re-emission), then the table lookup
        if (sample != 2) {
            const bool lam = (sample == 1);
            const F3 e3 = lam ? bh.n : f3(0.0f, 0.0f, 1.0f);
            const F3 e1 = lam ? forth(bh.n) : f3(1.0f, 0.0f, 0.0f);
            const F3 e2 = lam ? fcross(bh.n, e1) : f3(0.0f, 1.0f, 0.0f);
            FKin kin;
            F3 kd;
            for (int trial = 0;; ++trial) {
                const float u1 = g.u();
                const float u2 = g.u();
                const float ct = lam ? sqrtf(u1) : 2.0f * u1 - 1.0f;  // Lambertian: cos theta = sqrt(u)
                const float st_ = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
                float sphi, cphi;
                __sincosf(kTwoPiF * u2, &sphi, &cphi);
                kd = e1 * (st_ * cphi) + e2 * (st_ * sphi) + e3 * ct;
                if (lam) kd = funit(kd);
                kin = fmapk<kKin>(L, trk.mode, kd);
                if (!lam || fdot(kin.dir, bh.n) > 1e-6f) break;
                if (trial == 15) {
                    kd = bh.n;
                    kin = fmapk<kKin>(L, trk.mode, kd);
                    break;
                }
            }
            trk.k = kd;
            trk.vg = kin.dir;
            trk.vmag = kin.mag;
        }
    }
    if (err) atomicOr(a.err, err);
}

template <bool kSink, bool kSur, bool kSplit = false, int kKin = 0>
__global__ void __launch_bounds__(128, 6) k_batched_fp32(const __grid_constant__ FLat L,
                                                         const __grid_constant__ Detector D,
                                                         const __grid_constant__ RunArgs a,
                                                         const uint32_t* __restrict__ unit_event) {
    const AdjArgs none{};
    batched_loop<false, kSrcInput, kSink, kSur, kSplit, kKin>(L, D, a, unit_event, nullptr, none, nullptr, nullptr);
}

// A phonon queue (Luke phonons, film re-emissions): one unit per queue entry
template <bool kSur, bool kSplit = false, int kKin = 0>
__global__ void __launch_bounds__(128, 6) k_queue_fp32(const __grid_constant__ FLat L,
                                                       const __grid_constant__ Detector D,
                                                       const __grid_constant__ RunArgs a,
                                                       const QPhonon* __restrict__ queue) {
    const AdjArgs none{};
    batched_loop<false, kSrcQueue, true, kSur, kSplit, kKin>(L, D, a, nullptr, queue, none, nullptr, nullptr);
}

// The film kernel of the wavefront split: one queued film entry per thread. It runs the
// Kaplan cascade (or the surrogate lookup) from the entry's own substream, records the hit
// and the ledger in the entry's event, and queues the re-emitted phonons, each inward
// Lambertian with a DOS mode and its own substream (the first keeps the bounce count).
template <bool kSur, int kKin = 0>
__global__ void __launch_bounds__(128, 8) k_film_fp32(const __grid_constant__ FLat L,
                                                      const __grid_constant__ Detector D,
                                                      const __grid_constant__ RunArgs a,
                                                      const FilmRec* __restrict__ film, uint64_t n_film) {
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    unsigned err = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n_film;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const FilmRec r = film[i];
        const Surface& s = D.surf[r.surf];
        R128 g;
        int n_refl = 0;
        double edep;
        {
            R128 g_c;  // the only generator whose address is taken (see the step loop)
            g_c.seed(r.key);
            if constexpr (kSur) {
                edep = s.lut_abs ? surrogate_call(&s, r.E, refl_buf, &n_refl, kwork, &g_c)
                                 : kaplan_call(&s.film, r.E, refl_buf, &n_refl, kwork, &g_c);
            } else {
                edep = kaplan_call(&s.film, r.E, refl_buf, &n_refl, kwork, &g_c);
            }
            g = g_c;
        }
        cmpmc_sim_stats& o = a.ev_stats[r.ev];
        if (edep > 0.0) {
            const double wedep = edep * static_cast<double>(r.w);
            atomicAdd(reinterpret_cast<unsigned long long*>(&o.sensor_hits), 1ull);
            atomicAdd(&o.total_deposited_eV, wedep);
            if (a.keep_hits) {
                atomicAdd(reinterpret_cast<unsigned long long*>(a.ev_nhits + r.ev), 1ull);
                const unsigned long long idx = atomicAdd(a.hit_count, 1ull);
                if (idx < a.hit_cap) {
                    cmpmc_sensor_hit h;
                    h.pos[0] = r.px; h.pos[1] = r.py; h.pos[2] = r.pz;
                    h.time = r.t;
                    h.edep = wedep;
                    h.incident_energy = r.E;
                    h.surface_id = r.surf;
                    h.excitation = 0;
                    h.mode = r.mode;
                    h._pad = 0;
                    h.channel_id = r.ch_id;
                    a.hit_stage[idx] = h;
                    a.hit_key[idx] = r.ev;
                }
            }
        }
        double sum_refl = 0.0;
        for (int j = 0; j < n_refl; ++j) sum_refl += refl_buf[j];
        const double esc = dmax(0.0, r.E - edep - sum_refl) * static_cast<double>(r.w);
        if (esc != 0.0) atomicAdd(&o.escaped_or_killed_eV, esc);
        if (n_refl == 0) continue;
        const unsigned long long base = atomicAdd(a.reemit_tail, static_cast<unsigned long long>(n_refl));
        if (base + n_refl > a.reemit_cap) {
            err |= kErrQueue;
            continue;
        }
        // inward normal of the face at the entry point (CylinderSolid, solids.hpp:46-93)
        F3 n;
        if (r.surf == 0) n = f3(0.0f, 0.0f, -1.0f);
        else if (r.surf == 1) n = f3(0.0f, 0.0f, 1.0f);
        else {
            const float rr = sqrtf(r.px * r.px + r.py * r.py);
            n = (rr > 1e-15f) ? f3(-r.px / rr, -r.py / rr, 0.0f) : f3(-1.0f, 0.0f, 0.0f);
        }
        const F3 re = f3(r.px, r.py, r.pz) + n * kNudge;
        for (int j = 0; j < n_refl; ++j) {
            const int mode = fdos(L, g.u());
            FKin kin;
            const F3 k = finward<kKin>(L, mode, n, g, kin);
            QPhonon q;
            q.px = re.x; q.py = re.y; q.pz = re.z;
            q.kx = k.x; q.ky = k.y; q.kz = k.z;
            q.w = r.w;
            q.mode = static_cast<uint32_t>(mode);
            q.E = refl_buf[j];
            q.t = r.t;
            q.key = mix64(r.key ^ (0x9e3779b97f4a7c15ULL * static_cast<uint64_t>(j + 1)));
            q.ev = r.ev;
            q.pad = (j == 0) ? r.bounces : 0u;
            a.reemit[base + j] = q;
        }
    }
    if (err) atomicOr(a.err, err);
}

// ---- shared-memory staging of the small tables by the TMA engine -----------------------
// One thread issues an untiled bulk copy (cp.async.bulk global -> shared, no multicast, the
// source is this GPU's own memory) whose completion is counted on an mbarrier; every thread
// then waits on the barrier's first phase. The wait is bounded: a copy that has not landed
// after kStageSpins polls is reported (false) and the block must not touch the destination.
constexpr int kStageSpins = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// src and dst 16-byte aligned, bytes a multiple of 16; called by every thread of the block
__device__ __forceinline__ bool stage_bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    const uint32_t b = smem_addr(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(b),
                     "r"(bytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(dst)),
                     "l"(src), "r"(bytes), "r"(b)
                     : "memory");
    }
    __syncthreads();  // the barrier is initialised before anyone polls it
    auto landed = [b]() {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(b)
                     : "memory");
        return done != 0;
    };
    bool done = false;
    for (int i = 0; i < kStageSpins && !done; ++i) {
        done = landed();
        if (!done) __nanosleep(32);
    }
    // the block agrees on the outcome; a copy that is late is still waited for (bounded)
    // before the caller gives up, so no copy into this block's shared memory outlives it
    if (!__syncthreads_or(!done)) return true;
    for (int i = 0; i < kStageSpins && !done; ++i) {
        done = landed();
        if (!done) __nanosleep(32);
    }
    return false;
}

// inverse-CDF sample from a table in either memory space (plain loads: the staged copy
// lives in shared memory)
__device__ __forceinline__ float fcdf_any(const float* cdf, R128& g) {
    const float u = g.u() * (kNCdf - 1);
    const int i = min(static_cast<int>(u), kNCdf - 2);
    const float f = u - i;
    return cdf[i] * (1.0f - f) + cdf[i + 1] * f;
}

// ---- warp pool form -------------------------------------------------------------------
// One persistent launch transports the whole batch. Each warp owns a private ring of
// pending phonons (film re-emissions and daughters, with their group velocity, so a refill
// needs no table lookup) and a private buffer of film entries. Every iteration:
//   1. refill: the lanes without a track (one ballot) take the ring's oldest entries, then
//      the next primaries of the batch (one atomicAdd per warp for all of them);
//   2. step: every live lane takes one transport step;
//   3. regroup: the lanes whose step ended at an active film append a film record, the lanes
//      that made a daughter (decay, surface down-conversion) append it to the ring, each
//      class through one ballot and prefix count;
//   4. when 32 film entries are waiting, the whole warp runs one cascade per lane (the
//      film step, converged) and appends the re-emitted phonons to the ring.
// A warp ends when the batch's primaries are handed out and its ring, film buffer and lanes
// are empty. Work never moves between warps, so nothing waits on another warp (no spin, no
// grid barrier); the batch ends with one tail instead of one per film / transport round.
// Every unit (primary, ring phonon) has its own substream, so the hits of an event are a
// fixed set whatever the launch shape; units add to per-event sinks.
constexpr int kPoolFilmCap = 64;  // film records per warp (a batch of 32 runs when 32 wait)

struct alignas(16) PoolPh {  // 80 B
    float px, py, pz, kx, ky, kz, vx, vy, vz, vmag, w;
    uint32_t bounces_mode;  // bounces << 2 | mode
    double E, t;
    uint64_t key;
    uint32_t ev, pad;
};

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ PoolPh pool_entry(const FTrack& t, uint64_t key, uint32_t ev) {
    PoolPh q;
    q.px = t.pos.x; q.py = t.pos.y; q.pz = t.pos.z;
    q.kx = t.k.x; q.ky = t.k.y; q.kz = t.k.z;
    q.vx = t.vg.x; q.vy = t.vg.y; q.vz = t.vg.z;
    q.vmag = t.vmag;
    q.w = t.w;
    q.bounces_mode = (t.bounces << 2) | static_cast<uint32_t>(t.mode);
    q.E = t.E;
    q.t = t.t;
    q.key = key;
    q.ev = ev;
    q.pad = 0;
    return q;
}

__device__ __forceinline__ uint64_t draw_key(R128& g) {
    const uint64_t hi = g.next();
    return (hi << 32) | g.next();
}

// anharmonic decay of an L phonon (engine.hpp:938-988), FP32 angles: the parent continues
// in *tp, the daughter is written to *dp (it runs later on a substream of its own)
template <int kKin, class ST>
__device__ __noinline__ void pool_decay(const FLat* Lp, const float* cdf, FTrack* tp, FTrack* dp, const ST* st,
                                        R128* gp) {
    const FLat& L = *Lp;
    FTrack& trk = *tp;
    R128& g = *gp;
    const F3 d1 = trk.k;
    const F3 perp = forth(d1);
    float sp, cp;
    __sincosf(kTwoPiF * g.u(), &sp, &cp);
    float x, th1, th2;
    int m1, m2;
    const float m = L.m_ratio, mm = m * m;
    if (g.u() < L.fTT) {
        ++st->tt();
        x = fcdf_any(cdf + kNCdf, g);
        const float y = 1.0f - x;
        th1 = facos_clamped((1.0f - mm * y * y + mm * x * x) / (2.0f * m * x));
        th2 = facos_clamped((1.0f - mm * x * x + mm * y * y) / (2.0f * m * y));
        m1 = ftrans(L, g);
        m2 = ftrans(L, g);
    } else {
        ++st->lt();
        x = fcdf_any(cdf, g);
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
    FTrack& d = *dp;
    d.pos = trk.pos;
    d.k = k2;
    const FKin kin2 = fmapk<kKin>(L, m2, k2);
    d.vg = kin2.dir;
    d.vmag = kin2.mag;
    d.E = (1.0 - xd) * trk.E;
    d.t = trk.t;
    d.w = trk.w;
    d.bounces = 0;
    d.mode = m2;
    trk.E = xd * trk.E;
    trk.mode = m1;
    trk.k = k1;
    const FKin kin = fmapk<kKin>(L, m1, k1);
    trk.vg = kin.dir;
    trk.vmag = kin.mag;
}

enum { kStepOn = 0, kStepEnd = 1, kStepFilm = 2 };

// A step's single output record (a film entry or a daughter), staged in shared memory so
// that it holds no registers across the step; the warp copies it to its buffer afterwards.
union PoolOut {
    FilmRec film;
    PoolPh ph;
};
// output of the warp pool's step: the record goes to the thread's staging slot
// The per-surface constants of the boundary branch (staged in shared memory by every block
// that runs pool_step: the branch reads them by the surface a lane hit, which differs between
// lanes; read from the kernel parameters, each field would be a separate constant-bank load
// per distinct surface)
enum { kHotFilm = 1, kHotAmm = 2, kHotMask = 4, kHotSplitConst = 8 };
struct alignas(16) SurfHot {
    float prob_abs, p_enter, prob_refl, p_anh;  // p_enter: the film's film_absorption
    float p_anh_spec;                           // p_anh + p_spec (constant split)
    int flags;                                  // kHot*
    int pad0, pad1;
};
__device__ __forceinline__ SurfHot surf_hot(const FLat& L, const Surface& s, int i) {
    SurfHot h;
    h.prob_abs = static_cast<float>(s.prob_abs);
    h.p_enter = static_cast<float>(s.film.film_absorption);
    h.prob_refl = static_cast<float>(s.prob_refl);
    h.p_anh = L.p_anh[i];
    h.p_anh_spec = L.p_anh_spec[i];
    h.flags = (s.has_film ? kHotFilm : 0) | (s.has_amm ? kHotAmm : 0) | (s.n_pads > 0 ? kHotMask : 0) |
              (L.split_const[i] ? kHotSplitConst : 0);
    h.pad0 = h.pad1 = 0;
    return h;
}
// threads 0-2 of the block fill hot[3]; the caller synchronizes the block before use
__device__ __forceinline__ void stage_surf_hot(const FLat& L, const Detector& D, SurfHot* hot) {
    if (threadIdx.x < 3) hot[threadIdx.x] = surf_hot(L, D.surf[threadIdx.x], static_cast<int>(threadIdx.x));
}

struct WarpSink {
    PoolOut* o;
    bool has_d;
    const RunArgs* a;
    __device__ __forceinline__ void film(const FilmRec& r) { o->film = r; }
    __device__ __forceinline__ void hit(uint32_t ev, const cmpmc_sensor_hit& h) { stage_hit(*a, ev, h); }
    __device__ __forceinline__ void daughter(const PoolPh& q) {
        o->ph = q;
        has_d = true;
    }
};

// One transport step of a live track (the physics of batched_loop's step): returns whether
// the track goes on, ended (counters and ledger updated), or entered an active film (the
// film record handed to out.film). A daughter made in the step is handed to out.daughter
// with a substream key drawn from the track's stream.
// The step has no early return: every lane that entered meets the others again before the
// new-direction sampling, which the bulk scatters and the diffuse reflections of a warp then
// run together (with early returns in the boundary branch the two groups ran it one after
// the other).
template <int kKin, bool kSur, class ST, class Sink>
__device__ __forceinline__ int pool_step(const FLat& L, const float* cdf, const Detector& D, const SurfHot* hot,
                                         FTrack& trk, R128& g, const ST& st, uint32_t ev, Sink& out) {
    const unsigned m_in = __activemask();
    int outcome = kStepOn;
    int sample = 2;  // 0: isotropic (bulk scatter), 1: Lambertian about bh.n, 2: nothing more
    FBHit bh;
    if (trk.E < D.min_phonon_eV || trk.bounces >= D.max_bounces) {
        ++st.killed();
        st.esc() += trk.E * trk.w;
        outcome = kStepEnd;
    } else if (D.rr_bounces != 0 && trk.bounces > D.rr_bounces && (trk.bounces - D.rr_bounces) % 32 == 0) {
        if (g.u() < static_cast<float>(D.rr_survival)) {
            trk.w /= static_cast<float>(D.rr_survival);
        } else {
            ++st.killed();
            outcome = kStepEnd;
        }
    }
    if (outcome == kStepOn) {
        ++st.steps();
        const float R = static_cast<float>(D.radius), H = static_cast<float>(D.half_z);
        const float nu = static_cast<float>(trk.E) * L.inv_h_thz;
        const float nu2 = nu * nu;
        const float r_iso = L.b4 * (nu2 * nu2);
        const float r_poly = trk.vmag * L.poly_inv;
        const float r_down = (trk.mode == 0) ? L.a5 * (nu2 * nu2 * nu) : 0.0f;
        const float r_tot = r_iso + r_poly + r_down;
        const float d_phys = (r_tot > 1e-12f) ? (-logf(g.u()) * trk.vmag / r_tot) : __int_as_float(0x7f800000);
        bh = fexit_d(R, H, trk.pos, trk.vg);
        const bool bulk = d_phys < bh.d;
        const float d = bulk ? d_phys : bh.d;
        trk.pos = trk.pos + trk.vg * d;
        trk.t += static_cast<double>(d / trk.vmag);
        if (bulk) {
            const float u_proc = g.u() * r_tot;
            if (r_down > 0.0f && u_proc < r_down) {
                FTrack t_c = trk, d_c;
                R128 g_c = g;
                pool_decay<kKin>(&L, cdf, &t_c, &d_c, &st, &g_c);
                trk = t_c;
                g = g_c;
                out.daughter(pool_entry(d_c, draw_key(g), ev));
            } else {
                if (u_proc < r_down + r_iso) ++st.iso();
                else ++st.poly();
                trk.mode = fdos(L, g.u());
                sample = 0;
            }
        } else {
            bh.n = fnormal(bh.surf, trk.pos);
            trk.bounces++;
            const SurfHot hs = hot[bh.surf];
            const Surface& s = D.surf[bh.surf];  // read by the out-of-line calls only
            bool enter = false;
            int ch_id = -1;
            bool active_pad = true;
            if (hs.flags & kHotMask) {  // electrode mask (engine.hpp:483-488)
                R128 g_c = g;
                ch_id = mask_call(s.pads, s.n_pads, trk.pos.x, trk.pos.y, &g_c);
                g = g_c;
                active_pad = ch_id >= 0;
            }
            if (active_pad && (hs.flags & kHotFilm) && g.u() < hs.prob_abs) {
                const float p_enter =
                    (hs.flags & kHotAmm) ? amm_call(&s, trk.mode == 0, fdot(trk.k, bh.n)) : hs.p_enter;
                enter = g.u() < p_enter;
            }
            if (enter) {
                R128 g_c = g;
                const int film = film_quick<kSur>(&s.film, trk.E, &g_c);
                g = g_c;
                if (film == kFilmAbsorbed) {
                    const double wedep = trk.E * trk.w;
                    ++st.hits();
                    st.dep() += wedep;
                    cmpmc_sensor_hit h;
                    h.pos[0] = trk.pos.x; h.pos[1] = trk.pos.y; h.pos[2] = trk.pos.z;
                    h.time = trk.t;
                    h.edep = wedep;
                    h.incident_energy = trk.E;
                    h.surface_id = static_cast<uint8_t>(bh.surf);
                    h.excitation = 0;
                    h.mode = static_cast<uint8_t>(trk.mode);
                    h._pad = 0;
                    h.channel_id = ch_id;
                    out.hit(ev, h);
                    outcome = kStepEnd;
                } else if (film == kFilmCascade) {
                    FilmRec fr;
                    fr.px = trk.pos.x; fr.py = trk.pos.y; fr.pz = trk.pos.z;
                    fr.w = trk.w;
                    fr.E = trk.E;
                    fr.t = trk.t;
                    fr.key = draw_key(g);
                    fr.ev = ev;
                    fr.ch_id = ch_id;
                    fr.bounces = trk.bounces;
                    fr.surf = static_cast<uint8_t>(bh.surf);
                    fr.mode = static_cast<uint8_t>(trk.mode);
                    fr.pad0 = fr.pad1 = 0;
                    out.film(fr);
                    outcome = kStepFilm;
                } else {
                    // re-emitted unchanged: back into the crystal (bounces kept), a DOS mode and an
                    // inward Lambertian direction from the shared sampling below
                    trk.pos = trk.pos + bh.n * kNudge;
                    trk.mode = fdos(L, g.u());
                    sample = 1;
                }
            } else if (g.u() > hs.prob_refl) {
                ++st.killed();
                st.esc() += trk.E * trk.w;
                outcome = kStepEnd;
            } else {  // a surface reflection
                ++st.refl();
                trk.pos = trk.pos + bh.n * kNudge;
                float p_anh, p_anh_spec;
                if (hs.flags & kHotSplitConst) {
                    p_anh = hs.p_anh;
                    p_anh_spec = hs.p_anh_spec;
                } else {
                    const Split sp = reflection_split(s, trk.E);
                    p_anh = static_cast<float>(sp.p_anh);
                    p_anh_spec = static_cast<float>(sp.p_anh + sp.p_spec);
                }
                const float u_refl = g.u();
                if (u_refl < p_anh) {
                    ++st.down();
                    const bool tt = g.u() < L.fTT;
                    const float x = fcdf_any(tt ? cdf + kNCdf : cdf, g);
                    const int m1 = tt ? ftrans(L, g) : 0;
                    const int m2 = ftrans(L, g);
                    FTrack dtr;
                    FKin k2kin;
                    dtr.k = finward<kKin>(L, m2, bh.n, g, k2kin);
                    dtr.pos = trk.pos;
                    dtr.vg = k2kin.dir;
                    dtr.vmag = k2kin.mag;
                    dtr.E = (1.0 - static_cast<double>(x)) * trk.E;
                    dtr.t = trk.t;
                    dtr.w = trk.w;
                    dtr.bounces = 0;
                    dtr.mode = m2;
                    out.daughter(pool_entry(dtr, draw_key(g), ev));
                    trk.E = static_cast<double>(x) * trk.E;
                    trk.mode = m1;
                    sample = 1;
                } else if (u_refl < p_anh_spec) {
                    F3 kr = trk.k - bh.n * (2.0f * fdot(trk.k, bh.n));
                    FKin kin = fmapk<kKin>(L, trk.mode, kr);
                    if (fdot(kin.dir, bh.n) <= 1e-6f) kr = finward<kKin>(L, trk.mode, bh.n, g, kin);
                    trk.k = kr;
                    trk.vg = kin.dir;
                    trk.vmag = kin.mag;
                } else {
                    sample = 1;
                }
            }
        }
    }
    __syncwarp(m_in);
    // shared new-direction path: isotropic (bulk scatter) or Lambertian about the inward
    // normal (diffuse reflection, film re-emission), then the table lookup
    if (sample != 2) {
        const bool lam = (sample == 1);
        const F3 e3 = lam ? bh.n : f3(0.0f, 0.0f, 1.0f);
        const F3 e1 = lam ? forth(bh.n) : f3(1.0f, 0.0f, 0.0f);
        const F3 e2 = lam ? fcross(bh.n, e1) : f3(0.0f, 1.0f, 0.0f);
        FKin kin;
        F3 kd;
        for (int trial = 0;; ++trial) {
            const float u1 = g.u();
            const float u2 = g.u();
            const float ct = lam ? sqrtf(u1) : 2.0f * u1 - 1.0f;
            const float st_ = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
            float sphi, cphi;
            __sincosf(kTwoPiF * u2, &sphi, &cphi);
            kd = e1 * (st_ * cphi) + e2 * (st_ * sphi) + e3 * ct;
            if (lam) kd = funit(kd);
            kin = fmapk<kKin>(L, trk.mode, kd);
            if (!lam || fdot(kin.dir, bh.n) > 1e-6f) break;
            if (trial == 15) {
                kd = bh.n;
                kin = fmapk<kKin>(L, trk.mode, kd);
                break;
            }
        }
        trk.k = kd;
        trk.vg = kin.dir;
        trk.vmag = kin.mag;
    }
    return outcome;
}

struct PoolArgs {
    PoolPh* ring;           // [warps][ring_cap]
    FilmRec* film;          // [warps][kPoolFilmCap]
    uint32_t ring_cap;      // a power of two
    const uint32_t* unit_event;
    const QPhonon* queue;   // queue units (kQueue kernels)
    int stage_tables;       // decay CDF tables read from a shared-memory copy staged by TMA
};

// The film step of a warp, converged: lane l < n_rec runs the cascade of film record
// fb[(f_head + l) % kPoolFilmCap] (from the record's own substream), records the hit and
// the ledger in the record's event (hit slots reserved once per warp) and appends the
// re-emitted phonons, inward Lambertian with DOS modes and their own substreams (the first
// keeps the bounce count), to the warp's ring. Returns the new ring tail.
template <bool kSur, int kKin>
__device__ __noinline__ uint32_t pool_film_step(const FLat* Lp, const Detector* Dp, const RunArgs* ap,
                                                const FilmRec* fb, uint32_t f_head, int n_rec, PoolPh* ring,
                                                uint32_t ring_mask, uint32_t r_head, uint32_t r_tail,
                                                double* refl_buf, double* kwork, unsigned* err) {
    const FLat& L = *Lp;
    const Detector& D = *Dp;
    const RunArgs& a = *ap;
    const int lane = threadIdx.x & 31;
    const bool has = lane < n_rec;
    FilmRec r;
    double edep = 0.0;
    int n_refl = 0;
    R128 g;
    if (has) {
        r = fb[(f_head + lane) & (kPoolFilmCap - 1)];
        const Surface& s = D.surf[r.surf];
        R128 g_c;
        g_c.seed(r.key);
        // the entry step was drawn by the transport step (film_quick): the cascade starts at once
        if constexpr (kSur) {
            edep = s.lut_abs ? surrogate_call(&s, r.E, refl_buf, &n_refl, kwork, &g_c)
                             : kaplan_call(&s.film, r.E, refl_buf, &n_refl, kwork, &g_c);
        } else {
            edep = kaplan_cascade_call(&s.film, r.E, refl_buf, &n_refl, kwork, &g_c);
        }
        g = g_c;
    }
    // hits: one reservation for the warp
    const bool hit = has && edep > 0.0;
    const unsigned hit_mask = __ballot_sync(0xffffffffu, hit);
    if (hit_mask) {
        unsigned long long base = 0;
        if (lane == 0 && a.keep_hits) base = atomicAdd(a.hit_count, static_cast<unsigned long long>(__popc(hit_mask)));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (hit) {
            cmpmc_sim_stats& o = a.ev_stats[r.ev];
            const double wedep = edep * static_cast<double>(r.w);
            atomicAdd(reinterpret_cast<unsigned long long*>(&o.sensor_hits), 1ull);
            atomicAdd(&o.total_deposited_eV, wedep);
            if (a.keep_hits) {
                atomicAdd(reinterpret_cast<unsigned long long*>(a.ev_nhits + r.ev), 1ull);
                const unsigned long long idx = base + __popc(hit_mask & lanemask_lt());
                if (idx < a.hit_cap) {
                    cmpmc_sensor_hit h;
                    h.pos[0] = r.px; h.pos[1] = r.py; h.pos[2] = r.pz;
                    h.time = r.t;
                    h.edep = wedep;
                    h.incident_energy = r.E;
                    h.surface_id = r.surf;
                    h.excitation = 0;
                    h.mode = r.mode;
                    h._pad = 0;
                    h.channel_id = r.ch_id;
                    a.hit_stage[idx] = h;
                    a.hit_key[idx] = r.ev;
                }
            }
        }
    }
    if (has) {
        double sum_refl = 0.0;
        for (int j = 0; j < n_refl; ++j) sum_refl += refl_buf[j];
        const double esc = dmax(0.0, r.E - edep - sum_refl) * static_cast<double>(r.w);
        if (esc != 0.0) atomicAdd(&a.ev_stats[r.ev].escaped_or_killed_eV, esc);
    }
    // re-emissions: an exclusive warp scan of the counts places them in the ring
    int incl = n_refl;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t total = static_cast<uint32_t>(__shfl_sync(0xffffffffu, incl, 31));
    if (r_tail + total - r_head > ring_mask + 1) {  // ring full: the call reruns with a larger ring
        if (lane == 0) *err |= kErrQueue;
        return r_tail;
    }
    if (n_refl > 0) {
        uint32_t pos = r_tail + static_cast<uint32_t>(incl - n_refl);
        F3 n;
        if (r.surf == 0) n = f3(0.0f, 0.0f, -1.0f);
        else if (r.surf == 1) n = f3(0.0f, 0.0f, 1.0f);
        else {
            const float rr = sqrtf(r.px * r.px + r.py * r.py);
            n = (rr > 1e-15f) ? f3(-r.px / rr, -r.py / rr, 0.0f) : f3(-1.0f, 0.0f, 0.0f);
        }
        FTrack t;
        t.pos = f3(r.px, r.py, r.pz) + n * kNudge;
        t.t = r.t;
        t.w = r.w;
        for (int j = 0; j < n_refl; ++j, ++pos) {
            t.mode = fdos(L, g.u());
            FKin kin;
            t.k = finward<kKin>(L, t.mode, n, g, kin);
            t.vg = kin.dir;
            t.vmag = kin.mag;
            t.E = refl_buf[j];
            t.bounces = (j == 0) ? r.bounces : 0u;
            ring[pos & ring_mask] = pool_entry(t, mix64(r.key ^ (0x9e3779b97f4a7c15ULL * static_cast<uint64_t>(j + 1))),
                                               r.ev);
        }
    }
    return r_tail + total;
}

// kQueue: the units are the entries of a phonon queue (the Luke phonons of the charge form,
// p.queue; reserved-but-empty slots are skipped) instead of the batch's primary records
template <bool kSur, int kKin = 0, bool kQueue = false>
__global__ void __launch_bounds__(128, 6) k_pool_fp32(const __grid_constant__ FLat L,
                                                      const __grid_constant__ Detector D,
                                                      const __grid_constant__ RunArgs a,
                                                      const __grid_constant__ PoolArgs p) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    PoolPh* ring = p.ring + warp * p.ring_cap;
    const FilmRec* fb_c = p.film + warp * kPoolFilmCap;
    FilmRec* fb = p.film + warp * kPoolFilmCap;
    const uint32_t ring_mask = p.ring_cap - 1;
    uint32_t r_head = 0, r_tail = 0, f_head = 0, f_tail = 0;  // warp-uniform
    bool input_left = true;                                    // warp-uniform
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    unsigned err = 0;
    const uint64_t seed_key = mix64(a.seed ^ 0x5851f42d4c957f2dULL);
    __shared__ uint32_t s_cnt[kNCnt][kMaxBlock];
    __shared__ double s_led[2][kMaxBlock];
    __shared__ PoolOut s_out[kMaxBlock];
    __shared__ alignas(128) float s_cdf[2 * kNCdf];  // the decay CDF tables (L-LT, then TT)
    __shared__ alignas(8) uint64_t s_bar;
    __shared__ SurfHot s_hot[3];
    const UStats st{&s_cnt[0][threadIdx.x], &s_led[0][threadIdx.x]};
    PoolOut& my_out = s_out[threadIdx.x];
    stage_surf_hot(L, D, s_hot);
    __syncthreads();
    const float* cdf = L.cdf_lt;  // the two tables are contiguous in global memory
    if (p.stage_tables) {
        if (!stage_bulk(s_cdf, L.cdf_lt, 2 * kNCdf * sizeof(float), &s_bar)) {
            if (threadIdx.x == 0) atomicOr(a.err, kErrStage);
            return;
        }
        cdf = s_cdf;
    }
    FTrack trk;
    R128 g;
    uint32_t ev_cur = 0;
    bool live = false;
    for (;;) {
        // ring and film entries written by other lanes of the warp are visible after this
        __syncwarp();
        // 1. refill the empty lanes: the ring first, then new primaries
        const unsigned empty = __ballot_sync(full, !live);
        if (empty) {
            const int n_empty = __popc(empty);
            const int rank = __popc(empty & lanemask_lt());
            const uint32_t from_ring = min(r_tail - r_head, static_cast<uint32_t>(n_empty));
            if (!live && rank < static_cast<int>(from_ring)) {
                const PoolPh q = ring[(r_head + rank) & ring_mask];
                trk.pos = f3(q.px, q.py, q.pz);
                trk.k = f3(q.kx, q.ky, q.kz);
                trk.vg = f3(q.vx, q.vy, q.vz);
                trk.vmag = q.vmag;
                trk.w = q.w;
                trk.bounces = q.bounces_mode >> 2;
                trk.mode = static_cast<int>(q.bounces_mode & 3u);
                trk.E = q.E;
                trk.t = q.t;
                g.seed(q.key);
                ev_cur = q.ev;
                st.clear();
                live = true;
            }
            r_head += from_ring;
            const int need = n_empty - static_cast<int>(from_ring);
            if (need > 0 && input_left) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(a.next_work, static_cast<unsigned long long>(need));
                base = __shfl_sync(full, base, 0);
                if (base + need >= a.n_events) input_left = false;
                const uint64_t unit = base + static_cast<uint64_t>(rank - static_cast<int>(from_ring));
                if constexpr (kQueue) {
                    if (!live && rank >= static_cast<int>(from_ring) && unit < a.n_events) {
                        const QPhonon q = p.queue[unit];
                        if (q.ev != kQEmpty) {
                            ev_cur = q.ev;
                            g.seed(q.key);
                            trk.pos = f3(q.px, q.py, q.pz);
                            trk.k = f3(q.kx, q.ky, q.kz);
                            trk.mode = static_cast<int>(q.mode);
                            const FKin kin = fmapk<kKin>(L, trk.mode, trk.k);
                            trk.vg = kin.dir;
                            trk.vmag = kin.mag;
                            trk.E = q.E;
                            trk.t = q.t;
                            trk.w = q.w;
                            trk.bounces = q.pad;
                            st.clear();
                            live = true;
                        }
                    }
                } else if (!live && rank >= static_cast<int>(from_ring) && unit < a.n_events) {
                    const uint32_t ev = p.unit_event[unit];
                    ev_cur = ev;
                    const uint64_t j = unit - a.ph_off[ev];
                    g.seed(seed_key ^ mix64(((a.first_event + ev) << 20) | j));
                    const cmpmc_phonon_track& in = a.ph[unit];
                    trk.pos = f3(static_cast<float>(in.pos[0]), static_cast<float>(in.pos[1]),
                                 static_cast<float>(in.pos[2]));
                    trk.k = f3(static_cast<float>(in.k_dir[0]), static_cast<float>(in.k_dir[1]),
                               static_cast<float>(in.k_dir[2]));
                    trk.vg = f3(static_cast<float>(in.vg_dir[0]), static_cast<float>(in.vg_dir[1]),
                                static_cast<float>(in.vg_dir[2]));
                    trk.vmag = static_cast<float>(in.vg_mag);
                    trk.E = in.energy;
                    trk.t = in.time;
                    trk.w = static_cast<float>(in.weight);
                    trk.bounces = in.bounces;
                    trk.mode = in.mode;
                    st.clear();
                    live = true;
                }
            }
        }
        if (__ballot_sync(full, live) == 0) {
            // no transport work left in this warp: drain the film buffer, then stop
            if (f_tail != f_head) {
                const int n_rec = static_cast<int>(min(f_tail - f_head, 32u));
                r_tail = pool_film_step<kSur, kKin>(&L, &D, &a, fb_c, f_head, n_rec, ring, ring_mask, r_head, r_tail,
                                                    refl_buf, kwork, &err);
                f_head += n_rec;
                if (__any_sync(full, err != 0)) break;
                continue;
            }
            if (r_tail == r_head) break;
            continue;
        }
        // 2. one step of every live track
        int outcome = kStepOn;
        WarpSink sink{&my_out, false, &a};
        if (live) {
            outcome = pool_step<kKin, kSur>(L, cdf, D, s_hot, trk, g, st, ev_cur, sink);
            if (outcome != kStepOn) {
                sink_unit(&a, ev_cur, st);
                live = false;
            }
        }
        const bool has_d = sink.has_d;
        // 3. regroup: daughters to the ring, film entries to the film buffer
        const unsigned d_mask = __ballot_sync(full, has_d);
        if (d_mask) {
            if (r_tail + __popc(d_mask) - r_head > p.ring_cap) {
                err |= kErrQueue;
                break;
            }
            if (has_d) ring[(r_tail + __popc(d_mask & lanemask_lt())) & ring_mask] = my_out.ph;
            r_tail += __popc(d_mask);
        }
        const unsigned f_mask = __ballot_sync(full, outcome == kStepFilm);
        if (f_mask) {
            if (outcome == kStepFilm) fb[(f_tail + __popc(f_mask & lanemask_lt())) & (kPoolFilmCap - 1)] = my_out.film;
            f_tail += __popc(f_mask);
        }
        // 4. the film step, converged, once 32 entries wait
        if (f_tail - f_head >= 32) {
            __syncwarp();
            r_tail = pool_film_step<kSur, kKin>(&L, &D, &a, fb_c, f_head, 32, ring, ring_mask, r_head, r_tail,
                                                refl_buf, kwork, &err);
            f_head += 32;
            if (__any_sync(full, err != 0)) break;
        }
    }
    if (err && lane == 0) atomicOr(a.err, err);
}

// ---- SM-phase pool ----------------------------------------------------------------------
// The warp pool runs a warp's film cascades among the other warps' transport steps, and the
// two code paths then compete for the SM's instruction cache: measured, the transport
// machinery alone steps 2.4e10 times a second, the mix half as fast as separate kernels.
// Here one block of 512 threads (16 warps) owns an SM and alternates two phases, so the SM
// runs one code path at a time:
//   transport phase: every warp steps its lanes, refilling them from the block's ring of
//     pending phonons (entries published at the last phase boundary) and then from the
//     batch's primaries; a step that reaches an active film appends its record to the
//     block's film buffer, a daughter goes to the ring (both reserved by shared-memory
//     atomics, consumable after the boundary). A warp leaves the phase when the film buffer
//     holds film_trigger records or when it has no work left;
//   film phase: every thread takes film records from the buffer (a shared-memory counter)
//     and runs their cascades, hits reserved once per coalesced group, re-emissions appended
//     to the ring.
// The block ends when a boundary finds no live lane, no published phonon and no primary
// left. Nothing waits on another block; every wait is a block barrier that all threads
// reach (each phase ends by itself).
// Threads of the block (build-time, per precision). FP32: 512 threads keep the step loop's
// state in 128 registers with no spills; measured on the 1M-primary batch, 384 threads (168
// registers) 231 ms, 512 (128) 204 ms, 576 (96) 228 ms, 768 (80) 223 ms, 1024 (64) 263 ms.
// FP64: 768 threads (1,481 ms; 512 threads 1,564 ms).
#ifndef CMPMC_SM_THREADS
#define CMPMC_SM_THREADS 512
#endif
#ifndef CMPMC_SM_THREADS_FP64
#define CMPMC_SM_THREADS_FP64 768
#endif
// the block's shape: threads, warps and the per-lane unit counters and ledgers (dynamic
// shared memory: [warps][kNCnt][32] u32, then [warps][2][32] f64)
template <int kThreads>
struct SmShape {
    static constexpr int kWarps = kThreads / 32;
    static constexpr int kCntBytes = kWarps * kNCnt * 32 * 4;
    static constexpr int kDynBytes = kCntBytes + kWarps * 2 * 32 * 8;
};

struct SmPoolArgs {
    void* ring;              // [blocks][ring_cap] entries of the precision's ring type
    void* film;              // [blocks][film_cap] film records of the precision's type
    uint32_t ring_cap;       // a power of two
    uint32_t film_cap;       // film records per block and phase
    uint32_t film_trigger;   // records that end a transport phase (<= film_cap - threads)
    const uint32_t* unit_event;
    const QPhonon* queue;    // queue units (kQueue kernels)
    int stage_tables;
};

struct SmShared {
    uint32_t r_head, r_tail, r_pub;  // ring: consumable [r_head, r_pub), appended at r_tail
    uint32_t f_tail, f_next;         // film buffer: records [0, f_tail), next to run
    uint32_t input_left;             // the batch still has primaries
    uint32_t n_dry;                  // warps of this phase that ran out of work
};

// output of the SM pool's step: reserved in the block's buffers by shared-memory atomics
template <class Film, class Entry>
struct SmSink {
    SmShared* sh;
    Film* fbuf;
    Entry* ring;
    uint32_t film_cap, ring_mask, r_floor;
    unsigned* err;
    const RunArgs* a;
    __device__ __forceinline__ void hit(uint32_t ev, const cmpmc_sensor_hit& h) { stage_hit(*a, ev, h); }
    __device__ __forceinline__ void film(const Film& r) {
        const uint32_t i = atomicAdd(&sh->f_tail, 1u);
        if (i < film_cap) fbuf[i] = r;
        else *err |= kErrFilmQueue;
    }
    __device__ __forceinline__ void daughter(const Entry& q) {
        const uint32_t i = atomicAdd(&sh->r_tail, 1u);
        if (i + 1u - r_floor <= ring_mask + 1u) ring[i & ring_mask] = q;
        else *err |= kErrQueue;
    }
};

// the cascade of one film record (from the record's own substream) with its hit and ledger
// in the record's event; returns the energies to re-emit in refl[0, n_refl) and the record's
// generator, positioned after the cascade
template <bool kSur, class Film>
__device__ __forceinline__ int film_cascade(const Detector& D, const RunArgs& a, const Film& r, double hx, double hy,
                                            double hz, double* refl_buf, double* kwork, R128& g) {
    const Surface& s = D.surf[r.surf];
    int n_refl = 0;
    double edep;
    {
        R128 g_c;
        g_c.seed(r.key);
        // the entry step was drawn by the transport step (film_quick): the cascade starts at once
        if constexpr (kSur) {
            edep = s.lut_abs ? surrogate_call(&s, r.E, refl_buf, &n_refl, kwork, &g_c)
                             : kaplan_call(&s.film, r.E, refl_buf, &n_refl, kwork, &g_c);
        } else {
            edep = kaplan_cascade_call(&s.film, r.E, refl_buf, &n_refl, kwork, &g_c);
        }
        g = g_c;
    }
    cmpmc_sim_stats& o = a.ev_stats[r.ev];
    if (edep > 0.0) {
        const double wedep = edep * static_cast<double>(r.w);
        atomicAdd(reinterpret_cast<unsigned long long*>(&o.sensor_hits), 1ull);
        atomicAdd(&o.total_deposited_eV, wedep);
        cmpmc_sensor_hit h;
        h.pos[0] = hx; h.pos[1] = hy; h.pos[2] = hz;
        h.time = r.t;
        h.edep = wedep;
        h.incident_energy = r.E;
        h.surface_id = r.surf;
        h.excitation = 0;
        h.mode = r.mode;
        h._pad = 0;
        h.channel_id = r.ch_id;
        stage_hit(a, r.ev, h);
    }
    double sum_refl = 0.0;
    for (int j = 0; j < n_refl; ++j) sum_refl += refl_buf[j];
    const double esc = dmax(0.0, r.E - edep - sum_refl) * static_cast<double>(r.w);
    if (esc != 0.0) atomicAdd(&o.escaped_or_killed_eV, esc);
    return n_refl;
}

__device__ __forceinline__ uint64_t reemit_key(uint64_t key, int j) {
    return mix64(key ^ (0x9e3779b97f4a7c15ULL * static_cast<uint64_t>(j + 1)));
}

// ---- precision policies of the SM-phase pool ----------------------------------------------
// PF32: the batched FP32 form (FP32 geometry, directions and table blend; FP64 energy,
// time and ledger). PF64: the same process in FP64 throughout on the same substreams (the
// geometry, rates and samplers of the reference's FP64 code, 53-bit uniforms, the
// reference's 1e-11 m inward nudge, the lattice's own map_k_to_vg in every kinematics
// mode): the comparison point that isolates what FP32 buys.
struct PF32 {
    static constexpr int kThreads = CMPMC_SM_THREADS;
    using Track = FTrack;
    using Entry = PoolPh;
    using Film = FilmRec;
    using Lat = FLat;
    static constexpr bool kStage = true;
    __device__ static __forceinline__ void from_entry(const Entry& q, Track& t) {
        t.pos = f3(q.px, q.py, q.pz);
        t.k = f3(q.kx, q.ky, q.kz);
        t.vg = f3(q.vx, q.vy, q.vz);
        t.vmag = q.vmag;
        t.w = q.w;
        t.bounces = q.bounces_mode >> 2;
        t.mode = static_cast<int>(q.bounces_mode & 3u);
        t.E = q.E;
        t.t = q.t;
    }
    __device__ static __forceinline__ void from_primary(const cmpmc_phonon_track& in, Track& t) {
        t.pos = f3(static_cast<float>(in.pos[0]), static_cast<float>(in.pos[1]), static_cast<float>(in.pos[2]));
        t.k = f3(static_cast<float>(in.k_dir[0]), static_cast<float>(in.k_dir[1]), static_cast<float>(in.k_dir[2]));
        t.vg = f3(static_cast<float>(in.vg_dir[0]), static_cast<float>(in.vg_dir[1]),
                  static_cast<float>(in.vg_dir[2]));
        t.vmag = static_cast<float>(in.vg_mag);
        t.E = in.energy;
        t.t = in.time;
        t.w = static_cast<float>(in.weight);
        t.bounces = in.bounces;
        t.mode = in.mode;
    }
    template <int kKin>
    __device__ static __forceinline__ void from_queue(const Lat& L, const QPhonon& q, Track& t) {
        t.pos = f3(q.px, q.py, q.pz);
        t.k = f3(q.kx, q.ky, q.kz);
        t.mode = static_cast<int>(q.mode);
        const FKin kin = fmapk<kKin>(L, t.mode, t.k);
        t.vg = kin.dir;
        t.vmag = kin.mag;
        t.E = q.E;
        t.t = q.t;
        t.w = q.w;
        t.bounces = q.pad;
    }
    template <int kKin, bool kSur, class ST, class Sink>
    __device__ static __forceinline__ int step(const Lat& L, const float* cdf, const Detector& D, const SurfHot* hot,
                                               Track& trk, R128& g, const ST& st, uint32_t ev, Sink& out) {
        return pool_step<kKin, kSur>(L, cdf, D, hot, trk, g, st, ev, out);
    }
    // one film record of the film phase: cascade, then the re-emissions into the ring
    template <bool kSur, int kKin>
    __device__ static __forceinline__ void film_record(const Lat& L, const Detector& D, const RunArgs& a,
                                                       const Film& r, double* refl_buf, double* kwork, SmShared* sh,
                                                       Entry* ring, uint32_t ring_mask, uint32_t r_floor,
                                                       unsigned* err) {
        R128 g;
        const int n_refl = film_cascade<kSur>(D, a, r, r.px, r.py, r.pz, refl_buf, kwork, g);
        if (n_refl == 0) return;
        const uint32_t base = atomicAdd(&sh->r_tail, static_cast<uint32_t>(n_refl));
        if (base + static_cast<uint32_t>(n_refl) - r_floor > ring_mask + 1u) {
            *err |= kErrQueue;
            return;
        }
        F3 n;
        if (r.surf == 0) n = f3(0.0f, 0.0f, -1.0f);
        else if (r.surf == 1) n = f3(0.0f, 0.0f, 1.0f);
        else {
            const float rr = sqrtf(r.px * r.px + r.py * r.py);
            n = (rr > 1e-15f) ? f3(-r.px / rr, -r.py / rr, 0.0f) : f3(-1.0f, 0.0f, 0.0f);
        }
        FTrack t;
        t.pos = f3(r.px, r.py, r.pz) + n * kNudge;
        t.t = r.t;
        t.w = r.w;
        for (int j = 0; j < n_refl; ++j) {
            t.mode = fdos(L, g.u());
            FKin kin;
            t.k = finward<kKin>(L, t.mode, n, g, kin);
            t.vg = kin.dir;
            t.vmag = kin.mag;
            t.E = refl_buf[j];
            t.bounces = (j == 0) ? r.bounces : 0u;
            ring[(base + j) & ring_mask] = pool_entry(t, reemit_key(r.key, j), r.ev);
        }
    }
};

// ---- the FP64 policy ----------------------------------------------------------------------
constexpr double kNudge64 = 1e-11;  // the reference's inward move after a boundary event

struct DTrack {
    V3 pos, k, vg;
    double vmag, E, t, w;
    uint32_t bounces;
    int mode;
};

struct alignas(16) PoolPh64 {  // 128 B
    double px, py, pz, kx, ky, kz, vx, vy, vz, vmag, w, E, t;
    uint64_t key;
    uint32_t ev;
    uint32_t bounces_mode;  // bounces << 2 | mode
};

struct alignas(16) FilmRec64 {  // 80 B
    double px, py, pz, w, E, t;
    uint64_t key;
    uint32_t ev;
    int32_t ch_id;
    uint32_t bounces;
    uint8_t surf, mode, pad0, pad1;
};

__device__ __forceinline__ PoolPh64 pool_entry64(const DTrack& t, uint64_t key, uint32_t ev) {
    PoolPh64 q;
    q.px = t.pos.x; q.py = t.pos.y; q.pz = t.pos.z;
    q.kx = t.k.x; q.ky = t.k.y; q.kz = t.k.z;
    q.vx = t.vg.x; q.vy = t.vg.y; q.vz = t.vg.z;
    q.vmag = t.vmag;
    q.w = t.w;
    q.E = t.E;
    q.t = t.t;
    q.key = key;
    q.ev = ev;
    q.bounces_mode = (t.bounces << 2) | static_cast<uint32_t>(t.mode);
    return q;
}

// the reference's samplers (rng.hpp:78-96, phonon_kernels.hpp:53-63, crystal_lattice.hpp:200-212)
// on a substream's 53-bit uniforms
__device__ __forceinline__ V3 iso_dir64(R128& g) {
    const double cos_theta = 2.0 * g.uniform() - 1.0;
    const double sin_theta = sqrt(dmax(0.0, 1.0 - cos_theta * cos_theta));
    double s, c;
    sincos(kTwoPi * g.uniform(), &s, &c);
    return v3(sin_theta * c, sin_theta * s, cos_theta);
}
__device__ __forceinline__ V3 lambert_dir64(V3 n, R128& g) {
    double s, c;
    sincos(kTwoPi * g.uniform(), &s, &c);
    const double sin_theta = sqrt(g.uniform());
    const double cos_theta = sqrt(dmax(0.0, 1.0 - sin_theta * sin_theta));
    const V3 u = orthogonal_unit(n);
    const V3 v = cross(n, u);
    return unit(u * (sin_theta * c) + v * (sin_theta * s) + n * cos_theta);
}
__device__ __forceinline__ int dos64(const Lattice& L, double u) {
    return (u < L.fLDOS) ? 0 : ((u < L.fLDOS + L.fSTDOS) ? 2 : 1);
}
__device__ __forceinline__ int trans64(const Lattice& L, R128& g) {
    return (g.uniform() < L.fSTDOS / (L.fSTDOS + L.fFTDOS)) ? 2 : 1;
}
__device__ __forceinline__ double cdf64(const double* cdf, R128& g) {
    const double u = g.uniform() * (kNCdf - 1);
    const int i = imin(static_cast<int>(u), kNCdf - 2);
    const double f = u - i;
    return cdf[i] * (1.0 - f) + cdf[i + 1] * f;
}
// SimulationEngine::sample_inward_wavevector (engine.hpp:927-936)
__device__ __noinline__ V3 inward64(const Lattice* Lp, int mode, V3 n, R128* gp, Kin* kin) {
    for (int trial = 0; trial < 16; ++trial) {
        const V3 kd = lambert_dir64(n, *gp);
        *kin = map_k_to_vg(*Lp, mode, kd);
        if (dot(kin->vg_dir, n) > 1e-6) return kd;
    }
    *kin = map_k_to_vg(*Lp, mode, n);
    return n;
}
__device__ __noinline__ Kin map64_call(const Lattice* Lp, int mode, V3 k) { return map_k_to_vg(*Lp, mode, k); }

// anharmonic decay of an L phonon (engine.hpp:938-988) in FP64; the daughter goes to *dp
template <class ST>
__device__ __noinline__ void decay64(const Lattice* Lp, DTrack* tp, DTrack* dp, const ST* st, R128* gp) {
    const Lattice& L = *Lp;
    DTrack& trk = *tp;
    R128& g = *gp;
    const V3 d1 = trk.k;
    const V3 perp = orthogonal_unit(d1);
    const double phi = kTwoPi * g.uniform();
    double sp, cp;
    sincos(phi, &sp, &cp);
    double x, th1, th2;
    int m1, m2;
    if (g.uniform() < L.fTT_frac) {
        ++st->tt();
        x = cdf64(L.cdf_tt, g);
        th1 = decay_angle_TT(x, L.v_sound, L.v_trans);
        th2 = decay_angle_TT(1.0 - x, L.v_sound, L.v_trans);
        m1 = trans64(L, g);
        m2 = trans64(L, g);
    } else {
        ++st->lt();
        x = cdf64(L.cdf_lt, g);
        th1 = decay_angle_L_to_LT(x, L.v_sound, L.v_trans);
        th2 = decay_angle_T_from_LT(x, L.v_sound, L.v_trans);
        m1 = 0;
        m2 = trans64(L, g);
    }
    double s1, c1, s2, c2;
    sincos(th1, &s1, &c1);
    sincos(-th2, &s2, &c2);
    const V3 k1 = unit(rotate_around(rotate_around(d1, perp, c1, s1), d1, cp, sp));
    const V3 k2 = unit(rotate_around(rotate_around(d1, perp, c2, s2), d1, cp, sp));
    DTrack& d = *dp;
    d.pos = trk.pos;
    d.k = k2;
    const Kin kin2 = map_k_to_vg(L, m2, k2);
    d.vg = kin2.vg_dir;
    d.vmag = kin2.vg_mag;
    d.E = (1.0 - x) * trk.E;
    d.t = trk.t;
    d.w = trk.w;
    d.bounces = 0;
    d.mode = m2;
    trk.E = x * trk.E;
    trk.mode = m1;
    trk.k = k1;
    const Kin kin = map_k_to_vg(L, m1, k1);
    trk.vg = kin.vg_dir;
    trk.vmag = kin.vg_mag;
}

// one transport step in FP64: the branches and draws of pool_step
template <bool kSur, class ST, class Sink>
__device__ __forceinline__ int pool_step64(const Lattice& L, const Detector& D, DTrack& trk, R128& g, const ST& st,
                                           uint32_t ev, Sink& out) {
    if (trk.E < D.min_phonon_eV || trk.bounces >= D.max_bounces) {
        ++st.killed();
        st.esc() += trk.E * trk.w;
        return kStepEnd;
    }
    if (D.rr_bounces != 0 && trk.bounces > D.rr_bounces && (trk.bounces - D.rr_bounces) % 32 == 0) {
        if (g.uniform() < D.rr_survival) {
            trk.w /= D.rr_survival;
        } else {
            ++st.killed();
            return kStepEnd;
        }
    }
    ++st.steps();
    const double r_iso = isotope_rate(L, trk.E);
    const double r_poly = polycrystal_rate(L, trk.vmag);
    const double r_down = downconversion_rate(L, trk.mode, trk.E);
    const double r_tot = r_iso + r_poly + r_down;
    const double d_phys = (r_tot > 1e-12) ? (-log(g.uniform()) * trk.vmag / r_tot) : kInf;
    const BHit bh = intersect_exit(D.radius, D.half_z, trk.pos, trk.vg);
    const bool bulk = d_phys < bh.distance;
    const double d = bulk ? d_phys : bh.distance;
    trk.pos = trk.pos + trk.vg * d;
    trk.t += d / trk.vmag;
    int sample = 2;  // 0: isotropic, 1: Lambertian about bh.n_in, 2: nothing more
    if (bulk) {
        const double u_proc = g.uniform() * r_tot;
        if (r_down > 0.0 && u_proc < r_down) {
            DTrack t_c = trk, d_c;
            R128 g_c = g;
            decay64(&L, &t_c, &d_c, &st, &g_c);
            trk = t_c;
            g = g_c;
            out.daughter(pool_entry64(d_c, draw_key(g), ev));
        } else {
            if (u_proc < r_down + r_iso) ++st.iso();
            else ++st.poly();
            trk.mode = dos64(L, g.uniform());
            sample = 0;
        }
    } else {
        const V3 n = bh.n_in;
        trk.bounces++;
        const Surface& s = D.surf[bh.surf];
        bool enter = false;
        int ch_id = -1;
        bool active_pad = true;
        if (s.n_pads > 0) {
            R128 g_c = g;
            ch_id = mask_call(s.pads, s.n_pads, static_cast<float>(trk.pos.x), static_cast<float>(trk.pos.y), &g_c);
            g = g_c;
            active_pad = ch_id >= 0;
        }
        if (active_pad && s.has_film && g.uniform() < s.prob_abs) {
            const double p_enter = s.has_amm ? amm_transmission(s.amm_sub, s.amm_film, trk.mode == 0, dot(trk.k, n))
                                             : s.film.film_absorption;
            enter = g.uniform() < p_enter;
        }
        if (enter) {
            R128 g_c = g;
            const int film = film_quick<kSur>(&s.film, trk.E, &g_c);
            g = g_c;
            if (film == kFilmAbsorbed) {
                const double wedep = trk.E * trk.w;
                ++st.hits();
                st.dep() += wedep;
                cmpmc_sensor_hit h;
                h.pos[0] = trk.pos.x; h.pos[1] = trk.pos.y; h.pos[2] = trk.pos.z;
                h.time = trk.t;
                h.edep = wedep;
                h.incident_energy = trk.E;
                h.surface_id = static_cast<uint8_t>(bh.surf);
                h.excitation = 0;
                h.mode = static_cast<uint8_t>(trk.mode);
                h._pad = 0;
                h.channel_id = ch_id;
                out.hit(ev, h);
                return kStepEnd;
            }
            if (film == kFilmCascade) {
                FilmRec64 fr;
                fr.px = trk.pos.x; fr.py = trk.pos.y; fr.pz = trk.pos.z;
                fr.w = trk.w;
                fr.E = trk.E;
                fr.t = trk.t;
                fr.key = draw_key(g);
                fr.ev = ev;
                fr.ch_id = ch_id;
                fr.bounces = trk.bounces;
                fr.surf = static_cast<uint8_t>(bh.surf);
                fr.mode = static_cast<uint8_t>(trk.mode);
                fr.pad0 = fr.pad1 = 0;
                out.film(fr);
                return kStepFilm;
            }
            trk.pos = trk.pos + n * kNudge64;
            trk.mode = dos64(L, g.uniform());
            sample = 1;
        } else if (g.uniform() > s.prob_refl) {
            ++st.killed();
            st.esc() += trk.E * trk.w;
            return kStepEnd;
        }
        if (!enter) {
            ++st.refl();
            trk.pos = trk.pos + n * kNudge64;
            const Split sp = reflection_split(s, trk.E);
            const double u_refl = g.uniform();
            if (u_refl < sp.p_anh) {
                ++st.down();
                const bool tt = g.uniform() < L.fTT_frac;
                const double x = cdf64(tt ? L.cdf_tt : L.cdf_lt, g);
                const int m1 = tt ? trans64(L, g) : 0;
                const int m2 = trans64(L, g);
                DTrack dtr;
                Kin k2kin;
                R128 g_c = g;
                dtr.k = inward64(&L, m2, n, &g_c, &k2kin);
                g = g_c;
                dtr.pos = trk.pos;
                dtr.vg = k2kin.vg_dir;
                dtr.vmag = k2kin.vg_mag;
                dtr.E = (1.0 - x) * trk.E;
                dtr.t = trk.t;
                dtr.w = trk.w;
                dtr.bounces = 0;
                dtr.mode = m2;
                out.daughter(pool_entry64(dtr, draw_key(g), ev));
                trk.E = x * trk.E;
                trk.mode = m1;
                sample = 1;
            } else if (u_refl < sp.p_anh + sp.p_spec) {
                V3 kr = trk.k - n * (2.0 * dot(trk.k, n));
                Kin kin = map64_call(&L, trk.mode, kr);
                if (dot(kin.vg_dir, n) <= 1e-6) {
                    R128 g_c = g;
                    kr = inward64(&L, trk.mode, n, &g_c, &kin);
                    g = g_c;
                }
                trk.k = kr;
                trk.vg = kin.vg_dir;
                trk.vmag = kin.vg_mag;
            } else {
                sample = 1;
            }
        }
        if (sample == 1) {
            Kin kin;
            R128 g_c = g;
            trk.k = inward64(&L, trk.mode, n, &g_c, &kin);
            g = g_c;
            trk.vg = kin.vg_dir;
            trk.vmag = kin.vg_mag;
        }
        return kStepOn;
    }
    if (sample == 0) {
        trk.k = iso_dir64(g);
        const Kin kin = map_k_to_vg(L, trk.mode, trk.k);
        trk.vg = kin.vg_dir;
        trk.vmag = kin.vg_mag;
    }
    return kStepOn;
}

struct PF64 {
    static constexpr int kThreads = CMPMC_SM_THREADS_FP64;
    using Track = DTrack;
    using Entry = PoolPh64;
    using Film = FilmRec64;
    using Lat = Lattice;
    static constexpr bool kStage = false;
    __device__ static __forceinline__ void from_entry(const Entry& q, Track& t) {
        t.pos = v3(q.px, q.py, q.pz);
        t.k = v3(q.kx, q.ky, q.kz);
        t.vg = v3(q.vx, q.vy, q.vz);
        t.vmag = q.vmag;
        t.w = q.w;
        t.bounces = q.bounces_mode >> 2;
        t.mode = static_cast<int>(q.bounces_mode & 3u);
        t.E = q.E;
        t.t = q.t;
    }
    __device__ static __forceinline__ void from_primary(const cmpmc_phonon_track& in, Track& t) {
        t.pos = v3(in.pos[0], in.pos[1], in.pos[2]);
        t.k = v3(in.k_dir[0], in.k_dir[1], in.k_dir[2]);
        t.vg = v3(in.vg_dir[0], in.vg_dir[1], in.vg_dir[2]);
        t.vmag = in.vg_mag;
        t.E = in.energy;
        t.t = in.time;
        t.w = in.weight;
        t.bounces = in.bounces;
        t.mode = in.mode;
    }
    template <int kKin>
    __device__ static __forceinline__ void from_queue(const Lat& L, const QPhonon& q, Track& t) {
        t.pos = v3(q.px, q.py, q.pz);
        t.k = v3(q.kx, q.ky, q.kz);
        t.mode = static_cast<int>(q.mode);
        const Kin kin = map64_call(&L, t.mode, t.k);
        t.vg = kin.vg_dir;
        t.vmag = kin.vg_mag;
        t.E = q.E;
        t.t = q.t;
        t.w = q.w;
        t.bounces = q.pad;
    }
    template <int kKin, bool kSur, class ST, class Sink>
    __device__ static __forceinline__ int step(const Lat& L, const float*, const Detector& D, const SurfHot*,
                                               Track& trk, R128& g, const ST& st, uint32_t ev, Sink& out) {
        return pool_step64<kSur>(L, D, trk, g, st, ev, out);
    }
    template <bool kSur, int kKin>
    __device__ static __forceinline__ void film_record(const Lat& L, const Detector& D, const RunArgs& a,
                                                       const Film& r, double* refl_buf, double* kwork, SmShared* sh,
                                                       Entry* ring, uint32_t ring_mask, uint32_t r_floor,
                                                       unsigned* err) {
        R128 g;
        const int n_refl = film_cascade<kSur>(D, a, r, r.px, r.py, r.pz, refl_buf, kwork, g);
        if (n_refl == 0) return;
        const uint32_t base = atomicAdd(&sh->r_tail, static_cast<uint32_t>(n_refl));
        if (base + static_cast<uint32_t>(n_refl) - r_floor > ring_mask + 1u) {
            *err |= kErrQueue;
            return;
        }
        V3 n;
        if (r.surf == 0) n = v3(0.0, 0.0, -1.0);
        else if (r.surf == 1) n = v3(0.0, 0.0, 1.0);
        else {
            const double rr = m_hypot(r.px, r.py);
            n = (rr > 1e-15) ? v3(-r.px / rr, -r.py / rr, 0.0) : v3(-1.0, 0.0, 0.0);
        }
        DTrack t;
        t.pos = v3(r.px, r.py, r.pz) + n * kNudge64;
        t.t = r.t;
        t.w = r.w;
        for (int j = 0; j < n_refl; ++j) {
            t.mode = dos64(L, g.uniform());
            Kin kin;
            t.k = inward64(&L, t.mode, n, &g, &kin);
            t.vg = kin.vg_dir;
            t.vmag = kin.vg_mag;
            t.E = refl_buf[j];
            t.bounces = (j == 0) ? r.bounces : 0u;
            ring[(base + j) & ring_mask] = pool_entry64(t, reemit_key(r.key, j), r.ev);
        }
    }
};

// the film phase of one thread: records from the block's buffer until it is drained
template <class P, bool kSur, int kKin>
__device__ __noinline__ void sm_film_phase(const typename P::Lat* Lp, const Detector* Dp, const RunArgs* ap,
                                           const typename P::Film* film, uint32_t n_film, SmShared* sh,
                                           typename P::Entry* ring, uint32_t ring_mask, uint32_t r_floor,
                                           unsigned* err) {
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    for (;;) {
        const uint32_t i = atomicAdd(&sh->f_next, 1u);
        if (i >= n_film) break;
        const typename P::Film r = film[i];
        P::template film_record<kSur, kKin>(*Lp, *Dp, *ap, r, refl_buf, kwork, sh, ring, ring_mask, r_floor, err);
    }
}

template <class P, bool kSur, int kKin = 0, bool kQueue = false>
__global__ void __launch_bounds__(P::kThreads, 1) k_sm_pool(const __grid_constant__ typename P::Lat L,
                                                           const __grid_constant__ Detector D,
                                                           const __grid_constant__ RunArgs a,
                                                           const __grid_constant__ SmPoolArgs p) {
    using Entry = typename P::Entry;
    using Film = typename P::Film;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    extern __shared__ __align__(16) unsigned char sm_dyn[];
    uint32_t(*s_cnt)[kNCnt][32] = reinterpret_cast<uint32_t(*)[kNCnt][32]>(sm_dyn);
    double(*s_led)[2][32] = reinterpret_cast<double(*)[2][32]>(sm_dyn + SmShape<P::kThreads>::kCntBytes);
    __shared__ alignas(128) float s_cdf[P::kStage ? 2 * kNCdf : 4];  // decay CDF tables (L-LT, then TT)
    __shared__ alignas(8) uint64_t s_bar;
    __shared__ SmShared sh;
    __shared__ SurfHot s_hot[3];
    const UStatsT<32> st{&s_cnt[wid][0][lane], &s_led[wid][0][lane]};
    Entry* ring = static_cast<Entry*>(p.ring) + static_cast<uint64_t>(blockIdx.x) * p.ring_cap;
    Film* film = static_cast<Film*>(p.film) + static_cast<uint64_t>(blockIdx.x) * p.film_cap;
    const uint32_t ring_mask = p.ring_cap - 1;
    if constexpr (P::kStage) stage_surf_hot(L, D, s_hot);  // FP32 policy (the FP64 step reads D)
    if (threadIdx.x == 0) {
        sh.r_head = sh.r_tail = sh.r_pub = 0;
        sh.f_tail = sh.f_next = 0;
        sh.input_left = 1;
        sh.n_dry = 0;
    }
    const float* cdf = nullptr;
    if constexpr (P::kStage) {
        cdf = L.cdf_lt;  // the two tables are contiguous in global memory
        if (p.stage_tables) {  // (stage_bulk synchronizes the block)
            if (!stage_bulk(s_cdf, L.cdf_lt, 2 * kNCdf * sizeof(float), &s_bar)) {
                if (threadIdx.x == 0) atomicOr(a.err, kErrStage);
                return;
            }
            cdf = s_cdf;
        }
    }
    __syncthreads();
    const uint64_t seed_key = mix64(a.seed ^ 0x5851f42d4c957f2dULL);
    volatile SmShared* vsh = &sh;
    typename P::Track trk;
    R128 g;
    uint32_t ev_cur = 0;
    bool live = false;
    unsigned err = 0;
    for (;;) {
        // ---- transport phase --------------------------------------------------------
        const uint32_t r_floor = vsh->r_head;  // ring slots below it are free
        const uint32_t r_pub = vsh->r_pub;
        SmSink<Film, Entry> sink{&sh, film, ring, p.film_cap, ring_mask, r_floor, &err, &a};
        for (;;) {
            uint32_t ft = 0, inp = 0, dry = 0, unpub = 0;
            if (lane == 0) {
                ft = vsh->f_tail;
                inp = vsh->input_left;
                dry = vsh->n_dry;
                unpub = vsh->r_tail - r_pub;
            }
            ft = __shfl_sync(full, ft, 0);
            inp = __shfl_sync(full, inp, 0);
            dry = __shfl_sync(full, dry, 0);
            unpub = __shfl_sync(full, unpub, 0);
            // the film phase starts once enough records wait, or earlier when half the
            // block has run dry and the waiting cascades or the phonons appended to the ring
            // since the last boundary would give it work
            if (ft >= p.film_trigger || ((ft > 0 || unpub > 0) && 2 * dry >= SmShape<P::kThreads>::kWarps)) break;
            const unsigned empty = __ballot_sync(full, !live);
            if (empty) {
                const int n_empty = __popc(empty);
                const int rank = __popc(empty & lanemask_lt());
                uint32_t base = 0, got = 0;
                if (lane == 0 && vsh->r_head < r_pub) {
                    base = atomicAdd(&sh.r_head, static_cast<uint32_t>(n_empty));
                    got = (base < r_pub) ? min(static_cast<uint32_t>(n_empty), r_pub - base) : 0u;
                }
                base = __shfl_sync(full, base, 0);
                got = __shfl_sync(full, got, 0);
                if (!live && rank < static_cast<int>(got)) {
                    const Entry q = ring[(base + rank) & ring_mask];
                    P::from_entry(q, trk);
                    g.seed(q.key);
                    ev_cur = q.ev;
                    st.clear();
                    live = true;
                }
                const int need = n_empty - static_cast<int>(got);
                if (need > 0 && inp) {
                    unsigned long long ub = 0;
                    if (lane == 0) {
                        ub = atomicAdd(a.next_work, static_cast<unsigned long long>(need));
                        if (ub + need >= a.n_events) vsh->input_left = 0;
                    }
                    ub = __shfl_sync(full, ub, 0);
                    const uint64_t unit = ub + static_cast<uint64_t>(rank - static_cast<int>(got));
                    if (!live && rank >= static_cast<int>(got) && unit < a.n_events) {
                        if constexpr (kQueue) {
                            const QPhonon q = p.queue[unit];
                            if (q.ev != kQEmpty) {
                                ev_cur = q.ev;
                                g.seed(q.key);
                                P::template from_queue<kKin>(L, q, trk);
                                st.clear();
                                live = true;
                            }
                        } else {
                            const uint32_t ev = p.unit_event[unit];
                            ev_cur = ev;
                            const uint64_t j = unit - a.ph_off[ev];
                            g.seed(seed_key ^ mix64(((a.first_event + ev) << 20) | j));
                            P::from_primary(a.ph[unit], trk);
                            st.clear();
                            live = true;
                        }
                    }
                }
            }
            if (__ballot_sync(full, live) == 0) {  // nothing more until the boundary
                if (lane == 0) atomicAdd(&sh.n_dry, 1u);
                break;
            }
            if (live) {
                const int outcome = P::template step<kKin, kSur>(L, cdf, D, s_hot, trk, g, st, ev_cur, sink);
                if (outcome != kStepOn) {
                    sink_unit(&a, ev_cur, st);
                    live = false;
                }
            }
        }
        __syncthreads();
        // ---- film phase -------------------------------------------------------------
        const uint32_t n_film = min(vsh->f_tail, p.film_cap);
        if (n_film) sm_film_phase<P, kSur, kKin>(&L, &D, &a, film, n_film, &sh, ring, ring_mask, r_floor, &err);
        __syncthreads();
        // ---- boundary: publish what the phases appended ---------------------------------
        if (threadIdx.x == 0) {
            if (sh.r_head > sh.r_pub) sh.r_head = sh.r_pub;  // claims past the published entries were void
            sh.r_pub = sh.r_tail;
            sh.f_tail = 0;
            sh.f_next = 0;
            sh.n_dry = 0;
        }
        __syncthreads();
        if (__syncthreads_or(err != 0)) break;  // an overflow: the call reruns with more room
        if (!__syncthreads_or(live || vsh->r_pub != vsh->r_head || vsh->input_left != 0)) break;
    }
    if (err) atomicOr(a.err, err);
}

// Adjoint of the hit-time histogram: the batched transport with per-track scores. Bin
// weights (dLoss/dh_b) and the block's histogram live in shared memory; the histogram is
// added to the global FP64 bins once per block.
__global__ void __launch_bounds__(128, 6) k_adjoint_fp32(const __grid_constant__ FLat L,
                                                         const __grid_constant__ Detector D,
                                                         const __grid_constant__ RunArgs a,
                                                         const __grid_constant__ AdjArgs adj,
                                                         const uint32_t* __restrict__ unit_event) {
    __shared__ float s_w[kAdjMaxBins];
    __shared__ float s_hist[kAdjMaxBins];
    for (int b = threadIdx.x; b < kAdjMaxBins; b += blockDim.x) {
        s_w[b] = (b < adj.n_bins) ? adj.bin_w[b] : 0.0f;
        s_hist[b] = 0.0f;
    }
    __syncthreads();
    batched_loop<true>(L, D, a, unit_event, nullptr, adj, s_w, s_hist);
    __syncthreads();
    for (int b = threadIdx.x; b < adj.n_bins; b += blockDim.x)
        if (s_hist[b] != 0.0f) atomicAdd(adj.hist + b, static_cast<double>(s_hist[b]));
}

}  // namespace

cudaError_t launch_unit_event(const uint64_t* ph_off, uint64_t n_events, uint32_t* unit_event, cudaStream_t s) {
    k_unit_event<<<4 * 148, 128, 0, s>>>(ph_off, n_events, unit_event);
    return cudaGetLastError();
}

cudaError_t launch_batched_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const uint32_t* unit_event, int grid, int block, cudaStream_t s) {
    const FLat f = make_flat(L, cdf_f, D);
    if (L.kin_mode != kKinOctahedral) {  // Exact / Bilinear kinematics (no surrogate tables)
        if (a.film) k_batched_fp32<true, false, true, 1><<<grid, block, 0, s>>>(f, D, a, unit_event);
        else if (a.ev_sink) k_batched_fp32<true, false, false, 1><<<grid, block, 0, s>>>(f, D, a, unit_event);
        else k_batched_fp32<false, false, false, 1><<<grid, block, 0, s>>>(f, D, a, unit_event);
    } else if (a.film) {
        if (a.surrogate) k_batched_fp32<true, true, true><<<grid, block, 0, s>>>(f, D, a, unit_event);
        else k_batched_fp32<true, false, true><<<grid, block, 0, s>>>(f, D, a, unit_event);
    } else if (a.ev_sink) {
        if (a.surrogate) k_batched_fp32<true, true><<<grid, block, 0, s>>>(f, D, a, unit_event);
        else k_batched_fp32<true, false><<<grid, block, 0, s>>>(f, D, a, unit_event);
    } else {
        if (a.surrogate) k_batched_fp32<false, true><<<grid, block, 0, s>>>(f, D, a, unit_event);
        else k_batched_fp32<false, false><<<grid, block, 0, s>>>(f, D, a, unit_event);
    }
    return cudaGetLastError();
}

cudaError_t batched_fp32_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_batched_fp32<false, false>, block, 0);
}

size_t batched_stack_entry_bytes() { return sizeof(GFTrack); }

cudaError_t launch_film_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                             const FilmRec* film, uint64_t n_film, int grid, int block, cudaStream_t s) {
    const FLat f = make_flat(L, cdf_f, D);
    if (L.kin_mode != kKinOctahedral) k_film_fp32<false, 1><<<grid, block, 0, s>>>(f, D, a, film, n_film);
    else if (a.surrogate) k_film_fp32<true><<<grid, block, 0, s>>>(f, D, a, film, n_film);
    else k_film_fp32<false><<<grid, block, 0, s>>>(f, D, a, film, n_film);
    return cudaGetLastError();
}

cudaError_t film_fp32_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_film_fp32<false>, block, 0);
}

cudaError_t launch_queue_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                              const QPhonon* queue, int grid, int block, cudaStream_t s) {
    const FLat f = make_flat(L, cdf_f, D);
    if (L.kin_mode != kKinOctahedral) {
        if (a.film) k_queue_fp32<false, true, 1><<<grid, block, 0, s>>>(f, D, a, queue);
        else k_queue_fp32<false, false, 1><<<grid, block, 0, s>>>(f, D, a, queue);
    } else if (a.film) {
        if (a.surrogate) k_queue_fp32<true, true><<<grid, block, 0, s>>>(f, D, a, queue);
        else k_queue_fp32<false, true><<<grid, block, 0, s>>>(f, D, a, queue);
    } else {
        if (a.surrogate) k_queue_fp32<true><<<grid, block, 0, s>>>(f, D, a, queue);
        else k_queue_fp32<false><<<grid, block, 0, s>>>(f, D, a, queue);
    }
    return cudaGetLastError();
}

cudaError_t launch_pool_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a, void* ring,
                             uint32_t ring_cap, void* film, const uint32_t* unit_event, const QPhonon* queue,
                             int stage_tables, int grid, int block, cudaStream_t s) {
    if (ring_cap < 64 || (ring_cap & (ring_cap - 1u)) != 0) return cudaErrorInvalidValue;  // indexed by masking
    const FLat f = make_flat(L, cdf_f, D);
    PoolArgs p;
    p.ring = static_cast<PoolPh*>(ring);
    p.film = static_cast<FilmRec*>(film);
    p.ring_cap = ring_cap;
    p.unit_event = unit_event;
    p.queue = queue;
    p.stage_tables = stage_tables;
    if (queue) {
        if (L.kin_mode != kKinOctahedral) k_pool_fp32<false, 1, true><<<grid, block, 0, s>>>(f, D, a, p);
        else if (a.surrogate) k_pool_fp32<true, 0, true><<<grid, block, 0, s>>>(f, D, a, p);
        else k_pool_fp32<false, 0, true><<<grid, block, 0, s>>>(f, D, a, p);
    } else {
        if (L.kin_mode != kKinOctahedral) k_pool_fp32<false, 1><<<grid, block, 0, s>>>(f, D, a, p);
        else if (a.surrogate) k_pool_fp32<true><<<grid, block, 0, s>>>(f, D, a, p);
        else k_pool_fp32<false><<<grid, block, 0, s>>>(f, D, a, p);
    }
    return cudaGetLastError();
}

template <class P, bool kSur, int kKin = 0, bool kQueue = false>
cudaError_t sm_launch(const typename P::Lat& L, const Detector& D, const RunArgs& a, const SmPoolArgs& p, int grid,
                      cudaStream_t s) {
    constexpr int kDyn = SmShape<P::kThreads>::kDynBytes;
    if (kDyn > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k_sm_pool<P, kSur, kKin, kQueue>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, kDyn);
        if (e != cudaSuccess) return e;
    }
    k_sm_pool<P, kSur, kKin, kQueue><<<grid, P::kThreads, kDyn, s>>>(L, D, a, p);
    return cudaGetLastError();
}

cudaError_t launch_sm_pool_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a, void* ring,
                                uint32_t ring_cap, void* film, uint32_t film_cap, const uint32_t* unit_event,
                                const QPhonon* queue, int stage_tables, int fp64, int grid, cudaStream_t s) {
    // the ring is indexed by masking: its capacity must be a power of two
    const uint32_t threads = static_cast<uint32_t>(fp64 ? PF64::kThreads : PF32::kThreads);
    if (ring_cap < 2u * threads || (ring_cap & (ring_cap - 1u)) != 0 || film_cap < 4u * threads)
        return cudaErrorInvalidValue;
    SmPoolArgs p;
    p.ring = ring;
    p.film = film;
    p.ring_cap = ring_cap;
    p.film_cap = film_cap;
    p.film_trigger = film_cap > 2u * threads ? film_cap - 2u * threads : film_cap / 2u;
    p.unit_event = unit_event;
    p.queue = queue;
    p.stage_tables = stage_tables;
    if (fp64) {  // the FP64 comparison form: phonon batches, every kinematics mode, full cascades
        if (queue || a.surrogate) return cudaErrorInvalidValue;
        return sm_launch<PF64, false>(L, D, a, p, grid, s);
    }
    const FLat f = make_flat(L, cdf_f, D);
    if (queue) {
        if (L.kin_mode != kKinOctahedral) return sm_launch<PF32, false, 1, true>(f, D, a, p, grid, s);
        if (a.surrogate) return sm_launch<PF32, true, 0, true>(f, D, a, p, grid, s);
        if (flat_identity_orientation(f)) return sm_launch<PF32, false, 2, true>(f, D, a, p, grid, s);
        return sm_launch<PF32, false, 0, true>(f, D, a, p, grid, s);
    }
    if (L.kin_mode != kKinOctahedral) return sm_launch<PF32, false, 1>(f, D, a, p, grid, s);
    if (a.surrogate) return sm_launch<PF32, true>(f, D, a, p, grid, s);
    if (flat_identity_orientation(f)) return sm_launch<PF32, false, 2>(f, D, a, p, grid, s);
    return sm_launch<PF32, false>(f, D, a, p, grid, s);
}

size_t sm_pool_entry_bytes(int fp64) { return fp64 ? sizeof(PoolPh64) : sizeof(PoolPh); }
size_t sm_pool_film_bytes(int fp64) { return fp64 ? sizeof(FilmRec64) : sizeof(FilmRec); }

int sm_pool_threads(int fp64) { return fp64 ? PF64::kThreads : PF32::kThreads; }

cudaError_t pool_fp32_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_pool_fp32<false>, block, 0);
}

size_t pool_ring_entry_bytes() { return sizeof(PoolPh); }
size_t pool_film_bytes_per_warp() { return sizeof(FilmRec) * kPoolFilmCap; }

cudaError_t launch_adjoint_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const AdjArgs& adj, const uint32_t* unit_event, int grid, int block, cudaStream_t s) {
    k_adjoint_fp32<<<grid, block, 0, s>>>(make_flat(L, cdf_f, D), D, a, adj, unit_event);
    return cudaGetLastError();
}

cudaError_t adjoint_fp32_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_adjoint_fp32, block, 0);
}

size_t adjoint_stack_entry_bytes() { return sizeof(GFTrackA); }

}  // namespace cmpmc_gpu
