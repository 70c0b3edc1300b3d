// transport_plain.cu -- the plain FP64 form: one event per device thread, bit-exact
// event streams.
//
// Each thread takes the next event from a global work counter, restores the event's
// post-generator xoshiro256** state, and runs transport_charges then transport_phonons
// (engine.hpp:192-380, 403-582) exactly as run_events does on the CPU
// (parallel.hpp:102-114). The LIFO stacks of pushed tracks live in a per-thread
// region of global memory; the event's initial tracks are read in place as the bottom
// of the stack. The Kaplan cascade buffers are per-thread local arrays.
//
// This translation unit is compiled with --fmad=false: every + - * / rounds exactly as
// on x86-64 SSE, so only transcendental ulps can differ from the CPU.
#include "device.cuh"

namespace cmpmc_gpu {

namespace {

struct PlainCtx {
    // phonon stack = initial records [ph0, ph0 + n_init) under the pushed region
    const cmpmc_phonon_track* init;
    uint64_t n_init;
    GTrack* stk;
    uint32_t n_stk;
    uint32_t cap;
    // charge stack
    const cmpmc_charge_track* cinit;
    uint64_t n_cinit;
    GCharge* cstk;
    uint32_t n_cstk;
    uint32_t ccap;
    // hits
    cmpmc_sensor_hit* hit_stage;
    uint64_t* hit_key;
    uint64_t hit_cap;
    unsigned long long* hit_count;
    int keep_hits;
    uint64_t ev;
    uint32_t n_hits;
    V3 field_value;
    unsigned err;
    KBuf refl;
    double* kwork;

    __device__ bool pop(Track& t) {
        if (n_stk > 0) {
            t = unpack_track(stk[--n_stk]);
            return true;
        }
        if (n_init > 0) {
            t = track_from_input(init[--n_init]);
            return true;
        }
        return false;
    }
    __device__ void push(const Track& t) {
        if (n_stk < cap) stk[n_stk++] = pack_track(t);
        else err |= kErrPhononStack;
    }
    __device__ bool pop_charge(Charge& c) {
        if (n_cstk > 0) {
            const GCharge& g = cstk[--n_cstk];
            c.pos = v3(g.px, g.py, g.pz);
            c.p = v3(g.qx, g.qy, g.qz);
            c.ekin = g.ekin; c.t = g.t; c.w = g.w;
            c.valley = g.valley;
            c.type = g.type;
            return true;
        }
        if (n_cinit > 0) {
            c = charge_from_input(cinit[--n_cinit]);
            return true;
        }
        return false;
    }
    __device__ void push_charge(const Charge& c) {
        if (n_cstk < ccap) {
            GCharge g;
            g.px = c.pos.x; g.py = c.pos.y; g.pz = c.pos.z;
            g.qx = c.p.x; g.qy = c.p.y; g.qz = c.p.z;
            g.ekin = c.ekin; g.t = c.t; g.w = c.w;
            g.valley = c.valley;
            g.type = c.type;
            cstk[n_cstk++] = g;
        } else {
            err |= kErrChargeStack;
        }
    }
    __device__ V3 field(V3, Charge&) { return field_value; }
    __device__ void hit(const Hit& h, int channel) {
        const uint32_t local = n_hits++;
        if (!keep_hits) return;
        const unsigned long long idx = atomicAdd(hit_count, 1ull);
        if (idx >= hit_cap) return;
        cmpmc_sensor_hit r;
        r.pos[0] = h.pos.x; r.pos[1] = h.pos.y; r.pos[2] = h.pos.z;
        r.time = h.t;
        r.edep = h.edep;
        r.incident_energy = h.incident;
        r.surface_id = static_cast<uint8_t>(h.surf);
        r.excitation = static_cast<uint8_t>(h.excitation);
        r.mode = static_cast<uint8_t>(h.mode);
        r._pad = 0;
        r.channel_id = channel;
        hit_stage[idx] = r;
        hit_key[idx] = (ev << 32) | local;
    }
};

__global__ void __launch_bounds__(128) k_plain_fp64(const Lattice L, const Detector D, const RunArgs a) {
    const uint64_t slot = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    PlainCtx ctx;
    ctx.hit_stage = a.hit_stage;
    ctx.hit_key = a.hit_key;
    ctx.hit_cap = a.hit_cap;
    ctx.hit_count = a.hit_count;
    ctx.keep_hits = a.keep_hits;
    ctx.stk = a.stack + slot * a.stack_cap;
    ctx.cap = a.stack_cap;
    ctx.cstk = a.cstack + slot * a.cstack_cap;
    ctx.ccap = a.cstack_cap;
    ctx.refl.d = refl_buf;
    ctx.refl.n = 0;
    ctx.kwork = kwork;
    ctx.field_value = D.e_field;
    for (;;) {
        const unsigned long long ev = atomicAdd(a.next_work, 1ull);
        if (ev >= a.n_events) break;
        const uint64_t p0 = a.ph_off[ev], p1 = a.ph_off[ev + 1];
        ctx.init = a.ph + p0;
        ctx.n_init = p1 - p0;
        ctx.n_stk = 0;
        if (a.ch_off) {
            const uint64_t c0 = a.ch_off[ev], c1 = a.ch_off[ev + 1];
            ctx.cinit = a.ch + c0;
            ctx.n_cinit = c1 - c0;
        } else {
            ctx.cinit = nullptr;
            ctx.n_cinit = 0;
        }
        ctx.n_cstk = 0;
        ctx.ev = ev;
        ctx.n_hits = 0;
        ctx.err = 0;
        Rng rng;
        for (int k = 0; k < 4; ++k) rng.s[k] = a.rng_state[4 * ev + k];
        EvStats st;
        memset(&st, 0, sizeof(st));
        if (ctx.n_cinit > 0) transport_charges(L, D, ctx, st, rng);
        if (ctx.n_init > 0 || ctx.n_stk > 0) transport_phonons(L, D, ctx, st, rng);
        stats_from_event(st, a.injected[ev], a.ev_stats[ev]);
        a.ev_nhits[ev] = a.keep_hits ? ctx.n_hits : 0;
        if (ctx.err) atomicOr(a.err, ctx.err);
    }
}

}  // namespace

__global__ void k_math_check(uint64_t n, const double* __restrict__ x, double* __restrict__ out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        out[3 * i + 0] = crmath::log(x[i]);
        out[3 * i + 1] = crmath::sin(x[i]);
        out[3 * i + 2] = crmath::cos(x[i]);
    }
}

cudaError_t launch_math_check(uint64_t n, const double* x, double* out) {
    k_math_check<<<148, 256>>>(n, x, out);
    return cudaGetLastError();
}

cudaError_t launch_plain_fp64(const Lattice& L, const Detector& D, const RunArgs& a, int grid, int block,
                              cudaStream_t s) {
    k_plain_fp64<<<grid, block, 0, s>>>(L, D, a);
    return cudaGetLastError();
}

cudaError_t plain_fp64_occupancy(int block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_plain_fp64, block, 0);
}

}  // namespace cmpmc_gpu
