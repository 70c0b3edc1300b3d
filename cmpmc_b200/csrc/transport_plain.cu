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
#include <algorithm>
#include <cstring>
#include <string>

#include "device.cuh"
#include "internal.hpp"

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
    MeshView mesh;
    int32_t tet_hint;  // walk hint of this device thread, kept across carriers and events
    MeshView2 mesh2;
    int32_t tri_hint;  // the same for the 2D mesh
    unsigned err;
    KBuf refl;
    double* kwork;

    __device__ bool pop(Track& t) {
        if (err) return false;  // a stack overflowed: the event is rerun with more room
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
        if (err) return false;
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
    // DetectorModel::electric_field_at (engine.hpp:151-155)
    __device__ V3 field(V3 p, Charge&) {
        if (mesh.tet) return mesh_field(mesh, p, tet_hint);
        if (mesh2.tri) return mesh2_field(mesh2, p, tri_hint);
        return field_value;
    }
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
    ctx.mesh = D.mesh;
    ctx.tet_hint = 0;
    ctx.mesh2 = D.mesh2;
    ctx.tri_hint = 0;
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

// ---- allocation-free variant ---------------------------------------------------------
//
// cmpmc_gpu_run_events_noalloc runs the plain FP64 transport for phonon-only events
// without allocating device memory, for callers that cannot call cudaMalloc (code inside a
// framework whose caching allocator owns the device memory, code with a fixed memory
// budget, or latency-critical loops where an allocation may block or fail). The caller
// passes every input and output as device memory; the per-thread LIFO stacks and the
// run's counters live in the file-scope array below, and the lattice tables in another.
// Both are part of the loaded module: every GPU that loads this library holds them
// (about 32 MiB) until the process exits.
//
// Hits are written in two passes of the same deterministic transport: the first counts
// each event's hits into hit_offsets, an in-place scan turns the counts into offsets, and
// the second writes every hit at its final position. No staging buffer is needed, at the
// cost of running the transport twice.
//
// The first call on a device resolves the arrays' device addresses (cudaGetSymbolAddress)
// and uploads the tables; that first call must come before any stream capture. Every call
// shares the arrays and clears the counters it needs, so calls whose work overlaps on the
// GPU (two streams, two host threads) race and must be serialized by the caller.
namespace cmpmc_gpu {
namespace {

constexpr int kNoAllocBlocks = 32;
constexpr int kNoAllocThreads = 128;
constexpr int kNoAllocSlots = kNoAllocBlocks * kNoAllocThreads;  // 4096 device threads
constexpr int kNoAllocStackCap = 64;                              // pushed tracks per event
constexpr size_t kNoAllocStackBytes = sizeof(GTrack) * kNoAllocSlots * kNoAllocStackCap;

struct NoAllocCounters {
    unsigned long long next_work;
    unsigned err;
    unsigned pad;
    cmpmc_sim_stats total;
};

// scratch: [per-thread stacks | counters]
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocStackBytes + sizeof(NoAllocCounters)];
// octahedral table (float4 [3][256][256]) followed by the two decay CDF tables
static __device__ __align__(256) unsigned char
    g_noalloc_tables[3 * kNOct * kNOct * sizeof(OctEntry) + 2 * kNCdf * sizeof(double)];

struct NoAllocCtx {
    const cmpmc_phonon_track* init;
    uint64_t n_init;
    GTrack* stk;
    uint32_t n_stk;
    unsigned err;
    uint32_t n_hits;
    cmpmc_sensor_hit* out;  // nullptr in the counting pass
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
        if (n_stk < kNoAllocStackCap) stk[n_stk++] = pack_track(t);
        else err |= kErrPhononStack;
    }
    __device__ void hit(const Hit& h, int channel) {
        const uint32_t local = n_hits++;
        if (!out) return;
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
        out[local] = r;
    }
};

// pass 0 counts hits into hit_offsets[ev + 1]; pass 1 writes them at hit_offsets[ev]
__global__ void __launch_bounds__(kNoAllocThreads)
    k_plain_fp64_noalloc(const Lattice L, const Detector D, uint64_t n_events, const uint64_t* __restrict__ rng_state,
                         const double* __restrict__ injected, const uint64_t* __restrict__ ph_off,
                         const cmpmc_phonon_track* __restrict__ ph, cmpmc_sim_stats* __restrict__ ev_stats,
                         uint64_t* __restrict__ hit_offsets, cmpmc_sensor_hit* __restrict__ hits, int pass,
                         GTrack* stacks, NoAllocCounters* cnt) {
    const uint64_t slot = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    double refl_buf[kKaplanCap];
    double kwork[4 * kKaplanCap];
    NoAllocCtx ctx;
    ctx.stk = stacks + slot * kNoAllocStackCap;
    ctx.refl.d = refl_buf;
    ctx.refl.n = 0;
    ctx.kwork = kwork;
    unsigned err = 0;
    for (;;) {
        const unsigned long long ev = atomicAdd(&cnt->next_work, 1ull);
        if (ev >= n_events) break;
        ctx.init = ph + ph_off[ev];
        ctx.n_init = ph_off[ev + 1] - ph_off[ev];
        ctx.n_stk = 0;
        ctx.n_hits = 0;
        ctx.err = 0;
        ctx.out = pass ? hits + hit_offsets[ev] : nullptr;
        Rng rng;
        for (int k = 0; k < 4; ++k) rng.s[k] = rng_state[4 * ev + k];
        EvStats st;
        memset(&st, 0, sizeof(st));
        transport_phonons(L, D, ctx, st, rng);
        if (pass == 0) {
            stats_from_event(st, injected[ev], ev_stats[ev]);
            hit_offsets[ev + 1] = ctx.n_hits;
        }
        err |= ctx.err;
    }
    if (err) atomicOr(&cnt->err, err);
}

// hit_offsets[1..n] hold counts; turn them into offsets in place (hit_offsets[0] = 0)
__global__ void __launch_bounds__(1024) k_scan_inplace(uint64_t* __restrict__ a, uint64_t n) {
    __shared__ uint64_t part[1024];
    const int t = threadIdx.x;
    const uint64_t chunk = (n + 1023) / 1024;
    const uint64_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    uint64_t s = 0;
    for (uint64_t i = lo; i < hi; ++i) s += a[i + 1];
    part[t] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const uint64_t v = (t >= d) ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint64_t run = part[t] - s;
    for (uint64_t i = lo; i < hi; ++i) {
        run += a[i + 1];
        a[i + 1] = run;
    }
    if (t == 0) a[0] = 0;
}

// run totals over the per-event records: one block of kTotThreads threads, each summing a
// contiguous slice in event order, then a fixed-order pairwise tree over the slices (the
// result does not depend on scheduling; it may differ from a serial sum in the last bits)
constexpr int kTotThreads = 128;  // 128 x 208 B of shared memory
__device__ __forceinline__ void add_stats(cmpmc_sim_stats& t, const cmpmc_sim_stats& s) {
    t.total_steps += s.total_steps;
    t.isotope_scatters += s.isotope_scatters;
    t.polycrystal_scatters += s.polycrystal_scatters;
    t.decays_L_to_TT += s.decays_L_to_TT;
    t.decays_L_to_LT += s.decays_L_to_LT;
    t.surface_refls += s.surface_refls;
    t.surface_downconversions += s.surface_downconversions;
    t.sensor_hits += s.sensor_hits;
    t.killed_tracks += s.killed_tracks;
    t.total_injected_eV += s.total_injected_eV;
    t.total_deposited_eV += s.total_deposited_eV;
    t.escaped_or_killed_eV += s.escaped_or_killed_eV;
}
__global__ void __launch_bounds__(kTotThreads)
    k_total_noalloc(const cmpmc_sim_stats* __restrict__ ev, uint64_t n, NoAllocCounters* cnt) {
    __shared__ cmpmc_sim_stats part[kTotThreads];
    const int t = threadIdx.x;
    const uint64_t chunk = (n + kTotThreads - 1) / kTotThreads;
    const uint64_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    cmpmc_sim_stats acc;
    memset(&acc, 0, sizeof(acc));
    for (uint64_t i = lo; i < hi; ++i) add_stats(acc, ev[i]);
    part[t] = acc;
    __syncthreads();
    for (int d = kTotThreads / 2; d > 0; d >>= 1) {
        if (t < d) add_stats(part[t], part[t + d]);
        __syncthreads();
    }
    if (t == 0) cnt->total = part[0];
}

struct NoAllocDevice {
    bool ready = false;
    void* scratch = nullptr;
    void* tables = nullptr;
    uint64_t uploaded = 0;  // id of the lattice whose tables are in g_noalloc_tables (0: none)
};
NoAllocDevice g_noalloc_dev[64];

}  // namespace

}  // namespace cmpmc_gpu

using namespace cmpmc_gpu;

extern "C" int cmpmc_gpu_run_events_noalloc(const cmpmc_lattice* lat, const cmpmc_detector* det, int device,
                                            uint64_t n_events, const uint64_t* rng_state, const double* injected_eV,
                                            const uint64_t* phonon_offsets, const cmpmc_phonon_track* phonons,
                                            cmpmc_sim_stats* event_stats, uint64_t* hit_offsets,
                                            cmpmc_sensor_hit* hits, uint64_t hit_capacity, void* stream,
                                            cmpmc_sim_stats* total, uint64_t* n_hits) {
    if (!lat || !det || !total || !n_hits || device < 0 || device >= 64) return CMPMC_ERR_INVALID;
    if (n_events > 0 && (!rng_state || !injected_eV || !phonon_offsets || !phonons || !event_stats || !hit_offsets))
        return CMPMC_ERR_INVALID;
    if (n_events > (1ull << 31)) return CMPMC_ERR_INVALID;
    // only the octahedral table is staged in the module array: the Exact and Bilinear modes
    // read tables that live in host memory here, so they are refused before any device work
    if (lat->view.kin_mode != kKinOctahedral) return CMPMC_ERR_INVALID;
    std::string err;
    if (validate_config(lat->cfg, *det, false, err) != CMPMC_OK) return CMPMC_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return CMPMC_ERR_NO_DEVICE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NoAllocDevice& nd = g_noalloc_dev[device];
    if (!nd.ready) {
        // once per device, with the device current: device addresses of the module arrays
        if (cudaGetSymbolAddress(&nd.scratch, g_noalloc_scratch) != cudaSuccess) return CMPMC_ERR_CUDA;
        if (cudaGetSymbolAddress(&nd.tables, g_noalloc_tables) != cudaSuccess) return CMPMC_ERR_CUDA;
        nd.ready = true;
    }
    const size_t oct_bytes = lat->oct.size() * sizeof(OctEntry);
    if (nd.uploaded != lat->id) {
        if (cudaMemcpyAsync(nd.tables, lat->oct.data(), oct_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(static_cast<char*>(nd.tables) + oct_bytes, lat->cdf_lt.data(), kNCdf * sizeof(double),
                            cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(static_cast<char*>(nd.tables) + oct_bytes + kNCdf * sizeof(double), lat->cdf_tt.data(),
                            kNCdf * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
            return CMPMC_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return CMPMC_ERR_CUDA;
        nd.uploaded = lat->id;
    }
    Lattice L = lat->view;
    L.stiff = nullptr;
    L.bil = nullptr;
    L.oct = static_cast<const OctEntry*>(nd.tables);
    L.cdf_lt = reinterpret_cast<const double*>(static_cast<char*>(nd.tables) + oct_bytes);
    L.cdf_tt = L.cdf_lt + kNCdf;
    const Detector D = detector_view(*det);
    GTrack* stacks = static_cast<GTrack*>(nd.scratch);
    NoAllocCounters* cnt = reinterpret_cast<NoAllocCounters*>(static_cast<char*>(nd.scratch) + kNoAllocStackBytes);
    NoAllocCounters hc;
    std::memset(&hc, 0, sizeof(hc));
    if (n_events == 0) {
        *total = hc.total;
        *n_hits = 0;
        return (!hit_offsets || cudaMemsetAsync(hit_offsets, 0, 8, s) == cudaSuccess) &&
                       cudaStreamSynchronize(s) == cudaSuccess
                   ? CMPMC_OK
                   : CMPMC_ERR_CUDA;
    }
    const int grid = static_cast<int>(std::min<uint64_t>(kNoAllocBlocks, (n_events + kNoAllocThreads - 1) / kNoAllocThreads));
    for (int pass = 0; pass < 2; ++pass) {
        if (cudaMemsetAsync(cnt, 0, 16, s) != cudaSuccess) return CMPMC_ERR_CUDA;  // next_work, err
        k_plain_fp64_noalloc<<<grid, kNoAllocThreads, 0, s>>>(L, D, n_events, rng_state, injected_eV, phonon_offsets,
                                                             phonons, event_stats, hit_offsets, hits, pass, stacks, cnt);
        if (cudaGetLastError() != cudaSuccess) return CMPMC_ERR_CUDA;
        if (pass == 0) {
            k_scan_inplace<<<1, 1024, 0, s>>>(hit_offsets, n_events);
            k_total_noalloc<<<1, kTotThreads, 0, s>>>(event_stats, n_events, cnt);
            if (cudaGetLastError() != cudaSuccess) return CMPMC_ERR_CUDA;
            if (cudaMemcpyAsync(&hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaMemcpyAsync(n_hits, hit_offsets + n_events, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return CMPMC_ERR_CUDA;
            *total = hc.total;
            if (hc.err) return CMPMC_ERR_CAPACITY;  // an event pushed more than kNoAllocStackCap tracks
            if (*n_hits > hit_capacity || (*n_hits > 0 && !hits)) return CMPMC_ERR_CAPACITY;
            if (*n_hits == 0) break;
        }
    }
    if (cudaMemcpyAsync(&hc.err, &cnt->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CMPMC_ERR_CUDA;
    return hc.err ? CMPMC_ERR_CAPACITY : CMPMC_OK;
}
