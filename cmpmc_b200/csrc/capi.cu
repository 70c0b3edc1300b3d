// capi.cu -- device context and the run_events entry point of the C ABI.
//
// cmpmc_gpu_run_events is the device half of run_events (transport/parallel.hpp:76-148):
// the caller has already run the generator on the host (one Rng::for_stream(seed, ev)
// per event) and passes each event's post-generator Rng state with its initial stacks.
// The call uploads them (unless they are already on the device), runs the transport
// kernel, then the merge kernels (hit_offsets scan, hit scatter into event order, stats
// reduction), and returns RunResult's content. Buffers grow on demand and are reused
// across calls; a capacity overflow reruns the (deterministic) transport with more room.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"
#include "internal.hpp"

using namespace cmpmc_gpu;

namespace {

thread_local std::string g_create_error;
thread_local int g_create_status = CMPMC_OK;

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 8, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 8, 256);
        cudaError_t e = cudaMallocHost(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct Counters {
    unsigned long long hit_count;
    unsigned long long next_work;
    unsigned err;
    unsigned pad;
};

}  // namespace

struct cmpmc_gpu_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cmpmc_crystal_config cfg{};
    cmpmc_detector det{};
    Lattice L{};
    Detector D{};
    DevBuf tables;  // oct LUT + CDF tables
    DevBuf mesh;    // MeshTet records of the attached field mesh
    DevBuf kin;     // stiffness tensor and bilinear table of the lattice's kinematics mode
    int tpb = 128;
    int bps = 0;  // 0: occupancy-derived
    uint32_t stack_cap = 1024;        // plain form: tracks per device thread
    uint32_t stack_cap_batched = 256;  // batched form: one primary's lineage per thread
    uint32_t cstack_cap = 64;
    uint64_t hit_cap = 0;
    DevBuf in_rng, in_inj, in_phoff, in_ph, in_choff, in_ch;
    DevBuf stack, cstack, hit_stage, hit_key, counters, ev_stats, ev_nhits, offsets, hits_out, total;
    DevBuf unit_event, ev_offsets, ev_stats2, partials;  // batched form: unit -> event map, event offsets / stats
    DevBuf adj_prim, adj_hist, adj_w, adj_partials, adj_sums;  // adjoint: per-primary rows, bins, reductions
    DevBuf mesh32;                                      // FP32 mesh records (batched charge form)
    DevBuf mesh2, mesh2_32;                             // 2D field mesh records, FP64 and FP32
    DevBuf pads[3];                                     // electrode masks of the three surfaces
    DevBuf lut[3];                                      // Kaplan surrogate tables of the films
    bool lut_ready = false;
    DevBuf queue, resume_a, resume_b, ccounters, carrier_event, cursor;  // batched charge form
    DevBuf rel;                                         // batched charge release records
    DevBuf part_plans, part_counts;                     // device partition: plans, per-deposit counts
    DevBuf film_a, queue_b;                             // wavefront split: film entries, second phonon queue
    uint64_t film_cap = 1ull << 22;                     // film entries per phase (64 B each)
    uint32_t phase_steps = 0;                           // steps a track takes per transport phase (0: any)
    int pool = 1;                                       // batched phonon form: 1 SM-phase pool, 2 warp pool,
                                                        // 0 host-driven rounds, 3 SM-phase pool in FP64
    int stage_tables = 1;                               // pool forms: decay CDF tables staged in shared memory
    uint32_t pool_ring_cap = 1024;                      // pending phonons per warp (warp pool)
    uint32_t sm_ring_cap = 1u << 17;                    // pending phonons per block (SM-phase pool)
    uint32_t sm_film_cap = 8192;                        // film records per block and phase (SM-phase pool)
    DevBuf pool_ring, pool_film;                        // warp pool: per-warp rings and film buffers
    uint64_t queue_cap = 1ull << 24;                    // Luke-phonon queue entries (64 B each)
    // CUDA-graph replay of the batched phonon call (cmpmc_gpu_configure_graph)
    bool graph_enabled = false;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<uint64_t> graph_key;
    uint64_t graph_hits_cap = 0;                        // hit records the captured merge can write
    uint64_t graph_stage_cap = 0;                       // hit staging records of the captured transport
    int graph_launches = 0;
    const float* cdf_f = nullptr;              // FP32 copies of the decay tables (in `tables`)
    HostBuf h_hits, h_offsets, h_evstats, h_total, h_counters;
    cudaEvent_t e_start = nullptr, e_k0 = nullptr, e_k1 = nullptr, e_end = nullptr;
    std::string last_error;
    int last_status = CMPMC_OK;
};

namespace {

int fail(cmpmc_gpu_ctx* ctx, int status, const std::string& msg) {
    if (ctx) {
        ctx->last_error = msg;
        ctx->last_status = status;
    } else {
        g_create_error = msg;
        g_create_status = status;
    }
    return status;
}

int cuda_fail(cmpmc_gpu_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, CMPMC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                                     \
    do {                                                   \
        cudaError_t _e = (call);                           \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); \
    } while (0)

void drop_graph(cmpmc_gpu_ctx* ctx) {
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    ctx->graph_exec = nullptr;
    ctx->graph_key.clear();
}

// The call signature a captured graph is valid for: the descriptor's pointers and sizes (the
// number of phonon records too: it is read from the device offsets and baked into the launch),
// the context's launch configuration, and the address and capacity of every device and host
// buffer a captured call touches (a call of another form may grow, and so move, a shared
// buffer without recapturing: the key then no longer matches and the next call runs eagerly
// and recaptures).
std::vector<uint64_t> graph_key_of(const cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* d, uint64_t n_ph) {
    std::vector<uint64_t> k = {d->n_events, n_ph, d->first_event, reinterpret_cast<uint64_t>(d->rng_state),
                               reinterpret_cast<uint64_t>(d->injected_eV), reinterpret_cast<uint64_t>(d->phonon_offsets),
                               reinterpret_cast<uint64_t>(d->phonons), static_cast<uint64_t>(d->keep_hits), d->seed,
                               static_cast<uint64_t>(d->want_event_stats), static_cast<uint64_t>(d->kaplan_surrogate),
                               static_cast<uint64_t>(d->form), static_cast<uint64_t>(ctx->tpb),
                               static_cast<uint64_t>(ctx->bps), ctx->stack_cap_batched, ctx->hit_cap,
                               static_cast<uint64_t>(ctx->pool), static_cast<uint64_t>(ctx->stage_tables),
                               ctx->sm_ring_cap, ctx->sm_film_cap, ctx->pool_ring_cap};
    for (const DevBuf* b : {&ctx->stack, &ctx->cstack, &ctx->hit_stage, &ctx->hit_key, &ctx->counters, &ctx->ev_stats,
                            &ctx->ev_nhits, &ctx->offsets, &ctx->hits_out, &ctx->total, &ctx->unit_event,
                            &ctx->ev_offsets, &ctx->ev_stats2, &ctx->partials, &ctx->cursor, &ctx->pool_ring,
                            &ctx->pool_film}) {
        k.push_back(reinterpret_cast<uint64_t>(b->p));
        k.push_back(b->cap);
    }
    for (const HostBuf* b : {&ctx->h_counters, &ctx->h_total}) {
        k.push_back(reinterpret_cast<uint64_t>(b->p));
        k.push_back(b->cap);
    }
    return k;
}

// Builds (once per context) the Kaplan surrogate table of every film on the host
// (KaplanSurrogateLUT, reference seed 1337) and copies it to the device
int ensure_surrogate(cmpmc_gpu_ctx* ctx) {
    if (ctx->lut_ready) return CMPMC_OK;
    for (int i = 0; i < 3; ++i) {
        Surface& sf = ctx->D.surf[i];
        sf.lut_abs = nullptr;
        sf.lut_off = nullptr;
        sf.lut_refl = nullptr;
        if (!ctx->det.surfaces[i].has_film) continue;
        cmpmc_kaplan_lut* t = nullptr;
        const int st = cmpmc_kaplan_surrogate_create(&ctx->det.surfaces[i].film, 1337ull, &t);
        if (st != CMPMC_OK) return fail(ctx, st, "surrogate table");
        const size_t b_abs = t->abs.size() * 4, b_off = t->off.size() * 4, b_refl = std::max<size_t>(t->refl.size(), 1) * 4;
        const size_t o_off = (b_abs + 255) / 256 * 256, o_refl = o_off + (b_off + 255) / 256 * 256;
        cudaError_t e = ctx->lut[i].ensure(o_refl + b_refl);
        char* base = ctx->lut[i].as<char>();
        if (e == cudaSuccess) e = cudaMemcpy(base, t->abs.data(), b_abs, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(base + o_off, t->off.data(), b_off, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !t->refl.empty())
            e = cudaMemcpy(base + o_refl, t->refl.data(), t->refl.size() * 4, cudaMemcpyHostToDevice);
        cmpmc_kaplan_surrogate_destroy(t);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "copy surrogate table");
        sf.lut_abs = reinterpret_cast<const float*>(base);
        sf.lut_off = reinterpret_cast<const uint32_t*>(base + o_off);
        sf.lut_refl = reinterpret_cast<const float*>(base + o_refl);
    }
    ctx->lut_ready = true;
    return CMPMC_OK;
}

// ---- the persistent pool launches (SM-phase pool or warp pool) ----------------------
bool sm_pool(const cmpmc_gpu_ctx* ctx) { return ctx->pool == 1 || ctx->pool == 3; }
int pool_fp64(const cmpmc_gpu_ctx* ctx) { return ctx->pool == 3 ? 1 : 0; }

// grid of a pool launch over `units` units: one block per SM (SM-phase pool; 512 threads in
// FP32, 768 in FP64), or the occupancy's 128-thread blocks (warp pool), never more than the
// units can start
int pool_grid(cmpmc_gpu_ctx* ctx, uint64_t units, uint64_t* grid) {
    if (sm_pool(ctx)) {
        const uint64_t per = static_cast<uint64_t>(sm_pool_threads(pool_fp64(ctx)));
        *grid = std::max<uint64_t>(1, std::min<uint64_t>(ctx->num_sms, (units + per - 1) / per));
        return CMPMC_OK;
    }
    int bps = ctx->bps;
    if (!bps) {
        CK(pool_fp32_occupancy(128, &bps), "occupancy");
        bps = std::max(bps, 1);
    }
    *grid = std::max<uint64_t>(1, std::min<uint64_t>(static_cast<uint64_t>(ctx->num_sms) * bps, (units + 127) / 128));
    return CMPMC_OK;
}

// ring and film buffers for launches of up to `grid` blocks
int ensure_pool_buffers(cmpmc_gpu_ctx* ctx, uint64_t grid) {
    if (sm_pool(ctx)) {
        CK(ctx->pool_ring.ensure(grid * ctx->sm_ring_cap * sm_pool_entry_bytes(pool_fp64(ctx))), "alloc block rings");
        CK(ctx->pool_film.ensure(grid * ctx->sm_film_cap * sm_pool_film_bytes(pool_fp64(ctx))), "alloc film buffers");
    } else {
        CK(ctx->pool_ring.ensure(grid * 4 * ctx->pool_ring_cap * pool_ring_entry_bytes()), "alloc warp rings");
        CK(ctx->pool_film.ensure(grid * 4 * pool_film_bytes_per_warp()), "alloc film buffers");
    }
    return CMPMC_OK;
}

cudaError_t launch_pool(cmpmc_gpu_ctx* ctx, const RunArgs& a, uint64_t grid, const QPhonon* queue, cudaStream_t s) {
    const uint32_t* ue = ctx->unit_event.as<uint32_t>();
    if (sm_pool(ctx))
        return launch_sm_pool_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ctx->pool_ring.p, ctx->sm_ring_cap, ctx->pool_film.p,
                                   ctx->sm_film_cap, ue, queue, ctx->stage_tables, pool_fp64(ctx),
                                   static_cast<int>(grid), s);
    return launch_pool_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ctx->pool_ring.p, ctx->pool_ring_cap, ctx->pool_film.p, ue,
                            queue, ctx->stage_tables, static_cast<int>(grid), 128, s);
}

// after an overflow of a pool's ring or film buffer: more room for the rerun
void grow_pool(cmpmc_gpu_ctx* ctx, unsigned err) {
    if (err & kErrQueue) {
        if (sm_pool(ctx)) ctx->sm_ring_cap = std::min<uint32_t>(ctx->sm_ring_cap * 4, 1u << 24);
        else ctx->pool_ring_cap = std::min<uint32_t>(ctx->pool_ring_cap * 4, 1u << 20);
    }
    if ((err & kErrFilmQueue) && sm_pool(ctx)) ctx->sm_film_cap = std::min<uint32_t>(ctx->sm_film_cap * 2, 1u << 20);
}

// Device counters of the batched charge form (reset per phase except next_carrier)
struct ChargeCounters {
    unsigned long long q_tail, resume_next, n_resume_out, next_carrier, rel_tail;
    unsigned long long film_tail, reemit_tail;  // wavefront split inside the queue phases
};

// The batched FP32 form of events with charges: phase 0 transports the generator's
// phonons; then charge phases (carriers drift and queue their Luke phonons) alternate
// with queue phases (the queued phonons are transported) until every carrier is done.
// All units add their counters and hits to per-event sinks, merged at the end. A stack
// or hit-staging overflow reruns the whole call with more room (every unit owns its
// substream, so the rerun reproduces the same hits).
int run_charges_batched(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* d, RunArgs& a, uint64_t n, uint64_t n_ph,
                        uint64_t n_ch, int& launches, Counters& hc, float& kms, uint64_t& n_hits,
                        uint64_t*& ev_offsets, cmpmc_sim_stats*& ev_stats) {
    cudaStream_t s = ctx->stream;
    if (pool_fp64(ctx)) return fail(ctx, CMPMC_ERR_INVALID, "the FP64 pool form runs phonon-only batches");
    const int tpb = ctx->tpb;
    int bps_ph = ctx->bps, bps_ch = ctx->bps;
    if (!bps_ph) {
        CK(batched_fp32_occupancy(tpb, &bps_ph), "occupancy");
        bps_ph = std::max(bps_ph, 1);
    }
    if (!bps_ch) {
        CK(charges_fp32_occupancy(tpb, &bps_ch), "occupancy");
        bps_ch = std::max(bps_ch, 1);
    }
    const uint64_t grid_ph = static_cast<uint64_t>(ctx->num_sms) * bps_ph;
    const uint64_t grid_ch = std::max<uint64_t>(
        1, std::min<uint64_t>(static_cast<uint64_t>(ctx->num_sms) * bps_ch, (n_ch + tpb - 1) / tpb));
    const uint64_t resume_cap = grid_ch * tpb * 9;  // a carrier and up to 8 knock-ons per thread
    uint64_t q_cap = std::max<uint64_t>(ctx->queue_cap, 64);
    // collections with a release mode (BulkDebye / ElectrodeFilm) wait in a record buffer
    // for the release kernel of their round: at most every carrier and knock-on of the call
    const bool release = ctx->det.charge_release != 0;
    const uint64_t rel_cap = release ? std::max<uint64_t>(4 * n_ch, 1024) + resume_cap : 0;

    CK(ctx->ev_stats2.ensure(std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats)), "alloc event stats");
    CK(ctx->ev_nhits.ensure(std::max<uint64_t>(n, 1) * 8), "alloc event hit counts");
    CK(ctx->ev_offsets.ensure((n + 1) * 8), "alloc event offsets");
    CK(ctx->cursor.ensure(std::max<uint64_t>(n, 1) * 8), "alloc event cursors");
    CK(ctx->counters.ensure(sizeof(Counters)), "alloc counters");
    CK(ctx->ccounters.ensure(sizeof(ChargeCounters)), "alloc charge counters");
    CK(ctx->total.ensure(sizeof(cmpmc_sim_stats)), "alloc totals");
    CK(ctx->partials.ensure(kReducePartials * sizeof(cmpmc_sim_stats)), "alloc partial totals");
    CK(ctx->h_counters.ensure(sizeof(Counters) + sizeof(ChargeCounters)), "alloc host counters");
    if (release) CK(ctx->rel.ensure(rel_cap * sizeof(ReleaseRec)), "alloc release records");
    CK(ctx->resume_a.ensure(resume_cap * sizeof(QCharge)), "alloc parked carriers");
    CK(ctx->resume_b.ensure(resume_cap * sizeof(QCharge)), "alloc parked carriers");
    CK(ctx->carrier_event.ensure(std::max<uint64_t>(n_ch, 1) * 4), "alloc carrier map");
    if (n_ph) CK(ctx->unit_event.ensure(n_ph * 4), "alloc unit map");
    CK(launch_carrier_event(a.ch_off, n, ctx->carrier_event.as<uint32_t>(), s), "carrier map");
    ++launches;
    if (n_ph) {
        CK(launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), "unit map");
        ++launches;
    }
    a.ev_sink = 1;
    a.ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
    a.ev_nhits = ctx->ev_nhits.as<uint64_t>();
    Counters* dc = ctx->counters.as<Counters>();
    a.hit_count = &dc->hit_count;
    a.next_work = &dc->next_work;
    a.err = &dc->err;
    ChargeCounters* cc = ctx->ccounters.as<ChargeCounters>();
    ChargeArgs ca;
    std::memset(&ca, 0, sizeof(ca));
    ca.n_carriers = n_ch;
    ca.carrier_event = ctx->carrier_event.as<uint32_t>();
    ca.carrier_seed = mix64(d->seed ^ 0x2545f4914f6cdd1dULL);
    ca.q_tail = &cc->q_tail;
    ca.resume_next = &cc->resume_next;
    ca.n_resume_out = &cc->n_resume_out;
    ca.next_carrier = &cc->next_carrier;
    ca.resume_cap = resume_cap;
    ca.rel = release ? ctx->rel.as<ReleaseRec>() : nullptr;
    ca.rel_cap = rel_cap;
    ca.rel_tail = &cc->rel_tail;

    // wavefront split (the default batched form): the phonon phases end a track at film
    // entry; film phases run the cascades and queue the re-emissions, as in the phonon-only
    // split form, until the round's phonons are done
    // warp pool (the default batched form): each phonon phase (the generator's phonons, then
    // each round's queued Luke and released phonons) is one persistent pool launch with its
    // film cascades inside; the host-driven rounds (configure_pool 0) split them instead
    const bool pool = d->form == CMPMC_FORM_BATCHED_FP32 && ctx->pool != 0;
    const bool split = d->form == CMPMC_FORM_BATCHED_FP32 && !pool;
    uint64_t grid_pool = 1;
    if (pool) {
        const int st = pool_grid(ctx, ~0ull >> 1, &grid_pool);
        if (st != CMPMC_OK) return st;
    }
    int bps_f = ctx->bps;
    if (split && !bps_f) {
        CK(film_fp32_occupancy(tpb, &bps_f), "occupancy");
        bps_f = std::max(bps_f, 1);
    }
    const uint64_t grid_f = static_cast<uint64_t>(ctx->num_sms) * std::max(bps_f, 1);
    a.film_tail = &cc->film_tail;
    a.reemit_tail = &cc->reemit_tail;
    a.phase_steps = 0;

    uint64_t hit_cap = ctx->hit_cap;
    if (!hit_cap) hit_cap = std::max<uint64_t>(1u << 20, (n_ph + n_ch) * 64);
    uint32_t& stack_cap = ctx->stack_cap_batched;
    const uint64_t slots = grid_ph * tpb;
    char* hbuf = ctx->h_counters.as<char>();
    for (int attempt = 0;; ++attempt) {
        if (!d->keep_hits) hit_cap = 1;
        // split phases: film entries and re-emissions of one phase get their own capacity
        // (f_cap entries each); the Luke-queue buffer doubles as a re-emission queue, so it
        // holds max(q_cap, f_cap) entries while the Luke reservations stay below q_cap
        const uint64_t f_cap = split ? std::max<uint64_t>(q_cap, ctx->film_cap) : 0;
        CK(ctx->queue.ensure(std::max(q_cap, f_cap) * sizeof(QPhonon)), "alloc Luke-phonon queue");
        ca.queue = ctx->queue.as<QPhonon>();
        ca.q_cap = q_cap;
        bool split_over = false;
        if (split) {
            CK(ctx->queue_b.ensure(f_cap * sizeof(QPhonon)), "alloc re-emission queue");
            CK(ctx->film_a.ensure(f_cap * sizeof(FilmRec)), "alloc film queue");
            a.film = ctx->film_a.as<FilmRec>();
            a.film_cap = f_cap;
            a.reemit = ctx->queue_b.as<QPhonon>();
            a.reemit_cap = f_cap;
        }
        // After a transport launch that wrote its film entries to a.film and read `q_read`:
        // film phases and transport phases alternate until no phonon is left. q_read is
        // free again; a.reemit is where the film phase appends.
        auto drain = [&](QPhonon* q_read) -> int {
            QPhonon* q_free = q_read;
            for (;;) {
                CK(cudaMemcpyAsync(hbuf + sizeof(Counters), cc, sizeof(ChargeCounters), cudaMemcpyDeviceToHost, s),
                   "copy counters");
                CK(cudaStreamSynchronize(s), "transport phase");
                ChargeCounters h = *reinterpret_cast<const ChargeCounters*>(hbuf + sizeof(Counters));
                if (h.film_tail > f_cap || h.reemit_tail > f_cap) {
                    split_over = true;
                    return CMPMC_OK;
                }
                if (h.film_tail > 0) {
                    CK(launch_film_fp32(ctx->L, ctx->cdf_f, ctx->D, a, a.film, h.film_tail,
                                        static_cast<int>(std::min<uint64_t>(grid_f, (h.film_tail + tpb - 1) / tpb)),
                                        tpb, s),
                       "film launch");
                    ++launches;
                    CK(cudaMemcpyAsync(hbuf + sizeof(Counters), cc, sizeof(ChargeCounters), cudaMemcpyDeviceToHost,
                                       s),
                       "copy counters");
                    CK(cudaStreamSynchronize(s), "film phase");
                    h = *reinterpret_cast<const ChargeCounters*>(hbuf + sizeof(Counters));
                    if (h.reemit_tail > f_cap) {
                        split_over = true;
                        return CMPMC_OK;
                    }
                }
                const uint64_t n_r = h.reemit_tail;
                if (n_r == 0) return CMPMC_OK;
                QPhonon* q_in = a.reemit;
                a.reemit = q_free;
                q_free = q_in;
                CK(cudaMemsetAsync(&cc->film_tail, 0, 2 * sizeof(unsigned long long), s), "memset counters");
                CK(cudaMemsetAsync(&dc->next_work, 0, sizeof(unsigned long long), s), "memset work counter");
                a.n_events = n_r;
                CK(launch_queue_fp32(ctx->L, ctx->cdf_f, ctx->D, a, q_in,
                                     static_cast<int>(std::min<uint64_t>(grid_ph, (n_r + tpb - 1) / tpb)), tpb, s),
                   "queue launch");
                ++launches;
            }
        };
        if (pool) {
            const int st = ensure_pool_buffers(ctx, grid_pool);
            if (st != CMPMC_OK) return st;
        }
        // one pool launch over `units` units: the primaries (queue == nullptr) or a queue
        auto pool_phase = [&](uint64_t units, const QPhonon* queue) -> int {
            CK(cudaMemsetAsync(&dc->next_work, 0, sizeof(unsigned long long), s), "memset work counter");
            a.n_events = units;
            uint64_t grid = 1;
            const int st = pool_grid(ctx, units, &grid);
            if (st != CMPMC_OK) return st;
            CK(launch_pool(ctx, a, std::min(grid, grid_pool), queue, s), "pool launch");
            ++launches;
            return CMPMC_OK;
        };
        CK(ctx->stack.ensure(slots * stack_cap * batched_stack_entry_bytes()), "alloc phonon stacks");
        CK(ctx->hit_stage.ensure(hit_cap * sizeof(cmpmc_sensor_hit)), "alloc hit staging");
        CK(ctx->hit_key.ensure(hit_cap * 8), "alloc hit keys");
        a.stack = ctx->stack.as<GTrack>();
        a.stack_cap = stack_cap;
        a.hit_stage = ctx->hit_stage.as<cmpmc_sensor_hit>();
        a.hit_key = ctx->hit_key.as<uint64_t>();
        a.hit_cap = hit_cap;
        CK(cudaMemsetAsync(ctx->ev_stats2.p, 0, std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats), s), "memset");
        CK(cudaMemsetAsync(ctx->ev_nhits.p, 0, std::max<uint64_t>(n, 1) * 8, s), "memset");
        CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s), "memset counters");
        CK(cudaMemsetAsync(ctx->ccounters.p, 0, sizeof(ChargeCounters), s), "memset counters");
        CK(cudaEventRecord(ctx->e_k0, s), "event");
        // phase 0: the generator's phonons
        if (n_ph && pool) {
            const int st = pool_phase(n_ph, nullptr);
            if (st != CMPMC_OK) return st;
        } else if (n_ph) {
            a.n_events = n_ph;
            CK(launch_batched_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ctx->unit_event.as<uint32_t>(),
                                   static_cast<int>(std::min<uint64_t>(grid_ph, (n_ph + tpb - 1) / tpb)), tpb, s),
               "phonon launch");
            ++launches;
            if (split) {
                const int st = drain(ctx->queue.as<QPhonon>());  // the Luke queue is still free here
                if (st != CMPMC_OK) return st;
            }
        }
        // charge / queue phases
        QCharge* r_in = ctx->resume_a.as<QCharge>();
        QCharge* r_out = ctx->resume_b.as<QCharge>();
        uint64_t n_resume = 0, carriers_started = 0;
        for (int round = 0; !split_over; ++round) {
            CK(cudaMemsetAsync(ctx->queue.p, 0xff, q_cap * sizeof(QPhonon), s), "memset queue");
            CK(cudaMemsetAsync(&cc->q_tail, 0, 3 * sizeof(unsigned long long), s), "memset counters");
            CK(cudaMemsetAsync(&cc->rel_tail, 0, sizeof(unsigned long long), s), "memset counters");
            ca.resume_in = r_in;
            ca.n_resume_in = n_resume;
            ca.resume_out = r_out;
            CK(launch_charges_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ca, static_cast<int>(grid_ch), tpb, s),
               "charge launch");
            ++launches;
            CK(cudaMemcpyAsync(hbuf + sizeof(Counters), cc, sizeof(ChargeCounters), cudaMemcpyDeviceToHost, s),
               "copy counters");
            CK(cudaMemcpyAsync(hbuf, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s), "copy counters");
            CK(cudaStreamSynchronize(s), "charge kernel");
            ChargeCounters hcc = *reinterpret_cast<const ChargeCounters*>(hbuf + sizeof(Counters));
            // a pool phase that overflowed its ring: the call reruns with more room, so the
            // remaining rounds are not run
            if (pool && (reinterpret_cast<const Counters*>(hbuf)->err & (kErrQueue | kErrFilmQueue)) != 0) break;
            if (release && hcc.rel_tail > 0) {
                // the round's collections release their energy into the phonon queue
                if (hcc.rel_tail > rel_cap) return fail(ctx, CMPMC_ERR_CAPACITY, "release-record buffer overflow");
                CK(launch_release_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ca, hcc.rel_tail,
                                       static_cast<int>(std::min<uint64_t>(grid_ph, (hcc.rel_tail + tpb - 1) / tpb)),
                                       tpb, s),
                   "release launch");
                ++launches;
                CK(cudaMemcpyAsync(hbuf + sizeof(Counters), cc, sizeof(ChargeCounters), cudaMemcpyDeviceToHost, s),
                   "copy counters");
                CK(cudaStreamSynchronize(s), "release kernel");
                hcc = *reinterpret_cast<const ChargeCounters*>(hbuf + sizeof(Counters));
            }
            const uint64_t n_q = std::min<uint64_t>(hcc.q_tail, q_cap);
            if (n_q && pool) {
                const int st = pool_phase(n_q, ca.queue);
                if (st != CMPMC_OK) return st;
            } else if (n_q && !split_over) {
                CK(cudaMemsetAsync(&dc->next_work, 0, sizeof(unsigned long long), s), "memset work counter");
                a.n_events = n_q;
                if (split) {
                    a.reemit = ctx->queue_b.as<QPhonon>();
                    CK(cudaMemsetAsync(&cc->film_tail, 0, 2 * sizeof(unsigned long long), s), "memset counters");
                }
                CK(launch_queue_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ca.queue,
                                     static_cast<int>(std::min<uint64_t>(grid_ph, (n_q + tpb - 1) / tpb)), tpb, s),
                   "queue launch");
                ++launches;
                if (split) {
                    const int st = drain(ca.queue);
                    if (st != CMPMC_OK) return st;
                }
            }
            if (split_over) break;
            const uint64_t started = std::min<uint64_t>(hcc.next_carrier, n_ch);
            const uint64_t parked = hcc.n_resume_out;
            if (parked > resume_cap) return fail(ctx, CMPMC_ERR_CAPACITY, "parked-carrier buffer overflow");
            if (parked == 0 && started >= n_ch) break;
            if (n_q == 0 && parked >= n_resume && started == carriers_started)
                return fail(ctx, CMPMC_ERR_DEVICE, "charge phases make no progress (queue too small)");
            n_resume = parked;
            carriers_started = started;
            std::swap(r_in, r_out);
        }
        CK(cudaEventRecord(ctx->e_k1, s), "event");
        CK(cudaMemcpyAsync(hbuf, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s), "copy counters");
        CK(cudaStreamSynchronize(s), "transport kernels");
        hc = *reinterpret_cast<const Counters*>(hbuf);
        CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
        const bool stack_over = (hc.err & kErrPhononStack) != 0;
        const bool hits_over = d->keep_hits && hc.hit_count > hit_cap;
        const bool queue_over = (hc.err & kErrRelease) != 0;  // released phonons did not fit the queue
        const bool ring_over = pool && (hc.err & (kErrQueue | kErrFilmQueue)) != 0;  // a pool's ring or film buffer
        split_over = split_over || (!pool && (hc.err & (kErrQueue | kErrFilmQueue)) != 0);
        if (!stack_over && !hits_over && !queue_over && !split_over && !ring_over) break;
        if (ring_over) grow_pool(ctx, hc.err);
        if (attempt >= 8) return fail(ctx, CMPMC_ERR_CAPACITY, "device stack, hit or queue overflow persists");
        if (stack_over) stack_cap = std::min<uint32_t>(stack_cap * 8, 1u << 20);
        if (hits_over) hit_cap = hc.hit_count + hc.hit_count / 16 + 1024;
        if (queue_over) {
            q_cap *= 8;
            ctx->queue_cap = std::max<uint64_t>(ctx->queue_cap, q_cap);
        }
        if (split_over) {  // only the split phases' buffers grow (64 B per entry and buffer)
            if (f_cap >= (1ull << 28))
                return fail(ctx, CMPMC_ERR_CAPACITY, "film / re-emission phase exceeds 2^28 entries");
            ctx->film_cap = std::max<uint64_t>(ctx->film_cap, 4 * f_cap);
        }
        hc.err = 0;
    }
    a.film = nullptr;
    a.reemit = nullptr;
    if (d->keep_hits) ctx->hit_cap = std::max<uint64_t>(ctx->hit_cap, hit_cap);
    if (hc.err) return fail(ctx, CMPMC_ERR_DEVICE, "transport kernels reported error word " + std::to_string(hc.err));
    n_hits = d->keep_hits ? hc.hit_count : 0;
    CK(ctx->hits_out.ensure(std::max<uint64_t>(n_hits, 1) * sizeof(cmpmc_sensor_hit)), "alloc hits");
    CK(cudaMemsetAsync(ctx->cursor.p, 0, std::max<uint64_t>(n, 1) * 8, s), "memset cursors");
    ev_offsets = ctx->ev_offsets.as<uint64_t>();
    ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
    a.n_events = n;
    CK(launch_sink_finish(a, n, ev_offsets, ctx->cursor.as<unsigned long long>(), ctx->hits_out.as<cmpmc_sensor_hit>(),
                          n_hits, ctx->total.as<cmpmc_sim_stats>(), ctx->partials.as<cmpmc_sim_stats>(), s, &launches),
       "merge kernels");
    return CMPMC_OK;
}

// The batched phonon form with the wavefront split: phase 0 transports the generator's
// phonons until each one dies or reaches an active film (queued as a FilmRec); then film
// phases (cascades, hits, re-emitted phonons queued as QPhonon) alternate with transport
// phases over the re-emitted phonons until both queues are empty. Every unit owns its
// substream, so the phases' order does not change any track; units add to per-event sinks.
// A queue, stack or hit-staging overflow reruns the whole call with more room.
int run_split_batched(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* d, RunArgs& a, uint64_t n, uint64_t n_ph,
                      int& launches, Counters& hc, float& kms, uint64_t& n_hits, uint64_t*& ev_offsets,
                      cmpmc_sim_stats*& ev_stats) {
    cudaStream_t s = ctx->stream;
    const int tpb = ctx->tpb;
    int bps_ph = ctx->bps, bps_f = ctx->bps;
    if (!bps_ph) {
        CK(batched_fp32_occupancy(tpb, &bps_ph), "occupancy");
        bps_ph = std::max(bps_ph, 1);
    }
    if (!bps_f) {
        CK(film_fp32_occupancy(tpb, &bps_f), "occupancy");
        bps_f = std::max(bps_f, 1);
    }
    const uint64_t grid_ph = static_cast<uint64_t>(ctx->num_sms) * bps_ph;
    const uint64_t grid_f = static_cast<uint64_t>(ctx->num_sms) * bps_f;
    CK(ctx->ev_stats2.ensure(std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats)), "alloc event stats");
    CK(ctx->ev_nhits.ensure(std::max<uint64_t>(n, 1) * 8), "alloc event hit counts");
    CK(ctx->ev_offsets.ensure((n + 1) * 8), "alloc event offsets");
    CK(ctx->cursor.ensure(std::max<uint64_t>(n, 1) * 8), "alloc event cursors");
    CK(ctx->counters.ensure(sizeof(Counters)), "alloc counters");
    CK(ctx->ccounters.ensure(sizeof(ChargeCounters)), "alloc phase counters");
    CK(ctx->total.ensure(sizeof(cmpmc_sim_stats)), "alloc totals");
    CK(ctx->partials.ensure(kReducePartials * sizeof(cmpmc_sim_stats)), "alloc partial totals");
    CK(ctx->h_counters.ensure(sizeof(Counters) + sizeof(ChargeCounters)), "alloc host counters");
    if (n_ph) CK(ctx->unit_event.ensure(n_ph * 4), "alloc unit map");
    if (n_ph) {
        CK(launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), "unit map");
        ++launches;
    }
    a.ev_sink = 1;
    a.ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
    a.ev_nhits = ctx->ev_nhits.as<uint64_t>();
    Counters* dc = ctx->counters.as<Counters>();
    a.hit_count = &dc->hit_count;
    a.next_work = &dc->next_work;
    a.err = &dc->err;
    ChargeCounters* pc = ctx->ccounters.as<ChargeCounters>();  // q_tail: re-emissions, resume_next: film entries
    a.reemit_tail = &pc->q_tail;
    a.film_tail = &pc->resume_next;
    char* hbuf = ctx->h_counters.as<char>();

    uint64_t hit_cap = ctx->hit_cap;
    if (!hit_cap) hit_cap = std::max<uint64_t>(1u << 20, n_ph * 32);
    uint32_t& stack_cap = ctx->stack_cap_batched;
    const uint64_t slots = grid_ph * tpb;
    for (int attempt = 0;; ++attempt) {
        if (!d->keep_hits) hit_cap = 1;
        // a primary's lineage (decay daughters included) reaches a film a few times per round
        ctx->film_cap = std::max<uint64_t>(ctx->film_cap, std::min<uint64_t>(8 * n_ph, 1ull << 26));
        const uint64_t q_cap = std::max<uint64_t>(ctx->queue_cap, 64), f_cap = std::max<uint64_t>(ctx->film_cap, 64);
        CK(ctx->queue.ensure(q_cap * sizeof(QPhonon)), "alloc phonon queue");
        CK(ctx->queue_b.ensure(q_cap * sizeof(QPhonon)), "alloc phonon queue");
        CK(ctx->film_a.ensure(f_cap * sizeof(FilmRec)), "alloc film queue");
        CK(ctx->stack.ensure(slots * stack_cap * batched_stack_entry_bytes()), "alloc phonon stacks");
        CK(ctx->hit_stage.ensure(hit_cap * sizeof(cmpmc_sensor_hit)), "alloc hit staging");
        CK(ctx->hit_key.ensure(hit_cap * 8), "alloc hit keys");
        a.stack = ctx->stack.as<GTrack>();
        a.stack_cap = stack_cap;
        a.hit_stage = ctx->hit_stage.as<cmpmc_sensor_hit>();
        a.hit_key = ctx->hit_key.as<uint64_t>();
        a.hit_cap = hit_cap;
        a.reemit_cap = q_cap;
        a.film_cap = f_cap;
        a.film = ctx->film_a.as<FilmRec>();
        a.phase_steps = ctx->phase_steps;
        // the transport phase reads q_in and parks long tracks in q_out; the film phase
        // appends its re-emissions to q_out; then the queues swap
        QPhonon* q_in = ctx->queue.as<QPhonon>();
        QPhonon* q_out = ctx->queue_b.as<QPhonon>();
        CK(cudaMemsetAsync(ctx->ev_stats2.p, 0, std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats), s), "memset");
        CK(cudaMemsetAsync(ctx->ev_nhits.p, 0, std::max<uint64_t>(n, 1) * 8, s), "memset");
        CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s), "memset counters");
        CK(cudaMemsetAsync(ctx->ccounters.p, 0, sizeof(ChargeCounters), s), "memset counters");
        CK(cudaEventRecord(ctx->e_k0, s), "event");
        // phase 0: the generator's phonons
        a.reemit = q_out;
        if (n_ph) {
            a.n_events = n_ph;
            CK(launch_batched_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ctx->unit_event.as<uint32_t>(),
                                   static_cast<int>(std::min<uint64_t>(grid_ph, (n_ph + tpb - 1) / tpb)), tpb, s),
               "phonon launch");
            ++launches;
        }
        bool overflow = false;
        for (int round = 0;; ++round) {
            CK(cudaMemcpyAsync(hbuf + sizeof(Counters), pc, sizeof(ChargeCounters), cudaMemcpyDeviceToHost, s),
               "copy counters");
            CK(cudaStreamSynchronize(s), "transport phase");
            const ChargeCounters h1 = *reinterpret_cast<const ChargeCounters*>(hbuf + sizeof(Counters));
            if (h1.resume_next > f_cap || h1.q_tail > q_cap) {
                overflow = true;
                break;
            }
            const uint64_t n_f = h1.resume_next;
            if (n_f > 0) {
                // film phase: cascades of the queued film entries, re-emissions appended to q_out
                CK(launch_film_fp32(ctx->L, ctx->cdf_f, ctx->D, a, a.film, n_f,
                                    static_cast<int>(std::min<uint64_t>(grid_f, (n_f + tpb - 1) / tpb)), tpb, s),
                   "film launch");
                ++launches;
                CK(cudaMemcpyAsync(hbuf + sizeof(Counters), pc, sizeof(ChargeCounters), cudaMemcpyDeviceToHost, s),
                   "copy counters");
                CK(cudaStreamSynchronize(s), "film phase");
            }
            const ChargeCounters h2 = *reinterpret_cast<const ChargeCounters*>(hbuf + sizeof(Counters));
            if (h2.q_tail > q_cap) {
                overflow = true;
                break;
            }
            const uint64_t n_q = h2.q_tail;
            if (n_q == 0) break;
            // transport phase over q_out (parked tracks and re-emissions)
            std::swap(q_in, q_out);
            a.reemit = q_out;
            CK(cudaMemsetAsync(&pc->q_tail, 0, 2 * sizeof(unsigned long long), s), "memset counters");
            CK(cudaMemsetAsync(&dc->next_work, 0, sizeof(unsigned long long), s), "memset work counter");
            a.n_events = n_q;
            CK(launch_queue_fp32(ctx->L, ctx->cdf_f, ctx->D, a, q_in,
                                 static_cast<int>(std::min<uint64_t>(grid_ph, (n_q + tpb - 1) / tpb)), tpb, s),
               "queue launch");
            ++launches;
        }
        CK(cudaEventRecord(ctx->e_k1, s), "event");
        CK(cudaMemcpyAsync(hbuf, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s), "copy counters");
        CK(cudaStreamSynchronize(s), "transport kernels");
        hc = *reinterpret_cast<const Counters*>(hbuf);
        CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
        const bool stack_over = (hc.err & kErrPhononStack) != 0;
        const bool hits_over = d->keep_hits && hc.hit_count > hit_cap;
        overflow = overflow || (hc.err & (kErrQueue | kErrFilmQueue)) != 0;
        if (!stack_over && !hits_over && !overflow) break;
        if (attempt >= 6) return fail(ctx, CMPMC_ERR_CAPACITY, "device queue, stack or hit buffer overflow persists");
        if (stack_over) stack_cap = std::min<uint32_t>(stack_cap * 8, 1u << 20);
        if (hits_over) hit_cap = hc.hit_count + hc.hit_count / 16 + 1024;
        if (overflow) {
            ctx->queue_cap *= 2;
            ctx->film_cap *= 2;
        }
        hc.err = 0;
    }
    a.film = nullptr;
    if (d->keep_hits) ctx->hit_cap = std::max<uint64_t>(ctx->hit_cap, hit_cap);
    if (hc.err) return fail(ctx, CMPMC_ERR_DEVICE, "transport kernels reported error word " + std::to_string(hc.err));
    n_hits = d->keep_hits ? hc.hit_count : 0;
    CK(ctx->hits_out.ensure(std::max<uint64_t>(n_hits, 1) * sizeof(cmpmc_sensor_hit)), "alloc hits");
    CK(cudaMemsetAsync(ctx->cursor.p, 0, std::max<uint64_t>(n, 1) * 8, s), "memset cursors");
    ev_offsets = ctx->ev_offsets.as<uint64_t>();
    ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
    a.n_events = n;
    CK(launch_sink_finish(a, n, ev_offsets, ctx->cursor.as<unsigned long long>(), ctx->hits_out.as<cmpmc_sensor_hit>(),
                          n_hits, ctx->total.as<cmpmc_sim_stats>(), ctx->partials.as<cmpmc_sim_stats>(), s, &launches),
       "merge kernels");
    return CMPMC_OK;
}

// The batched FP32 form of phonon-only events as one persistent launch (k_pool_fp32): every
// warp refills its lanes from its own ring of pending phonons and from the batch's
// primaries, queues film entries in its own buffer and runs them 32 at a time, and appends
// re-emissions and daughters to its ring. The host only launches, reads the counters once
// and merges; a ring, stack or hit-staging overflow reruns the call with more room (every
// unit owns its substream, so the rerun reproduces the same hits).
int run_pool_batched(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* d, RunArgs& a, uint64_t n, uint64_t n_ph,
                     int& launches, Counters& hc, float& kms, uint64_t& n_hits, uint64_t*& ev_offsets,
                     cmpmc_sim_stats*& ev_stats) {
    cudaStream_t s = ctx->stream;
    if (pool_fp64(ctx) && a.surrogate)
        return fail(ctx, CMPMC_ERR_INVALID, "the FP64 pool form runs the full film cascades (no surrogate)");
    // ---- CUDA-graph replay: the same device-resident batch again (the persistent transport
    // launch with its counter resets, unit map and merge as one graph launch) ---------------
    const bool graph_ok = ctx->graph_enabled && n > 0 && n_ph > 0 && d->inputs_on_device && d->outputs_on_device;
    if (graph_ok && ctx->graph_exec && ctx->graph_key == graph_key_of(ctx, d, n_ph)) {
        CK(cudaGraphLaunch(ctx->graph_exec, s), "graph launch");
        CK(cudaStreamSynchronize(s), "graph");
        hc = *ctx->h_counters.as<Counters>();
        const bool over = hc.err != 0 || (d->keep_hits && (hc.hit_count > ctx->graph_stage_cap ||
                                                          hc.hit_count > ctx->graph_hits_cap));
        if (!over) {
            CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
            n_hits = d->keep_hits ? hc.hit_count : 0;
            ev_offsets = ctx->ev_offsets.as<uint64_t>();
            ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
            launches += ctx->graph_launches;
            return CMPMC_OK;
        }
        drop_graph(ctx);  // a ring, film buffer or hit buffer overflowed: rerun eagerly with more room
        if (hc.err & (kErrQueue | kErrFilmQueue)) grow_pool(ctx, hc.err);
        hc = Counters{};
    }
    uint64_t grid = 1;
    {
        const int st = pool_grid(ctx, n_ph, &grid);
        if (st != CMPMC_OK) return st;
    }
    CK(ctx->ev_stats2.ensure(std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats)), "alloc event stats");
    CK(ctx->ev_nhits.ensure(std::max<uint64_t>(n, 1) * 8), "alloc event hit counts");
    CK(ctx->ev_offsets.ensure((n + 1) * 8), "alloc event offsets");
    CK(ctx->cursor.ensure(std::max<uint64_t>(n, 1) * 8), "alloc event cursors");
    CK(ctx->counters.ensure(sizeof(Counters)), "alloc counters");
    CK(ctx->total.ensure(sizeof(cmpmc_sim_stats)), "alloc totals");
    CK(ctx->partials.ensure(kReducePartials * sizeof(cmpmc_sim_stats)), "alloc partial totals");
    CK(ctx->h_counters.ensure(sizeof(Counters)), "alloc host counters");
    if (n_ph) {
        CK(ctx->unit_event.ensure(n_ph * 4), "alloc unit map");
        CK(launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), "unit map");
        ++launches;
    }
    a.ev_sink = 1;
    a.ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
    a.ev_nhits = ctx->ev_nhits.as<uint64_t>();
    Counters* dc = ctx->counters.as<Counters>();
    a.hit_count = &dc->hit_count;
    a.next_work = &dc->next_work;
    a.err = &dc->err;
    a.film = nullptr;
    a.phase_steps = 0;
    a.n_events = n_ph;
    uint64_t hit_cap = ctx->hit_cap;
    if (!hit_cap) hit_cap = std::max<uint64_t>(1u << 20, n_ph * 32);
    for (int attempt = 0;; ++attempt) {
        if (!d->keep_hits) hit_cap = 1;
        {
            const int st = ensure_pool_buffers(ctx, grid);
            if (st != CMPMC_OK) return st;
        }
        CK(ctx->hit_stage.ensure(hit_cap * sizeof(cmpmc_sensor_hit)), "alloc hit staging");
        CK(ctx->hit_key.ensure(hit_cap * 8), "alloc hit keys");
        a.hit_stage = ctx->hit_stage.as<cmpmc_sensor_hit>();
        a.hit_key = ctx->hit_key.as<uint64_t>();
        a.hit_cap = hit_cap;
        CK(cudaMemsetAsync(ctx->ev_stats2.p, 0, std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats), s), "memset");
        CK(cudaMemsetAsync(ctx->ev_nhits.p, 0, std::max<uint64_t>(n, 1) * 8, s), "memset");
        CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s), "memset counters");
        CK(cudaEventRecord(ctx->e_k0, s), "event");
        if (n_ph) {
            CK(launch_pool(ctx, a, grid, nullptr, s), "pool launch");
            ++launches;
        }
        CK(cudaEventRecord(ctx->e_k1, s), "event");
        CK(cudaMemcpyAsync(ctx->h_counters.p, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s),
           "copy counters");
        CK(cudaStreamSynchronize(s), "transport kernel");
        hc = *ctx->h_counters.as<Counters>();
        CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
        const bool ring_over = (hc.err & (kErrQueue | kErrFilmQueue)) != 0;
        const bool hits_over = d->keep_hits && hc.hit_count > hit_cap;
        if (!ring_over && !hits_over) break;
        if (attempt >= 6) return fail(ctx, CMPMC_ERR_CAPACITY, "pool ring or hit buffer overflow persists");
        if (ring_over) grow_pool(ctx, hc.err);
        if (hits_over) hit_cap = hc.hit_count + hc.hit_count / 16 + 1024;
        hc.err = 0;
    }
    if (d->keep_hits) ctx->hit_cap = std::max<uint64_t>(ctx->hit_cap, hit_cap);
    if (hc.err) return fail(ctx, CMPMC_ERR_DEVICE, "transport kernel reported error word " + std::to_string(hc.err));
    n_hits = d->keep_hits ? hc.hit_count : 0;
    CK(ctx->hits_out.ensure(std::max<uint64_t>(n_hits, 1) * sizeof(cmpmc_sensor_hit)), "alloc hits");
    CK(cudaMemsetAsync(ctx->cursor.p, 0, std::max<uint64_t>(n, 1) * 8, s), "memset cursors");
    ev_offsets = ctx->ev_offsets.as<uint64_t>();
    ev_stats = ctx->ev_stats2.as<cmpmc_sim_stats>();
    a.n_events = n;
    CK(launch_sink_finish(a, n, ev_offsets, ctx->cursor.as<unsigned long long>(), ctx->hits_out.as<cmpmc_sensor_hit>(),
                          n_hits, ctx->total.as<cmpmc_sim_stats>(), ctx->partials.as<cmpmc_sim_stats>(), s, &launches),
       "merge kernels");
    // ---- capture the clean call for replay: counter and sink resets, unit map, the pool
    // launch (between external timing events), the copy of the counters and the merge ------
    if (graph_ok) {
        drop_graph(ctx);
        const uint64_t out_cap = ctx->hits_out.cap / sizeof(cmpmc_sensor_hit);
        RunArgs ag = a;  // the transport's view (n_events = units), as the eager launch had it
        ag.n_events = n_ph;
        int gl = 0;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t e = cudaMemsetAsync(ctx->ev_stats2.p, 0, n * sizeof(cmpmc_sim_stats), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->ev_nhits.p, 0, n * 8, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s);
        if (e == cudaSuccess) e = launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), ++gl;
        if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->e_k0, s, cudaEventRecordExternal);
        if (e == cudaSuccess) e = launch_pool(ctx, ag, grid, nullptr, s), ++gl;
        if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->e_k1, s, cudaEventRecordExternal);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ctx->h_counters.p, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->cursor.p, 0, n * 8, s);
        if (e == cudaSuccess)
            e = launch_sink_finish(a, n, ev_offsets, ctx->cursor.as<unsigned long long>(),
                                   ctx->hits_out.as<cmpmc_sensor_hit>(), out_cap, ctx->total.as<cmpmc_sim_stats>(),
                                   ctx->partials.as<cmpmc_sim_stats>(), s, &gl);
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        if (e == cudaSuccess) e = ec;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            ctx->graph_exec = nullptr;
            return cuda_fail(ctx, e, "graph capture");
        }
        ctx->graph_key = graph_key_of(ctx, d, n_ph);
        ctx->graph_hits_cap = out_cap;
        ctx->graph_stage_cap = d->keep_hits ? a.hit_cap : 0;
        ctx->graph_launches = gl;
    }
    return CMPMC_OK;
}

}  // namespace

extern "C" {

int cmpmc_gpu_device_count(int* count) {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (count) *count = (e == cudaSuccess) ? n : 0;
    return (e == cudaSuccess && n > 0) ? CMPMC_OK : CMPMC_ERR_NO_DEVICE;
}

int cmpmc_gpu_memcpy(void* dst, const void* src, size_t bytes) {
    if (!bytes) return CMPMC_OK;
    if (!dst || !src) return CMPMC_ERR_INVALID;
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) == cudaSuccess ? CMPMC_OK : CMPMC_ERR_CUDA;
}

int cmpmc_gpu_math_check(int device, uint64_t n, const double* x, double* out) {
    if (!x || !out) return CMPMC_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return CMPMC_ERR_NO_DEVICE;
    double *dx = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&dx, std::max<uint64_t>(n, 1) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&dout, std::max<uint64_t>(n, 1) * 24);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = launch_math_check(n, dx, dout);
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * 24, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    return e == cudaSuccess ? CMPMC_OK : CMPMC_ERR_CUDA;
}

int cmpmc_gpu_create(const cmpmc_lattice* lat, const cmpmc_detector* det, int device, cmpmc_gpu_ctx** out) {
    cmpmc_gpu_ctx* ctx = nullptr;
    if (!out) return fail(nullptr, CMPMC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!lat || !det) return fail(nullptr, CMPMC_ERR_INVALID, "lattice and detector are required");
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
        return fail(nullptr, CMPMC_ERR_NO_DEVICE, "no CUDA device is visible");
    if (device < 0 || device >= n_dev) return fail(nullptr, CMPMC_ERR_INVALID, "device index out of range");
    std::string err;
    const int st = validate_config(lat->cfg, *det, false, err);
    if (st != CMPMC_OK) return fail(nullptr, st, err);

    ctx = new cmpmc_gpu_ctx();
    ctx->device = device;
    ctx->cfg = lat->cfg;
    ctx->det = *det;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->e_start);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->e_k0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->e_k1);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->e_end);
    const size_t oct_bytes = lat->oct.size() * sizeof(OctEntry);
    const size_t cdf_bytes = 2 * kNCdf * sizeof(double);
    const size_t cdf_f_bytes = 2 * kNCdf * sizeof(float);
    float cdf_f[2 * kNCdf];
    for (int i = 0; i < kNCdf; ++i) {
        cdf_f[i] = static_cast<float>(lat->cdf_lt[i]);
        cdf_f[kNCdf + i] = static_cast<float>(lat->cdf_tt[i]);
    }
    if (e == cudaSuccess) e = ctx->tables.ensure(oct_bytes + cdf_bytes + cdf_f_bytes);
    if (e == cudaSuccess)
        e = cudaMemcpy(static_cast<char*>(ctx->tables.p) + oct_bytes + cdf_bytes, cdf_f, cdf_f_bytes,
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ctx->tables.p, lat->oct.data(), oct_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(static_cast<char*>(ctx->tables.p) + oct_bytes, lat->cdf_lt.data(), kNCdf * sizeof(double),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(static_cast<char*>(ctx->tables.p) + oct_bytes + kNCdf * sizeof(double), lat->cdf_tt.data(),
                       kNCdf * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        const std::string msg = std::string("context setup: ") + cudaGetErrorString(e);
        cmpmc_gpu_destroy(ctx);
        return fail(nullptr, CMPMC_ERR_CUDA, msg);
    }
    ctx->L = lat->view;
    if (e == cudaSuccess && lat->view.kin_mode != kKinOctahedral) {
        // the exact and bilinear modes read the stiffness tensor / the bilinear table
        const size_t b_st = sizeof(Stiffness), b_bil = lat->bil.size() * sizeof(double);
        e = ctx->kin.ensure(b_st + b_bil);
        if (e == cudaSuccess) e = cudaMemcpy(ctx->kin.p, &lat->stiff, b_st, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && b_bil)
            e = cudaMemcpy(static_cast<char*>(ctx->kin.p) + b_st, lat->bil.data(), b_bil, cudaMemcpyHostToDevice);
        ctx->L.stiff = ctx->kin.as<Stiffness>();
        ctx->L.bil = b_bil ? reinterpret_cast<const double*>(static_cast<char*>(ctx->kin.p) + b_st) : nullptr;
        if (e != cudaSuccess) {
            const std::string msg = std::string("context setup: ") + cudaGetErrorString(e);
            cmpmc_gpu_destroy(ctx);
            return fail(nullptr, CMPMC_ERR_CUDA, msg);
        }
    }
    ctx->L.oct = static_cast<const OctEntry*>(ctx->tables.p);
    ctx->L.cdf_lt = reinterpret_cast<const double*>(static_cast<char*>(ctx->tables.p) + oct_bytes);
    ctx->L.cdf_tt = ctx->L.cdf_lt + kNCdf;
    ctx->cdf_f = reinterpret_cast<const float*>(static_cast<char*>(ctx->tables.p) + oct_bytes + cdf_bytes);
    ctx->D = detector_view(*det);
    // Keep the 3 MiB group-velocity table resident in L2 (it is gathered on every step).
    cudaStreamAttrValue attr;
    std::memset(&attr, 0, sizeof(attr));
    attr.accessPolicyWindow.base_ptr = ctx->tables.p;
    attr.accessPolicyWindow.num_bytes = oct_bytes + cdf_bytes;
    attr.accessPolicyWindow.hitRatio = 1.0f;
    attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    if (cudaStreamSetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &attr) != cudaSuccess)
        (void)cudaGetLastError();  // optional: not every configuration grants a persisting L2 window
    *out = ctx;
    return CMPMC_OK;
}

void cmpmc_gpu_destroy(cmpmc_gpu_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (DevBuf* b : {&ctx->kin, &ctx->film_a, &ctx->queue_b, &ctx->rel, &ctx->part_plans, &ctx->part_counts, &ctx->lut[0], &ctx->lut[1], &ctx->lut[2], &ctx->pads[0], &ctx->pads[1], &ctx->pads[2], &ctx->tables, &ctx->mesh, &ctx->mesh32, &ctx->mesh2, &ctx->mesh2_32, &ctx->queue, &ctx->resume_a, &ctx->resume_b,
                      &ctx->ccounters, &ctx->carrier_event, &ctx->cursor, &ctx->in_rng, &ctx->in_inj, &ctx->in_phoff, &ctx->in_ph, &ctx->in_choff,
                      &ctx->in_ch, &ctx->stack, &ctx->cstack, &ctx->hit_stage, &ctx->hit_key, &ctx->counters,
                      &ctx->ev_stats, &ctx->ev_nhits, &ctx->offsets, &ctx->hits_out, &ctx->total,
                      &ctx->unit_event, &ctx->ev_offsets, &ctx->ev_stats2, &ctx->partials, &ctx->adj_prim,
                      &ctx->adj_hist, &ctx->adj_w, &ctx->adj_partials, &ctx->adj_sums})
        b->release();
    for (HostBuf* b : {&ctx->h_hits, &ctx->h_offsets, &ctx->h_evstats, &ctx->h_total, &ctx->h_counters})
        b->release();
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    for (cudaEvent_t ev : {ctx->e_start, ctx->e_k0, ctx->e_k1, ctx->e_end})
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int cmpmc_gpu_last_error(const cmpmc_gpu_ctx* ctx, char* buf, size_t size) {
    const std::string& m = ctx ? ctx->last_error : g_create_error;
    const int st = ctx ? ctx->last_status : g_create_status;
    if (buf && size) {
        const size_t n = std::min(size - 1, m.size());
        std::memcpy(buf, m.data(), n);
        buf[n] = '\0';
    }
    return st;
}

int cmpmc_gpu_configure(cmpmc_gpu_ctx* ctx, int threads_per_block, int blocks_per_sm, uint64_t stack_capacity,
                        uint64_t hit_capacity) {
    if (!ctx) return CMPMC_ERR_INVALID;
    if (threads_per_block < 0 || threads_per_block > 128 || (threads_per_block % 32) != 0 || blocks_per_sm < 0)
        return fail(ctx, CMPMC_ERR_INVALID, "threads_per_block must be a multiple of 32 in [32, 128]");
    drop_graph(ctx);  // a captured call holds the launch configuration and kernel arguments
    if (threads_per_block) ctx->tpb = threads_per_block;
    if (blocks_per_sm) ctx->bps = blocks_per_sm;
    if (stack_capacity) {
        ctx->stack_cap = static_cast<uint32_t>(std::min<uint64_t>(stack_capacity, 1u << 24));
        ctx->stack_cap_batched = ctx->stack_cap;
    }
    if (hit_capacity) ctx->hit_cap = hit_capacity;
    return CMPMC_OK;
}

int cmpmc_gpu_set_electrode_mask(cmpmc_gpu_ctx* ctx, int surface, const cmpmc_electrode_pad* pads, uint64_t n) {
    if (!ctx) return CMPMC_ERR_INVALID;
    ctx->last_status = CMPMC_OK;
    ctx->last_error.clear();
    if (surface < 0 || surface > 2) return fail(ctx, CMPMC_ERR_INVALID, "surface must be 0 (top), 1 (bottom) or 2 (side)");
    if (n && !pads) return fail(ctx, CMPMC_ERR_INVALID, "pads is NULL");
    if (n > 4096) return fail(ctx, CMPMC_ERR_INVALID, "at most 4096 pads per surface");
    drop_graph(ctx);  // the detector view (its mask pointers) is a kernel argument of a captured call
    std::vector<Pad> p(n);
    for (uint64_t i = 0; i < n; ++i) {
        if (pads[i].shape < 0 || pads[i].shape > 2)
            return fail(ctx, CMPMC_ERR_INVALID, "pad shape must be disk, annular sector or rectangle");
        p[i] = pad_view(pads[i]);
    }
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    ctx->D.surf[surface].pads = nullptr;
    ctx->D.surf[surface].n_pads = 0;
    if (n == 0) return CMPMC_OK;
    CK(ctx->pads[surface].ensure(n * sizeof(Pad)), "alloc pads");
    CK(cudaMemcpy(ctx->pads[surface].p, p.data(), n * sizeof(Pad), cudaMemcpyHostToDevice), "copy pads");
    ctx->D.surf[surface].pads = ctx->pads[surface].as<Pad>();
    ctx->D.surf[surface].n_pads = static_cast<int>(n);
    return CMPMC_OK;
}

int cmpmc_gpu_autotune(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* sample, int repeats, cmpmc_tune_result* out) {
    if (!ctx || !sample || !out) return CMPMC_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    repeats = std::max(1, std::min(repeats, 16));
    const bool batched = sample->form == CMPMC_FORM_BATCHED_FP32;
    const bool charges = batched && sample->charge_offsets != nullptr;
    const int tpb0 = ctx->tpb, bps0 = ctx->bps;
    const uint64_t q0 = ctx->queue_cap;
    auto time_run = [&](double& best) -> int {
        best = 1e300;
        for (int r = 0; r < repeats; ++r) {
            cmpmc_run_out o;
            const int st = cmpmc_gpu_run_events(ctx, sample, &o);
            if (st != CMPMC_OK) return st;
            best = std::min(best, static_cast<double>(o.kernel_ms));
        }
        return CMPMC_OK;
    };
    auto record = [&](int tpb, int bps, uint64_t q, double ms) {
        if (out->n_tried < CMPMC_TUNE_MAX) {
            out->tried_tpb[out->n_tried] = tpb;
            out->tried_bps[out->n_tried] = bps;
            out->tried_queue[out->n_tried] = q;
            out->tried_ms[out->n_tried] = ms;
            ++out->n_tried;
        }
    };
    // the configuration in place first (it also sizes every buffer)
    double ms = 0.0;
    int st = time_run(ms);
    if (st != CMPMC_OK) return st;
    out->first_ms = ms;
    int best_tpb = tpb0, best_bps = bps0;
    uint64_t best_q = q0;
    double best_ms = ms;
    record(tpb0, bps0, q0, ms);
    // block shapes: 64 or 128 threads, the occupancy limit and three quarters / half of it
    for (int tpb : {64, 128}) {
        int occ = 1;
        CK(charges ? charges_fp32_occupancy(tpb, &occ)
                   : (batched ? batched_fp32_occupancy(tpb, &occ) : plain_fp64_occupancy(tpb, &occ)),
           "occupancy");
        occ = std::max(occ, 1);
        int tried[3] = {occ, std::max(1, (3 * occ) / 4), std::max(1, occ / 2)};
        for (int k = 0; k < 3; ++k) {
            const int bps = tried[k];
            if ((k > 0 && bps == tried[k - 1]) || (k > 1 && bps == tried[0])) continue;
            ctx->tpb = tpb;
            ctx->bps = bps;
            st = time_run(ms);
            if (st != CMPMC_OK) break;
            record(tpb, bps, ctx->queue_cap, ms);
            if (ms < best_ms) {
                best_ms = ms;
                best_tpb = tpb;
                best_bps = bps;
            }
        }
        if (st != CMPMC_OK) break;
    }
    const uint32_t best_ps = ctx->phase_steps;  // not tuned: it changes the substream layout
    // queue depth of the charge phases, with the best block shape
    if (st == CMPMC_OK && charges) {
        ctx->tpb = best_tpb;
        ctx->bps = best_bps;
        for (uint64_t q : {1ull << 20, 1ull << 22, 1ull << 24}) {
            if (q == q0) continue;
            ctx->queue_cap = q;
            st = time_run(ms);
            if (st != CMPMC_OK) break;
            record(best_tpb, best_bps, q, ms);
            if (ms < best_ms) {
                best_ms = ms;
                best_q = q;
            }
        }
    }
    ctx->tpb = best_tpb;
    ctx->bps = best_bps;
    ctx->queue_cap = best_q;
    drop_graph(ctx);
    if (st != CMPMC_OK) return st;
    out->threads_per_block = best_tpb;
    out->blocks_per_sm = best_bps;
    out->queue_capacity = best_q;
    out->phase_steps = best_ps;
    out->best_ms = best_ms;
    return CMPMC_OK;
}

int cmpmc_gpu_configure_phases(cmpmc_gpu_ctx* ctx, uint32_t phase_steps) {
    if (!ctx) return CMPMC_ERR_INVALID;
    drop_graph(ctx);
    ctx->phase_steps = phase_steps;
    return CMPMC_OK;
}

int cmpmc_gpu_configure_staging(cmpmc_gpu_ctx* ctx, int enable) {
    if (!ctx || enable < 0 || enable > 1) return CMPMC_ERR_INVALID;
    drop_graph(ctx);
    ctx->stage_tables = enable;
    return CMPMC_OK;
}

int cmpmc_gpu_configure_pool(cmpmc_gpu_ctx* ctx, int form, uint32_t ring_capacity) {
    if (!ctx || form < 0 || form > 3) return CMPMC_ERR_INVALID;
    if (ring_capacity != 0 && (ring_capacity < 64 || (ring_capacity & (ring_capacity - 1)) != 0))
        return fail(ctx, CMPMC_ERR_INVALID, "ring capacity: a power of two, at least 64");
    drop_graph(ctx);
    ctx->pool = form;
    if (ring_capacity) {
        if (form == 1 || form == 3) ctx->sm_ring_cap = std::max<uint32_t>(ring_capacity, 2048);  // a block appends up to 2 x 512 at once
        else ctx->pool_ring_cap = ring_capacity;
    }
    return CMPMC_OK;
}

int cmpmc_gpu_configure_graph(cmpmc_gpu_ctx* ctx, int enable) {
    if (!ctx) return CMPMC_ERR_INVALID;
    ctx->graph_enabled = enable != 0;
    if (!ctx->graph_enabled) drop_graph(ctx);
    return CMPMC_OK;
}

int cmpmc_gpu_configure_queue(cmpmc_gpu_ctx* ctx, uint64_t queue_capacity) {
    if (!ctx) return CMPMC_ERR_INVALID;
    drop_graph(ctx);
    if (queue_capacity) ctx->queue_cap = std::max<uint64_t>(queue_capacity, 64);
    return CMPMC_OK;
}

int cmpmc_gpu_set_mesh(cmpmc_gpu_ctx* ctx, const cmpmc_mesh* mesh) {
    if (!ctx) return CMPMC_ERR_INVALID;
    ctx->last_status = CMPMC_OK;
    ctx->last_error.clear();
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    drop_graph(ctx);
    ctx->D.mesh.tet = nullptr;
    ctx->D.mesh.n_tets = 0;
    ctx->D.mesh32.tet = nullptr;
    ctx->D.mesh32.n_tets = 0;
    if (!mesh || mesh->rec.empty()) return CMPMC_OK;
    const size_t bytes = mesh->rec.size() * sizeof(MeshTet);
    CK(ctx->mesh.ensure(bytes), "alloc mesh");
    CK(cudaMemcpy(ctx->mesh.p, mesh->rec.data(), bytes, cudaMemcpyHostToDevice), "copy mesh");
    std::vector<MeshTet32> r32(mesh->rec.size());
    for (size_t i = 0; i < r32.size(); ++i) {
        const MeshTet& t = mesh->rec[i];
        MeshTet32& o = r32[i];
        for (int j = 0; j < 9; ++j) o.tinv[j] = static_cast<float>(t.tinv[j]);
        for (int j = 0; j < 3; ++j) {
            o.x3[j] = static_cast<float>(t.x3[j]);
            o.e[j] = static_cast<float>(t.e[j]);
        }
        for (int j = 0; j < 4; ++j) o.nb[j] = t.nb[j];
        o.pad = 0.0f;
    }
    CK(ctx->mesh32.ensure(r32.size() * sizeof(MeshTet32)), "alloc FP32 mesh");
    CK(cudaMemcpy(ctx->mesh32.p, r32.data(), r32.size() * sizeof(MeshTet32), cudaMemcpyHostToDevice),
       "copy FP32 mesh");
    ctx->D.mesh.tet = ctx->mesh.as<MeshTet>();
    ctx->D.mesh.n_tets = static_cast<int32_t>(mesh->rec.size());
    ctx->D.mesh32.tet = ctx->mesh32.as<MeshTet32>();
    ctx->D.mesh32.n_tets = static_cast<int32_t>(mesh->rec.size());
    return CMPMC_OK;
}

int cmpmc_gpu_set_mesh2d(cmpmc_gpu_ctx* ctx, const cmpmc_mesh2d* mesh) {
    if (!ctx) return CMPMC_ERR_INVALID;
    ctx->last_status = CMPMC_OK;
    ctx->last_error.clear();
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    drop_graph(ctx);
    ctx->D.mesh2 = MeshView2{nullptr, 0, 1};
    ctx->D.mesh2_32 = MeshView2_32{nullptr, 0, 1};
    if (!mesh || mesh->rec.empty()) return CMPMC_OK;
    const size_t n = mesh->rec.size();
    CK(ctx->mesh2.ensure(n * sizeof(MeshTri)), "alloc 2D mesh");
    CK(cudaMemcpy(ctx->mesh2.p, mesh->rec.data(), n * sizeof(MeshTri), cudaMemcpyHostToDevice), "copy 2D mesh");
    std::vector<MeshTri32> r32(n);
    for (size_t i = 0; i < n; ++i) {
        const MeshTri& t = mesh->rec[i];
        MeshTri32& o = r32[i];
        for (int j = 0; j < 4; ++j) o.tinv[j] = static_cast<float>(t.tinv[j]);
        for (int j = 0; j < 2; ++j) {
            o.x2[j] = static_cast<float>(t.x2[j]);
            o.e[j] = static_cast<float>(t.e[j]);
        }
        for (int j = 0; j < 3; ++j) o.nb[j] = t.nb[j];
        o.pad = 0;
    }
    CK(ctx->mesh2_32.ensure(n * sizeof(MeshTri32)), "alloc FP32 2D mesh");
    CK(cudaMemcpy(ctx->mesh2_32.p, r32.data(), n * sizeof(MeshTri32), cudaMemcpyHostToDevice), "copy FP32 2D mesh");
    ctx->D.mesh2 = MeshView2{ctx->mesh2.as<MeshTri>(), static_cast<int32_t>(n), mesh->axisym};
    ctx->D.mesh2_32 = MeshView2_32{ctx->mesh2_32.as<MeshTri32>(), static_cast<int32_t>(n), mesh->axisym};
    return CMPMC_OK;
}

int cmpmc_gpu_partition_deposits(cmpmc_gpu_ctx* ctx, const cmpmc_deposit* deposits, uint64_t n,
                                 const cmpmc_partition_options* opts, uint64_t* rng_state, uint64_t* charge_offsets,
                                 uint64_t* phonon_offsets, cmpmc_charge_track* charges, uint64_t charge_cap,
                                 cmpmc_phonon_track* phonons, uint64_t phonon_cap, uint64_t* n_charges,
                                 uint64_t* n_phonons) {
    if (!ctx || !n_charges || !n_phonons || !charge_offsets || !phonon_offsets) return CMPMC_ERR_INVALID;
    ctx->last_status = CMPMC_OK;
    ctx->last_error.clear();
    *n_charges = *n_phonons = 0;
    const cmpmc_partition_options o = opts ? *opts : default_partition_options();
    if (o.niel_model < CMPMC_NIEL_LINDHARD || o.niel_model > CMPMC_NIEL_EMPIRICAL || o.max_sampled_pairs == 0 ||
        o.max_sampled_phonons == 0)
        return fail(ctx, CMPMC_ERR_INVALID, "partition options");
    if (n > 0 && (!deposits || !rng_state)) return fail(ctx, CMPMC_ERR_INVALID, "deposits and generator states");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = ctx->stream;
    CK(ctx->part_plans.ensure(std::max<uint64_t>(n, 1) * partition_plan_bytes()), "alloc partition plans");
    CK(ctx->part_counts.ensure((2 * n + 1) * 8), "alloc partition counts");
    uint64_t* cnt = ctx->part_counts.as<uint64_t>();
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(cnt + 2 * n);  // non-finite deposits
    CK(cudaMemsetAsync(bad, 0, 8, s), "memset");
    CK(launch_partition_plan(ctx->cfg, o, deposits, n, rng_state, ctx->part_plans.p, cnt, cnt + n, bad, s),
       "plan launch");
    CK(launch_scan_u64(cnt, n, charge_offsets, s), "scan");
    CK(launch_scan_u64(cnt + n, n, phonon_offsets, s), "scan");
    uint64_t tot[3] = {0, 0, 0};
    CK(cudaMemcpyAsync(&tot[0], charge_offsets + n, 8, cudaMemcpyDeviceToHost, s), "copy totals");
    CK(cudaMemcpyAsync(&tot[1], phonon_offsets + n, 8, cudaMemcpyDeviceToHost, s), "copy totals");
    CK(cudaMemcpyAsync(&tot[2], bad, 8, cudaMemcpyDeviceToHost, s), "copy totals");
    CK(cudaStreamSynchronize(s), "partition plan");
    if (tot[2] > 0)  // nothing was filled and rng_state is unchanged
        return fail(ctx, CMPMC_ERR_INVALID,
                    std::to_string(tot[2]) + " deposit(s) with a non-finite energy, position or time");
    *n_charges = tot[0];
    *n_phonons = tot[1];
    if (tot[0] > charge_cap || tot[1] > phonon_cap || (tot[0] && !charges) || (tot[1] && !phonons))
        return fail(ctx, CMPMC_ERR_CAPACITY, "record capacity (the totals are set)");
    CK(launch_partition_fill(ctx->L, ctx->cfg, o, deposits, n, ctx->part_plans.p, charge_offsets, phonon_offsets,
                             charges, phonons, rng_state, s),
       "fill launch");
    CK(cudaStreamSynchronize(s), "partition fill");
    return CMPMC_OK;
}

int cmpmc_gpu_run_events(cmpmc_gpu_ctx* ctx, const cmpmc_run_desc* d, cmpmc_run_out* out) {
    if (!ctx || !d || !out) return CMPMC_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    ctx->last_status = CMPMC_OK;
    ctx->last_error.clear();
    const uint64_t n = d->n_events;
    if (d->form != CMPMC_FORM_PLAIN_FP64 && d->form != CMPMC_FORM_BATCHED_FP32 &&
        d->form != CMPMC_FORM_BATCHED_FP32_INLINE)
        return fail(ctx, CMPMC_ERR_INVALID, "unknown transport form");
    if (n > (1ull << 31)) return fail(ctx, CMPMC_ERR_INVALID, "too many events in one call");
    if (n > 0 && (!d->rng_state || !d->injected_eV || !d->phonon_offsets))
        return fail(ctx, CMPMC_ERR_INVALID, "rng_state, injected_eV and phonon_offsets are required");
    const bool batched = d->form == CMPMC_FORM_BATCHED_FP32 || d->form == CMPMC_FORM_BATCHED_FP32_INLINE;
    const bool split = d->form == CMPMC_FORM_BATCHED_FP32;
    const bool has_charges = d->charge_offsets != nullptr;
    std::string err;
    const int vst = validate_config(ctx->cfg, ctx->det, has_charges, err);
    if (vst != CMPMC_OK) return fail(ctx, vst, err);
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = ctx->stream;
    int launches = 0;

    CK(cudaEventRecord(ctx->e_start, s), "event");
    // ---- inputs ------------------------------------------------------------------
    RunArgs a;
    std::memset(&a, 0, sizeof(a));
    a.first_event = d->first_event;
    a.keep_hits = d->keep_hits;
    a.seed = d->seed;
    if (d->kaplan_surrogate && batched) {
        const int st = ensure_surrogate(ctx);
        if (st != CMPMC_OK) return st;
        a.surrogate = 1;
    }
    uint64_t n_ph = 0, n_ch = 0;
    if (d->inputs_on_device) {
        a.rng_state = d->rng_state;
        a.injected = d->injected_eV;
        a.ph_off = d->phonon_offsets;
        a.ph = d->phonons;
        a.ch_off = d->charge_offsets;
        a.ch = d->charges;
        if (n > 0) {
            CK(cudaMemcpyAsync(&n_ph, d->phonon_offsets + n, 8, cudaMemcpyDeviceToHost, s), "read track count");
            if (has_charges)
                CK(cudaMemcpyAsync(&n_ch, d->charge_offsets + n, 8, cudaMemcpyDeviceToHost, s), "read charge count");
            CK(cudaStreamSynchronize(s), "read track count");
        }
    } else if (n > 0) {
        n_ph = d->phonon_offsets[n];
        n_ch = has_charges ? d->charge_offsets[n] : 0;
        if ((n_ph && !d->phonons) || (n_ch && !d->charges))
            return fail(ctx, CMPMC_ERR_INVALID, "track arrays are required for non-empty stacks");
        CK(ctx->in_rng.ensure(n * 32), "alloc rng");
        CK(ctx->in_inj.ensure(n * 8), "alloc injected");
        CK(ctx->in_phoff.ensure((n + 1) * 8), "alloc offsets");
        CK(ctx->in_ph.ensure(std::max<uint64_t>(n_ph, 1) * sizeof(cmpmc_phonon_track)), "alloc phonons");
        CK(cudaMemcpyAsync(ctx->in_rng.p, d->rng_state, n * 32, cudaMemcpyHostToDevice, s), "copy rng");
        CK(cudaMemcpyAsync(ctx->in_inj.p, d->injected_eV, n * 8, cudaMemcpyHostToDevice, s), "copy injected");
        CK(cudaMemcpyAsync(ctx->in_phoff.p, d->phonon_offsets, (n + 1) * 8, cudaMemcpyHostToDevice, s),
           "copy offsets");
        if (n_ph)
            CK(cudaMemcpyAsync(ctx->in_ph.p, d->phonons, n_ph * sizeof(cmpmc_phonon_track), cudaMemcpyHostToDevice, s),
               "copy phonons");
        a.rng_state = ctx->in_rng.as<uint64_t>();
        a.injected = ctx->in_inj.as<double>();
        a.ph_off = ctx->in_phoff.as<uint64_t>();
        a.ph = ctx->in_ph.as<cmpmc_phonon_track>();
        if (has_charges) {
            CK(ctx->in_choff.ensure((n + 1) * 8), "alloc charge offsets");
            CK(ctx->in_ch.ensure(std::max<uint64_t>(n_ch, 1) * sizeof(cmpmc_charge_track)), "alloc charges");
            CK(cudaMemcpyAsync(ctx->in_choff.p, d->charge_offsets, (n + 1) * 8, cudaMemcpyHostToDevice, s),
               "copy charge offsets");
            if (n_ch)
                CK(cudaMemcpyAsync(ctx->in_ch.p, d->charges, n_ch * sizeof(cmpmc_charge_track), cudaMemcpyHostToDevice,
                                   s),
                   "copy charges");
            a.ch_off = ctx->in_choff.as<uint64_t>();
            a.ch = ctx->in_ch.as<cmpmc_charge_track>();
        }
    }
    Counters hc{};
    float kms = 0.0f;
    uint64_t n_hits = 0;
    uint64_t* ev_offsets = nullptr;
    cmpmc_sim_stats* ev_stats = nullptr;
    if (batched && ctx->L.kin_mode != kKinOctahedral && d->kaplan_surrogate)
        return fail(ctx, CMPMC_ERR_INVALID,
                    "the Kaplan surrogate runs with octahedral kinematics (Exact / Bilinear: full cascades)");
    if (batched && n_ch > 0) {
        // carriers and their Luke phonons: alternating charge / queue phases, event sinks
        const int st = run_charges_batched(ctx, d, a, n, n_ph, n_ch, launches, hc, kms, n_hits, ev_offsets, ev_stats);
        if (st != CMPMC_OK) return st;
    } else if (split && ctx->pool) {
        // phonons, warp pool: one persistent launch, event sinks
        const int st = run_pool_batched(ctx, d, a, n, n_ph, launches, hc, kms, n_hits, ev_offsets, ev_stats);
        if (st != CMPMC_OK) return st;
    } else if (split) {
        // phonons, wavefront split: host-driven transport and film rounds, event sinks
        const int st = run_split_batched(ctx, d, a, n, n_ph, launches, hc, kms, n_hits, ev_offsets, ev_stats);
        if (st != CMPMC_OK) return st;
    } else {
        // ---- CUDA-graph replay: the same device-resident batch again ----------------------
        const bool graph_ok = ctx->graph_enabled && batched && n > 0 && d->inputs_on_device && d->outputs_on_device;
        if (graph_ok && ctx->graph_exec && ctx->graph_key == graph_key_of(ctx, d, n_ph)) {
            CK(cudaGraphLaunch(ctx->graph_exec, s), "graph launch");
            CK(cudaStreamSynchronize(s), "graph");
            hc = *ctx->h_counters.as<Counters>();
            const bool over = hc.err != 0 || (d->keep_hits && (hc.hit_count > ctx->hit_cap ||
                                                              hc.hit_count > ctx->graph_hits_cap));
            if (!over) {
                CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
                float tms = 0.0f;
                CK(cudaEventElapsedTime(&tms, ctx->e_start, ctx->e_end), "event time");
                out->stats = *ctx->h_total.as<cmpmc_sim_stats>();
                out->n_hits = d->keep_hits ? hc.hit_count : 0;
                out->hits = ctx->hits_out.as<cmpmc_sensor_hit>();
                out->hit_offsets = ctx->ev_offsets.as<uint64_t>();
                out->event_stats = d->want_event_stats ? ctx->ev_stats2.as<cmpmc_sim_stats>() : nullptr;
                out->kernel_ms = kms;
                out->total_ms = tms;
                out->device_error = 0;
                out->kernel_launches = static_cast<uint32_t>(ctx->graph_launches);
                return CMPMC_OK;
            }
            drop_graph(ctx);  // a buffer overflowed: rerun eagerly with more room (and recapture)
        }

        // ---- work units: events (plain form) or primary phonons (batched form) ---------
        const uint64_t units = batched ? n_ph : n;
        a.n_events = units;
        int bps = ctx->bps;
        if (!bps) {
            CK(batched ? batched_fp32_occupancy(ctx->tpb, &bps) : plain_fp64_occupancy(ctx->tpb, &bps), "occupancy");
            bps = std::max(bps, 1);
        }
        uint64_t grid = static_cast<uint64_t>(ctx->num_sms) * bps;
        grid = std::min<uint64_t>(grid, (std::max<uint64_t>(units, 1) + ctx->tpb - 1) / ctx->tpb);
        grid = std::max<uint64_t>(grid, 1);
        const uint64_t slots = grid * ctx->tpb;
        const size_t stack_entry = batched ? batched_stack_entry_bytes() : sizeof(GTrack);

        CK(ctx->ev_stats.ensure(std::max<uint64_t>(units, 1) * sizeof(cmpmc_sim_stats)), "alloc unit stats");
        CK(ctx->ev_nhits.ensure(std::max<uint64_t>(units, 1) * 8), "alloc unit hit counts");
        CK(ctx->offsets.ensure((units + 1) * 8), "alloc unit offsets");
        CK(ctx->counters.ensure(sizeof(Counters)), "alloc counters");
        CK(ctx->total.ensure(sizeof(cmpmc_sim_stats)), "alloc totals");
        CK(ctx->partials.ensure(kReducePartials * sizeof(cmpmc_sim_stats)), "alloc partial totals");
        CK(ctx->h_counters.ensure(sizeof(Counters)), "alloc host counters");
        CK(ctx->cstack.ensure(slots * ctx->cstack_cap * sizeof(GCharge)), "alloc charge stacks");
        if (batched) {
            CK(ctx->unit_event.ensure(std::max<uint64_t>(units, 1) * 4), "alloc unit map");
            CK(ctx->ev_offsets.ensure((n + 1) * 8), "alloc event offsets");
            if (d->want_event_stats) CK(ctx->ev_stats2.ensure(std::max<uint64_t>(n, 1) * sizeof(cmpmc_sim_stats)),
                                        "alloc event stats");
            if (n > 0) {
                CK(launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), "unit map");
                ++launches;
            }
        }
        a.cstack = ctx->cstack.as<GCharge>();
        a.cstack_cap = ctx->cstack_cap;
        a.ev_stats = ctx->ev_stats.as<cmpmc_sim_stats>();
        a.ev_nhits = ctx->ev_nhits.as<uint64_t>();
        Counters* dc = ctx->counters.as<Counters>();
        a.hit_count = &dc->hit_count;
        a.next_work = &dc->next_work;
        a.err = &dc->err;

        uint64_t hit_cap = ctx->hit_cap;
        if (!hit_cap) hit_cap = std::max<uint64_t>(4096, std::max<uint64_t>(n, n_ph + n_ch) * 32);
        uint32_t& stack_cap = batched ? ctx->stack_cap_batched : ctx->stack_cap;
        for (int attempt = 0;; ++attempt) {
            if (!d->keep_hits) hit_cap = 1;
            CK(ctx->stack.ensure(slots * stack_cap * stack_entry), "alloc phonon stacks");
            CK(ctx->hit_stage.ensure(hit_cap * sizeof(cmpmc_sensor_hit)), "alloc hit staging");
            CK(ctx->hit_key.ensure(hit_cap * 8), "alloc hit keys");
            a.stack = ctx->stack.as<GTrack>();
            a.stack_cap = stack_cap;
            a.hit_stage = ctx->hit_stage.as<cmpmc_sensor_hit>();
            a.hit_key = ctx->hit_key.as<uint64_t>();
            a.hit_cap = hit_cap;
            CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s), "memset counters");
            CK(cudaEventRecord(ctx->e_k0, s), "event");
            if (units > 0) {
                CK(batched ? launch_batched_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ctx->unit_event.as<uint32_t>(),
                                                 static_cast<int>(grid), ctx->tpb, s)
                           : launch_plain_fp64(ctx->L, ctx->D, a, static_cast<int>(grid), ctx->tpb, s),
                   "transport launch");
                ++launches;
            }
            CK(cudaEventRecord(ctx->e_k1, s), "event");
            CK(cudaMemcpyAsync(ctx->h_counters.p, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s),
               "copy counters");
            CK(cudaStreamSynchronize(s), "transport kernel");
            hc = *ctx->h_counters.as<Counters>();
            CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
            const bool stack_over = (hc.err & (kErrPhononStack | kErrChargeStack)) != 0;
            const bool hits_over = d->keep_hits && hc.hit_count > hit_cap;
            if (!stack_over && !hits_over) break;
            if (attempt >= 10) return fail(ctx, CMPMC_ERR_CAPACITY, "device stack or hit buffer overflow persists");
            if (hc.err & kErrPhononStack) stack_cap = std::min<uint32_t>(stack_cap * 8, 1u << 24);
            if (hc.err & kErrChargeStack) {
                ctx->cstack_cap = std::min<uint32_t>(ctx->cstack_cap * 8, 1u << 20);
                CK(ctx->cstack.ensure(slots * ctx->cstack_cap * sizeof(GCharge)), "alloc charge stacks");
                a.cstack = ctx->cstack.as<GCharge>();
                a.cstack_cap = ctx->cstack_cap;
            }
            if (hits_over) hit_cap = hc.hit_count + hc.hit_count / 16 + 1024;
        }
        if (d->keep_hits) ctx->hit_cap = std::max<uint64_t>(ctx->hit_cap, hit_cap);
        if (hc.err) return fail(ctx, CMPMC_ERR_DEVICE, "transport kernel reported error word " + std::to_string(hc.err));

        // ---- merge ------------------------------------------------------------------------
        n_hits = d->keep_hits ? hc.hit_count : 0;
        CK(ctx->hits_out.ensure(std::max<uint64_t>(n_hits, 1) * sizeof(cmpmc_sensor_hit)), "alloc hits");
        ev_offsets = batched ? ctx->ev_offsets.as<uint64_t>() : ctx->offsets.as<uint64_t>();
        ev_stats = batched ? ctx->ev_stats2.as<cmpmc_sim_stats>() : ctx->ev_stats.as<cmpmc_sim_stats>();
        if (n > 0 && batched) {
            CK(launch_batched_finish(a, n, a.ph_off, a.injected, ctx->offsets.as<uint64_t>(), ev_offsets,
                                     ctx->hits_out.as<cmpmc_sensor_hit>(), n_hits, ctx->total.as<cmpmc_sim_stats>(),
                                     ctx->partials.as<cmpmc_sim_stats>(), d->want_event_stats ? ev_stats : nullptr, s,
                                     &launches),
               "merge kernels");
        } else if (n > 0) {
            CK(launch_finish(a, ctx->offsets.as<uint64_t>(), ctx->hits_out.as<cmpmc_sensor_hit>(), n_hits,
                             ctx->total.as<cmpmc_sim_stats>(), ctx->partials.as<cmpmc_sim_stats>(), s, &launches),
               "merge kernels");
        } else {
            CK(cudaMemsetAsync(ev_offsets, 0, 8, s), "memset offsets");
            CK(cudaMemsetAsync(ctx->total.p, 0, sizeof(cmpmc_sim_stats), s), "memset totals");
        }
        // ---- capture the clean call for replay: counters, unit map, transport, merge, and
        // the copies of the counters and totals, as one graph; the timing events are
        // external event-record nodes, so a replay can be timed like the eager call --------
        if (graph_ok) {
            drop_graph(ctx);
            CK(ctx->h_total.ensure(sizeof(cmpmc_sim_stats)), "alloc host totals");
            const uint64_t out_cap = ctx->hits_out.cap / sizeof(cmpmc_sensor_hit);
            int gl = 0;
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
            cudaError_t e = cudaEventRecordWithFlags(ctx->e_start, s, cudaEventRecordExternal);
            if (e == cudaSuccess) e = cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s);
            if (e == cudaSuccess) e = launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), ++gl;
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->e_k0, s, cudaEventRecordExternal);
            if (e == cudaSuccess)
                e = launch_batched_fp32(ctx->L, ctx->cdf_f, ctx->D, a, ctx->unit_event.as<uint32_t>(),
                                        static_cast<int>(grid), ctx->tpb, s), ++gl;
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->e_k1, s, cudaEventRecordExternal);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ctx->h_counters.p, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess)
                e = launch_batched_finish(a, n, a.ph_off, a.injected, ctx->offsets.as<uint64_t>(), ev_offsets,
                                          ctx->hits_out.as<cmpmc_sensor_hit>(), out_cap, ctx->total.as<cmpmc_sim_stats>(),
                                          ctx->partials.as<cmpmc_sim_stats>(), d->want_event_stats ? ev_stats : nullptr,
                                          s, &gl);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ctx->h_total.p, ctx->total.p, sizeof(cmpmc_sim_stats), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->e_end, s, cudaEventRecordExternal);
            const cudaError_t ec = cudaStreamEndCapture(s, &g);
            if (e == cudaSuccess) e = ec;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                ctx->graph_exec = nullptr;
                return cuda_fail(ctx, e, "graph capture");
            }
            ctx->graph_key = graph_key_of(ctx, d, n_ph);
            ctx->graph_hits_cap = out_cap;
            ctx->graph_launches = gl;
        }
    }
    CK(ctx->h_total.ensure(sizeof(cmpmc_sim_stats)), "alloc host totals");
    CK(cudaMemcpyAsync(ctx->h_total.p, ctx->total.p, sizeof(cmpmc_sim_stats), cudaMemcpyDeviceToHost, s),
       "copy totals");
    if (d->outputs_on_device) {
        out->hits = ctx->hits_out.as<cmpmc_sensor_hit>();
        out->hit_offsets = ev_offsets;
        out->event_stats = d->want_event_stats ? ev_stats : nullptr;
    } else {
        CK(ctx->h_hits.ensure(std::max<uint64_t>(n_hits, 1) * sizeof(cmpmc_sensor_hit)), "alloc host hits");
        CK(ctx->h_offsets.ensure((n + 1) * 8), "alloc host offsets");
        if (n_hits)
            CK(cudaMemcpyAsync(ctx->h_hits.p, ctx->hits_out.p, n_hits * sizeof(cmpmc_sensor_hit),
                               cudaMemcpyDeviceToHost, s),
               "copy hits");
        CK(cudaMemcpyAsync(ctx->h_offsets.p, ev_offsets, (n + 1) * 8, cudaMemcpyDeviceToHost, s), "copy offsets");
        if (d->want_event_stats && n > 0) {
            CK(ctx->h_evstats.ensure(n * sizeof(cmpmc_sim_stats)), "alloc host event stats");
            CK(cudaMemcpyAsync(ctx->h_evstats.p, ev_stats, n * sizeof(cmpmc_sim_stats), cudaMemcpyDeviceToHost, s),
               "copy event stats");
        }
        out->hits = ctx->h_hits.as<cmpmc_sensor_hit>();
        out->hit_offsets = ctx->h_offsets.as<uint64_t>();
        out->event_stats = d->want_event_stats ? ctx->h_evstats.as<cmpmc_sim_stats>() : nullptr;
    }
    CK(cudaEventRecord(ctx->e_end, s), "event");
    CK(cudaStreamSynchronize(s), "merge kernels");
    float tms = 0.0f;
    CK(cudaEventElapsedTime(&tms, ctx->e_start, ctx->e_end), "event time");
    out->stats = *ctx->h_total.as<cmpmc_sim_stats>();
    out->n_hits = n_hits;
    out->kernel_ms = kms;
    out->total_ms = tms;
    out->device_error = hc.err;
    out->kernel_launches = static_cast<uint32_t>(launches);
    return CMPMC_OK;
}

// Adjoint of the hit-time histogram (batched FP32 form with per-track scores). theta
// replaces the context's isotope and anharmonic coefficients, the reflection split of every
// surface and the absorption of every film for this call only.
int cmpmc_gpu_adjoint(cmpmc_gpu_ctx* ctx, const cmpmc_adjoint_desc* d, cmpmc_adjoint_out* out) {
    if (!ctx || !d || !out) return CMPMC_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    ctx->last_status = CMPMC_OK;
    ctx->last_error.clear();
    const uint64_t n = d->n_events;
    if (n > (1ull << 31)) return fail(ctx, CMPMC_ERR_INVALID, "too many events in one call");
    if (n > 0 && !d->phonon_offsets) return fail(ctx, CMPMC_ERR_INVALID, "phonon_offsets is required");
    if (d->n_bins < 1 || d->n_bins > CMPMC_ADJ_MAX_BINS) return fail(ctx, CMPMC_ERR_INVALID, "n_bins out of range");
    if (!(d->t_max > d->t_min)) return fail(ctx, CMPMC_ERR_INVALID, "t_max must exceed t_min");
    const double* th = d->theta;
    if (!(th[0] > 0.0) || !(th[1] > 0.0) || !(th[2] > 0.0 && th[2] <= 1.0) || !(th[3] > 0.0 && th[3] <= 1.0))
        return fail(ctx, CMPMC_ERR_INVALID, "theta: B_iso > 0, A_anh > 0, diffuse fraction and film absorption in (0, 1]");
    std::string err;
    const int vst = validate_config(ctx->cfg, ctx->det, false, err);
    if (vst != CMPMC_OK) return fail(ctx, vst, err);
    for (int i = 0; i < 3; ++i)
        if (ctx->det.surfaces[i].has_amm)
            return fail(ctx, CMPMC_ERR_INVALID, "the adjoint's film parameter is film_absorption: no AMM interfaces");
    if (ctx->L.kin_mode != kKinOctahedral)
        return fail(ctx, CMPMC_ERR_INVALID, "the adjoint runs with octahedral kinematics");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = ctx->stream;
    int launches = 0;
    CK(cudaEventRecord(ctx->e_start, s), "event");

    // ---- parameters ------------------------------------------------------------------
    Lattice L = ctx->L;
    L.B_iso = th[0];
    L.A_anh = th[1];
    Detector D = ctx->D;
    for (int i = 0; i < 3; ++i) {
        Surface& sf = D.surf[i];
        sf.n_spec = 1;
        sf.spec[0] = 1.0 - th[2];
        sf.n_diff = 1;
        sf.diff[0] = th[2];
        sf.n_anh = 0;
        sf.spec_prob_const = 1.0 - th[2];
        if (sf.has_film) sf.film.film_absorption = th[3];
    }

    // ---- inputs --------------------------------------------------------------------
    RunArgs a;
    std::memset(&a, 0, sizeof(a));
    a.first_event = d->first_event;
    a.keep_hits = 0;
    a.seed = d->seed;
    uint64_t n_ph = 0;
    if (d->inputs_on_device) {
        a.ph_off = d->phonon_offsets;
        a.ph = d->phonons;
        if (n > 0) {
            CK(cudaMemcpyAsync(&n_ph, d->phonon_offsets + n, 8, cudaMemcpyDeviceToHost, s), "read track count");
            CK(cudaStreamSynchronize(s), "read track count");
        }
    } else if (n > 0) {
        n_ph = d->phonon_offsets[n];
        if (n_ph && !d->phonons) return fail(ctx, CMPMC_ERR_INVALID, "phonons are required for non-empty stacks");
        CK(ctx->in_phoff.ensure((n + 1) * 8), "alloc offsets");
        CK(ctx->in_ph.ensure(std::max<uint64_t>(n_ph, 1) * sizeof(cmpmc_phonon_track)), "alloc phonons");
        CK(cudaMemcpyAsync(ctx->in_phoff.p, d->phonon_offsets, (n + 1) * 8, cudaMemcpyHostToDevice, s),
           "copy offsets");
        if (n_ph)
            CK(cudaMemcpyAsync(ctx->in_ph.p, d->phonons, n_ph * sizeof(cmpmc_phonon_track), cudaMemcpyHostToDevice, s),
               "copy phonons");
        a.ph_off = ctx->in_phoff.as<uint64_t>();
        a.ph = ctx->in_ph.as<cmpmc_phonon_track>();
    }
    if (n_ph >= (1ull << 32)) return fail(ctx, CMPMC_ERR_INVALID, "too many primaries in one call");
    const uint64_t units = n_ph;
    a.n_events = units;

    int bps = ctx->bps;
    if (!bps) {
        CK(adjoint_fp32_occupancy(ctx->tpb, &bps), "occupancy");
        bps = std::max(bps, 1);
    }
    uint64_t grid = static_cast<uint64_t>(ctx->num_sms) * bps;
    grid = std::min<uint64_t>(grid, (std::max<uint64_t>(units, 1) + ctx->tpb - 1) / ctx->tpb);
    grid = std::max<uint64_t>(grid, 1);
    const uint64_t slots = grid * ctx->tpb;

    CK(ctx->ev_stats.ensure(std::max<uint64_t>(units, 1) * sizeof(cmpmc_sim_stats)), "alloc unit stats");
    CK(ctx->ev_nhits.ensure(std::max<uint64_t>(units, 1) * 8), "alloc unit hit counts");
    CK(ctx->counters.ensure(sizeof(Counters)), "alloc counters");
    CK(ctx->total.ensure(sizeof(cmpmc_sim_stats)), "alloc totals");
    CK(ctx->partials.ensure(kReducePartials * sizeof(cmpmc_sim_stats)), "alloc partial totals");
    CK(ctx->h_counters.ensure(sizeof(Counters)), "alloc host counters");
    CK(ctx->unit_event.ensure(std::max<uint64_t>(units, 1) * 4), "alloc unit map");
    CK(ctx->adj_prim.ensure(std::max<uint64_t>(units, 1) * kAdjCols * 8), "alloc per-primary rows");
    CK(ctx->adj_hist.ensure(CMPMC_ADJ_MAX_BINS * 8), "alloc histogram");
    CK(ctx->adj_w.ensure(CMPMC_ADJ_MAX_BINS * 4), "alloc bin weights");
    CK(ctx->adj_partials.ensure(kColPartials * 2 * kAdjCols * 8), "alloc partial sums");
    CK(ctx->adj_sums.ensure(2 * kAdjCols * 8), "alloc sums");
    CK(ctx->h_total.ensure(sizeof(cmpmc_sim_stats) + (CMPMC_ADJ_MAX_BINS + 2 * kAdjCols) * 8), "alloc host totals");
    float w[CMPMC_ADJ_MAX_BINS];
    for (int b = 0; b < d->n_bins; ++b) w[b] = d->bin_weight ? static_cast<float>(d->bin_weight[b]) : 0.0f;
    CK(cudaMemcpyAsync(ctx->adj_w.p, w, d->n_bins * 4, cudaMemcpyHostToDevice, s), "copy bin weights");
    CK(cudaStreamSynchronize(s), "copy bin weights");  // w lives on this stack frame
    if (n > 0) {
        CK(launch_unit_event(a.ph_off, n, ctx->unit_event.as<uint32_t>(), s), "unit map");
        ++launches;
    }
    a.ev_stats = ctx->ev_stats.as<cmpmc_sim_stats>();
    a.ev_nhits = ctx->ev_nhits.as<uint64_t>();
    Counters* dc = ctx->counters.as<Counters>();
    a.hit_count = &dc->hit_count;
    a.next_work = &dc->next_work;
    a.err = &dc->err;
    a.hit_cap = 0;

    AdjArgs adj;
    std::memset(&adj, 0, sizeof(adj));
    adj.n_bins = d->n_bins;
    adj.t0 = d->t_min;
    adj.inv_dt = d->n_bins / (d->t_max - d->t_min);
    adj.bin_w = ctx->adj_w.as<float>();
    adj.hist = ctx->adj_hist.as<double>();
    adj.prim = ctx->adj_prim.as<double>();
    adj.spec_score = th[2] < 1.0 ? static_cast<float>(-th[2] / (1.0 - th[2])) : 0.0f;
    adj.film_miss_score = th[3] < 1.0 ? static_cast<float>(-th[3] / (1.0 - th[3])) : 0.0f;
    for (int k = 0; k < 4; ++k) adj.inv_theta[k] = 1.0 / th[k];

    Counters hc{};
    float kms = 0.0f;
    uint32_t& stack_cap = ctx->stack_cap_batched;
    for (int attempt = 0;; ++attempt) {
        CK(ctx->stack.ensure(slots * stack_cap * adjoint_stack_entry_bytes()), "alloc phonon stacks");
        a.stack = ctx->stack.as<GTrack>();
        a.stack_cap = stack_cap;
        CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(Counters), s), "memset counters");
        CK(cudaMemsetAsync(ctx->adj_hist.p, 0, CMPMC_ADJ_MAX_BINS * 8, s), "memset histogram");
        CK(cudaEventRecord(ctx->e_k0, s), "event");
        if (units > 0) {
            CK(launch_adjoint_fp32(L, ctx->cdf_f, D, a, adj, ctx->unit_event.as<uint32_t>(), static_cast<int>(grid),
                                   ctx->tpb, s),
               "adjoint launch");
            ++launches;
        }
        CK(cudaEventRecord(ctx->e_k1, s), "event");
        CK(cudaMemcpyAsync(ctx->h_counters.p, ctx->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s),
           "copy counters");
        CK(cudaStreamSynchronize(s), "adjoint kernel");
        hc = *ctx->h_counters.as<Counters>();
        CK(cudaEventElapsedTime(&kms, ctx->e_k0, ctx->e_k1), "event time");
        if (!(hc.err & kErrPhononStack)) break;
        if (attempt >= 10) return fail(ctx, CMPMC_ERR_CAPACITY, "device stack overflow persists");
        stack_cap = std::min<uint32_t>(stack_cap * 8, 1u << 24);
    }
    if (hc.err) return fail(ctx, CMPMC_ERR_DEVICE, "adjoint kernel reported error word " + std::to_string(hc.err));

    // ---- reductions (fixed order) and outputs -------------------------------------------
    char* hbuf = static_cast<char*>(ctx->h_total.p);
    if (units > 0) {
        CK(launch_reduce_cols(adj.prim, units, kAdjCols, ctx->adj_partials.as<double>(), ctx->adj_sums.as<double>(), s,
                              &launches),
           "reduce per-primary rows");
        CK(launch_reduce_stats(a.ev_stats, units, ctx->partials.as<cmpmc_sim_stats>(), ctx->total.as<cmpmc_sim_stats>(),
                               s, &launches),
           "reduce stats");
    } else {
        CK(cudaMemsetAsync(ctx->adj_sums.p, 0, 2 * kAdjCols * 8, s), "memset sums");
        CK(cudaMemsetAsync(ctx->total.p, 0, sizeof(cmpmc_sim_stats), s), "memset totals");
    }
    CK(cudaMemcpyAsync(hbuf, ctx->total.p, sizeof(cmpmc_sim_stats), cudaMemcpyDeviceToHost, s), "copy totals");
    CK(cudaMemcpyAsync(hbuf + sizeof(cmpmc_sim_stats), ctx->adj_hist.p, CMPMC_ADJ_MAX_BINS * 8,
                       cudaMemcpyDeviceToHost, s),
       "copy histogram");
    CK(cudaMemcpyAsync(hbuf + sizeof(cmpmc_sim_stats) + CMPMC_ADJ_MAX_BINS * 8, ctx->adj_sums.p, 2 * kAdjCols * 8,
                       cudaMemcpyDeviceToHost, s),
       "copy sums");
    if (d->per_primary && units > 0)
        CK(cudaMemcpyAsync(d->per_primary, adj.prim, units * kAdjCols * 8,
                           d->per_primary_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s),
           "copy per-primary rows");
    CK(cudaEventRecord(ctx->e_end, s), "event");
    CK(cudaStreamSynchronize(s), "adjoint outputs");
    float tms = 0.0f;
    CK(cudaEventElapsedTime(&tms, ctx->e_start, ctx->e_end), "event time");
    std::memcpy(&out->stats, hbuf, sizeof(cmpmc_sim_stats));
    const double* hist = reinterpret_cast<const double*>(hbuf + sizeof(cmpmc_sim_stats));
    const double* sums = hist + CMPMC_ADJ_MAX_BINS;
    for (int b = 0; b < d->n_bins; ++b) out->hist[b] = hist[b];
    const double nu = static_cast<double>(units);
    auto var_of_sum = [&](int c) {  // n / (n - 1) * (sum x^2 - (sum x)^2 / n)
        if (units < 2) return 0.0;
        const double v = sums[kAdjCols + c] - sums[c] * sums[c] / nu;
        return std::max(0.0, v) * nu / (nu - 1.0);
    };
    out->value = sums[0];
    out->value_var = var_of_sum(0);
    for (int k = 0; k < 4; ++k) {
        out->grad[k] = sums[1 + k];
        out->grad_var[k] = var_of_sum(1 + k);
    }
    out->n_primaries = units;
    out->kernel_ms = kms;
    out->total_ms = tms;
    out->device_error = hc.err;
    out->kernel_launches = static_cast<uint32_t>(launches);
    return CMPMC_OK;
}

}  // extern "C"
