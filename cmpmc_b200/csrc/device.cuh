// device.cuh -- device-side data structures shared by the kernels and the context.
#pragma once

#include <cuda_runtime.h>

#include "../../include/cmpmc_gpu.h"
#include "transport.cuh"

namespace cmpmc_gpu {

// error word bits written by the kernels (never a trap)
enum : unsigned {
    kErrPhononStack = 1u,
    kErrChargeStack = 2u,
    kErrQueue = 4u,
    kErrResume = 8u,
    kErrFilmQueue = 16u,
    kErrRelease = 32u,     // batched charge release: release records or their phonons overflowed
    kErrStage = 64u,       // a shared-memory staging copy did not complete within its wait limit
};

// A pushed phonon in a per-thread global-memory LIFO (112 B, 16-byte aligned)
struct alignas(16) GTrack {
    double px, py, pz, kx, ky, kz, vx, vy, vz, E, vmag, t, w;
    uint32_t bounces;
    int mode;
};

struct alignas(16) GCharge {
    double px, py, pz, qx, qy, qz, ekin, t, w;
    int valley, type;
};

// Per-event output record: SimStats of the event plus its hit count
struct EventOut {
    cmpmc_sim_stats st;
};

// Everything the transport kernels read or write for one run
struct RunArgs {
    uint64_t n_events;
    uint64_t first_event;
    const uint64_t* rng_state;        // [n][4]
    const double* injected;           // [n]
    const uint64_t* ph_off;           // [n+1]
    const cmpmc_phonon_track* ph;     // initial phonons
    const uint64_t* ch_off;           // [n+1] or nullptr
    const cmpmc_charge_track* ch;     // initial charges
    int keep_hits;
    uint64_t seed;                    // substream seed of the batched form
    // per-slot stacks
    GTrack* stack;
    uint32_t stack_cap;
    GCharge* cstack;
    uint32_t cstack_cap;
    // hit staging: record + (event << 32 | index within event)
    cmpmc_sensor_hit* hit_stage;
    uint64_t* hit_key;
    uint64_t hit_cap;
    unsigned long long* hit_count;
    unsigned long long* next_work;
    // outputs
    cmpmc_sim_stats* ev_stats;        // [n]
    uint64_t* ev_nhits;               // [n]
    unsigned* err;
    // event sink (batched form with charges): units add their counters to ev_stats[event]
    // and their hit counts to ev_nhits[event]; staged hits carry the event as key
    int ev_sink;
    // batched form: film cascades from the surfaces' surrogate tables (Surface::lut_*)
    int surrogate;
    // wavefront split of the batched form: film entries are queued (film, film_tail, up to
    // film_cap) for the film kernel, which queues the re-emitted phonons (reemit, ...)
    struct FilmRec* film;
    uint64_t film_cap;
    unsigned long long* film_tail;
    struct QPhonon* reemit;
    uint64_t reemit_cap;
    unsigned long long* reemit_tail;
    // wavefront split: a track that has taken this many steps in the current phase is parked
    // in `reemit` (next phase) on a substream derived from its own (0: no limit)
    uint32_t phase_steps;
};

// Phonon queue entry of the batched forms (64 B): Luke phonons of the charge form and
// film re-emissions of the wavefront split. ev == kQEmpty marks a slot that was reserved
// but not filled; `pad` carries the bounce count of a continuing track.
constexpr uint32_t kQEmpty = 0xffffffffu;
struct alignas(16) QPhonon {
    float px, py, pz, kx, ky, kz;
    float w;
    uint32_t mode;
    double E, t;
    uint64_t key;  // substream key of this phonon
    uint32_t ev;   // event index within the call
    uint32_t pad;
};

// A film entry of the wavefront-split batched form (64 B): the phonon that reached an
// active film, waiting for the film kernel. `key` seeds the cascade and the re-emissions.
struct alignas(16) FilmRec {
    float px, py, pz;
    float w;
    double E, t;
    uint64_t key;
    uint32_t ev;
    int32_t ch_id;
    uint32_t bounces;
    uint8_t surf, mode, pad0, pad1;
};

// A carrier of the batched charge form between phases (96 B): a carrier whose queue
// reservation failed is parked here with its generator state and resumed next phase.
struct alignas(16) QCharge {
    float px, py, pz, qx, qy, qz, ekin, w;
    double t;
    uint64_t ckey;      // lineage key: Luke phonon i of this carrier uses mix(ckey, i)
    uint32_t rng[4];
    uint32_t ev, luke_idx, n_knock;
    int32_t hint;       // mesh walk hint
    uint32_t valley_type;  // valley | type << 16
    uint32_t pad[3];
};

// A collected carrier whose released energy (DetectorModel::ChargeRelease BulkDebye or
// ElectrodeFilm, engine.hpp:302-313) is handed from the charge kernel to the release
// kernel of the batched charge form, with its own substream key.
struct ReleaseRec {
    float px, py, pz;  // contact point
    float w;
    double e_rel;      // collection_release_energy
    double t;
    uint64_t key;
    uint32_t ev;
    int32_t ch_id;
    uint8_t surf, type, pad0, pad1;
    uint32_t pad2;
};

struct ChargeArgs {
    uint64_t n_carriers;              // initial carriers (RunArgs::ch)
    const uint32_t* carrier_event;    // [n_carriers]
    uint64_t carrier_seed;            // substream seed of the carriers
    QPhonon* queue;
    uint64_t q_cap;
    unsigned long long* q_tail;
    const QCharge* resume_in;
    uint64_t n_resume_in;
    unsigned long long* resume_next;
    QCharge* resume_out;
    uint64_t resume_cap;
    unsigned long long* n_resume_out;
    unsigned long long* next_carrier;
    ReleaseRec* rel;                  // collections with a release mode (null: RecordOnly)
    uint64_t rel_cap;
    unsigned long long* rel_tail;
};

// Adjoint of a binned hit-time histogram (batched FP32 form, k_adjoint_fp32)
constexpr int kAdjMaxBins = 256;
constexpr int kAdjCols = 5;  // per primary: value, d value / d theta_0..3
struct AdjArgs {
    int n_bins;
    double t0, inv_dt;        // bin b covers [t0 + b / inv_dt, t0 + (b + 1) / inv_dt)
    const float* bin_w;       // [n_bins] dLoss/dh_b
    double* hist;             // [n_bins] weighted hit counts (accumulated)
    double* prim;             // [units][kAdjCols]
    float spec_score;         // d log(1 - p_d) / d log p_d = -p_d / (1 - p_d)
    float film_miss_score;    // d log(1 - f) / d log f = -f / (1 - f)
    double inv_theta[4];      // log-derivatives -> derivatives
};

CMPMC_HD GTrack pack_track(const Track& t) {
    GTrack g;
    g.px = t.pos.x; g.py = t.pos.y; g.pz = t.pos.z;
    g.kx = t.k.x; g.ky = t.k.y; g.kz = t.k.z;
    g.vx = t.vg.x; g.vy = t.vg.y; g.vz = t.vg.z;
    g.E = t.E; g.vmag = t.vmag; g.t = t.t; g.w = t.w;
    g.bounces = t.bounces;
    g.mode = t.mode;
    return g;
}
CMPMC_HD Track unpack_track(const GTrack& g) {
    Track t;
    t.pos = v3(g.px, g.py, g.pz);
    t.k = v3(g.kx, g.ky, g.kz);
    t.vg = v3(g.vx, g.vy, g.vz);
    t.E = g.E; t.vmag = g.vmag; t.t = g.t; t.w = g.w;
    t.bounces = g.bounces;
    t.mode = g.mode;
    return t;
}
CMPMC_HD Track track_from_input(const cmpmc_phonon_track& r) {
    Track t;
    t.pos = v3(r.pos[0], r.pos[1], r.pos[2]);
    t.k = v3(r.k_dir[0], r.k_dir[1], r.k_dir[2]);
    t.vg = v3(r.vg_dir[0], r.vg_dir[1], r.vg_dir[2]);
    t.E = r.energy; t.vmag = r.vg_mag; t.t = r.time; t.w = r.weight;
    t.bounces = r.bounces;
    t.mode = r.mode;
    return t;
}
CMPMC_HD Charge charge_from_input(const cmpmc_charge_track& r) {
    Charge c;
    c.pos = v3(r.pos[0], r.pos[1], r.pos[2]);
    c.p = v3(r.p_eV[0], r.p_eV[1], r.p_eV[2]);
    c.ekin = r.ekin; c.t = r.time; c.w = r.weight;
    c.valley = r.valley;
    c.type = r.type;
    return c;
}

CMPMC_HD void stats_from_event(const EvStats& e, double injected, cmpmc_sim_stats& s) {
    s.total_steps = e.total_steps;
    s.isotope_scatters = e.isotope_scatters;
    s.polycrystal_scatters = e.polycrystal_scatters;
    s.decays_L_to_TT = e.decays_TT;
    s.decays_L_to_LT = e.decays_LT;
    s.surface_refls = e.surface_refls;
    s.surface_downconversions = e.surface_downconversions;
    s.sensor_hits = e.sensor_hits;
    s.killed_tracks = e.killed_tracks;
    s.charge_steps = e.charge_steps;
    s.luke_phonons_emitted = e.luke_emitted;
    s.intervalley_scatters = e.intervalley_scatters;
    s.charges_trapped = e.charges_trapped;
    s.trap_ionizations = e.trap_ionizations;
    s.charge_surface_refls = e.charge_surface_refls;
    s.charges_collected = e.charges_collected;
    s.total_luke_phonon_eV = e.luke_eV;
    s.charge_recomb_edep_eV = e.recomb_eV;
    s.sc_pair_breakings = 0;
    s.qp_diffusion_steps = 0;
    s.qp_phonons_radiated = 0;
    s.qp_recombinations = 0;
    s.qp_local_traps = 0;
    s.total_injected_eV = injected;
    s.total_deposited_eV = e.deposited_eV;
    s.escaped_or_killed_eV = e.escaped_eV;
}

// kernels (launch wrappers return the cudaError_t of the launch)
cudaError_t launch_plain_fp64(const Lattice& L, const Detector& D, const RunArgs& a, int grid, int block,
                              cudaStream_t s);
cudaError_t plain_fp64_occupancy(int block, int* blocks_per_sm);
cudaError_t launch_batched_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const uint32_t* unit_event, int grid, int block, cudaStream_t s);
cudaError_t batched_fp32_occupancy(int block, int* blocks_per_sm);
cudaError_t launch_unit_event(const uint64_t* ph_off, uint64_t n_events, uint32_t* unit_event, cudaStream_t s);
size_t batched_stack_entry_bytes();
cudaError_t launch_adjoint_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const AdjArgs& adj, const uint32_t* unit_event, int grid, int block, cudaStream_t s);
cudaError_t adjoint_fp32_occupancy(int block, int* blocks_per_sm);
size_t adjoint_stack_entry_bytes();
// fixed-order column sums and sums of squares of a row-major [rows][cols] FP64 array
// (cols <= 8): out[c] = sum, out[cols + c] = sum of squares
cudaError_t launch_reduce_cols(const double* x, uint64_t rows, int cols, double* partials, double* out,
                               cudaStream_t s, int* launches);
constexpr int kColPartials = 296;
// fixed-order SimStats sum of n records (two levels through `partials` above 65,536 records)
cudaError_t launch_reduce_stats(const cmpmc_sim_stats* rec, uint64_t n, cmpmc_sim_stats* partials,
                                cmpmc_sim_stats* total, cudaStream_t s, int* launches);
// merge of the batched form: units are primaries; event offsets / stats derive from them
cudaError_t launch_batched_finish(const RunArgs& a, uint64_t n_events, const uint64_t* ph_off,
                                  const double* injected, uint64_t* unit_offsets, uint64_t* ev_offsets,
                                  cmpmc_sensor_hit* hits_out, uint64_t out_cap, cmpmc_sim_stats* total,
                                  cmpmc_sim_stats* partials, cmpmc_sim_stats* ev_stats_out, cudaStream_t s,
                                  int* launches);
cudaError_t launch_math_check(uint64_t n, const double* x, double* out);
// batched charge form: carriers (FP32 drift) filling the Luke-phonon queue, then the
// phonon kernel over the queue entries; both add to per-event sinks
cudaError_t launch_charges_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const ChargeArgs& c, int grid, int block, cudaStream_t s);
cudaError_t charges_fp32_occupancy(int block, int* blocks_per_sm);
// Exclusive scan of n counts into offsets[0..n] (single block)
cudaError_t launch_scan_u64(const uint64_t* counts, uint64_t n, uint64_t* offsets, cudaStream_t s);

// EnergyPartition::partition_deposit on the device (partition_gpu.cu): the plan pass writes
// per-deposit counts and plans, the fill pass the records and the final generator states
struct PartitionPlanRec;
cudaError_t launch_partition_plan(const cmpmc_crystal_config& cfg, const cmpmc_partition_options& o,
                                  const cmpmc_deposit* dep, uint64_t n, const uint64_t* rng, void* plans,
                                  uint64_t* n_charges, uint64_t* n_phonons, unsigned long long* n_bad,
                                  cudaStream_t s);
cudaError_t launch_partition_fill(const Lattice& L, const cmpmc_crystal_config& cfg, const cmpmc_partition_options& o,
                                  const cmpmc_deposit* dep, uint64_t n, const void* plans, const uint64_t* ch_off,
                                  const uint64_t* ph_off, cmpmc_charge_track* ch, cmpmc_phonon_track* ph,
                                  uint64_t* rng, cudaStream_t s);
size_t partition_plan_bytes();

// The release phase of the batched charge form: c.rel[0, n_rel) into c.queue, hits and ledgers
cudaError_t launch_release_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                                const ChargeArgs& c, uint64_t n_rel, int grid, int block, cudaStream_t s);
cudaError_t launch_queue_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                              const QPhonon* queue, int grid, int block, cudaStream_t s);
// wavefront split of the batched form: the phonon kernels with a.film set stop a track at
// film entry and queue it; the film kernel runs the queued cascades and queues the
// re-emitted phonons in a.reemit
cudaError_t launch_film_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a,
                             const FilmRec* film, uint64_t n_film, int grid, int block, cudaStream_t s);
cudaError_t film_fp32_occupancy(int block, int* blocks_per_sm);
// warp pool form of the batched phonon transport (one persistent launch): `ring` holds
// ring_cap pending-phonon entries (pool_ring_entry_bytes) per warp, `film`
// pool_film_bytes_per_warp bytes per warp; grid * block / 32 warps
// (queue != nullptr: the units are the a.n_events entries of a phonon queue instead of the
// primary records)
cudaError_t launch_pool_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a, void* ring,
                             uint32_t ring_cap, void* film, const uint32_t* unit_event, const QPhonon* queue,
                             int stage_tables, int grid, int block, cudaStream_t s);
cudaError_t pool_fp32_occupancy(int block, int* blocks_per_sm);
// SM-phase pool (one block of sm_pool_threads(fp64) threads per SM alternating transport and
// film phases): `ring` holds ring_cap entries (pool_ring_entry_bytes) per block, `film`
// film_cap film records (64 B) per block
// (fp64 = 1: the FP64 comparison form of the same pool, phonon batches without the
// surrogate; its ring entries and film records are sm_pool_entry_bytes(1) and
// sm_pool_film_bytes(1) bytes)
cudaError_t launch_sm_pool_fp32(const Lattice& L, const float* cdf_f, const Detector& D, const RunArgs& a, void* ring,
                                uint32_t ring_cap, void* film, uint32_t film_cap, const uint32_t* unit_event,
                                const QPhonon* queue, int stage_tables, int fp64, int grid, cudaStream_t s);
int sm_pool_threads(int fp64);
size_t sm_pool_entry_bytes(int fp64);
size_t sm_pool_film_bytes(int fp64);
size_t pool_ring_entry_bytes();
size_t pool_film_bytes_per_warp();
cudaError_t launch_carrier_event(const uint64_t* ch_off, uint64_t n_events, uint32_t* carrier_event,
                                 cudaStream_t s);
// merge of the event-sink runs: injected energies, hit offsets, hits into event order
// (order within an event follows staging), run totals
cudaError_t launch_sink_finish(const RunArgs& a, uint64_t n_events, uint64_t* ev_offsets,
                               unsigned long long* cursor, cmpmc_sensor_hit* hits_out, uint64_t out_cap,
                               cmpmc_sim_stats* total, cmpmc_sim_stats* partials, cudaStream_t s, int* launches);
constexpr int kReducePartials = 592;  // blocks of the first reduction level
cudaError_t launch_finish(const RunArgs& a, uint64_t* offsets, cmpmc_sensor_hit* hits_out, uint64_t out_cap,
                          cmpmc_sim_stats* total, cmpmc_sim_stats* partials, cudaStream_t s, int* launches);

}  // namespace cmpmc_gpu
