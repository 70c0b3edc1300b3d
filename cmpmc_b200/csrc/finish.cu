// finish.cu -- the merge step of run_events on the device (parallel.hpp:133-145):
// per-event hit counts -> hit_offsets (exclusive scan), staged hits -> event order,
// per-event SimStats -> run totals. All three are deterministic (fixed summation order).
#include "device.cuh"

namespace cmpmc_gpu {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kReduceThreads = 128;
constexpr int kStatsWords = sizeof(cmpmc_sim_stats) / 8;
constexpr uint64_t kReduceTwoLevel = 65536;  // above this many records, reduce in two levels

// SimStats word kinds: doubles at 16, 17, 23, 24, 25 (engine.hpp:49-50, 60-62)
__host__ __device__ constexpr bool stats_word_is_double(int i) {
    return i == 16 || i == 17 || i == 23 || i == 24 || i == 25;
}

// Single-block chunked exclusive scan: thread t owns a contiguous slice of events.
__global__ void __launch_bounds__(kScanThreads) k_scan(const uint64_t* __restrict__ counts, uint64_t n,
                                                       uint64_t* __restrict__ offsets) {
    __shared__ uint64_t part[kScanThreads];
    const int t = threadIdx.x;
    const uint64_t chunk = (n + kScanThreads - 1) / kScanThreads;
    const uint64_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    uint64_t s = 0;
    for (uint64_t i = lo; i < hi; ++i) s += counts[i];
    part[t] = s;
    __syncthreads();
    // Hillis-Steele inclusive scan over the 1024 partial sums
    for (int d = 1; d < kScanThreads; d <<= 1) {
        const uint64_t v = (t >= d) ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint64_t run = part[t] - s;
    if (t == 0) offsets[0] = 0;
    for (uint64_t i = lo; i < hi; ++i) {
        run += counts[i];
        offsets[i + 1] = run;
    }
}

__global__ void k_scatter(const cmpmc_sensor_hit* __restrict__ stage, const uint64_t* __restrict__ key,
                          const unsigned long long* __restrict__ count, uint64_t stage_cap,
                          const uint64_t* __restrict__ offsets, cmpmc_sensor_hit* __restrict__ out,
                          uint64_t out_cap) {
    const uint64_t n = min(static_cast<uint64_t>(*count), stage_cap);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t k = key[i];
        const uint64_t dst = offsets[k >> 32] + (k & 0xffffffffull);
        if (dst < out_cap) out[dst] = stage[i];
    }
}

// event-sink runs: staged hits carry their event; each lands at the event's offset plus a
// per-event cursor (within an event the order is the staging order)
__global__ void k_scatter_sink(const cmpmc_sensor_hit* __restrict__ stage, const uint64_t* __restrict__ key,
                               const unsigned long long* __restrict__ count, uint64_t stage_cap,
                               const uint64_t* __restrict__ offsets, unsigned long long* __restrict__ cursor,
                               cmpmc_sensor_hit* __restrict__ out, uint64_t out_cap) {
    const uint64_t n = min(static_cast<uint64_t>(*count), stage_cap);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t ev = key[i];
        const uint64_t dst = offsets[ev] + atomicAdd(cursor + ev, 1ull);
        if (dst < out_cap) out[dst] = stage[i];
    }
}

__global__ void k_set_injected(cmpmc_sim_stats* __restrict__ ev_stats, const double* __restrict__ injected,
                               uint64_t n) {
    for (uint64_t ev = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; ev < n;
         ev += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        ev_stats[ev].total_injected_eV = injected[ev];
}

// Block b reduces records [b n / B, (b + 1) n / B) into total[b] in a fixed order (each
// thread a contiguous slice, then a tree over the threads).
__global__ void __launch_bounds__(kReduceThreads) k_reduce_stats(const cmpmc_sim_stats* __restrict__ ev_all,
                                                                 uint64_t n_all, cmpmc_sim_stats* total_all) {
    __shared__ uint64_t acc[kReduceThreads][kStatsWords];
    const uint64_t b0 = n_all * blockIdx.x / gridDim.x, b1 = n_all * (blockIdx.x + 1) / gridDim.x;
    const cmpmc_sim_stats* ev = ev_all + b0;
    const uint64_t n = b1 - b0;
    cmpmc_sim_stats* total = total_all + blockIdx.x;
    const int t = threadIdx.x;
    const uint64_t chunk = (n + kReduceThreads - 1) / kReduceThreads;
    const uint64_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    uint64_t u[kStatsWords];
    double d[kStatsWords];
#pragma unroll
    for (int w = 0; w < kStatsWords; ++w) {
        u[w] = 0;
        d[w] = 0.0;
    }
    for (uint64_t i = lo; i < hi; ++i) {
        const uint64_t* src = reinterpret_cast<const uint64_t*>(ev + i);
#pragma unroll
        for (int w = 0; w < kStatsWords; ++w) {
            const uint64_t x = src[w];
            if (stats_word_is_double(w)) d[w] += __longlong_as_double(static_cast<long long>(x));
            else u[w] += x;
        }
    }
#pragma unroll
    for (int w = 0; w < kStatsWords; ++w)
        acc[t][w] = stats_word_is_double(w) ? static_cast<uint64_t>(__double_as_longlong(d[w])) : u[w];
    __syncthreads();
    for (int stride = kReduceThreads / 2; stride > 0; stride >>= 1) {
        if (t < stride) {
            for (int w = 0; w < kStatsWords; ++w) {
                if (stats_word_is_double(w)) {
                    const double a = __longlong_as_double(static_cast<long long>(acc[t][w]));
                    const double b = __longlong_as_double(static_cast<long long>(acc[t + stride][w]));
                    acc[t][w] = static_cast<uint64_t>(__double_as_longlong(a + b));
                } else {
                    acc[t][w] += acc[t + stride][w];
                }
            }
        }
        __syncthreads();
    }
    if (t < kStatsWords) reinterpret_cast<uint64_t*>(total)[t] = acc[0][t];
}

__global__ void k_event_offsets(const uint64_t* __restrict__ unit_offsets, const uint64_t* __restrict__ ph_off,
                                uint64_t n_events, uint64_t* __restrict__ ev_offsets) {
    for (uint64_t ev = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; ev <= n_events;
         ev += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        ev_offsets[ev] = unit_offsets[ph_off[ev]];
}

// per-event SimStats of the batched form: the event's primaries summed in order
__global__ void k_event_stats(const cmpmc_sim_stats* __restrict__ unit_stats, const uint64_t* __restrict__ ph_off,
                              const double* __restrict__ injected, uint64_t n_events,
                              cmpmc_sim_stats* __restrict__ out) {
    for (uint64_t ev = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; ev < n_events;
         ev += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t u[kStatsWords];
        double d[kStatsWords];
        for (int w = 0; w < kStatsWords; ++w) {
            u[w] = 0;
            d[w] = 0.0;
        }
        for (uint64_t j = ph_off[ev]; j < ph_off[ev + 1]; ++j) {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(unit_stats + j);
            for (int w = 0; w < kStatsWords; ++w) {
                if (stats_word_is_double(w)) d[w] += __longlong_as_double(static_cast<long long>(src[w]));
                else u[w] += src[w];
            }
        }
        d[23] = injected[ev];
        uint64_t* dst = reinterpret_cast<uint64_t*>(out + ev);
        for (int w = 0; w < kStatsWords; ++w)
            dst[w] = stats_word_is_double(w) ? static_cast<uint64_t>(__double_as_longlong(d[w])) : u[w];
    }
}

// total injected energy (deterministic single-block sum) into total->total_injected_eV
__global__ void __launch_bounds__(kReduceThreads) k_sum_injected(const double* __restrict__ injected, uint64_t n,
                                                                 cmpmc_sim_stats* total) {
    __shared__ double acc[kReduceThreads];
    const int t = threadIdx.x;
    const uint64_t chunk = (n + kReduceThreads - 1) / kReduceThreads;
    const uint64_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    double s = 0.0;
    for (uint64_t i = lo; i < hi; ++i) s += injected[i];
    acc[t] = s;
    __syncthreads();
    for (int stride = kReduceThreads / 2; stride > 0; stride >>= 1) {
        if (t < stride) acc[t] += acc[t + stride];
        __syncthreads();
    }
    if (t == 0) total->total_injected_eV = acc[0];
}

// Column sums (and sums of squares when `squares`) of rows [b n / B, (b + 1) n / B) of a
// row-major [n][cols] array into out[b][2 cols]: each thread a contiguous slice, then a
// fixed tree over the threads, so the result does not depend on scheduling.
constexpr int kMaxCols = 8;
__global__ void __launch_bounds__(kReduceThreads) k_reduce_cols(const double* __restrict__ x_all, uint64_t n_all,
                                                                int cols, int in_stride, bool squares,
                                                                double* __restrict__ out_all) {
    __shared__ double acc[kReduceThreads][2 * kMaxCols];
    const uint64_t b0 = n_all * blockIdx.x / gridDim.x, b1 = n_all * (blockIdx.x + 1) / gridDim.x;
    const uint64_t n = b1 - b0;
    const int t = threadIdx.x;
    const uint64_t chunk = (n + kReduceThreads - 1) / kReduceThreads;
    const uint64_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    double sum[2 * kMaxCols];
#pragma unroll
    for (int c = 0; c < 2 * kMaxCols; ++c) sum[c] = 0.0;
    for (uint64_t i = lo; i < hi; ++i) {
        const double* row = x_all + (b0 + i) * in_stride;
#pragma unroll
        for (int c = 0; c < kMaxCols; ++c) {
            if (c < cols) {
                const double v = row[c];
                sum[c] += v;
                sum[kMaxCols + c] += squares ? v * v : row[cols + c];
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 2 * kMaxCols; ++c) acc[t][c] = sum[c];
    __syncthreads();
    for (int stride = kReduceThreads / 2; stride > 0; stride >>= 1) {
        if (t < stride)
            for (int c = 0; c < 2 * kMaxCols; ++c) acc[t][c] += acc[t + stride][c];
        __syncthreads();
    }
    if (t < cols) {
        out_all[blockIdx.x * 2 * cols + t] = acc[0][t];
        out_all[blockIdx.x * 2 * cols + cols + t] = acc[0][kMaxCols + t];
    }
}

}  // namespace

cudaError_t launch_reduce_cols(const double* x, uint64_t rows, int cols, double* partials, double* out,
                               cudaStream_t s, int* launches) {
    if (cols < 1 || cols > kMaxCols) return cudaErrorInvalidValue;
    // level 1: row blocks -> [kColPartials][sum, sum of squares]; level 2: one block over them
    k_reduce_cols<<<kColPartials, kReduceThreads, 0, s>>>(x, rows, cols, cols, true, partials);
    k_reduce_cols<<<1, kReduceThreads, 0, s>>>(partials, kColPartials, cols, 2 * cols, false, out);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_batched_finish(const RunArgs& a, uint64_t n_events, const uint64_t* ph_off,
                                  const double* injected, uint64_t* unit_offsets, uint64_t* ev_offsets,
                                  cmpmc_sensor_hit* hits_out, uint64_t out_cap, cmpmc_sim_stats* total,
                                  cmpmc_sim_stats* partials, cmpmc_sim_stats* ev_stats_out, cudaStream_t s,
                                  int* launches) {
    cudaError_t e = launch_finish(a, unit_offsets, hits_out, out_cap, total, partials, s, launches);
    if (e != cudaSuccess) return e;
    k_event_offsets<<<148, 256, 0, s>>>(unit_offsets, ph_off, n_events, ev_offsets);
    k_sum_injected<<<1, kReduceThreads, 0, s>>>(injected, n_events, total);
    *launches += 2;
    if (ev_stats_out) {
        k_event_stats<<<148, 128, 0, s>>>(a.ev_stats, ph_off, injected, n_events, ev_stats_out);
        *launches += 1;
    }
    return cudaGetLastError();
}

cudaError_t launch_finish(const RunArgs& a, uint64_t* offsets, cmpmc_sensor_hit* hits_out, uint64_t out_cap,
                          cmpmc_sim_stats* total, cmpmc_sim_stats* partials, cudaStream_t s, int* launches) {
    k_scan<<<1, kScanThreads, 0, s>>>(a.ev_nhits, a.n_events, offsets);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    *launches += 1;
    if (a.keep_hits) {
        k_scatter<<<4 * 148, 256, 0, s>>>(a.hit_stage, a.hit_key, a.hit_count, a.hit_cap, offsets, hits_out,
                                          out_cap);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        *launches += 1;
    }
    return launch_reduce_stats(a.ev_stats, a.n_events, partials, total, s, launches);
}

cudaError_t launch_scan_u64(const uint64_t* counts, uint64_t n, uint64_t* offsets, cudaStream_t s) {
    k_scan<<<1, kScanThreads, 0, s>>>(counts, n, offsets);
    return cudaGetLastError();
}

cudaError_t launch_sink_finish(const RunArgs& a, uint64_t n_events, uint64_t* ev_offsets,
                               unsigned long long* cursor, cmpmc_sensor_hit* hits_out, uint64_t out_cap,
                               cmpmc_sim_stats* total, cmpmc_sim_stats* partials, cudaStream_t s, int* launches) {
    if (n_events == 0) {
        cudaError_t e = cudaMemsetAsync(ev_offsets, 0, 8, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(total, 0, sizeof(cmpmc_sim_stats), s);
        return e;
    }
    k_set_injected<<<148, 256, 0, s>>>(a.ev_stats, a.injected, n_events);
    k_scan<<<1, kScanThreads, 0, s>>>(a.ev_nhits, n_events, ev_offsets);
    *launches += 2;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.keep_hits) {
        k_scatter_sink<<<4 * 148, 256, 0, s>>>(a.hit_stage, a.hit_key, a.hit_count, a.hit_cap, ev_offsets, cursor,
                                               hits_out, out_cap);
        *launches += 1;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return launch_reduce_stats(a.ev_stats, n_events, partials, total, s, launches);
}

cudaError_t launch_reduce_stats(const cmpmc_sim_stats* rec, uint64_t n, cmpmc_sim_stats* partials,
                                cmpmc_sim_stats* total, cudaStream_t s, int* launches) {
    if (n > kReduceTwoLevel && partials) {
        k_reduce_stats<<<kReducePartials, kReduceThreads, 0, s>>>(rec, n, partials);
        k_reduce_stats<<<1, kReduceThreads, 0, s>>>(partials, kReducePartials, total);
        *launches += 2;
    } else {
        k_reduce_stats<<<1, kReduceThreads, 0, s>>>(rec, n, total);
        *launches += 1;
    }
    return cudaGetLastError();
}

}  // namespace cmpmc_gpu
