// partition_gpu.cu -- EnergyPartition::partition_deposit (energy_partition.hpp:78-167) on
// the device: one deposit per thread from its own generator state, with the same code as
// the host (partition.cuh). Two passes: the plan (the yield and the draws up to the pair
// count, which fix the sizes) writes per-deposit counts, the host scans them into CSR
// offsets, and the fill writes the carrier and phonon records and the final states.
// Compiled without FMA contraction, like the plain transport form, so the arithmetic
// rounds as on the host; the transcendentals are the correctly rounded ones.
#include "device.cuh"
#include "partition.cuh"

namespace cmpmc_gpu {

namespace {

// a deposit whose energy, position or time is not finite is refused (the reference's NIEL
// yields and pair counts are undefined there)
__device__ __forceinline__ bool deposit_finite(const cmpmc_deposit& e) {
    return isfinite(e.edep_eV) && isfinite(e.pos[0]) && isfinite(e.pos[1]) && isfinite(e.pos[2]) &&
           isfinite(e.time_s);
}

struct PlanRec {
    PartitionPlan d;
    uint64_t s[4];  // generator state after the plan's draws
};

__global__ void __launch_bounds__(128) k_partition_plan(const cmpmc_crystal_config cfg,
                                                        const cmpmc_partition_options o,
                                                        const cmpmc_deposit* __restrict__ dep, uint64_t n,
                                                        const uint64_t* __restrict__ rng, PlanRec* __restrict__ plans,
                                                        uint64_t* __restrict__ n_ch, uint64_t* __restrict__ n_ph,
                                                        unsigned long long* __restrict__ bad) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const cmpmc_deposit& e = dep[i];
        if (!deposit_finite(e)) {  // counted and skipped: the call fails before the fill
            atomicAdd(bad, 1ull);
            n_ch[i] = 0;
            n_ph[i] = 0;
            continue;
        }
        Rng r;
        for (int k = 0; k < 4; ++k) r.s[k] = rng[4 * i + k];
        PlanRec p;
        p.d = plan_partition(cfg, dep[i].edep_eV, dep[i].is_nuclear_recoil != 0, o, r);
        for (int k = 0; k < 4; ++k) p.s[k] = r.s[k];
        plans[i] = p;
        n_ch[i] = 2 * p.d.pairs_sampled;
        n_ph[i] = p.d.phonons_sampled;
    }
}

__global__ void __launch_bounds__(128) k_partition_fill(const Lattice L, const cmpmc_crystal_config cfg,
                                                        const cmpmc_partition_options o,
                                                        const cmpmc_deposit* __restrict__ dep, uint64_t n,
                                                        const PlanRec* __restrict__ plans,
                                                        const uint64_t* __restrict__ ch_off,
                                                        const uint64_t* __restrict__ ph_off,
                                                        cmpmc_charge_track* __restrict__ ch,
                                                        cmpmc_phonon_track* __restrict__ ph, uint64_t* __restrict__ rng) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const PlanRec p = plans[i];
        Rng r;
        for (int k = 0; k < 4; ++k) r.s[k] = p.s[k];
        const cmpmc_deposit e = dep[i];
        fill_partition(L, cfg, p.d, o, v3(e.pos[0], e.pos[1], e.pos[2]), e.time_s, r, ch + ch_off[i], ph + ph_off[i]);
        for (int k = 0; k < 4; ++k) rng[4 * i + k] = r.s[k];
    }
}

int grid_for(uint64_t n) { return static_cast<int>(std::min<uint64_t>((n + 127) / 128, 148ull * 16)); }

}  // namespace

size_t partition_plan_bytes() { return sizeof(PlanRec); }

cudaError_t launch_partition_plan(const cmpmc_crystal_config& cfg, const cmpmc_partition_options& o,
                                  const cmpmc_deposit* dep, uint64_t n, const uint64_t* rng, void* plans,
                                  uint64_t* n_charges, uint64_t* n_phonons, unsigned long long* n_bad,
                                  cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_partition_plan<<<grid_for(n), 128, 0, s>>>(cfg, o, dep, n, rng, static_cast<PlanRec*>(plans), n_charges,
                                                 n_phonons, n_bad);
    return cudaGetLastError();
}

cudaError_t launch_partition_fill(const Lattice& L, const cmpmc_crystal_config& cfg, const cmpmc_partition_options& o,
                                  const cmpmc_deposit* dep, uint64_t n, const void* plans, const uint64_t* ch_off,
                                  const uint64_t* ph_off, cmpmc_charge_track* ch, cmpmc_phonon_track* ph,
                                  uint64_t* rng, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_partition_fill<<<grid_for(n), 128, 0, s>>>(L, cfg, o, dep, n, static_cast<const PlanRec*>(plans), ch_off, ph_off,
                                                 ch, ph, rng);
    return cudaGetLastError();
}

}  // namespace cmpmc_gpu
