// kernels.cuh -- declarations of the device kernels (pairlist.cu, forces.cu)
// used by the host runtime (api.cu).
#pragma once
#include "nb_common.cuh"

namespace gnb {
__global__ void k_refpos(const SysDev* __restrict__ sys, unsigned long long* __restrict__ cg_key);
__global__ void k_scatter(const SysDev* __restrict__ sys, const unsigned long long* __restrict__ cg_key);
__global__ void k_cell_sort(const SysDev* __restrict__ sys);
__global__ void k_cluster_setup(const SysDev* __restrict__ sys);
__global__ void k_cell_candidates(const SysDev* __restrict__ sys);
struct SearchParams;
template <int W, bool POPSORT>
__global__ void k_water_search(const SysDev* __restrict__ sys, const SearchParams P);
__global__ void k_solute_search(const SysDev* __restrict__ sys);
__global__ void k_pert_pairs(const SysDev* __restrict__ sys);
__global__ void k_expand_cgpairs(const SysDev* __restrict__ sys, int long_range);

__global__ void k_water_prep(const SysDev* __restrict__ sys);
struct WaterParams;
struct WaterScaled;
template <bool LJ00, bool LONG>
__global__ void k_water_force(const SysDev* __restrict__ sys, const WaterParams wp);
template <bool LJ00, bool LONG>
__global__ void k_water_deferred(const SysDev* __restrict__ sys, const WaterParams wp);
template <int W, bool LJ00, bool LONG, bool PK>
__global__ void k_water_force_it(const SysDev* __restrict__ sys, const WaterParams wp, const WaterScaled ws);
template <bool LONG>
__global__ void k_solute_force(const SysDev* __restrict__ sys);
__global__ void k_pos32(const SysDev* __restrict__ sys);
__global__ void k_plain_force(const SysDev* __restrict__ sys, int long_range);
__global__ void k_excluded_14(const SysDev* __restrict__ sys);
__global__ void k_pert_pairs_force(const SysDev* __restrict__ sys);
__global__ void k_pert_terms(const SysDev* __restrict__ sys);
__global__ void k_finalize(const SysDev* __restrict__ sys, int plain);
__global__ void k_finalize_plain_energies(const SysDev* __restrict__ sys);
__global__ void k_ffma_peak(float* out, int iters, float a, float b);
}  // namespace gnb
