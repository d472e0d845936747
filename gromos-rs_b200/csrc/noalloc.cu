// noalloc.cu -- gr_lj_crf_innerloop_noalloc: the explicit pair-list LJ + RF
// inner loop without any device allocation.
//
// Who needs it: callers that may not call cudaMalloc while they compute
// forces, for example an integrator that records its whole step into a CUDA
// graph, a real-time loop that must not stall on the allocator, or a host
// program whose device memory is owned by another allocator.  They pass
// device pointers for all inputs and outputs and a stream.
//
// Where its scratch lives: the kernel needs two scratch buffers, the FP32
// (c6, c12) table and the FP64 energy / virial accumulators.  Both live in one
// file-scope __device__ array (g_noalloc_scratch), which every GPU that loads
// this library holds until the process exits; the maximum is 64 atom types
// (32 KiB of table plus 88 bytes of accumulators).  Host code cannot use the
// array's name as a device address: the first call on each device looks the
// address up with cudaGetSymbolAddress while that device is current, so that
// first call must come before any stream capture.  Every call shares the
// array and leaves the previous call's contents in it: each call clears the
// accumulators first, and calls whose work overlaps on the GPU (different
// streams, no ordering between them) race on the array.
//
// What the caller guarantees: every pointer except box_data (3 host doubles,
// passed to the kernel by value) is device memory of the calling thread's
// current device; pair indices are < n_atoms and iac values are
// < n_types (the inputs stay on the device, so they are not checked here).
// The forces output is cleared by the call (it does not need to start at
// zero); energies and virial are overwritten.
#include <cuda_runtime.h>

#include <mutex>

namespace gnb {

constexpr uint32_t kNoAllocMaxTypes = 64;

struct NoAllocScratch {
    float2 lj[kNoAllocMaxTypes * kNoAllocMaxTypes];  // (c6, c12) per type pair
    double acc[11];                                   // e_lj, e_crf, virial[9]
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

__global__ void k_noalloc_prepare(NoAllocScratch* __restrict__ scr, const double* __restrict__ lj_params,
                                  uint32_t n_types) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_types * n_types) scr->lj[t] = make_float2(float(lj_params[2 * t]), float(lj_params[2 * t + 1]));
    if (t < 11) scr->acc[t] = 0.0;
}

__global__ void k_noalloc_finish(const NoAllocScratch* __restrict__ scr, double* __restrict__ energies,
                                 double* __restrict__ virial) {
    const int t = threadIdx.x;
    if (t < 2) energies[t] = scr->acc[t];
    if (t < 9) virial[t] = scr->acc[2 + t];
}

// Device address of g_noalloc_scratch for the current device, looked up once
// per device (cudaGetSymbolAddress) and cached.
static gr_status noalloc_scratch(NoAllocScratch** out) {
    static std::mutex mu;
    static NoAllocScratch* addr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("gr_lj_crf_innerloop_noalloc: ") + cudaGetErrorString(e));
        return GR_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= 64) {
        set_error("gr_lj_crf_innerloop_noalloc: device index beyond 63");
        return GR_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("gr_lj_crf_innerloop_noalloc: cudaGetSymbolAddress failed: ") +
                      cudaGetErrorString(e));
            return GR_ERR_CUDA;
        }
        addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = addr[dev];
    return GR_OK;
}

}  // namespace gnb

extern "C" gr_status gr_lj_crf_innerloop_noalloc(const float* positions, const float* charges, const uint32_t* iac,
                                                 uint32_t n_atoms, const uint32_t* pairlist, uint32_t n_pairs,
                                                 const double* lj_params, uint32_t n_types, const double* box_data,
                                                 uint32_t boundary_type, double crf_cut, double crf_2cut3i,
                                                 double crf_cut3i, float* forces, double* energies, double* virial,
                                                 void* stream) {
    using namespace gnb;
    if (n_types == 0 || n_types > kNoAllocMaxTypes) {
        set_error("gr_lj_crf_innerloop_noalloc: n_types must be 1..64 (the static scratch holds a 64 x 64 table)");
        return GR_ERR_INVALID;
    }
    if (boundary_type > 1) {
        set_error("gr_lj_crf_innerloop_noalloc: boundary_type must be 0 (vacuum) or 1 (rectangular)");
        return GR_ERR_UNSUPPORTED;
    }
    if (!forces || !energies || !virial || !lj_params || (n_pairs > 0 && (!positions || !charges || !iac || !pairlist)) ||
        (boundary_type == 1 && !box_data)) {
        set_error("gr_lj_crf_innerloop_noalloc: null pointer argument");
        return GR_ERR_INVALID;
    }
    NoAllocScratch* scr = nullptr;
    gr_status st = noalloc_scratch(&scr);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(forces, 0, sizeof(float) * 3 * size_t(n_atoms), s);
    if (e == cudaSuccess) {
        const uint32_t nt2 = n_types * n_types, n_prep = nt2 > 11 ? nt2 : 11;
        k_noalloc_prepare<<<(n_prep + 255) / 256, 256, 0, s>>>(scr, lj_params, n_types);
        if (n_pairs > 0) {
            const float bx = boundary_type ? float(box_data[0]) : 1.f, by = boundary_type ? float(box_data[1]) : 1.f;
            const float bz = boundary_type ? float(box_data[2]) : 1.f;
            unsigned grid = (n_pairs + 255) / 256;
            if (grid > 4096) grid = 4096;
            k_innerloop_pairs<<<grid, 256, 0, s>>>(positions, charges, iac, pairlist, n_pairs, scr->lj, n_types, bx,
                                                   by, bz, int(boundary_type), float(crf_cut), float(crf_2cut3i),
                                                   float(crf_cut3i), 138.9354f, forces, scr->acc);
        }
        k_noalloc_finish<<<1, 32, 0, s>>>(scr, energies, virial);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_error(std::string("gr_lj_crf_innerloop_noalloc: ") + cudaGetErrorString(e));
        return GR_ERR_CUDA;
    }
    return GR_OK;
}
