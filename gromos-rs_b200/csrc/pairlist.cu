// pairlist.cu -- cell-grid charge-group pairlist on the device.
//
// Semantics are those of gromos-rs StandardPairlistAlgorithm::
// update_chargegroup_based (crates/gromos-core/src/pairlist.rs:183-442); the
// candidate generation follows the cell-list idea of
// CellListPairlistAlgorithm (pairlist.rs:537-777) but the pair SET, not the
// order, is what is reproduced, and the distance test is the reference's
// FP64 arithmetic bit for bit (nb_common.cuh):
//   * solute CG reference = centre of geometry (topology.rs:408-417),
//     solvent CG reference = its first atom;
//   * d2 = |nearest_image(ref_1, ref_2)|^2; d2 > (rcl+skin)^2 -> no pair,
//     d2 > (rcs+skin)^2 -> long range, else short range (strict '>').
//
// Stages: k_refpos (reference positions, cell keys) -> k_scan_cells ->
// k_scatter -> k_cell_sort (bitonic, per cell, deterministic) ->
// k_scan_clusters -> k_cluster_setup (solvent i-clusters of W CGs) ->
// k_water_search (water-water j-lists with W-bit masks) and
// k_solute_search (per solute CG j-lists with exclusion masks) ->
// k_pert_pairs (explicit perturbed atom pairs for the FEP correction).
#include "nb_common.cuh"

namespace gnb {

__device__ __forceinline__ int imod(int a, int m) {
    int r = a % m;
    return r < 0 ? r + m : r;
}

__device__ __forceinline__ int cell_coord(double x, double cs, int g, double* frac) {
    double q = x / cs;
    double f = floor(q);
    *frac = q - f;
    long long c = static_cast<long long>(f);
    long long r = c % g;
    if (r < 0) r += g;
    return static_cast<int>(r);
}

__device__ __forceinline__ unsigned spread3(unsigned v) {  // 3-bit Morton spread
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4);
}

// Reference positions + cell keys (pairlist.rs:196-198, 577-585, 658-663).
__global__ void k_refpos(const SysDev* __restrict__ sys, unsigned long long* __restrict__ cg_key) {
    const SysDev& s = sys[blockIdx.y];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= s.n_cg) return;
    int a0 = s.cg_off[c], a1 = s.cg_off[c + 1];
    double rx, ry, rz;
    if (c < s.n_solute_cg) {
        // ChargeGroup::center_of_geometry: sum from ZERO, then / len
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int a = a0; a < a1; ++a) {
            sx = __dadd_rn(sx, s.pos[3 * a]);
            sy = __dadd_rn(sy, s.pos[3 * a + 1]);
            sz = __dadd_rn(sz, s.pos[3 * a + 2]);
        }
        double len = static_cast<double>(a1 - a0);
        rx = __ddiv_rn(sx, len);
        ry = __ddiv_rn(sy, len);
        rz = __ddiv_rn(sz, len);
    } else {
        rx = s.pos[3 * a0];
        ry = s.pos[3 * a0 + 1];
        rz = s.pos[3 * a0 + 2];
    }
    s.ref[3 * c] = rx;
    s.ref[3 * c + 1] = ry;
    s.ref[3 * c + 2] = rz;
    double fx = 0, fy = 0, fz = 0;
    int cx = 0, cy = 0, cz = 0;
    if (s.boundary == 1) {
        cx = cell_coord(rx, s.cell_size[0], s.gdim[0], &fx);
        cy = cell_coord(ry, s.cell_size[1], s.gdim[1], &fy);
        cz = cell_coord(rz, s.cell_size[2], s.gdim[2], &fz);
    }
    int cell = cx + s.gdim[0] * (cy + s.gdim[1] * cz);
    unsigned sx3 = min(7u, static_cast<unsigned>(fx * 8.0));
    unsigned sy3 = min(7u, static_cast<unsigned>(fy * 8.0));
    unsigned sz3 = min(7u, static_cast<unsigned>(fz * 8.0));
    unsigned morton = spread3(sx3) | (spread3(sy3) << 1) | (spread3(sz3) << 2);
    unsigned long long solvent = c >= s.n_solute_cg ? 1ull : 0ull;
    cg_key[c] = (static_cast<unsigned long long>(cell) << 42) | (solvent << 41) |
                (static_cast<unsigned long long>(morton) << 32) | static_cast<unsigned>(c);
    s.cg_cell[c] = cell;
    s.cg_slot[c] = -1;
    atomicAdd(&s.cell_count[cell], 1);
}

// Exclusive scan of n values (single block, blockDim.x == 1024).  out has n+1
// entries; out may alias in.  Also returns the total in *total (if given).
__device__ void block_exclusive_scan(const int* in, int* out, int n, int* total) {
    __shared__ int warp_tot[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < n ? in[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int t = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        int excl = x - v + (wid > 0 ? warp_tot[wid - 1] : 0) + carry;
        __syncthreads();
        if (i < n) out[i] = excl;
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[n] = carry;
        if (total) *total = carry;
    }
}

__global__ void k_scan_cells(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    block_exclusive_scan(s.cell_count, s.cell_start, s.n_cells, nullptr);
}

__global__ void k_scatter(const SysDev* __restrict__ sys, const unsigned long long* __restrict__ cg_key) {
    const SysDev& s = sys[blockIdx.y];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= s.n_cg) return;
    int cell = s.cg_cell[c];
    int p = s.cell_start[cell] + atomicAdd(&s.cell_fill[cell], 1);
    s.keys[p] = cg_key[c];
}

// One block (1024 threads) per cell: bitonic sort of the cell's keys.
__global__ void k_cell_sort(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    __shared__ unsigned long long sk[kMaxCellCGs];
    int cell = blockIdx.x;
    int start = s.cell_start[cell], n = s.cell_start[cell + 1] - start;
    if (n > kMaxCellCGs) {
        if (threadIdx.x == 0) atomicOr(&s.err[0], ERR_CELL_TOO_DENSE);
        return;
    }
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = threadIdx.x; i < m; i += blockDim.x) sk[i] = i < n ? s.keys[start + i] : ~0ull;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    unsigned long long a = sk[i], b = sk[ixj];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        sk[i] = b;
                        sk[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    __shared__ int nsol;
    if (threadIdx.x == 0) nsol = 0;
    __syncthreads();
    int local = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        unsigned long long key = sk[i];
        int cg = static_cast<int>(key & 0xffffffffull);
        s.keys[start + i] = key;
        s.sorted_cg[start + i] = cg;
        s.cg_spos[cg] = start + i;
        const int stride = s.n_cg + 2;
        s.sref[start + i] = s.ref[3 * cg];
        s.sref[stride + start + i] = s.ref[3 * cg + 1];
        s.sref[2 * stride + start + i] = s.ref[3 * cg + 2];
        if (((key >> 41) & 1ull) == 0ull) ++local;
    }
    atomicAdd(&nsol, local);
    __syncthreads();
    if (threadIdx.x == 0) {
        s.cell_nsolute[cell] = nsol;
        int nsolv = n - nsol;
        s.cell_nclus[cell] = (nsolv + s.W - 1) / s.W;
        s.cell_part[cell] = (s.cell_nclus[cell] + kSearchWarps - 1) / kSearchWarps;
    }
}

__global__ void k_scan_clusters(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    __shared__ int total;
    block_exclusive_scan(s.cell_part, s.cell_part, s.n_cells, nullptr);
    __syncthreads();
    block_exclusive_scan(s.cell_nclus, s.cell_nclus, s.n_cells, &total);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (total > s.max_clusters) {
            atomicOr(&s.err[0], ERR_WLIST_OVERFLOW);
            total = s.max_clusters;
        }
        s.n_clusters[0] = total;
    }
}

// One warp per cell: write the cluster records and the slot <-> CG maps.
__global__ void k_cluster_setup(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    int cell = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (cell >= s.n_cells) return;
    int c0 = s.cell_nclus[cell], c1 = s.cell_nclus[cell + 1];
    int first_solv = s.cell_start[cell] + s.cell_nsolute[cell];
    int nsolv = s.cell_start[cell + 1] - first_solv;
    for (int k = c0 + lane; k < c1; k += 32) {
        if (k >= s.max_clusters) break;
        int local = k - c0;
        int first = first_solv + local * s.W;
        int n = min(s.W, nsolv - local * s.W);
        s.clus_cell[k] = cell;
        s.clus_first[k] = first;
        s.clus_n[k] = n;
        for (int m = 0; m < s.W; ++m) {
            int slot = k * s.W + m;
            if (m < n) {
                int cg = s.sorted_cg[first + m];
                s.slot_cg[slot] = cg;
                s.cg_slot[cg] = slot;
            } else {
                s.slot_cg[slot] = -1;
            }
        }
    }
}

// Neighbour cell offsets along one axis, de-duplicated for grids of 1 or 2
// cells (the reference de-duplicates with a HashSet, pairlist.rs:675-692).
__device__ __forceinline__ int axis_offsets(int g, int* off) {
    if (g >= 3) {
        off[0] = -1;
        off[1] = 0;
        off[2] = 1;
        return 3;
    }
    if (g == 2) {
        off[0] = 0;
        off[1] = 1;
        return 2;
    }
    off[0] = 0;
    return 1;
}

// Water-water search, tiled by cell.  One block per group of up to
// kSearchWarps clusters of one cell; the solvent CGs of each neighbour cell are
// staged in shared memory in tiles of kTile, the (cluster, chunk of 32) pairs
// of a tile that pass the bounding-sphere test are shared out over the
// block's warps, and each cluster's warp then appends its results in chunk
// order.  Pair {i_k, j} belongs to this
// cluster iff j's sorted position is after i_k's, so every unordered CG pair
// is listed once.  Bit k of the short (long) mask is set when the reference
// test puts (i_k, j) in the short (long) range; the solvent reference point
// is the first atom for both CGs (pairlist.rs:359-368).
//
// Candidates are staged with FP64 positions and FP32 min-image offsets from
// the centre of their chunk of 32; a warp skips a chunk whose bounding sphere
// is out of reach of its cluster.  The test runs in FP32 on
// cluster-to-chunk vectors (FP64 image, rounded once) minus the offsets; a
// squared distance within a relative 1e-5 of either cutoff,
// or a vector near half a box edge (image not certain in FP32), is decided by
// the exact FP64 test (nearest_image_exact + len2_exact).  The FP32 error is
// below 1e-6 relative, so the set is exactly the reference's.
//
// Each cluster's entries are collected in shared memory and written out
// sorted by mask value, so warp chunks of the force kernel see similar masks.
constexpr int kTile = 256;

// Per-launch constants of the water search (kernel parameters, constant bank).
struct SearchParams {
    double box[3], inv_box[3];
    float boxf[3], inv_boxf[3], half_boxf[3];
    double c2s, c2l;
    int boundary;
    int wcap;
};
constexpr int kEntBuf = 480;

__device__ __forceinline__ void sort_write_entries(const uint32_t* __restrict__ buf, int nbuf,
                                                   uint32_t* __restrict__ out, int lane) {
    int off[16];
    int hist[16];
#pragma unroll
    for (int v = 0; v < 16; ++v) hist[v] = 0;
    for (int c = 0; c < nbuf; c += 32) {
        const int e = c + lane;
        const unsigned m = e < nbuf ? (buf[e] & 0xfu) : 0u;
#pragma unroll
        for (int v = 1; v < 16; ++v) hist[v] += __popc(__ballot_sync(0xffffffffu, m == unsigned(v)));
    }
    off[0] = 0;
#pragma unroll
    for (int v = 1; v < 16; ++v) off[v] = off[v - 1] + hist[v - 1];
    const unsigned lt = (1u << lane) - 1u;
    for (int c = 0; c < nbuf; c += 32) {
        const int e = c + lane;
        const uint32_t ent = e < nbuf ? buf[e] : 0u;
        const unsigned m = ent & 0xfu;
#pragma unroll
        for (int v = 1; v < 16; ++v) {
            const unsigned b = __ballot_sync(0xffffffffu, m == unsigned(v));
            if (m == unsigned(v)) out[off[v] + __popc(b & lt)] = ent;
            off[v] += __popc(b);
        }
    }
}

// Stable counting sort of a cluster's entries by popcount of the mask (lanes of
// a warp chunk then iterate over the same number of bits).
template <int W>
__device__ __forceinline__ void sort_write_entries_pop(const uint32_t* __restrict__ buf, int nbuf,
                                                       uint32_t* __restrict__ out, int lane) {
    int off[W + 1];
    int hist[W + 1];
#pragma unroll
    for (int v = 0; v <= W; ++v) hist[v] = 0;
    for (int c = 0; c < nbuf; c += 32) {
        const int e = c + lane;
        const int m = e < nbuf ? __popc(buf[e] & 0xffu) : 0;
#pragma unroll
        for (int v = 1; v <= W; ++v) hist[v] += __popc(__ballot_sync(0xffffffffu, m == v));
    }
    off[0] = 0;
#pragma unroll
    for (int v = 1; v <= W; ++v) off[v] = off[v - 1] + hist[v - 1];
    const unsigned lt = (1u << lane) - 1u;
    for (int c = 0; c < nbuf; c += 32) {
        const int e = c + lane;
        const uint32_t ent = e < nbuf ? buf[e] : 0u;
        const int m = e < nbuf ? __popc(ent & 0xffu) : 0;
#pragma unroll
        for (int v = 1; v <= W; ++v) {
            const unsigned b = __ballot_sync(0xffffffffu, m == v);
            if (m == v) out[off[v] + __popc(b & lt)] = ent;
            off[v] += __popc(b);
        }
    }
}

template <int W, bool POPSORT>
__global__ void __launch_bounds__(kSearchWarps * 32, 3) k_water_search(const SysDev* __restrict__ sys, const SearchParams P) {
    const SysDev& s = sys[blockIdx.y];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = blockIdx.x;
    if (b >= s.cell_part[s.n_cells]) return;  // the whole block leaves together
    int lo = 0, hi = s.n_cells - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s.cell_part[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int cell = lo;
    const int ci = s.cell_nclus[cell] + (b - s.cell_part[cell]) * kSearchWarps + warp;
    const bool active = ci < s.cell_nclus[cell + 1];
    constexpr int kChunks = kTile / 32;

    __shared__ double tx[kTile], ty[kTile], tz[kTile];
    __shared__ float fx[kTile], fy[kTile], fz[kTile];       // offsets from the chunk centre (min image)
    __shared__ double chx[kChunks], chy[kChunks], chz[kChunks];  // chunk centres
    __shared__ float chr[kChunks];                          // chunk radii
    __shared__ uint32_t ebuf_s[kSearchWarps][kEntBuf], ebuf_l[kSearchWarps][kEntBuf];
    // the block's clusters (one per warp, all in this cell): FP64 first atoms
    // (exact tests), FP32 offsets from the first one, sizes, reach, counters
    __shared__ double cxs[kSearchWarps][3][8];
    __shared__ float cex[kSearchWarps][3][8];
    __shared__ int c_n[kSearchWarps], c_first[kSearchWarps];
    __shared__ float c_reach[kSearchWarps], c_rad[kSearchWarps];
    // (cluster, chunk) pairs of the current tile that survive the bounding
    // sphere test: the block's warps share them out, so a warp whose cluster
    // sees few chunks does not wait at the tile barrier for one that sees
    // many.  Their masks land at fixed places (res_*[cluster chunk][lane]) and
    // each cluster's warp appends them in chunk order afterwards, so the
    // lists come out in the same order on every run.
    __shared__ int n_items;
    __shared__ int it_cc[kSearchWarps * kChunks];
    __shared__ float it_C[kSearchWarps * kChunks][3];
    __shared__ uint8_t res_s[kSearchWarps * kChunks][32], res_l[kSearchWarps * kChunks][32];
    __shared__ unsigned c_surv[kSearchWarps];  // bit ch: chunk ch survived for this cluster

    {
        int n = 0, first = 0;
        if (active) {
            n = s.clus_n[ci];
            first = s.clus_first[ci];
        }
        if (lane < W) {
            double x = 0, y = 0, z = 0;
            if (lane < n) {
                const int cg = s.sorted_cg[first + lane];
                x = s.ref[3 * cg];
                y = s.ref[3 * cg + 1];
                z = s.ref[3 * cg + 2];
            }
            cxs[warp][0][lane] = x;
            cxs[warp][1][lane] = y;
            cxs[warp][2][lane] = z;
        }
        __syncwarp();
        if (lane < W) {
            const bool v = lane < n;
            const float ox = v ? float(cxs[warp][0][lane] - cxs[warp][0][0]) : 0.f;
            const float oy = v ? float(cxs[warp][1][lane] - cxs[warp][1][0]) : 0.f;
            const float oz = v ? float(cxs[warp][2][lane] - cxs[warp][2][0]) : 0.f;
            cex[warp][0][lane] = ox;
            cex[warp][1][lane] = oy;
            cex[warp][2][lane] = oz;
        }
        __syncwarp();
        if (lane == 0) {
            float rad = 0.f;
            for (int k = 0; k < n; ++k)
                rad = fmaxf(rad, sqrtf(cex[warp][0][k] * cex[warp][0][k] + cex[warp][1][k] * cex[warp][1][k] +
                                       cex[warp][2][k] * cex[warp][2][k]));
            c_n[warp] = n;
            c_first[warp] = first;
            c_rad[warp] = rad;
            c_reach[warp] = sqrtf(float(P.c2l)) + rad + 1e-3f;
        }
    }
    const float c2s = float(P.c2s), c2l = float(P.c2l);
    const float s_lo = c2s * (1.f - 1e-5f), s_hi = c2s * (1.f + 1e-5f);
    const float l_lo = c2l * (1.f - 1e-5f), l_hi = c2l * (1.f + 1e-5f);
    const float limx = P.boundary ? P.half_boxf[0] - 1e-4f : 3e38f;
    const float limy = P.boundary ? P.half_boxf[1] - 1e-4f : 3e38f;
    const float limz = P.boundary ? P.half_boxf[2] - 1e-4f : 3e38f;
    const int gx = s.gdim[0], gy = s.gdim[1], gz = s.gdim[2];
    const int cx = cell % gx, cy = (cell / gx) % gy, cz = cell / (gx * gy);
    int ox[3], oy[3], oz[3];
    const int nx = axis_offsets(gx, ox), ny = axis_offsets(gy, oy), nz = axis_offsets(gz, oz);
    const unsigned below = (1u << lane) - 1u;
    uint32_t* outs = s.wl_s + static_cast<size_t>(active ? ci : 0) * P.wcap;
    uint32_t* outl = s.wl_l + static_cast<size_t>(active ? ci : 0) * P.wcap;
    int cnt_s = 0, cnt_l = 0;
    // neighbour cells at or after this one (block-uniform), then the tiles of
    // their solvent CGs; the next tile is prefetched into registers while the
    // current one is processed
    __shared__ int ncell[27];
    __shared__ int n_nc;
    if (threadIdx.x == 0) {
        int m = 0;
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    const int nc = imod(cx + ox[ix], gx) + gx * (imod(cy + oy[iy], gy) + gy * imod(cz + oz[iz], gz));
                    if (nc >= cell) ncell[m++] = nc;
                }
        n_nc = m;
    }
    __syncthreads();
    const int stride = s.n_cg + 2;
    int ic = 0, t0 = 0;  // current tile: neighbour index ic, offset t0 into its solvent range
    auto tile_range = [&](int icc, int& j0, int& j1) {
        const int nc = ncell[icc];
        j0 = s.cell_start[nc] + s.cell_nsolute[nc];
        j1 = s.cell_start[nc + 1];
    };
    // skip empty neighbour ranges
    int j0 = 0, j1 = 0;
    while (ic < n_nc) {
        tile_range(ic, j0, j1);
        if (j1 > j0) break;
        ++ic;
    }
    double px = 0, py = 0, pz = 0;
    if (ic < n_nc && threadIdx.x < min(kTile, j1 - j0)) {
        px = s.sref[j0 + threadIdx.x];
        py = s.sref[stride + j0 + threadIdx.x];
        pz = s.sref[2 * stride + j0 + threadIdx.x];
    }
    while (ic < n_nc) {
        const int nc = ncell[ic];
        const int tbeg = j0 + t0;
        const int tn = min(kTile, j1 - tbeg);
        const int nch = (tn + 31) >> 5;
        const int slot0 = s.cell_nclus[nc] * W;
        __syncthreads();
        if (threadIdx.x == 0) n_items = 0;
        if (threadIdx.x < kSearchWarps) c_surv[threadIdx.x] = 0u;
        if (threadIdx.x < tn) {
            tx[threadIdx.x] = px;
            ty[threadIdx.x] = py;
            tz[threadIdx.x] = pz;
        }
        // chunk of 32 candidates per warp: centre = first member, FP32 min-image
        // offsets of the members, radius = largest offset
        {
            const int cbeg = warp * 32;
            if (cbeg < tn) {
                const double cx0 = __shfl_sync(0xffffffffu, px, 0);
                const double cy0 = __shfl_sync(0xffffffffu, py, 0);
                const double cz0 = __shfl_sync(0xffffffffu, pz, 0);
                float r = 0.f;
                if (threadIdx.x < tn) {
                    double dx = px - cx0, dy = py - cy0, dz = pz - cz0;
                    if (P.boundary) {
                        dx -= P.box[0] * rint(dx * P.inv_box[0]);
                        dy -= P.box[1] * rint(dy * P.inv_box[1]);
                        dz -= P.box[2] * rint(dz * P.inv_box[2]);
                    }
                    fx[threadIdx.x] = float(dx);
                    fy[threadIdx.x] = float(dy);
                    fz[threadIdx.x] = float(dz);
                    r = sqrtf(float(dx) * float(dx) + float(dy) * float(dy) + float(dz) * float(dz));
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, o));
                if (lane == 0) {
                    chx[warp] = cx0;
                    chy[warp] = cy0;
                    chz[warp] = cz0;
                    chr[warp] = r * (1.f + 1e-5f) + 1e-5f;
                }
            }
        }
        __syncthreads();
        // advance to the next tile and prefetch it
        int nic = ic, nt0 = t0 + kTile, nj0 = j0, nj1 = j1;
        if (nj0 + nt0 >= nj1) {
            nt0 = 0;
            ++nic;
            while (nic < n_nc) {
                tile_range(nic, nj0, nj1);
                if (nj1 > nj0) break;
                ++nic;
            }
        }
        if (nic < n_nc && threadIdx.x < min(kTile, nj1 - (nj0 + nt0))) {
            const int q = nj0 + nt0 + threadIdx.x;
            px = s.sref[q];
            py = s.sref[stride + q];
            pz = s.sref[2 * stride + q];
        }
        // bounding-sphere test of every (cluster, chunk) pair: cluster-to-chunk
        // vector with the FP64 image, rounded once; survivors are queued with
        // their vector and a flag for chunks near half a box edge
        for (int q = threadIdx.x; q < kSearchWarps * nch; q += blockDim.x) {
            const int c = q / nch, ch = q - c * nch;
            if (c_n[c] == 0) continue;
            double cdx = cxs[c][0][0] - chx[ch], cdy = cxs[c][1][0] - chy[ch], cdz = cxs[c][2][0] - chz[ch];
            if (P.boundary) {
                cdx -= P.box[0] * rint(cdx * P.inv_box[0]);
                cdy -= P.box[1] * rint(cdy * P.inv_box[1]);
                cdz -= P.box[2] * rint(cdz * P.inv_box[2]);
            }
            const float Cx = float(cdx), Cy = float(cdy), Cz = float(cdz);
            const float cd = sqrtf(Cx * Cx + Cy * Cy + Cz * Cz);
            if (cd - chr[ch] > c_reach[c]) continue;
            // |C - f| <= |C| + chunk radius, and a pair vector adds at most the
            // cluster radius: when that stays below half a box edge on every
            // axis, C - f is the minimum image and every pair is inside the box
            const float ext = chr[ch] + c_rad[c];
            const bool edge = P.boundary && !(fabsf(Cx) + ext < limx && fabsf(Cy) + ext < limy &&
                                              fabsf(Cz) + ext < limz);
            const int k = atomicAdd(&n_items, 1);
            atomicOr(&c_surv[c], 1u << ch);
            it_cc[k] = (c << 8) | (ch << 1) | (edge ? 1 : 0);
            it_C[k][0] = Cx;
            it_C[k][1] = Cy;
            it_C[k][2] = Cz;
        }
        __syncthreads();
        const int items = n_items;
        for (int it = warp; it < items; it += kSearchWarps) {
            const int cc = it_cc[it];
            const int c = cc >> 8, ch = (cc >> 1) & 0x7f;
            const bool edge = cc & 1;
            const float Cx = it_C[it][0], Cy = it_C[it][1], Cz = it_C[it][2];
            const int n = c_n[c], first = c_first[c];
            const float reach2 = c_reach[c] * c_reach[c];
            const int t = ch * 32 + lane;
            const int sp = tbeg + t;
            unsigned ms = 0, ml = 0, amb = 0;
            if (t < tn && sp > first) {
                float Dx = Cx - fx[t], Dy = Cy - fy[t], Dz = Cz - fz[t];
                if (edge) {  // the sum of two minimum images need not be one
                    Dx -= P.boxf[0] * rintf(Dx * P.inv_boxf[0]);
                    Dy -= P.boxf[1] * rintf(Dy * P.inv_boxf[1]);
                    Dz -= P.boxf[2] * rintf(Dz * P.inv_boxf[2]);
                }
                if (Dx * Dx + Dy * Dy + Dz * Dz <= reach2) {
                    // branch-free classification of the W pairs; pairs inside a
                    // band around a cutoff or near half a box edge are decided by
                    // the exact FP64 test; pairs {i_k, j} with k < n and i_k
                    // before j in sorted order
                    const int nv = min(n, sp - first);
                    const unsigned valid = (1u << nv) - 1u;
#pragma unroll
                    for (int k = 0; k < W; ++k) {
                        const float kx = cex[c][0][k] + Dx, ky = cex[c][1][k] + Dy, kz = cex[c][2][k] + Dz;
                        const float d2 = kx * kx + ky * ky + kz * kz;
                        ms |= unsigned(d2 < s_lo) << k;
                        ml |= unsigned(d2 > s_hi && d2 < l_lo) << k;
                        amb |= unsigned((d2 >= s_lo && d2 <= s_hi) || (d2 >= l_lo && d2 <= l_hi)) << k;
                        if (edge) {
                            const bool inbox = fabsf(kx) < limx && fabsf(ky) < limy && fabsf(kz) < limz;
                            amb |= unsigned(!inbox) << k;
                        }
                    }
                    ms &= valid & ~amb;
                    ml &= valid & ~amb;
                    amb &= valid;
                }
            }
            // the rare ambiguous pairs: one warp-uniform test, then the exact
            // FP64 decision (nearest_image_exact + len2_exact, box from the
            // kernel parameters) for the lanes that have some
            if (__any_sync(0xffffffffu, amb != 0u) && amb) {
#pragma unroll 1
                for (int k = 0; k < W; ++k) {
                    if (!((amb >> k) & 1u)) continue;
                    double rx = __dsub_rn(cxs[c][0][k], tx[t]);
                    double ry = __dsub_rn(cxs[c][1][k], ty[t]);
                    double rz = __dsub_rn(cxs[c][2][k], tz[t]);
                    if (P.boundary) {
                        rx = image_exact(rx, P.box[0], P.inv_box[0]);
                        ry = image_exact(ry, P.box[1], P.inv_box[1]);
                        rz = image_exact(rz, P.box[2], P.inv_box[2]);
                    }
                    const double e2 = len2_exact(rx, ry, rz);
                    if (!(e2 > P.c2l)) {
                        if (e2 > P.c2s)
                            ml |= 1u << k;
                        else
                            ms |= 1u << k;
                    }
                }
            }
            res_s[c * kChunks + ch][lane] = static_cast<uint8_t>(ms);
            res_l[c * kChunks + ch][lane] = static_cast<uint8_t>(ml);
        }
        __syncthreads();
        // each cluster's warp appends its surviving chunks in chunk order
        if (active) {
            unsigned surv = c_surv[warp];
            while (surv) {
                const int ch = __ffs(surv) - 1;
                surv &= surv - 1;
                const unsigned ms = res_s[warp * kChunks + ch][lane], ml = res_l[warp * kChunks + ch][lane];
                const uint32_t slot = static_cast<uint32_t>(slot0 + (tbeg + ch * 32 + lane - j0));
                const unsigned bs = __ballot_sync(0xffffffffu, ms != 0);
                const unsigned bl = __ballot_sync(0xffffffffu, ml != 0);
                if (ms) {
                    const int p = cnt_s + __popc(bs & below);
                    const uint32_t ent = (slot << 8) | ms;
                    if (p < kEntBuf)
                        ebuf_s[warp][p] = ent;
                    else if (p < P.wcap)
                        outs[p] = ent;
                }
                if (ml) {
                    const int p = cnt_l + __popc(bl & below);
                    const uint32_t ent = (slot << 8) | ml;
                    if (p < kEntBuf)
                        ebuf_l[warp][p] = ent;
                    else if (p < P.wcap)
                        outl[p] = ent;
                }
                cnt_s += __popc(bs);
                cnt_l += __popc(bl);
            }
        }
        ic = nic;
        t0 = nt0;
        j0 = nj0;
        j1 = nj1;
    }
    if (!active) return;
    __syncwarp();
    if (POPSORT) {
        sort_write_entries_pop<W>(ebuf_s[warp], min(cnt_s, kEntBuf), outs, lane);
        sort_write_entries_pop<W>(ebuf_l[warp], min(cnt_l, kEntBuf), outl, lane);
    } else {
        sort_write_entries(ebuf_s[warp], min(cnt_s, kEntBuf), outs, lane);
        sort_write_entries(ebuf_l[warp], min(cnt_l, kEntBuf), outl, lane);
    }
    if (lane == 0) {
        if (cnt_s > P.wcap || cnt_l > P.wcap) atomicOr(&s.err[0], ERR_WLIST_OVERFLOW);
        s.wn_s[ci] = min(cnt_s, P.wcap);
        s.wn_l[ci] = min(cnt_l, P.wcap);
    }
}

// Topology::is_excluded_or_14 (topology.rs:853-864).
__device__ bool excluded_or_14(const SysDev& s, int i, int j) {
    for (int pass = 0; pass < 2; ++pass) {
        int a = pass ? j : i, b = pass ? i : j;
        int lo = s.excl_off[a], hi = s.excl_off[a + 1] - 1;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            int v = s.excl[mid];
            if (v == b) return true;
            if (v < b)
                lo = mid + 1;
            else
                hi = mid - 1;
        }
        for (int k = s.o14_off[a]; k < s.o14_off[a + 1]; ++k)
            if (s.o14[k] == b) return true;
    }
    return false;
}

// Excluded atom pairs of CG pair (ci, cj) as bits a*8+b; for ci == cj the
// pairs with a >= b are marked too (only a < b is a pair).
__device__ unsigned long long excl_mask(const SysDev& s, int ci, int cj) {
    unsigned long long m = 0;
    int i0 = s.cg_off[ci], ni = s.cg_off[ci + 1] - i0;
    int j0 = s.cg_off[cj], nj = s.cg_off[cj + 1] - j0;
    for (int a = 0; a < ni; ++a)
        for (int b = 0; b < nj; ++b) {
            bool ex = (ci == cj && b <= a) || excluded_or_14(s, i0 + a, j0 + b);
            if (ex) m |= 1ull << (a * 8 + b);
        }
    return m;
}

// Solute CG i against every CG in the neighbour cells: solute j > i
// (COG-COG, with exclusions for the short range) and every solvent CG
// (COG-first atom, no exclusion check), pairlist.rs:237-350.  One warp per
// solute CG.  Entry = (j << 1 | long); the first entry is the CG itself
// (intra-CG pairs, pairlist.rs:239-249).
__global__ void k_solute_search(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int ci = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (ci >= s.n_solute_cg) return;
    if (s.cg_off[ci + 1] - s.cg_off[ci] > kMaxCGAtoms) {
        if (lane == 0) atomicOr(&s.err[0], ERR_CG_TOO_LARGE);
        return;
    }
    int* out = s.sl + static_cast<size_t>(ci) * s.scap;
    unsigned long long* outx = s.sl_excl + static_cast<size_t>(ci) * s.scap;
    int cnt = 0;
    if (lane == 0) {
        out[0] = ci << 1;
        outx[0] = excl_mask(s, ci, ci);
    }
    cnt = 1;
    double xi = s.ref[3 * ci], yi = s.ref[3 * ci + 1], zi = s.ref[3 * ci + 2];
    int cell = s.cg_cell[ci];
    int gx = s.gdim[0], gy = s.gdim[1], gz = s.gdim[2];
    int cx = cell % gx, cy = (cell / gx) % gy, cz = cell / (gx * gy);
    int ox[3], oy[3], oz[3];
    int nx = axis_offsets(gx, ox), ny = axis_offsets(gy, oy), nz = axis_offsets(gz, oz);
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                int nc = imod(cx + ox[ix], gx) + gx * (imod(cy + oy[iy], gy) + gy * imod(cz + oz[iz], gz));
                int j0 = s.cell_start[nc], j1 = s.cell_start[nc + 1];
                for (int base = j0; base < j1; base += 32) {
                    int sp = base + lane;
                    int entry = -1;
                    unsigned long long xm = 0;
                    if (sp < j1) {
                        int cj = s.sorted_cg[sp];
                        bool solute_j = cj < s.n_solute_cg;
                        if (!solute_j || cj > ci) {
                            double rx, ry, rz;
                            nearest_image_exact(s, xi, yi, zi, s.ref[3 * cj], s.ref[3 * cj + 1],
                                                s.ref[3 * cj + 2], rx, ry, rz);
                            double d2 = len2_exact(rx, ry, rz);
                            if (!(d2 > s.c2l)) {
                                int lr = d2 > s.c2s ? 1 : 0;
                                if (solute_j && s.cg_off[cj + 1] - s.cg_off[cj] > kMaxCGAtoms) {
                                    atomicOr(&s.err[0], ERR_CG_TOO_LARGE);
                                } else {
                                    entry = (cj << 1) | lr;
                                    if (solute_j && !lr) xm = excl_mask(s, ci, cj);
                                }
                            }
                        }
                    }
                    unsigned b = __ballot_sync(0xffffffffu, entry >= 0);
                    if (entry >= 0) {
                        int p = cnt + __popc(b & ((1u << lane) - 1u));
                        if (p < s.scap) {
                            out[p] = entry;
                            outx[p] = xm;
                        }
                    }
                    cnt += __popc(b);
                }
            }
    if (lane == 0) {
        if (cnt > s.scap) atomicOr(&s.err[0], ERR_SLIST_OVERFLOW);
        s.sn[ci] = min(cnt, s.scap);
    }
}

// Explicit list of atom pairs that the FEP correction visits: pairs of the
// solute lists whose first atom (the atom of the lower-index CG) is
// perturbed (perturbed.rs:324-332).  One thread per (solute CG, entry).
__global__ void k_pert_pairs(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    int ci = gid / s.scap, e = gid % s.scap;
    if (ci >= s.n_solute_cg || e >= s.sn[ci]) return;
    int entry = s.sl[static_cast<size_t>(ci) * s.scap + e];
    unsigned long long xm = s.sl_excl[static_cast<size_t>(ci) * s.scap + e];
    int cj = entry >> 1, lr = entry & 1;
    int i0 = s.cg_off[ci], i1 = s.cg_off[ci + 1];
    int j0 = s.cg_off[cj], j1 = s.cg_off[cj + 1];
    for (int a = i0; a < i1; ++a) {
        if (s.pert_idx[a] < 0) continue;
        for (int b = j0; b < j1; ++b) {
            if (xm & (1ull << ((a - i0) * 8 + (b - j0)))) continue;
            int p = atomicAdd(s.n_pert_pairs, 1);
            if (p < s.pcap) {
                s.pert_pairs[3 * p] = a;
                s.pert_pairs[3 * p + 1] = b;
                s.pert_pairs[3 * p + 2] = lr;
            } else {
                atomicOr(&s.err[0], ERR_PERT_OVERFLOW);
            }
        }
    }
}

// Explicit CG-pair list (i, j, long) + exclusion mask, for the plain kernel
// and for downloading the pair set.  Water-water pairs from the cluster
// masks, then solute entries.  One thread per (cluster, entry) / (solute
// CG, entry).
__global__ void k_expand_cgpairs(const SysDev* __restrict__ sys, int long_range) {
    const SysDev& s = sys[blockIdx.y];
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    int nclus = s.n_clusters[0];
    long long nwater = static_cast<long long>(nclus) * s.wcap;
    if (gid < nwater) {
        int ci = gid / s.wcap, e = gid % s.wcap;
        const int* wn = long_range ? s.wn_l : s.wn_s;
        if (e >= wn[ci]) return;
        uint32_t ent = (long_range ? s.wl_l : s.wl_s)[static_cast<size_t>(ci) * s.wcap + e];
        int cj = s.slot_cg[ent >> 8];
        unsigned mask = ent & 0xffu;
        for (int k = 0; k < s.W; ++k)
            if (mask & (1u << k)) {
                int cik = s.slot_cg[ci * s.W + k];
                int p = atomicAdd(&s.n_cgp[long_range], 1);
                int idx = long_range ? s.cgp_cap - 1 - p : p;
                if (p < s.cgp_cap) {
                    s.cgp[3 * idx] = min(cik, cj);
                    s.cgp[3 * idx + 1] = max(cik, cj);
                    s.cgp[3 * idx + 2] = long_range;
                    s.cgp_excl[idx] = 0ull;
                } else {
                    atomicOr(&s.err[0], ERR_CGPAIR_OVERFLOW);
                }
            }
        return;
    }
    long long g2 = gid - nwater;
    int ci = static_cast<int>(g2 / s.scap), e = static_cast<int>(g2 % s.scap);
    if (ci >= s.n_solute_cg || e >= s.sn[ci]) return;
    int entry = s.sl[static_cast<size_t>(ci) * s.scap + e];
    if ((entry & 1) != long_range) return;
    int p = atomicAdd(&s.n_cgp[long_range], 1);
    int idx = long_range ? s.cgp_cap - 1 - p : p;
    if (p < s.cgp_cap) {
        s.cgp[3 * idx] = ci;
        s.cgp[3 * idx + 1] = entry >> 1;
        s.cgp[3 * idx + 2] = long_range;
        s.cgp_excl[idx] = s.sl_excl[static_cast<size_t>(ci) * s.scap + e];
    } else {
        atomicOr(&s.err[0], ERR_CGPAIR_OVERFLOW);
    }
}

}  // namespace gnb

namespace gnb {
}  // namespace gnb

namespace gnb {
template __global__ void k_water_search<4, false>(const SysDev*, const SearchParams);
template __global__ void k_water_search<4, true>(const SysDev*, const SearchParams);
template __global__ void k_water_search<8, true>(const SysDev*, const SearchParams);
}  // namespace gnb
