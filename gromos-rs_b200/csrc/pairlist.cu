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
// Stages: k_refpos (reference positions, cell keys, counts; its last block
// scans the cell counts) -> k_scatter -> k_cell_sort (rank sort, per cell,
// deterministic; its last block scans the cluster counts) ->
// k_cluster_setup (solvent i-clusters of W CGs) ->
// k_cell_candidates (each cell's j-cluster candidates, contiguous) ->
// k_water_search (water-water j-lists with W-bit masks) and
// k_solute_search (per solute CG j-lists with exclusion masks) ->
// k_pert_pairs (explicit perturbed atom pairs for the FEP correction).
#include "nb_common.cuh"

namespace gnb {

__device__ __forceinline__ int imod(int a, int m) {
    int r = a % m;
    return r < 0 ? r + m : r;
}

// Cell of stencil lane l (0..26, offsets in z-y-x order, -1..1 per axis;
// grids of 1 or 2 cells along an axis use the de-duplicated offsets of
// axis_offsets), -1 for a lane a small grid does not use.  The stencil is
// symmetric: c is in the stencil of c' iff c' is in the stencil of c.
__device__ __forceinline__ int stencil_cell(int cell, int l, int gx, int gy, int gz) {
    const int ix = l % 3, iy = (l / 3) % 3, iz = l / 9;
    if (ix >= (gx >= 3 ? 3 : gx) || iy >= (gy >= 3 ? 3 : gy) || iz >= (gz >= 3 ? 3 : gz)) return -1;
    const int cx = cell % gx, cy = (cell / gx) % gy, cz = cell / (gx * gy);
    const int ox = gx >= 3 ? ix - 1 : ix, oy = gy >= 3 ? iy - 1 : iy, oz = gz >= 3 ? iz - 1 : iz;
    return imod(cx + ox, gx) + gx * (imod(cy + oy, gy) + gy * imod(cz + oz, gz));
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

// Reference positions + cell keys (pairlist.rs:196-198, 577-585, 658-663).
__device__ __forceinline__ void refpos_one(const SysDev& s, int c, unsigned long long* __restrict__ cg_key) {
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
    // order inside the cell: ncol[0] x ncol[1] columns visited row by row,
    // every other row backwards, and z along each column, every other column
    // downwards (64 levels), so that W consecutive CGs are close together
    const int ncx = s.ncol[0], ncy = s.ncol[1];
    int kx = min(ncx - 1, static_cast<int>(fx * ncx));
    const int ky = min(ncy - 1, static_cast<int>(fy * ncy));
    if (ky & 1) kx = ncx - 1 - kx;
    const unsigned col = static_cast<unsigned>(ky * ncx + kx);
    const unsigned zq = min(63u, static_cast<unsigned>(((col & 1u) ? 1.0 - fz : fz) * 64.0));
    const unsigned order = (col << 6) | zq;  // 10 bits
    unsigned long long solvent = c >= s.n_solute_cg ? 1ull : 0ull;
    // the cell's bits only label the key (keys are sorted within a cell)
    cg_key[c] = (static_cast<unsigned long long>(cell) << 43) | (solvent << 42) |
                (static_cast<unsigned long long>(order) << 32) | static_cast<unsigned>(c);
    s.cg_cell[c] = cell;
    s.cg_slot[c] = -1;
    atomicAdd(&s.cell_count[cell], 1);
}

// Exclusive scan of n ints by one block (blockDim a multiple of 32, at most
// 1024): each pass takes 8 consecutive values per thread, so a grid of up to
// 8 x blockDim cells is one pass.  out has n + 1 entries (out[n] = total) and
// may alias in (each thread reads its values before writing them).  The
// values are read past L1 (other blocks of the same kernel wrote them).
__device__ void block_scan8(const int* in, int* out, int n, int* total) {
    __shared__ int wsum[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int carry = 0;
    for (int base = 0; base < n; base += 8 * blockDim.x) {
        const int i0 = base + 8 * threadIdx.x;
        int v[8], t = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v[k] = i0 + k < n ? __ldcg(in + i0 + k) : 0;
            t += v[k];
        }
        int x = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = lane < nw ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        int e = carry + (wid > 0 ? wsum[wid - 1] : 0) + x - t;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (i0 + k < n) out[i0 + k] = e;
            e += v[k];
        }
        carry += wsum[nw - 1];
        __syncthreads();  // wsum is reused by the next pass
    }
    if (threadIdx.x == 0) {
        out[n] = carry;
        if (total) *total = carry;
    }
}

// Whether this block is the last of its grid to get here: every earlier
// block's global writes (and atomics) are visible to it afterwards.  The
// counter is left at zero for the next launch.
__device__ __forceinline__ bool last_block(int* ctr) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(ctr, 1) == int(gridDim.x * gridDim.y) - 1;
        if (last) *ctr = 0;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// The last block scans the cell counts into the cell starts and clears the
// counts and the scatter's fill counters for the next build.
__global__ void k_refpos(const SysDev* __restrict__ sys, unsigned long long* __restrict__ cg_key) {
    const SysDev& s = sys[blockIdx.y];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < s.n_cg) refpos_one(s, c, cg_key);
    if (last_block(s.build_ctr)) {
        block_scan8(s.cell_count, s.cell_start, s.n_cells, nullptr);
        __syncthreads();
        for (int i = threadIdx.x; i < s.n_cells; i += blockDim.x) {
            s.cell_count[i] = 0;
            s.cell_fill[i] = 0;
        }
    }
}

__global__ void k_scatter(const SysDev* __restrict__ sys, const unsigned long long* __restrict__ cg_key) {
    const SysDev& s = sys[blockIdx.y];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= s.n_cg) return;
    const int cell = s.cg_cell[c];
    const int p = s.cell_start[cell] + atomicAdd(&s.cell_fill[cell], 1);
    s.keys[p] = cg_key[c];
}

// One block per cell: rank sort of the cell's keys (keys are unique: they
// end in the CG index), one barrier; each key is then written at its rank
// with the sorted CG maps and the sorted FP64 reference positions.  The last
// block scans the cells' cluster counts into cluster starts.
__global__ void __launch_bounds__(256) k_cell_sort(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    __shared__ unsigned long long sk[kMaxCellCGs];
    __shared__ int nsol;
    const int cell = blockIdx.x;
    const int start = s.cell_start[cell], n = s.cell_start[cell + 1] - start;
    if (n > kMaxCellCGs) {
        if (threadIdx.x == 0) {
            atomicOr(&s.err[0], ERR_CELL_TOO_DENSE);
            s.cell_nsolute[cell] = 0;
            s.cell_nclus[cell] = 0;
        }
    } else {
        unsigned long long* __restrict__ keys = s.keys;
        int* __restrict__ sorted_cg = s.sorted_cg;
        int* __restrict__ cg_spos = s.cg_spos;
        double* __restrict__ sref = s.sref;
        const double* __restrict__ ref = s.ref;
        const int stride = s.n_cg + 2;
        if (threadIdx.x == 0) nsol = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) sk[i] = keys[start + i];
        __syncthreads();
        int local = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long key = sk[i];
            int rank = 0;
            int j = 0;
            for (; j + 4 <= n; j += 4)
                rank += int(sk[j] < key) + int(sk[j + 1] < key) + int(sk[j + 2] < key) + int(sk[j + 3] < key);
            for (; j < n; ++j) rank += int(sk[j] < key);
            const int cg = static_cast<int>(key & 0xffffffffull);
            const int p = start + rank;
            const double rx = ref[3 * cg], ry = ref[3 * cg + 1], rz = ref[3 * cg + 2];
            keys[p] = key;
            sorted_cg[p] = cg;
            cg_spos[cg] = p;
            sref[p] = rx;
            sref[stride + p] = ry;
            sref[2 * stride + p] = rz;
            if (((key >> 42) & 1ull) == 0ull) ++local;
        }
        if (local) atomicAdd(&nsol, local);
        __syncthreads();
        if (threadIdx.x == 0) {
            s.cell_nsolute[cell] = nsol;
            s.cell_nclus[cell] = (n - nsol + s.W - 1) / s.W;
        }
    }
    if (last_block(s.build_ctr + 1)) {
        __shared__ int total;
        block_scan8(s.cell_nclus, s.cell_nclus, s.n_cells, &total);
        __syncthreads();
        if (threadIdx.x == 0) {
            s.n_deferred[6] = 0;  // the water search's cluster counter
            s.n_deferred[7] = 0;  // the candidate lists' allocation counter
            if (total > s.max_clusters) {
                atomicOr(&s.err[0], ERR_WLIST_OVERFLOW);
                total = s.max_clusters;
            }
            s.n_clusters[0] = total;
        }
    }
}

// One block per cell, one thread per slot of the cell's clusters (the W
// slots of a cluster are W consecutive lanes): the slot <-> CG maps, the
// member offsets from the cluster's first atom and, reduced over the
// cluster's lanes, its record and search geometry (FP64 first atom, bounding
// box of the first atoms, radius of the offsets).
__global__ void __launch_bounds__(256) k_cluster_setup(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[blockIdx.y];
    const int cell = blockIdx.x;
    const int W = s.W;  // 4 or 8: a cluster's lanes are an aligned group
    const int c0 = s.cell_nclus[cell], c1 = s.cell_nclus[cell + 1];
    const int first_solv = s.cell_start[cell] + s.cell_nsolute[cell];
    const int nsolv = s.cell_start[cell + 1] - first_solv;
    const int max_clusters = s.max_clusters;
    const int stride = s.n_cg + 2;
    const double* __restrict__ sref = s.sref;
    const int* __restrict__ sorted_cg = s.sorted_cg;
    const int nslots = (c1 - c0) * W;
    for (int base = 0; base < nslots; base += blockDim.x) {  // block-uniform trip count
        const int t = base + threadIdx.x;
        const int local = t / W, m = t - local * W;
        const int k = c0 + local;
        const bool live = t < nslots && k < max_clusters;
        const int first = first_solv + local * W;
        const int n = live ? min(W, nsolv - local * W) : 0;
        double x = 0.0, y = 0.0, z = 0.0;
        int cg = -1;
        if (m < n) {
            cg = sorted_cg[first + m];
            x = sref[first + m];
            y = sref[stride + first + m];
            z = sref[2 * stride + first + m];
        }
        // the group's first atom (lane m = 0 of the group)
        const int g0 = (threadIdx.x & 31) & ~(W - 1);
        const double x0 = __shfl_sync(0xffffffffu, x, g0), y0 = __shfl_sync(0xffffffffu, y, g0);
        const double z0 = __shfl_sync(0xffffffffu, z, g0);
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        double lx = x0, ly = y0, lz = z0, hx = x0, hy = y0, hz = z0;
        if (m < n) {
            o.x = float(x - x0);
            o.y = float(y - y0);
            o.z = float(z - z0);
            lx = hx = x;
            ly = hy = y;
            lz = hz = z;
        }
        float rad = sqrtf(o.x * o.x + o.y * o.y + o.z * o.z);
        for (int d = 1; d < W; d <<= 1) {
            rad = fmaxf(rad, __shfl_xor_sync(0xffffffffu, rad, d));
            lx = fmin(lx, __shfl_xor_sync(0xffffffffu, lx, d));
            ly = fmin(ly, __shfl_xor_sync(0xffffffffu, ly, d));
            lz = fmin(lz, __shfl_xor_sync(0xffffffffu, lz, d));
            hx = fmax(hx, __shfl_xor_sync(0xffffffffu, hx, d));
            hy = fmax(hy, __shfl_xor_sync(0xffffffffu, hy, d));
            hz = fmax(hz, __shfl_xor_sync(0xffffffffu, hz, d));
        }
        if (live) {
            const int slot = k * W + m;
            s.slot_cg[slot] = cg;
            if (cg >= 0) s.cg_slot[cg] = slot;
            s.slot_off[slot] = o;
            if (m == 0) {
                s.clus_cell[k] = cell;
                s.clus_first[k] = first;
                s.clus_n[k] = n;
                s.clus_x64[4 * k] = x0;
                s.clus_x64[4 * k + 1] = y0;
                s.clus_x64[4 * k + 2] = z0;
                s.clus_x64[4 * k + 3] = 0.0;
                s.clus_geo[k] = make_float4(float(0.5 * (lx + hx)), float(0.5 * (ly + hy)), float(0.5 * (lz + hz)),
                                            rad * (1.f + 1e-5f) + 1e-5f);
                s.clus_ext[k] = make_float4(float(0.5 * (hx - lx)) * (1.f + 1e-6f) + 1e-6f,
                                            float(0.5 * (hy - ly)) * (1.f + 1e-6f) + 1e-6f,
                                            float(0.5 * (hz - lz)) * (1.f + 1e-6f) + 1e-6f, 0.f);
            }
        }
    }
}

// Grid (n_cells, 2): the candidate list of the water search for the
// clusters of parity p = blockIdx.y of one cell, the geometry and index of
// the j-clusters such a cluster can own.  A pair of clusters a < b belongs
// to a when a + b is even and to b when it is odd.  The list holds the own
// cell's clusters of parity p (run A; a cluster owns those from itself on),
// those of parity 1 - p (run B; it owns those before itself), then the
// owned clusters of the stencil cells: the clusters of another cell lie all
// before or all after this cell's, so from a cell after this one those of
// parity p, from a cell before it those of parity 1 - p.  Every cluster thus
// owns about half of the pairs around it in every direction, and all lists
// are about equally long.  The lists are placed by an atomic counter: where
// a list lies does not change what it holds.
__global__ void __launch_bounds__(256) k_cell_candidates(const SysDev* __restrict__ sys) {
    const SysDev& s = sys[0];
    const int cell = blockIdx.x, par = blockIdx.y;
    constexpr int kSegs = 29;  // runs A and B, 27 stencil lanes
    __shared__ int seg_lo[kSegs], seg_pre[kSegs + 1];
    __shared__ int base_s;
    const int gx = s.gdim[0], gy = s.gdim[1], gz = s.gdim[2];
    const int max_clusters = s.max_clusters;
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        int lo = 0, len = 0, c0 = 0, c1 = 0, q = 0;
        if (l < 2) {  // own cell: parity p (A), then 1 - p (B)
            c0 = s.cell_nclus[cell];
            c1 = min(s.cell_nclus[cell + 1], max_clusters);
            q = par + l;
        } else if (l < kSegs) {
            const int nc = stencil_cell(cell, l - 2, gx, gy, gz);
            if (nc >= 0 && nc != cell) {
                c0 = s.cell_nclus[nc];
                c1 = min(s.cell_nclus[nc + 1], max_clusters);
                q = nc > cell ? par : par + 1;
            }
        }
        if (c1 > c0) {
            lo = c0 + ((c0 - q) & 1);
            len = lo < c1 ? (c1 - lo + 1) >> 1 : 0;
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (l >= o) incl += y;
        }
        if (l < kSegs) {
            seg_lo[l] = lo;
            seg_pre[l] = incl - len;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        if (l == 0) {
            int n = total;
            int base = atomicAdd(s.n_deferred + 7, total);
            if (base + total > s.cand_cap) {
                atomicOr(&s.err[0], ERR_WLIST_OVERFLOW);
                base = 0;
                n = 0;
            }
            seg_pre[kSegs] = n;
            base_s = base;
            s.cell_cand[2 * cell + par] = base;
            s.cell_ncand[2 * cell + par] = n;
        }
    }
    __syncthreads();
    const int total = seg_pre[kSegs], base = base_s;
    const float4* __restrict__ geo = s.clus_geo;
    const float4* __restrict__ ext = s.clus_ext;
    float4* __restrict__ cgeo = s.cand_geo + base;
    float4* __restrict__ cext = s.cand_ext + base;
    // two entries per thread and pass, loads first
    for (int v0 = threadIdx.x; v0 < total; v0 += 2 * blockDim.x) {
        int jc[2];
        float4 g[2], e[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int v = v0 + u * blockDim.x;
            jc[u] = -1;
            if (v < total) {
                int lo = 0;  // run of v: binary search over the kSegs + 1 offsets
#pragma unroll
                for (int step = 16; step > 0; step >>= 1)
                    if (lo + step <= kSegs && seg_pre[lo + step] <= v) lo += step;
                jc[u] = seg_lo[lo] + 2 * (v - seg_pre[lo]);
                g[u] = geo[jc[u]];
                e[u] = ext[jc[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (jc[u] < 0) continue;
            const int v = v0 + u * blockDim.x;
            e[u].w = __int_as_float(jc[u]);
            cgeo[v] = g[u];
            cext[v] = e[u];
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

// Water-water search, one warp per i-cluster (clusters handed out by a
// counter, so every warp stays busy to the end).  Every unordered CG pair is
// listed once: a pair of two clusters a < b belongs to a when a + b is even,
// to b when it is odd; a pair inside one cluster to the member that comes
// first in sorted order.  Each cluster owns about half of the pairs around
// it in every direction, wherever it sits in its cell, so all lists (and the
// search's and the force kernels' work per cluster) are about equally long.
// (Listing a pair under the cluster that comes first in sorted order gives
// lists of 0 to 2.3 times the mean length.)  Bit k of the short (long) mask is set when the
// reference test puts (i_k, j) in the short (long) range; the solvent
// reference point is the first atom for both CGs (pairlist.rs:359-368).
//
// The candidates are the owned j-clusters: in the own cell every second
// cluster (two strided runs), in the stencil cells those of the cell's
// candidate list for this cluster's parity (k_cell_candidates: geometry and
// index, contiguous).  They are swept 32 at a time with a
// conservative FP32 test of the gap between the two clusters' axis-aligned
// bounding boxes (1e-3 nm margin).  Survivors queue in shared memory in
// candidate order; lane q takes survivor q of the next 32: the
// cluster-to-cluster vector C with the FP64 image of the two first atoms,
// rounded once, then all W x W member pairs, the pair vector being the i
// offset + C - the j offset (offsets from the cluster's first atom, FP32);
// the lanes' entries are compacted member by member.  A squared distance
// within a relative 1e-5 of either cutoff, or a vector near half a box edge
// (image not certain in FP32), is decided by the exact FP64 test
// (nearest_image_exact + len2_exact).  The FP32 error is below 1e-6
// relative, so the set is exactly the reference's.
//
// Each cluster's entries are collected in shared memory and written out
// sorted by mask value (or popcount), so warp chunks of the force kernel see
// similar masks.
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

// Stable counting sort of a cluster's entries by popcount of the mask, most
// bits first: lanes of a warp chunk then iterate over the same number of bits,
// and the last, partly filled chunk holds the cheapest entries.
template <int W>
__device__ __forceinline__ void sort_write_entries_pop(const uint32_t* __restrict__ buf, int nbuf,
                                                       uint32_t* __restrict__ out, int lane) {
    if constexpr (W == 4) {
        // popcount - 1 as two bits, one ballot each: the four class masks and
        // counts follow from three ballots, and each lane stores once
        const unsigned lt = (1u << lane) - 1u;
        int n[4] = {0, 0, 0, 0};
        for (int c = 0; c < nbuf; c += 32) {
            const int e = c + lane;
            const bool valid = e < nbuf;
            const int k = valid ? __popc(buf[e] & 0xffu) - 1 : 0;
            const unsigned bv = __ballot_sync(0xffffffffu, valid);
            const unsigned b0 = __ballot_sync(0xffffffffu, valid && (k & 1));
            const unsigned b1 = __ballot_sync(0xffffffffu, valid && (k & 2));
            n[3] += __popc(b0 & b1);
            n[2] += __popc(b1 & ~b0);
            n[1] += __popc(b0 & ~b1);
            n[0] += __popc(bv & ~(b0 | b1));
        }
        int o3 = 0, o2 = n[3], o1 = n[3] + n[2], o0 = n[3] + n[2] + n[1];  // most bits first
        for (int c = 0; c < nbuf; c += 32) {
            const int e = c + lane;
            const bool valid = e < nbuf;
            const uint32_t ent = valid ? buf[e] : 0u;
            const int k = valid ? __popc(ent & 0xffu) - 1 : 0;
            const unsigned bv = __ballot_sync(0xffffffffu, valid);
            const unsigned b0 = __ballot_sync(0xffffffffu, valid && (k & 1));
            const unsigned b1 = __ballot_sync(0xffffffffu, valid && (k & 2));
            const unsigned m3 = b0 & b1, m2 = b1 & ~b0, m1 = b0 & ~b1, m0 = bv & ~(b0 | b1);
            const unsigned mine = k == 3 ? m3 : k == 2 ? m2 : k == 1 ? m1 : m0;
            const int base = k == 3 ? o3 : k == 2 ? o2 : k == 1 ? o1 : o0;
            if (valid) out[base + __popc(mine & lt)] = ent;
            o3 += __popc(m3);
            o2 += __popc(m2);
            o1 += __popc(m1);
            o0 += __popc(m0);
        }
        return;
    }
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
    off[W] = 0;
#pragma unroll
    for (int v = W - 1; v >= 0; --v) off[v] = off[v + 1] + hist[v + 1];
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
__global__ void __launch_bounds__(kSearchWarps * 32, W == 4 ? 8 : 4) k_water_search(const SysDev* __restrict__ sys, const SearchParams P) {
    const SysDev& s = sys[blockIdx.y];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ uint32_t ebuf_s[kSearchWarps][kEntBuf], ebuf_l[kSearchWarps][kEntBuf];
    __shared__ int q_jc[kSearchWarps][64];          // surviving j-clusters, candidate order
    __shared__ float q_sp[kSearchWarps][64];        // their offset radii (clus_geo .w)
    const int nclus = s.n_clusters[0];
    const float4* __restrict__ geo = s.clus_geo;
    const float4* __restrict__ ext = s.clus_ext;
    const float4* __restrict__ soff = s.slot_off;
    const double* __restrict__ x64 = s.clus_x64;
    const double* __restrict__ sref = s.sref;
    const int stride = s.n_cg + 2;
    const float c2s = float(P.c2s), c2l = float(P.c2l);
    const float s_lo = c2s * (1.f - 1e-5f), s_hi = c2s * (1.f + 1e-5f);
    const float l_lo = c2l * (1.f - 1e-5f), l_hi = c2l * (1.f + 1e-5f);
    const float rcl = sqrtf(c2l) * (1.f + 1e-6f) + 1e-3f;
    const float limx = P.boundary ? P.half_boxf[0] - 1e-4f : 3e38f;
    const float limy = P.boundary ? P.half_boxf[1] - 1e-4f : 3e38f;
    const float limz = P.boundary ? P.half_boxf[2] - 1e-4f : 3e38f;
    const unsigned below = (1u << lane) - 1u;
    for (;;) {
        int ci = 0;
        if (lane == 0) ci = atomicAdd(s.n_deferred + 6, 1);
        ci = __shfl_sync(0xffffffffu, ci, 0);
        if (ci >= nclus) break;
        const int n_i = s.clus_n[ci], first_i = s.clus_first[ci], cell = s.clus_cell[ci];
        const float4 gi = geo[ci], hi = ext[ci];
        const double X0 = x64[4 * ci], Y0 = x64[4 * ci + 1], Z0 = x64[4 * ci + 2];
        float ex[W], ey[W], ez[W];
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const float4 o = soff[ci * W + k];
            ex[k] = o.x;
            ey[k] = o.y;
            ez[k] = o.z;
        }
        // candidates, from the list of this cell and parity: run A from ci
        // on (ci itself for its internal pairs), run B before ci, then the
        // stencil cells' clusters
        const int oc0 = s.cell_nclus[cell], oc1 = min(s.cell_nclus[cell + 1], s.max_clusters);
        const int a0 = oc0 + ((oc0 - ci) & 1), b0 = oc0 + ((oc0 - ci - 1) & 1);
        const int len_a = (oc1 - a0 + 1) >> 1, len_b = b0 < oc1 ? (oc1 - b0 + 1) >> 1 : 0;
        const int skip_a = (ci - a0) >> 1;                       // A entries before ci
        const int nb = b0 < ci ? (ci - b0 + 1) >> 1 : 0;         // B entries before ci
        const int n_ab = len_a - skip_a + nb;                     // own-cell candidates
        const int skip_ab = skip_a + len_b - nb;                  // + B entries after ci
        const int lidx = 2 * cell + (ci & 1);
        const int total = s.cell_ncand[lidx] - skip_ab;
        const float4* __restrict__ cgeo = s.cand_geo + s.cell_cand[lidx];
        const float4* __restrict__ cext = s.cand_ext + s.cell_cand[lidx];
        uint32_t* outs = s.wl_s + static_cast<size_t>(ci) * P.wcap;
        uint32_t* outl = s.wl_l + static_cast<size_t>(ci) * P.wcap;
        int cnt_s = 0, cnt_l = 0, qn = 0, v0 = 0;
        for (;;) {
            // sphere tests until 32 survivors are queued or the candidates end
            while (v0 < total && qn < 32) {
                const int v = v0 + lane;
                bool surv = false;
                int jc = 0;
                float rj = 0.f;
                if (v < total) {
                    // list position: skip A's entries before ci, and B's after it
                    const int pos = v + (v < n_ab ? skip_a : skip_ab);
                    const float4 gj = cgeo[pos], hj = cext[pos];
                    jc = min(max(__float_as_int(hj.w), 0), nclus - 1);
                    rj = gj.w;
                    float dx = gi.x - gj.x, dy = gi.y - gj.y, dz = gi.z - gj.z;
                    if (P.boundary) {
                        dx -= P.boxf[0] * rintf(dx * P.inv_boxf[0]);
                        dy -= P.boxf[1] * rintf(dy * P.inv_boxf[1]);
                        dz -= P.boxf[2] * rintf(dz * P.inv_boxf[2]);
                    }
                    // gap between the two boxes along each axis
                    dx = fmaxf(fabsf(dx) - hi.x - hj.x, 0.f);
                    dy = fmaxf(fabsf(dy) - hi.y - hj.y, 0.f);
                    dz = fmaxf(fabsf(dz) - hi.z - hj.z, 0.f);
                    surv = dx * dx + dy * dy + dz * dz <= rcl * rcl;
                }
                const unsigned b = __ballot_sync(0xffffffffu, surv);
                if (surv) {
                    q_jc[w][qn + __popc(b & below)] = jc;
                    q_sp[w][qn + __popc(b & below)] = rj;
                }
                qn += __popc(b);
                v0 += 32;
            }
            if (qn == 0) break;
            const int nq = min(qn, 32);
            __syncwarp();
            // lane q classifies survivor q: the cluster-to-cluster vector C
            // (FP64 image of the first atoms, rounded once), then per member
            // m the W x W pair vectors i offset + C - j offset (FP32)
            int jc = 0;
            unsigned ms[W], ml[W], am[W];
#pragma unroll
            for (int m = 0; m < W; ++m) ms[m] = ml[m] = am[m] = 0u;
            if (lane < nq) {
                jc = q_jc[w][lane];
                const int n_j = s.clus_n[jc];
                const float span = gi.w + q_sp[w][lane];
                double cdx = X0 - x64[4 * jc], cdy = Y0 - x64[4 * jc + 1], cdz = Z0 - x64[4 * jc + 2];
                if (P.boundary) {
                    cdx -= P.box[0] * rint(cdx * P.inv_box[0]);
                    cdy -= P.box[1] * rint(cdy * P.inv_box[1]);
                    cdz -= P.box[2] * rint(cdz * P.inv_box[2]);
                }
                const float Cx = float(cdx), Cy = float(cdy), Cz = float(cdz);
                // |C + i offset - j offset| per axis stays below |C| + both
                // radii: when that is below half a box edge, the sum is the
                // minimum image of every member pair
                const bool edge = P.boundary && !(fabsf(Cx) + span < limx && fabsf(Cy) + span < limy &&
                                                  fabsf(Cz) + span < limz);
                // pairs {i_k, j_m} with k < n_i, m < n_j and i_k before j_m in sorted order
                const unsigned valid_i = (1u << n_i) - 1u;
#pragma unroll
                for (int m = 0; m < W; ++m) {
                    const float4 o = soff[jc * W + m];
                    float Dx = Cx - o.x, Dy = Cy - o.y, Dz = Cz - o.z;
                    if (edge) {  // the sum of two minimum images need not be one
                        Dx -= P.boxf[0] * rintf(Dx * P.inv_boxf[0]);
                        Dy -= P.boxf[1] * rintf(Dy * P.inv_boxf[1]);
                        Dz -= P.boxf[2] * rintf(Dz * P.inv_boxf[2]);
                    }
                    unsigned valid = m < n_j ? valid_i : 0u;
                    if (jc == ci) valid &= (1u << m) - 1u;
                    unsigned s_m = 0, l_m = 0, a_m = 0;
#pragma unroll
                    for (int k = 0; k < W; ++k) {
                        const float kx = ex[k] + Dx, ky = ey[k] + Dy, kz = ez[k] + Dz;
                        const float d2 = kx * kx + ky * ky + kz * kz;
                        s_m |= unsigned(d2 < s_lo) << k;
                        l_m |= unsigned(d2 > s_hi && d2 < l_lo) << k;
                        a_m |= unsigned((d2 >= s_lo && d2 <= s_hi) || (d2 >= l_lo && d2 <= l_hi)) << k;
                        if (edge) {
                            const bool inbox = fabsf(kx) < limx && fabsf(ky) < limy && fabsf(kz) < limz;
                            a_m |= unsigned(!inbox) << k;
                        }
                    }
                    ms[m] = s_m & valid & ~a_m;
                    ml[m] = l_m & valid & ~a_m;
                    am[m] = a_m & valid;
                }
            }
            // the rare ambiguous pairs: the exact FP64 decision
            // (nearest_image_exact + len2_exact, box from the kernel
            // parameters) for the lanes that have some
            unsigned any_am = 0u;
#pragma unroll
            for (int m = 0; m < W; ++m) any_am |= am[m];
            if (__any_sync(0xffffffffu, any_am != 0u) && any_am) {
                const int fj = s.clus_first[jc];
#pragma unroll
                for (int m = 0; m < W; ++m) {
                    unsigned a = am[m];
                    if (!a) continue;
                    const int sp = fj + m;
                    const double tjx = sref[sp], tjy = sref[stride + sp], tjz = sref[2 * stride + sp];
                    unsigned add_s = 0u, add_l = 0u;
                    while (a) {
                        const int k = __ffs(a) - 1;
                        a &= a - 1u;
                        double rx = __dsub_rn(sref[first_i + k], tjx);
                        double ry = __dsub_rn(sref[stride + first_i + k], tjy);
                        double rz = __dsub_rn(sref[2 * stride + first_i + k], tjz);
                        if (P.boundary) {
                            rx = image_exact(rx, P.box[0], P.inv_box[0]);
                            ry = image_exact(ry, P.box[1], P.inv_box[1]);
                            rz = image_exact(rz, P.box[2], P.inv_box[2]);
                        }
                        const double e2 = len2_exact(rx, ry, rz);
                        if (!(e2 > P.c2l)) {
                            if (e2 > P.c2s)
                                add_l |= 1u << k;
                            else
                                add_s |= 1u << k;
                        }
                    }
                    ms[m] |= add_s;
                    ml[m] |= add_l;
                }
            }
            // entries of member m of every lane's survivor, compacted in lane order
#pragma unroll
            for (int m = 0; m < W; ++m) {
                const uint32_t slot = static_cast<uint32_t>(jc * W + m);
                const unsigned bs = __ballot_sync(0xffffffffu, ms[m] != 0u);
                const unsigned bl = __ballot_sync(0xffffffffu, ml[m] != 0u);
                if (ms[m]) {
                    const int p = cnt_s + __popc(bs & below);
                    const uint32_t ent = (slot << 8) | ms[m];
                    if (p < kEntBuf)
                        ebuf_s[w][p] = ent;
                    else if (p < P.wcap)
                        outs[p] = ent;
                }
                if (ml[m]) {
                    const int p = cnt_l + __popc(bl & below);
                    const uint32_t ent = (slot << 8) | ml[m];
                    if (p < kEntBuf)
                        ebuf_l[w][p] = ent;
                    else if (p < P.wcap)
                        outl[p] = ent;
                }
                cnt_s += __popc(bs);
                cnt_l += __popc(bl);
            }
            // keep the survivors beyond the 32 just classified
            const int rem = qn - nq;
            const int keep = lane < rem ? q_jc[w][32 + lane] : 0;
            const float keep_sp = lane < rem ? q_sp[w][32 + lane] : 0.f;
            __syncwarp();
            if (lane < rem) {
                q_jc[w][lane] = keep;
                q_sp[w][lane] = keep_sp;
            }
            qn = rem;
            __syncwarp();
        }
        __syncwarp();
        // an overflowing list (more entries than its capacity; the build is redone with
        // grown lists) writes no further than its capacity
        const int nws = min(min(cnt_s, kEntBuf), P.wcap), nwl = min(min(cnt_l, kEntBuf), P.wcap);
        if (POPSORT) {
            sort_write_entries_pop<W>(ebuf_s[w], nws, outs, lane);
            sort_write_entries_pop<W>(ebuf_l[w], nwl, outl, lane);
        } else {
            sort_write_entries(ebuf_s[w], nws, outs, lane);
            sort_write_entries(ebuf_l[w], nwl, outl, lane);
        }
        if (lane == 0) {
            if (cnt_s > P.wcap || cnt_l > P.wcap) atomicOr(&s.err[0], ERR_WLIST_OVERFLOW);
            s.wn_s[ci] = min(cnt_s, P.wcap);
            s.wn_l[ci] = min(cnt_l, P.wcap);
        }
        __syncwarp();  // the entry buffers and queues are reused by the next cluster
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
    // Candidates are swept 32 at a time through the neighbour cells in z-y-x
    // order; positions come from the sorted copy of the reference positions
    // (sref: the same FP64 values, stored at the sorted position) and the next
    // round's candidate is loaded while this round's is tested, so a round
    // waits for one memory latency instead of two chained ones.
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
    const double xi = s.ref[3 * ci], yi = s.ref[3 * ci + 1], zi = s.ref[3 * ci + 2];
    const int cell = s.cg_cell[ci];
    const int gx = s.gdim[0], gy = s.gdim[1], gz = s.gdim[2];
    const int cx = cell % gx, cy = (cell / gx) % gy, cz = cell / (gx * gy);
    int ox[3], oy[3], oz[3];
    const int nx = axis_offsets(gx, ox), ny = axis_offsets(gy, oy), nz = axis_offsets(gz, oz);
    int ncl[27];
    int nn = 0;
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix)
                ncl[nn++] = imod(cx + ox[ix], gx) + gx * (imod(cy + oy[iy], gy) + gy * imod(cz + oz[iz], gz));
    const int stride = s.n_cg + 2;
    const int* __restrict__ cell_start = s.cell_start;
    const int* __restrict__ sorted_cg = s.sorted_cg;
    const double* __restrict__ sref = s.sref;
    // sweep state: neighbour k, round start base within [cell_start[ncl[k]], cell_start[ncl[k] + 1])
    int k = 0, base = 0, end = 0;
    auto seek = [&]() {  // first non-empty cell at or after k
        while (k < nn) {
            base = cell_start[ncl[k]];
            end = cell_start[ncl[k] + 1];
            if (base < end) return;
            ++k;
        }
    };
    struct Cand {
        int cj;
        double x, y, z;
    };
    auto load = [&](int b, int e) {
        Cand c{-1, 0.0, 0.0, 0.0};
        const int sp = b + lane;
        if (sp < e) {
            c.cj = sorted_cg[sp];
            c.x = sref[sp];
            c.y = sref[stride + sp];
            c.z = sref[2 * stride + sp];
        }
        return c;
    };
    seek();
    Cand cur = k < nn ? load(base, end) : Cand{-1, 0.0, 0.0, 0.0};
    while (k < nn) {
        // the next round: advance, then load it before this round is tested
        int nb = base + 32, ne = end;
        if (nb >= end) {
            ++k;
            seek();
            nb = base;
            ne = end;
        }
        const bool more = k < nn;
        const Cand nxt = more ? load(nb, ne) : Cand{-1, 0.0, 0.0, 0.0};
        int entry = -1;
        unsigned long long xm = 0;
        const int cj = cur.cj;
        if (cj >= 0) {
            const bool solute_j = cj < s.n_solute_cg;
            if (!solute_j || cj > ci) {
                double rx, ry, rz;
                nearest_image_exact(s, xi, yi, zi, cur.x, cur.y, cur.z, rx, ry, rz);
                const double d2 = len2_exact(rx, ry, rz);
                if (!(d2 > s.c2l)) {
                    const int lr = d2 > s.c2s ? 1 : 0;
                    if (solute_j && s.cg_off[cj + 1] - s.cg_off[cj] > kMaxCGAtoms) {
                        atomicOr(&s.err[0], ERR_CG_TOO_LARGE);
                    } else {
                        entry = (cj << 1) | lr;
                        if (solute_j && !lr) xm = excl_mask(s, ci, cj);
                    }
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, entry >= 0);
        if (entry >= 0) {
            const int p = cnt + __popc(bal & ((1u << lane) - 1u));
            if (p < s.scap) {
                out[p] = entry;
                outx[p] = xm;
            }
        }
        cnt += __popc(bal);
        cur = nxt;
        base = nb;
        end = ne;
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
