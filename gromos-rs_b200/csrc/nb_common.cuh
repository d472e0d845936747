// nb_common.cuh -- device-side data layout and arithmetic helpers shared by
// the pairlist and force kernels of libgromos_nb.
//
// HBM layout (one system; a batch holds an array of these descriptors):
//   topology   : cg_off[n_cg+1] i32, charge f64, iac i32, lj64 [T*T*4] f64,
//                lj32 [T*T] float2 (c6, c12), exclusion / 1-4 CSR i32
//   positions  : pos [N*3] f64 (gromos-rs DVec3 layout)
//   pairlist   : ref [n_cg*3] f64 (COG for solute CGs, first atom for
//                solvent CGs), cell keys, CGs sorted by (cell, solute-first,
//                column, z, index), solvent i-clusters of W CGs,
//                per-cluster j-lists of packed (slot << 8 | mask) u32 entries
//                (short and long separately), per-solute-CG j-lists
//   per step   : water slots in cluster order: first-atom f64 position and
//                FP32 offsets of every atom from its CG's first atom
//   results    : 64-bit fixed-point force accumulators (short, long cache),
//                fixed-point energy-group / virial accumulators, f64 forces
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gnb {

constexpr int kMaxCGAtoms = 8;        // generic (solute) kernel: atoms per CG
constexpr int kMaxGroups = 16;        // energy groups
constexpr double kForceScale = 4294967296.0;   // 2^32: force fixed point
constexpr double kEnergyScale = 16777216.0;    // 2^24: energy / virial fixed point
constexpr int kMaxCellCGs = 2048;     // per-cell sort capacity (charge groups in one grid cell)
constexpr int kSearchWarps = 4;       // warps per block of the water search

// Error flags (bitwise OR into SysDev::err[0]).
enum : int {
    ERR_CELL_TOO_DENSE = 1,
    ERR_WLIST_OVERFLOW = 2,
    ERR_SLIST_OVERFLOW = 4,
    ERR_CG_TOO_LARGE = 8,
    ERR_PERT_OVERFLOW = 16,
    ERR_CGPAIR_OVERFLOW = 32,
    ERR_DEFER_OVERFLOW = 64,
};

// One water per slot, 48 bytes, read with three 16-byte loads: the FP64
// position of the first atom and the FP32 offsets of atoms 1 and 2 from it.
struct __align__(16) WaterRec {
    double x0, y0;
    double z0;
    float h1x, h1y;
    float h1z, h2x, h2y, h2z;
};

struct SysDev {
    // ---- sizes and flags
    int n_atoms, n_cg, n_solute_cg, n_solute_atoms, aps, n_types, n_egroups;
    int boundary;        // 0 vacuum, 1 rectangular
    int twin;            // twin-range active (rcutp < rcutl - 1e-10)
    int cg_grouped;      // use_cg_grouped_solute (forcefield.rs:267-283)
    int W;               // solvent cluster width
    int has_pert;
    int water_lj00_only; // solvent LJ only between site 0 and site 0
    int solvent_group;   // energy group of all solvent atoms (-1 = mixed)
    int excl_atoms;      // atoms [0, excl_atoms) go through k_excluded_14; the
                         // intra-molecular solvent exclusions are done in k_water_prep
    // ---- geometry (FP64, exact reference semantics)
    double box[3], inv_box[3];
    double c2s, c2l;     // (rcutp+skin)^2, (rcutl+skin)^2 (pairlist.rs:192-193)
    float boxf[3], inv_boxf[3], half_boxf[3];
    // ---- CRF (params.rs:78-96) and Coulomb prefactor
    double crf_cut, crf_2cut3i, crf_cut3i, cutoff_sq, fpe;
    float crf_cut_f, crf_2cut3i_f, crf_cut3i_f;
    // ---- cell grid
    int gdim[3], n_cells;
    double cell_size[3];
    int ncol[2];         // columns per cell along x and y (order inside a cell)
    // ---- solvent 3x3 parameter table from the first solvent molecule
    //      (innerloops.rs:241-255): c6, c12, q_i q_j fpe
    float w_c6[16], w_c12[16], w_qq[16];
    // ---- FEP lambda parameters (perturbed.rs:12-101), order of orc_lambda_params
    double lp[17];
    // ---- topology (device)
    const int* cg_off;
    const double* charge;
    const int* iac;
    const double* lj64;
    const float2* lj32;
    const int* excl_off;
    const int* excl;
    const int* o14_off;
    const int* o14;
    const int* egroup;
    const int* atom_cg;
    const int* pert_idx;       // n_atoms, -1 = unperturbed
    const int* pert_iac;       // [n_pert*2] a, b
    const double* pert_q;      // [n_pert*2] a, b
    const double* pert_alpha;  // [n_pert*2] lj, crf
    const int* pp;             // [n_pp*4] i, j, a_type, b_type
    int n_pert, n_pp;
    // ---- state
    double* pos;               // n_atoms*3
    // ---- pairlist build
    double* ref;               // n_cg*3
    unsigned long long* keys;  // n_cg (unsorted scatter, then sorted within cells)
    int* cg_cell;              // n_cg
    int* cell_count;           // n_cells (zero between builds)
    int* cell_fill;            // n_cells: the scatter's counters (zero between builds)
    int* build_ctr;            // [4] finished-block counters of the build kernels (zero between launches)
    int* cell_start;           // n_cells+1
    int* cell_nsolute;         // n_cells
    int* cell_nclus;           // n_cells+1 (scanned in place -> cluster start)
    int* cell_cand;            // 2*n_cells: start of each cell's candidate list per cluster parity
    int* cell_ncand;           // 2*n_cells: its length
    float4* cand_geo;          // [cand_cap] candidate j-clusters of the stencil cells: clus_geo
    float4* cand_ext;          // [cand_cap] clus_ext, .w = the j-cluster index (int bits)
    int cand_cap;
    int* sorted_cg;            // n_cg: sorted position -> CG
    double* sref;              // [3][n_cg + 2] sorted reference positions (x, y, z planes)
    int* cg_spos;              // n_cg: CG -> sorted position
    int* clus_cell;            // cluster -> cell
    int* clus_first;           // cluster -> first sorted position
    float4* clus_geo;          // cluster: FP32 bounding-box centre, radius of the offsets from the first atom
    float4* clus_ext;          // cluster: FP32 bounding-box half extents
    double* clus_x64;          // cluster*4: FP64 first-atom position (x, y, z, 0)
    float4* slot_off;          // slot: FP32 offset from the cluster's first atom
    int* clus_n;               // cluster -> #CGs (<= W)
    int* n_clusters;           // [1]
    int max_clusters;
    int* slot_cg;              // max_clusters*W: slot -> CG (-1 pad)
    int* cg_slot;              // n_cg: solvent CG -> slot (-1 for solute)
    uint32_t* wl_s;            // [max_clusters * wcap] packed (slot<<8 | mask)
    uint32_t* wl_l;
    int* wn_s;                 // [max_clusters]
    int* wn_l;
    int wcap;
    int* sl;                   // [n_solute_cg * scap] (j_cg << 1 | long)
    unsigned long long* sl_excl; // [n_solute_cg * scap] excluded atom-pair bits
    int* sn;                   // [n_solute_cg]
    int scap;
    int* pert_pairs;           // [pcap*3] (i, j, long)
    int* n_pert_pairs;         // [1]
    int pcap;
    // ---- per-step water data in slot order
    struct WaterRec* wrec;     // [max_clusters*W] per-slot FP64 first atom + FP32 offsets
    long long* fs_short;       // [max_clusters*W*9] water forces per slot (fixed 2^32)
    long long* fs_long;        // same, long-range cache
    int* deferred;             // [2 * 2 * defer_cap] (i slot, j slot): short, then long
    int* n_deferred;           // [8]: deferred pairs, water-kernel work counters, finished blocks (short, long each), search counter
    float* max_delta;          // [1] largest |offset| component of a water atom from its first atom (this step)
    int defer_cap;
    // ---- plain-kernel data
    float4* pos32;             // n_atoms (x, y, z, q)
    int* cgp;                  // [cgp_cap*3] explicit CG pairs (i_cg, j_cg, long)
    unsigned long long* cgp_excl; // [cgp_cap]
    int* n_cgp;                // [2] short count, long count (short first, long after)
    int cgp_cap;
    float* f32;                // n_atoms*3 plain-kernel float force accumulators
    float* f32_long;           // n_atoms*3 plain long-range cache
    double* e64;               // plain: [0] lj, [1] crf, [2..10] virial (short)
    double* e64_long;          // plain long cache: same layout
    // ---- accumulators
    long long* f_short;        // n_atoms*3 (fixed 2^32)
    long long* f_long;         // n_atoms*3 (fixed 2^32) twin-range cache
    long long* acc_short;      // [2*G*G + 9 + 1]: lj, crf group matrices, virial, dhdl (fixed 2^24)
    long long* acc_long;       // same layout (long-range cache)
    double* f_out;             // n_atoms*3 final forces
    double* e_out;             // [2*G*G + 9 + 1] final energies/virial/dhdl
    int* err;                  // [4] error flags, counters
};

__host__ __device__ inline int acc_size(int G) { return 2 * G * G + 9 + 1; }

// ---------------------------------------------------------------------------
// Exact FP64 arithmetic in the reference's operation order.  The __d*_rn
// intrinsics are never contracted into FMAs, so these reproduce the Rust
// (strict IEEE) results bit for bit.

// glam DVec3::length_squared: (x*x + y*y) + z*z
__device__ __forceinline__ double len2_exact(double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Rectangular::nearest_image (crates/gromos-core/src/math.rs:60-68):
// r = d - box * round(d * inv_box), round = half away from zero.
__device__ __forceinline__ double image_exact(double d, double box, double inv_box) {
    double k = round(__dmul_rn(d, inv_box));
    return __dsub_rn(d, __dmul_rn(box, k));
}

__device__ __forceinline__ void nearest_image_exact(const SysDev& s, double ax, double ay, double az,
                                                    double bx, double by, double bz, double& rx,
                                                    double& ry, double& rz) {
    rx = __dsub_rn(ax, bx);
    ry = __dsub_rn(ay, by);
    rz = __dsub_rn(az, bz);
    if (s.boundary == 1) {
        rx = image_exact(rx, s.box[0], s.inv_box[0]);
        ry = image_exact(ry, s.box[1], s.inv_box[1]);
        rz = image_exact(rz, s.box[2], s.inv_box[2]);
    }
}

// ---------------------------------------------------------------------------
// Fixed-point accumulation: deterministic regardless of the order in which
// blocks add their contributions (integer addition is associative).

__device__ __forceinline__ long long to_fixed_f(float v, float scale) {
    return __float2ll_rn(v * scale);
}
__device__ __forceinline__ long long to_fixed_d(double v, double scale) { return __double2ll_rn(v * scale); }

// Fire-and-forget reduction into global memory (red, not atom: no value comes
// back, so the issuing warp never waits on it).
__device__ __forceinline__ void red_add(long long* addr, long long v) {
    if (v != 0) asm volatile("red.global.add.u64 [%0], %1;" ::"l"(addr), "l"(v) : "memory");
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int group_slot(int G, int gi, int gj) {
    int a = gi < gj ? gi : gj, b = gi < gj ? gj : gi;
    return a * G + b;
}

}  // namespace gnb
