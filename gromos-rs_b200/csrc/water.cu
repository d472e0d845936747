// water.cu -- water-water LJ + reaction-field forces (the hot kernel).
//
// Physics per atom pair: lj_crf_interaction
// (crates/gromos-forces/src/nonbonded/innerloops.rs:21-55) with the solvent
// parameter table of process_solvent_pairs (innerloops.rs:241-255); one
// image per CG pair taken from the first atoms (innerloops.rs:264-267) for
// the short list, per-atom images for the long list (innerloops.rs:186).
//
// Two layouts, both one warp per i-cluster of W waters and one lane per
// j-water entry of the cluster's list (bit k of the entry mask selects the
// pair (i_k, j)):
//  - k_water_force (layout 1, W = 4): lanes share the mask bits of an entry;
//    the cluster's atoms live in registers, i-forces are reduced across lanes;
//  - k_water_force_it (layout 2, default, W = 4 or 8): each lane iterates over
//    its own bits; the cluster's atoms are read from shared memory by bit
//    index and i-forces accumulate in lane-private shared-memory rows; the
//    virial is assembled from per-atom force sums (j side per entry, i side
//    per cluster) instead of per pair.
// The CG-pair image comes from an FP64 difference of first oxygens; FP32
// arithmetic for the pairs; forces are accumulated in 64-bit fixed point
// (2^32 per kJ mol^-1 nm^-1) with fire-and-forget reductions.  A CG pair whose
// first-atom vector is not certainly inside half a box edge is re-imaged in
// FP32; if that is still not certain it is deferred to the exact FP64 images
// (process_deferred: k_water_deferred for layout 1, the last block of
// k_water_force_it for layout 2), so image choices are always those of the
// reference.
#include "nb_common.cuh"

namespace gnb {

// Per-launch constants (kernel parameters live in the constant bank, so the
// FP32 instructions read them without registers).
struct WaterParams {
    float qq[9];            // q_a q_b fpe of the first solvent molecule
    float c6[9], c12[9];    // solvent LJ table
    float crf2, crfc, crf3; // crf_2cut3i, crf_cut, crf_cut3i
    float lim[3];           // half box edge - margin: FP32 image certain below this
    double box[3], inv_box[3];
    float boxf[3], inv_boxf[3];
    int boundary;
    int slot;               // energy-group slot of solvent-solvent pairs
    int G;
};

// Force constants with the fixed-point scale 2^32 folded in (a power of two, so
// the scaling is exact): FP32 force sums then convert to fixed point without
// a multiply.  Energies keep the unscaled constants of WaterParams.
struct WaterScaled {
    float qf[9];     // q_a q_b fpe 2^32
    float qcf[9];    // q_a q_b fpe crf_cut3i 2^32
    float c6f[9];    // 6 c6 2^32
    float c12f[9];   // 12 c12 2^32
    float crfc_sumq; // crf_cut * sum over the 9 atom pairs of q_a q_b fpe (one water pair's constant CRF term)
    // The packed (FP32x2) kernel evaluates the eight atom pairs other than
    // first-first as four pairs of pairs ("units"), one per 64-bit register
    // pair: u = 0: (0,1)|(0,2), 1: (1,0)|(2,0), 2: (1,1)|(2,2), 3: (1,2)|(2,1)
    // (t = 3 a + b of the lo and hi half).  The constants of both halves:
    float2 pqf[4], pqcf[4], pqq[4];  // qf, qcf, qq (energy, unscaled)
    float2 pc12[4], pnc6[4];         // c12, -c6 (energy)
    float2 pc12f[4], pnc6f[4];       // 12 c12 2^32, -6 c6 2^32 (force)
    float2 ncrf2;                    // -crf_2cut3i in both halves
};

// The (lo, hi) atom-pair index t of packed unit u (see WaterScaled).
__host__ __device__ constexpr int unit_t(int u, int half) {
    return half == 0 ? (u == 0 ? 1 : u == 1 ? 3 : u == 2 ? 4 : 5) : (u == 0 ? 2 : u == 1 ? 6 : u == 2 ? 8 : 7);
}

__device__ __forceinline__ float rsqrt_fast(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The nine atom pairs of one water pair (lj_crf_interaction,
// innerloops.rs:21-55): x/y/z/r2 hold the atom-pair vectors and squared
// distances (t = 3 a + b); forces accumulate with FMAs into the i rows f[a]
// and the j sums g*[b] (forces carry 2^32, energies do not).  The common case
// is one branch-free block, so that the nine independent chains interleave;
// an atom pair at r^2 < 1e-10 (zeros in the reference) takes the slow path,
// which also cancels that pair's share of the CRF constant term.
template <bool LJ00>
__device__ __forceinline__ void water_pair_math(const float (&x)[9], const float (&y)[9], const float (&z)[9],
                                                const float (&r2)[9], float4 (&f)[3], float (&gx)[3], float (&gy)[3],
                                                float (&gz)[3], float& ecrf, float& elj, const WaterParams& wp,
                                                const WaterScaled& ws) {
    float m2 = r2[0];
#pragma unroll
    for (int t = 1; t < 9; ++t) m2 = fminf(m2, r2[t]);
    if (m2 >= 1e-10f) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int t = a * 3 + b;
                const float ri = rsqrt_fast(r2[t]);
                const float ri2 = ri * ri;
                float fs = fmaf(ws.qf[t], ri2 * ri, ws.qcf[t]);
                ecrf = fmaf(wp.qq[t], fmaf(-wp.crf2, r2[t], ri), ecrf);
                if (!LJ00 || t == 0) {
                    const float ri6 = ri2 * ri2 * ri2;
                    elj = fmaf(fmaf(wp.c12[t], ri6, -wp.c6[t]), ri6, elj);
                    fs = fmaf(fmaf(ws.c12f[t], ri6, -ws.c6f[t]), ri6 * ri2, fs);
                }
                f[a].x = fmaf(x[t], fs, f[a].x);
                f[a].y = fmaf(y[t], fs, f[a].y);
                f[a].z = fmaf(z[t], fs, f[a].z);
                gx[b] = fmaf(-x[t], fs, gx[b]);
                gy[b] = fmaf(-y[t], fs, gy[b]);
                gz[b] = fmaf(-z[t], fs, gz[b]);
            }
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int t = a * 3 + b;
                if (r2[t] < 1e-10f) {
                    ecrf = fmaf(wp.qq[t], wp.crfc, ecrf);
                    continue;
                }
                const float ri = rsqrt_fast(r2[t]);
                const float ri2 = ri * ri;
                float fs = fmaf(ws.qf[t], ri2 * ri, ws.qcf[t]);
                ecrf = fmaf(wp.qq[t], fmaf(-wp.crf2, r2[t], ri), ecrf);
                if (!LJ00 || t == 0) {
                    const float ri6 = ri2 * ri2 * ri2;
                    elj = fmaf(fmaf(wp.c12[t], ri6, -wp.c6[t]), ri6, elj);
                    fs = fmaf(fmaf(ws.c12f[t], ri6, -ws.c6f[t]), ri6 * ri2, fs);
                }
                f[a].x = fmaf(x[t], fs, f[a].x);
                f[a].y = fmaf(y[t], fs, f[a].y);
                f[a].z = fmaf(z[t], fs, f[a].z);
                gx[b] = fmaf(-x[t], fs, gx[b]);
                gy[b] = fmaf(-y[t], fs, gy[b]);
                gz[b] = fmaf(-z[t], fs, gz[b]);
            }
    }
}

struct PairAcc {
    float fi[9];  // i-water atoms a*3 + comp
    float fj[9];  // j-water atoms b*3 + comp
    float elj, ecrf, v[6];
};

// One CG pair (i water in slot islot, j water in slot jslot) with the
// reference's exact FP64 images: the first-atom shift (short list) or
// per-atom images (long list).  Used only for pairs near half a box edge.
template <bool LJ00, bool LONG>
__device__ __forceinline__ PairAcc water_slow_pair(const SysDev& s, const WaterParams& wp, int islot, int jslot) {
    PairAcc o;
    for (int k = 0; k < 9; ++k) o.fi[k] = o.fj[k] = 0.f;
    o.elj = o.ecrf = 0.f;
    for (int k = 0; k < 6; ++k) o.v[k] = 0.f;
    const int ai = s.cg_off[s.slot_cg[islot]], aj = s.cg_off[s.slot_cg[jslot]];
    double tx = 0, ty = 0, tz = 0;
    if (!LONG) {
        double dx, dy, dz;
        nearest_image_exact(s, s.pos[3 * ai], s.pos[3 * ai + 1], s.pos[3 * ai + 2], s.pos[3 * aj],
                            s.pos[3 * aj + 1], s.pos[3 * aj + 2], dx, dy, dz);
        tx = dx - s.pos[3 * ai] + s.pos[3 * aj];
        ty = dy - s.pos[3 * ai + 1] + s.pos[3 * aj + 1];
        tz = dz - s.pos[3 * ai + 2] + s.pos[3 * aj + 2];
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const int t = a * 3 + b;
            double dx, dy, dz;
            if (LONG) {
                nearest_image_exact(s, s.pos[3 * (ai + a)], s.pos[3 * (ai + a) + 1], s.pos[3 * (ai + a) + 2],
                                    s.pos[3 * (aj + b)], s.pos[3 * (aj + b) + 1], s.pos[3 * (aj + b) + 2], dx, dy,
                                    dz);
            } else {
                dx = s.pos[3 * (ai + a)] + tx - s.pos[3 * (aj + b)];
                dy = s.pos[3 * (ai + a) + 1] + ty - s.pos[3 * (aj + b) + 1];
                dz = s.pos[3 * (ai + a) + 2] + tz - s.pos[3 * (aj + b) + 2];
            }
            const float x = float(dx), y = float(dy), z = float(dz);
            const float r2 = fmaf(x, x, fmaf(y, y, z * z));
            if (r2 < 1e-10f) continue;
            const float ri = rsqrt_fast(r2), ri2 = ri * ri;
            const float q = wp.qq[t];
            o.ecrf = fmaf(q, fmaf(-wp.crf2, r2, ri) - wp.crfc, o.ecrf);
            float fs = q * fmaf(ri, ri2, wp.crf3);
            if (!LJ00 || t == 0) {
                const float ri6 = ri2 * ri2 * ri2;
                o.elj = fmaf(fmaf(wp.c12[t], ri6, -wp.c6[t]), ri6, o.elj);
                fs = fmaf(fmaf(12.f * wp.c12[t], ri6, -6.f * wp.c6[t]), ri6 * ri2, fs);
            }
            const float fx = x * fs, fy = y * fs, fz = z * fs;
            o.fi[a * 3] += fx;
            o.fi[a * 3 + 1] += fy;
            o.fi[a * 3 + 2] += fz;
            o.fj[b * 3] -= fx;
            o.fj[b * 3 + 1] -= fy;
            o.fj[b * 3 + 2] -= fz;
            o.v[0] = fmaf(x, fx, o.v[0]);
            o.v[1] = fmaf(x, fy, o.v[1]);
            o.v[2] = fmaf(x, fz, o.v[2]);
            o.v[3] = fmaf(y, fy, o.v[3]);
            o.v[4] = fmaf(y, fz, o.v[4]);
            o.v[5] = fmaf(z, fz, o.v[5]);
        }
    return o;
}

// Reduce-scatter of a per-lane array of 36 = 4 waters x 9 components over the
// warp: afterwards lane l (with (l & 7) == 0) holds the warp sum of the 9
// components of water l >> 3 in out[0..8].
__device__ __forceinline__ void reduce_scatter_36(const float (&v)[36], float (&out)[9], int lane) {
    float w[18];
    const bool h16 = lane & 16;
#pragma unroll
    for (int i = 0; i < 18; ++i) {
        const float keep = h16 ? v[i + 18] : v[i];
        const float send = h16 ? v[i] : v[i + 18];
        w[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    const bool h8 = lane & 8;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float keep = h8 ? w[i + 9] : w[i];
        const float send = h8 ? w[i] : w[i + 9];
        out[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        out[i] += __shfl_xor_sync(0xffffffffu, out[i], 4);
        out[i] += __shfl_xor_sync(0xffffffffu, out[i], 2);
        out[i] += __shfl_xor_sync(0xffffffffu, out[i], 1);
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ double rec_x(float4 v) { return __hiloint2double(__float_as_int(v.y), __float_as_int(v.x)); }
__device__ __forceinline__ double rec_y(float4 v) { return __hiloint2double(__float_as_int(v.w), __float_as_int(v.z)); }

constexpr int kWaterWarps = 4;

// Software pipeline per warp: the 32 j-records of chunk c+1 are copied into
// shared memory (cp.async, double buffer) while chunk c is computed, the
// entries are loaded two chunks ahead, and the next cluster's i-records are
// copied while the current cluster's forces are reduced.
template <bool LJ00, bool LONG>
__global__ void __launch_bounds__(128, 4) k_water_force(const SysDev* __restrict__ sys, const WaterParams wp) {
    constexpr int W = 4;
    const SysDev& s = sys[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nclus = s.n_clusters[0];
    long long* __restrict__ FS = LONG ? s.fs_long : s.fs_short;  // per slot: 3 atoms x 3 components
    const uint32_t* __restrict__ wl = LONG ? s.wl_l : s.wl_s;
    const int* __restrict__ wn = LONG ? s.wn_l : s.wn_s;
    const float4* __restrict__ wrec4 = reinterpret_cast<const float4*>(s.wrec);
    const int* __restrict__ clus_n = s.clus_n;
    const int wcap = s.wcap;
    // certain-image limits: the short list needs only the first-atom vector
    // inside half a box edge; per-atom images (long list) also need room for
    // both molecules' extents (measured this step by k_water_prep)
    float limx = wp.lim[0], limy = wp.lim[1], limz = wp.lim[2];
    if (LONG) {
        const float m = 2.f * (*s.max_delta) * 1.0001f + 1e-4f;
        limx -= m;
        limy -= m;
        limz -= m;
    }
    // per-lane fixed-point (2^24) accumulators of lj, crf, xx, xy, xz, yy, yz, zz
    __shared__ long long accs[kWaterWarps * 32 * 8];
    __shared__ float4 sp_all[kWaterWarps][W * 3];            // i atoms (offsets from the first oxygen)
    __shared__ float4 ibuf[kWaterWarps][2][W * 3];           // raw i-records, two clusters
    __shared__ float4 jbuf[kWaterWarps][2][32 * 3];          // raw j-records, two chunks
    long long* __restrict__ my = accs + threadIdx.x * 8;
#pragma unroll
    for (int v = 0; v < 8; ++v) my[v] = 0;
    float4* __restrict__ sp = sp_all[wid];
    const int stride = gridDim.x * kWaterWarps;
    int ci = blockIdx.x * kWaterWarps + wid;
    int ib = 0;
    // prologue: i-records of the first cluster
    if (ci < nclus && lane < W * 3) cp_async16(&ibuf[wid][0][lane], wrec4 + 3 * (ci * W) + lane);
    cp_async_commit();

    for (; ci < nclus; ci += stride) {
        const int n = clus_n[ci];
        const int base = ci * W;
        const int cnt = wn[ci];
        const uint32_t* __restrict__ list = wl + static_cast<size_t>(ci) * wcap;
        uint32_t e_cur = lane < cnt ? __ldg(list + lane) : 0u;
        uint32_t e_nx = 32 + lane < cnt ? __ldg(list + 32 + lane) : 0u;
        cp_async_wait<0>();  // this cluster's i-records
        __syncwarp();
        const double x00 = rec_x(ibuf[wid][ib][0]), y00 = rec_y(ibuf[wid][ib][0]);
        const double z00 = rec_x(ibuf[wid][ib][1]);
        if (lane < W * 3) {
            const int k = lane / 3, a = lane % 3;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < n) {
                const float4 v0 = ibuf[wid][ib][3 * k], v1 = ibuf[wid][ib][3 * k + 1], v2 = ibuf[wid][ib][3 * k + 2];
                const float dx = a == 0 ? 0.f : (a == 1 ? v1.z : v2.y);
                const float dy = a == 0 ? 0.f : (a == 1 ? v1.w : v2.z);
                const float dz = a == 0 ? 0.f : (a == 1 ? v2.x : v2.w);
                p.x = float(rec_x(v0) - x00) + dx;
                p.y = float(rec_y(v0) - y00) + dy;
                p.z = float(rec_x(v1) - z00) + dz;
            }
            sp[lane] = p;
        }
        // j-records of chunk 0
        if (e_cur & 0xffu) {
            const int js = static_cast<int>(e_cur >> 8);
#pragma unroll
            for (int q = 0; q < 3; ++q) cp_async16(&jbuf[wid][0][3 * lane + q], wrec4 + 3 * js + q);
        }
        cp_async_commit();
        __syncwarp();
        float fi[36];
#pragma unroll
        for (int i = 0; i < 36; ++i) fi[i] = 0.f;
        float elj = 0.f, ecrf = 0.f, v0s = 0.f, v1s = 0.f, v2s = 0.f, v3s = 0.f, v4s = 0.f, v5s = 0.f;
        const int nch = (cnt + 31) >> 5;
        for (int c = 0; c < nch; ++c) {
            const int jb = c & 1;
            if (c + 1 < nch && (e_nx & 0xffu)) {
                const int js = static_cast<int>(e_nx >> 8);
#pragma unroll
                for (int q = 0; q < 3; ++q) cp_async16(&jbuf[wid][jb ^ 1][3 * lane + q], wrec4 + 3 * js + q);
            }
            cp_async_commit();
            const int e2 = (c + 2) * 32 + lane;
            const uint32_t e_nn = e2 < cnt ? __ldg(list + e2) : 0u;
            cp_async_wait<1>();  // chunk c's records
            __syncwarp();
            const uint32_t ent = e_cur;
            const unsigned mask = ent & 0xffu;
            const int js = static_cast<int>(ent >> 8);
            float qx[3], qy[3], qz[3];
            float gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
            if (mask) {
                const float4 r0 = jbuf[wid][jb][3 * lane], r1 = jbuf[wid][jb][3 * lane + 1],
                             r2 = jbuf[wid][jb][3 * lane + 2];
                double dx = x00 - rec_x(r0), dy = y00 - rec_y(r0), dz = z00 - rec_x(r1);
                if (wp.boundary) {
                    dx -= wp.box[0] * rint(dx * wp.inv_box[0]);
                    dy -= wp.box[1] * rint(dy * wp.inv_box[1]);
                    dz -= wp.box[2] * rint(dz * wp.inv_box[2]);
                }
                const float Dx = float(dx), Dy = float(dy), Dz = float(dz);
                qx[0] = -Dx;
                qy[0] = -Dy;
                qz[0] = -Dz;
                qx[1] = r1.z - Dx;
                qy[1] = r1.w - Dy;
                qz[1] = r2.x - Dz;
                qx[2] = r2.y - Dx;
                qy[2] = r2.z - Dy;
                qz[2] = r2.w - Dz;
            } else {
#pragma unroll
                for (int b = 0; b < 3; ++b) qx[b] = qy[b] = qz[b] = 0.f;
            }
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const bool act = (mask >> k) & 1u;
                if (!__any_sync(0xffffffffu, act)) continue;
                if (!act) continue;
                const float4 p0 = sp[k * 3], p1 = sp[k * 3 + 1], p2 = sp[k * 3 + 2];
                const float pxk[3] = {p0.x, p1.x, p2.x}, pyk[3] = {p0.y, p1.y, p2.y}, pzk[3] = {p0.z, p1.z, p2.z};
                // first-atom vector: decides whether the FP32 image is certain; a
                // pair outside the certain range is re-imaged in FP32 (one shift
                // for the CG pair), and if still uncertain deferred to the exact
                // FP64 kernel (k_water_deferred)
                float r0x = pxk[0] - qx[0], r0y = pyk[0] - qy[0], r0z = pzk[0] - qz[0];
                float shx = 0.f, shy = 0.f, shz = 0.f;
                if (!(fabsf(r0x) < limx && fabsf(r0y) < limy && fabsf(r0z) < limz)) {
                    if (wp.boundary) {
                        shx = -wp.boxf[0] * rintf(r0x * wp.inv_boxf[0]);
                        shy = -wp.boxf[1] * rintf(r0y * wp.inv_boxf[1]);
                        shz = -wp.boxf[2] * rintf(r0z * wp.inv_boxf[2]);
                        r0x += shx;
                        r0y += shy;
                        r0z += shz;
                    }
                    if (!(fabsf(r0x) < limx && fabsf(r0y) < limy && fabsf(r0z) < limz)) {
                        const int d = atomicAdd(&s.n_deferred[LONG ? 1 : 0], 1);
                        if (d < s.defer_cap) {
                            s.deferred[2 * (LONG ? s.defer_cap + d : d)] = base + k;
                            s.deferred[2 * (LONG ? s.defer_cap + d : d) + 1] = js;
                        } else {
                            atomicOr(&s.err[0], ERR_DEFER_OVERFLOW);
                        }
                        continue;
                    }
                }
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const int t = a * 3 + b;
                        const float x = (a == 0 && b == 0) ? r0x : (pxk[a] + shx) - qx[b];
                        const float y = (a == 0 && b == 0) ? r0y : (pyk[a] + shy) - qy[b];
                        const float z = (a == 0 && b == 0) ? r0z : (pzk[a] + shz) - qz[b];
                        const float r2 = fmaf(x, x, fmaf(y, y, z * z));
                        // an atom pair at r^2 < 1e-10 contributes nothing (innerloops.rs:32):
                        // 1/r and the charge product (hence the CRF constant) are zero
                        const bool zero = r2 < 1e-10f;
                        const float ri = zero ? 0.f : rsqrt_fast(r2);
                        const float ri2 = ri * ri;
                        const float q = zero ? 0.f : wp.qq[t];
                        ecrf = fmaf(q, fmaf(-wp.crf2, r2, ri) - wp.crfc, ecrf);
                        float fs = q * fmaf(ri, ri2, wp.crf3);
                        if (!LJ00 || t == 0) {
                            const float ri6 = ri2 * ri2 * ri2;
                            elj = fmaf(fmaf(wp.c12[t], ri6, -wp.c6[t]), ri6, elj);
                            fs = fmaf(fmaf(12.f * wp.c12[t], ri6, -6.f * wp.c6[t]), ri6 * ri2, fs);
                        }
                        const float fxx = x * fs, fyy = y * fs, fzz = z * fs;
                        fi[k * 9 + a * 3] += fxx;
                        fi[k * 9 + a * 3 + 1] += fyy;
                        fi[k * 9 + a * 3 + 2] += fzz;
                        gx[b] -= fxx;
                        gy[b] -= fyy;
                        gz[b] -= fzz;
                        v0s = fmaf(x, fxx, v0s);
                        v1s = fmaf(x, fyy, v1s);
                        v2s = fmaf(x, fzz, v2s);
                        v3s = fmaf(y, fyy, v3s);
                        v4s = fmaf(y, fzz, v4s);
                        v5s = fmaf(z, fzz, v5s);
                    }
            }
            if (mask) {
                long long* __restrict__ fj = FS + static_cast<size_t>(js) * 9;
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    red_add(fj + 3 * b, to_fixed_f(gx[b], 4294967296.0f));
                    red_add(fj + 3 * b + 1, to_fixed_f(gy[b], 4294967296.0f));
                    red_add(fj + 3 * b + 2, to_fixed_f(gz[b], 4294967296.0f));
                }
            }
            e_cur = e_nx;
            e_nx = e_nn;
            __syncwarp();  // jbuf[jb] is refilled two chunks later
        }
        // next cluster's i-records, copied while this cluster's forces are reduced
        const int cn = ci + stride;
        if (cn < nclus && lane < W * 3) cp_async16(&ibuf[wid][ib ^ 1][lane], wrec4 + 3 * (cn * W) + lane);
        cp_async_commit();
        float red[9];
        reduce_scatter_36(fi, red, lane);
        const int k = lane >> 3;
        if ((lane & 7) == 0 && k < n) {
            long long* __restrict__ fi_out = FS + static_cast<size_t>(base + k) * 9;
#pragma unroll
            for (int cc = 0; cc < 9; ++cc) red_add(fi_out + cc, to_fixed_f(red[cc], 4294967296.0f));
        }
        my[0] += to_fixed_f(elj, 16777216.0f);
        my[1] += to_fixed_f(ecrf, 16777216.0f);
        my[2] += to_fixed_f(v0s, 16777216.0f);
        my[3] += to_fixed_f(v1s, 16777216.0f);
        my[4] += to_fixed_f(v2s, 16777216.0f);
        my[5] += to_fixed_f(v3s, 16777216.0f);
        my[6] += to_fixed_f(v4s, 16777216.0f);
        my[7] += to_fixed_f(v5s, 16777216.0f);
        ib ^= 1;
        __syncwarp();  // sp is rewritten by the next cluster
    }
    cp_async_wait<0>();
    long long acc[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[v] = warp_sum_ll(my[v]);
    __shared__ unsigned long long sh[8];
    if (threadIdx.x < 8) sh[threadIdx.x] = 0ull;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < 8; ++v)
            if (acc[v]) atomicAdd(&sh[v], static_cast<unsigned long long>(acc[v]));
    __syncthreads();
    if (threadIdx.x < 8 && sh[threadIdx.x]) {
        long long* dst = LONG ? s.acc_long : s.acc_short;
        const int G = wp.G, vb = 2 * G * G;
        const int v = threadIdx.x;
        const int idx0[8] = {wp.slot, G * G + wp.slot, vb + 0, vb + 1, vb + 2, vb + 4, vb + 5, vb + 8};
        const int idx1[8] = {-1, -1, -1, vb + 3, vb + 6, -1, vb + 7, -1};
        atomicAdd(reinterpret_cast<unsigned long long*>(dst + idx0[v]), sh[v]);
        if (idx1[v] >= 0) atomicAdd(reinterpret_cast<unsigned long long*>(dst + idx1[v]), sh[v]);
    }
}

// CG pairs the main kernels deferred: exact FP64 images (first-atom shift for
// the short list, per-atom images for the long list), FP32 pair arithmetic.
// Threads tid, tid + nthreads, ... of the caller take one pair each.  The
// list and its count were written by other blocks: read through L2.
template <bool LJ00, bool LONG>
__device__ __forceinline__ void process_deferred(const SysDev& s, const WaterParams& wp, int tid, int nthreads) {
    long long* __restrict__ FS = LONG ? s.fs_long : s.fs_short;
    const int nd = min(__ldcg(s.n_deferred + (LONG ? 1 : 0)), s.defer_cap);
    long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int d = tid; d < nd; d += nthreads) {
        const int e = LONG ? s.defer_cap + d : d;
        const int islot = __ldcg(s.deferred + 2 * e), jslot = __ldcg(s.deferred + 2 * e + 1);
        const PairAcc o = water_slow_pair<LJ00, LONG>(s, wp, islot, jslot);
        for (int c = 0; c < 9; ++c) {
            red_add(FS + static_cast<size_t>(islot) * 9 + c, to_fixed_f(o.fi[c], 4294967296.0f));
            red_add(FS + static_cast<size_t>(jslot) * 9 + c, to_fixed_f(o.fj[c], 4294967296.0f));
        }
        acc[0] += to_fixed_f(o.elj, 16777216.0f);
        acc[1] += to_fixed_f(o.ecrf, 16777216.0f);
        for (int v = 0; v < 6; ++v) acc[2 + v] += to_fixed_f(o.v[v], 16777216.0f);
    }
    long long* dst = LONG ? s.acc_long : s.acc_short;
    const int G = wp.G, vb = 2 * G * G;
    const int idx0[8] = {wp.slot, G * G + wp.slot, vb + 0, vb + 1, vb + 2, vb + 4, vb + 5, vb + 8};
    const int idx1[8] = {-1, -1, -1, vb + 3, vb + 6, -1, vb + 7, -1};
    for (int v = 0; v < 8; ++v) {
        const long long t = warp_sum_ll(acc[v]);
        if ((threadIdx.x & 31) == 0 && t) {
            atomicAdd(reinterpret_cast<unsigned long long*>(dst + idx0[v]), static_cast<unsigned long long>(t));
            if (idx1[v] >= 0)
                atomicAdd(reinterpret_cast<unsigned long long*>(dst + idx1[v]), static_cast<unsigned long long>(t));
        }
    }
}

// ---------------------------------------------------------------------------
// Packed FP32x2 evaluation (layout 4).  Blackwell executes one FP32x2
// instruction (fma/add/mul .f32x2) for two lanes' worth of FP32 work per
// issue slot, so the eight atom pairs of a water pair other than first-first
// are evaluated as four packed units (see WaterScaled) and the first-first
// pair, the only one with Lennard-Jones terms in SPC-like solvents, in scalar
// arithmetic.  Per unit the i and j operands sit in 64-bit register pairs:
//   u = 0 (0,1)|(0,2): i {p0, p0},  j {q1, q2};  i-force -> F00, j-force -> G12
//   u = 1 (1,0)|(2,0): i {p1, p2},  j {q0, q0};  i-force -> F12, j-force -> G00
//   u = 2 (1,1)|(2,2): i {p1, p2},  j {q1, q2};  i-force -> F12, j-force -> G12
//   u = 3 (1,2)|(2,1): i {p1, p2},  j {q2, q1};  i-force -> F12, j-force -> G21
// so that every accumulator is a register pair too: the i rows hold F00 =
// {f0 part, f0 part} and F12 = {f1, f2}; the j sums G00 = {g0 part, g0 part},
// G12 = {g1, g2}, G21 = {g2, g1} (accumulated with the i sign and negated once
// per entry).  The arithmetic per atom pair is that of water_pair_math.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <bool LJ00, int U>
__device__ __forceinline__ void packed_unit(float2 X, float2 Y, float2 Z, float2 R2, float2& Fx, float2& Fy,
                                            float2& Fz, float2& Gx, float2& Gy, float2& Gz, float2& E, float2& EL,
                                            const WaterScaled& ws) {
    const float2 RI = make_float2(rsqrt_fast(R2.x), rsqrt_fast(R2.y));
    const float2 RI2 = mul2(RI, RI);
    float2 FS = fma2(ws.pqf[U], mul2(RI2, RI), ws.pqcf[U]);
    E = fma2(ws.pqq[U], fma2(ws.ncrf2, R2, RI), E);
    if (!LJ00) {
        const float2 RI6 = mul2(mul2(RI2, RI2), RI2);
        EL = fma2(fma2(ws.pc12[U], RI6, ws.pnc6[U]), RI6, EL);
        FS = fma2(fma2(ws.pc12f[U], RI6, ws.pnc6f[U]), mul2(RI6, RI2), FS);
    }
    Fx = fma2(X, FS, Fx);
    Fy = fma2(Y, FS, Fy);
    Fz = fma2(Z, FS, Fz);
    Gx = fma2(X, FS, Gx);
    Gy = fma2(Y, FS, Gy);
    Gz = fma2(Z, FS, Gz);
}

// One j-water entry of the bit-iterating kernel, packed: the CG-pair image,
// every set bit of the mask (i water k of the cluster), the j-part of the
// virial and the j forces (reductions, or staged in st for the long range).
template <bool LJ00, bool LONG>
__device__ __forceinline__ void water_entry_packed(const SysDev& s, const WaterParams& wp, const WaterScaled& pp,
                                                   const float4* __restrict__ sp, float4* __restrict__ myrow,
                                                   const float4* __restrict__ jrec, double x00, double y00, double z00,
                                                   float limx, float limy, float limz, int base, int js, unsigned mask,
                                                   long long* __restrict__ FS, long long* __restrict__ st, float& ecrf,
                                                   float& elj, float2& ecrf2, float2& elj2, float& v0s, float& v1s,
                                                   float& v2s, float& v3s, float& v4s, float& v5s, int& n_wp) {
    const float4 r0 = jrec[0], r1 = jrec[1], r2 = jrec[2];
    double dx = x00 - rec_x(r0), dy = y00 - rec_y(r0), dz = z00 - rec_x(r1);
    if (wp.boundary) {
        dx -= wp.box[0] * rint(dx * wp.inv_box[0]);
        dy -= wp.box[1] * rint(dy * wp.inv_box[1]);
        dz -= wp.box[2] * rint(dz * wp.inv_box[2]);
    }
    // j atoms relative to the cluster origin: q0 = -D, q1, q2
    const float Dx = float(dx), Dy = float(dy), Dz = float(dz);
    const float q1x = r1.z - Dx, q1y = r1.w - Dy, q1z = r2.x - Dz;
    const float q2x = r2.y - Dx, q2y = r2.z - Dy, q2z = r2.w - Dz;
    // negated j operands: X = P + N equals P - Q exactly
    const float2 N0x = make_float2(Dx, Dx), N0y = make_float2(Dy, Dy), N0z = make_float2(Dz, Dz);
    const float2 N12x = make_float2(-q1x, -q2x), N12y = make_float2(-q1y, -q2y), N12z = make_float2(-q1z, -q2z);
    const float2 N21x = make_float2(-q2x, -q1x), N21y = make_float2(-q2y, -q1y), N21z = make_float2(-q2z, -q1z);
    const float2 zero2 = make_float2(0.f, 0.f);
    float2 G00x = zero2, G00y = zero2, G00z = zero2, G12x = zero2, G12y = zero2, G12z = zero2;
    float2 G21x = zero2, G21y = zero2, G21z = zero2;
    while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        const float4 B = sp[k * 3], C = sp[k * 3 + 1], E4 = sp[k * 3 + 2];
        float2 P0x = make_float2(B.x, B.y), P0y = make_float2(B.z, B.w), P0z = make_float2(C.x, C.y);
        float2 P12x = make_float2(C.z, C.w), P12y = make_float2(E4.x, E4.y), P12z = make_float2(E4.z, E4.w);
        // first-atom vector: decides whether the FP32 image is certain (as in
        // the scalar kernel: FP32 re-image, else deferred to exact FP64)
        float r0x = B.x + Dx, r0y = B.z + Dy, r0z = C.x + Dz;
        float shx = 0.f, shy = 0.f, shz = 0.f;
        bool shifted = false;
        if (!(fabsf(r0x) < limx && fabsf(r0y) < limy && fabsf(r0z) < limz)) {
            if (wp.boundary) {
                shx = -wp.boxf[0] * rintf(r0x * wp.inv_boxf[0]);
                shy = -wp.boxf[1] * rintf(r0y * wp.inv_boxf[1]);
                shz = -wp.boxf[2] * rintf(r0z * wp.inv_boxf[2]);
            }
            r0x += shx;
            r0y += shy;
            r0z += shz;
            if (!(fabsf(r0x) < limx && fabsf(r0y) < limy && fabsf(r0z) < limz)) {
                const int d = atomicAdd(&s.n_deferred[LONG ? 1 : 0], 1);
                if (d < s.defer_cap) {
                    s.deferred[2 * (LONG ? s.defer_cap + d : d)] = base + k;
                    s.deferred[2 * (LONG ? s.defer_cap + d : d) + 1] = js;
                } else {
                    atomicOr(&s.err[0], ERR_DEFER_OVERFLOW);
                }
                continue;
            }
            const float2 sx2 = make_float2(shx, shx), sy2 = make_float2(shy, shy), sz2 = make_float2(shz, shz);
            P0x = add2(P0x, sx2);
            P0y = add2(P0y, sy2);
            P0z = add2(P0z, sz2);
            P12x = add2(P12x, sx2);
            P12y = add2(P12y, sy2);
            P12z = add2(P12z, sz2);
            shifted = true;
        }
        const float4 R0 = myrow[k * 3], R1 = myrow[k * 3 + 1], R2 = myrow[k * 3 + 2];
        float2 F00x = make_float2(R0.x, R0.y), F00y = make_float2(R0.z, R0.w), F00z = make_float2(R1.x, R1.y);
        float2 F12x = make_float2(R1.z, R1.w), F12y = make_float2(R2.x, R2.y), F12z = make_float2(R2.z, R2.w);
        float gs0 = 0.f, gs1 = 0.f, gs2 = 0.f;
        if (shifted) {
            gs0 = G00x.x + G00x.y + G12x.x + G12x.y + G21x.x + G21x.y;
            gs1 = G00y.x + G00y.y + G12y.x + G12y.y + G21y.x + G21y.y;
            gs2 = G00z.x + G00z.y + G12z.x + G12z.y + G21z.x + G21z.y;
        }
        // atom-pair vectors i - j of the four units and the first-first pair
        const float2 XA = add2(P0x, N12x), YA = add2(P0y, N12y), ZA = add2(P0z, N12z);
        const float2 XB = add2(P12x, N0x), YB = add2(P12y, N0y), ZB = add2(P12z, N0z);
        const float2 XC = add2(P12x, N12x), YC = add2(P12y, N12y), ZC = add2(P12z, N12z);
        const float2 XD = add2(P12x, N21x), YD = add2(P12y, N21y), ZD = add2(P12z, N21z);
        const float2 R2A = fma2(XA, XA, fma2(YA, YA, mul2(ZA, ZA)));
        const float2 R2B = fma2(XB, XB, fma2(YB, YB, mul2(ZB, ZB)));
        const float2 R2C = fma2(XC, XC, fma2(YC, YC, mul2(ZC, ZC)));
        const float2 R2D = fma2(XD, XD, fma2(YD, YD, mul2(ZD, ZD)));
        const float r2s = fmaf(r0x, r0x, fmaf(r0y, r0y, r0z * r0z));
        const float m2 = fminf(fminf(fminf(r2s, fminf(R2A.x, R2A.y)), fminf(R2B.x, R2B.y)),
                               fminf(fminf(R2C.x, R2C.y), fminf(R2D.x, R2D.y)));
        if (m2 >= 1e-10f) {
            {  // first-first pair, scalar, with Lennard-Jones
                const float ri = rsqrt_fast(r2s);
                const float ri2 = ri * ri;
                float fs = fmaf(pp.qf[0], ri2 * ri, pp.qcf[0]);
                ecrf = fmaf(wp.qq[0], fmaf(-wp.crf2, r2s, ri), ecrf);
                const float ri6 = ri2 * ri2 * ri2;
                elj = fmaf(fmaf(wp.c12[0], ri6, -wp.c6[0]), ri6, elj);
                fs = fmaf(fmaf(pp.c12f[0], ri6, -pp.c6f[0]), ri6 * ri2, fs);
                F00x.x = fmaf(r0x, fs, F00x.x);
                F00y.x = fmaf(r0y, fs, F00y.x);
                F00z.x = fmaf(r0z, fs, F00z.x);
                G00x.x = fmaf(r0x, fs, G00x.x);
                G00y.x = fmaf(r0y, fs, G00y.x);
                G00z.x = fmaf(r0z, fs, G00z.x);
            }
            packed_unit<LJ00, 0>(XA, YA, ZA, R2A, F00x, F00y, F00z, G12x, G12y, G12z, ecrf2, elj2, pp);
            packed_unit<LJ00, 1>(XB, YB, ZB, R2B, F12x, F12y, F12z, G00x, G00y, G00z, ecrf2, elj2, pp);
            packed_unit<LJ00, 2>(XC, YC, ZC, R2C, F12x, F12y, F12z, G12x, G12y, G12z, ecrf2, elj2, pp);
            packed_unit<LJ00, 3>(XD, YD, ZD, R2D, F12x, F12y, F12z, G21x, G21y, G21z, ecrf2, elj2, pp);
        } else {
            // an atom pair at r^2 < 1e-10: scalar, with the reference's zeros
            const float xs[9] = {r0x, XA.x, XA.y, XB.x, XC.x, XD.x, XB.y, XD.y, XC.y};
            const float ys[9] = {r0y, YA.x, YA.y, YB.x, YC.x, YD.x, YB.y, YD.y, YC.y};
            const float zs[9] = {r0z, ZA.x, ZA.y, ZB.x, ZC.x, ZD.x, ZB.y, ZD.y, ZC.y};
            const float rs[9] = {r2s, R2A.x, R2A.y, R2B.x, R2C.x, R2D.x, R2B.y, R2D.y, R2C.y};
            float fx[9], fy[9], fz[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                fx[t] = fy[t] = fz[t] = 0.f;
                if (rs[t] < 1e-10f) {
                    ecrf = fmaf(wp.qq[t], wp.crfc, ecrf);
                    continue;
                }
                const float ri = rsqrt_fast(rs[t]);
                const float ri2 = ri * ri;
                float fs = fmaf(pp.qf[t], ri2 * ri, pp.qcf[t]);
                ecrf = fmaf(wp.qq[t], fmaf(-wp.crf2, rs[t], ri), ecrf);
                if (!LJ00 || t == 0) {
                    const float ri6 = ri2 * ri2 * ri2;
                    elj = fmaf(fmaf(wp.c12[t], ri6, -wp.c6[t]), ri6, elj);
                    fs = fmaf(fmaf(pp.c12f[t], ri6, -pp.c6f[t]), ri6 * ri2, fs);
                }
                fx[t] = xs[t] * fs;
                fy[t] = ys[t] * fs;
                fz[t] = zs[t] * fs;
            }
            // i: atom 0 <- t 0, 1, 2; atom 1 <- 3, 4, 5; atom 2 <- 6, 7, 8
            F00x.x += fx[0] + fx[1];
            F00y.x += fy[0] + fy[1];
            F00z.x += fz[0] + fz[1];
            F00x.y += fx[2];
            F00y.y += fy[2];
            F00z.y += fz[2];
            F12x.x += fx[3] + fx[4] + fx[5];
            F12y.x += fy[3] + fy[4] + fy[5];
            F12z.x += fz[3] + fz[4] + fz[5];
            F12x.y += fx[6] + fx[7] + fx[8];
            F12y.y += fy[6] + fy[7] + fy[8];
            F12z.y += fz[6] + fz[7] + fz[8];
            // j: atom 0 <- t 0, 3, 6; atom 1 <- 1, 4, 7; atom 2 <- 2, 5, 8
            G00x.x += fx[0] + fx[3];
            G00y.x += fy[0] + fy[3];
            G00z.x += fz[0] + fz[3];
            G00x.y += fx[6];
            G00y.y += fy[6];
            G00z.y += fz[6];
            G12x.x += fx[1] + fx[4];
            G12y.x += fy[1] + fy[4];
            G12z.x += fz[1] + fz[4];
            G12x.y += fx[2] + fx[8];
            G12y.y += fy[2] + fy[8];
            G12z.y += fz[2] + fz[8];
            G21x.x += fx[5];
            G21y.x += fy[5];
            G21z.x += fz[5];
            G21x.y += fx[7];
            G21y.y += fy[7];
            G21z.y += fz[7];
        }
        myrow[k * 3] = make_float4(F00x.x, F00x.y, F00y.x, F00y.y);
        myrow[k * 3 + 1] = make_float4(F00z.x, F00z.y, F12x.x, F12x.y);
        myrow[k * 3 + 2] = make_float4(F12y.x, F12y.y, F12z.x, F12z.y);
        ++n_wp;
        if (shifted) {  // shift (x) sum_a fi_a = shift (x) (change of the j sums with the i sign)
            const float sx = G00x.x + G00x.y + G12x.x + G12x.y + G21x.x + G21x.y - gs0;
            const float sy = G00y.x + G00y.y + G12y.x + G12y.y + G21y.x + G21y.y - gs1;
            const float sz = G00z.x + G00z.y + G12z.x + G12z.y + G21z.x + G21z.y - gs2;
            v0s = fmaf(shx, sx, v0s);
            v1s = fmaf(shx, sy, v1s);
            v2s = fmaf(shx, sz, v2s);
            v3s = fmaf(shy, sy, v3s);
            v4s = fmaf(shy, sz, v4s);
            v5s = fmaf(shz, sz, v5s);
        }
    }
    // the j forces g_b = -(sums with the i sign)
    const float gx[3] = {-(G00x.x + G00x.y), -(G12x.x + G21x.y), -(G12x.y + G21x.x)};
    const float gy[3] = {-(G00y.x + G00y.y), -(G12y.x + G21y.y), -(G12y.y + G21y.x)};
    const float gz[3] = {-(G00z.x + G00z.y), -(G12z.x + G21z.y), -(G12z.y + G21z.x)};
    const float qx[3] = {-Dx, q1x, q2x}, qy[3] = {-Dy, q1y, q2y}, qz[3] = {-Dz, q1z, q2z};
#pragma unroll
    for (int b = 0; b < 3; ++b) {  // the j-part of the virial: Q_b (x) g_b
        v0s = fmaf(qx[b], gx[b], v0s);
        v1s = fmaf(qx[b], gy[b], v1s);
        v2s = fmaf(qx[b], gz[b], v2s);
        v3s = fmaf(qy[b], gy[b], v3s);
        v4s = fmaf(qy[b], gz[b], v4s);
        v5s = fmaf(qz[b], gz[b], v5s);
    }
    if (LONG) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {  // the forces carry the 2^32 scale already
            st[3 * b] = __float2ll_rn(gx[b]);
            st[3 * b + 1] = __float2ll_rn(gy[b]);
            st[3 * b + 2] = __float2ll_rn(gz[b]);
        }
    } else {
        long long* __restrict__ fj = FS + static_cast<size_t>(js) * 9;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            red_add(fj + 3 * b, __float2ll_rn(gx[b]));
            red_add(fj + 3 * b + 1, __float2ll_rn(gy[b]));
            red_add(fj + 3 * b + 2, __float2ll_rn(gz[b]));
        }
    }
}

// Cluster end of the packed kernel: column sums of the lane rows (lane c < 3W
// sums float4 c of every row), per-atom i forces assembled from the packed
// halves, their reductions, and the i-part of the virial P (x) F.  Called by
// the whole warp (shuffles).
template <int W>
__device__ __forceinline__ void packed_column_sums(const float4* __restrict__ fis, const float4* __restrict__ sp,
                                                   long long* __restrict__ fo_base, int lane, int n, float& v0s,
                                                   float& v1s, float& v2s, float& v3s, float& v4s, float& v5s) {
    constexpr int ROW = W * 3 + 1;
    float4 S = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane < W * 3) {
#pragma unroll 8
        for (int r = 0; r < 32; ++r) {
            const float4 f = fis[r * ROW + lane];
            S.x += f.x;
            S.y += f.y;
            S.z += f.z;
            S.w += f.w;
        }
    }
    const int k3 = (lane / 3) * 3;
    float4 S0, S1, S2;
    S0.x = __shfl_sync(0xffffffffu, S.x, k3);
    S0.y = __shfl_sync(0xffffffffu, S.y, k3);
    S0.z = __shfl_sync(0xffffffffu, S.z, k3);
    S0.w = __shfl_sync(0xffffffffu, S.w, k3);
    S1.x = __shfl_sync(0xffffffffu, S.x, k3 + 1);
    S1.y = __shfl_sync(0xffffffffu, S.y, k3 + 1);
    S1.z = __shfl_sync(0xffffffffu, S.z, k3 + 1);
    S1.w = __shfl_sync(0xffffffffu, S.w, k3 + 1);
    S2.x = __shfl_sync(0xffffffffu, S.x, k3 + 2);
    S2.y = __shfl_sync(0xffffffffu, S.y, k3 + 2);
    S2.z = __shfl_sync(0xffffffffu, S.z, k3 + 2);
    S2.w = __shfl_sync(0xffffffffu, S.w, k3 + 2);
    if (lane < W * 3 && lane / 3 < n) {
        const int a = lane - k3;
        float sx, sy, sz, px, py, pz;
        const float4 B = sp[k3], C = sp[k3 + 1], E4 = sp[k3 + 2];
        if (a == 0) {
            sx = S0.x + S0.y;
            sy = S0.z + S0.w;
            sz = S1.x + S1.y;
            px = B.x;
            py = B.z;
            pz = C.x;
        } else if (a == 1) {
            sx = S1.z;
            sy = S2.x;
            sz = S2.z;
            px = C.z;
            py = E4.x;
            pz = E4.z;
        } else {
            sx = S1.w;
            sy = S2.y;
            sz = S2.w;
            px = C.w;
            py = E4.y;
            pz = E4.w;
        }
        long long* __restrict__ fo = fo_base + 3 * lane;
        red_add(fo, __float2ll_rn(sx));
        red_add(fo + 1, __float2ll_rn(sy));
        red_add(fo + 2, __float2ll_rn(sz));
        v0s = fmaf(px, sx, v0s);
        v1s = fmaf(px, sy, v1s);
        v2s = fmaf(px, sz, v2s);
        v3s = fmaf(py, sy, v3s);
        v4s = fmaf(py, sz, v4s);
        v5s = fmaf(pz, sz, v5s);
    }
}

// Bit-iterating layout: one warp per i-cluster of W waters, one lane per
// j-water entry; each lane loops over the set bits of its own mask only, so
// no lane idles on another lane's bits (entries are sorted by popcount, so
// the lanes of a chunk run the same number of iterations).  The i atoms are
// read from shared memory by bit index; i-forces accumulate in a lane-private
// shared-memory row (no atomics, so the result does not depend on the order
// of lanes) and the rows are summed once per cluster.
template <int W, bool LJ00, bool LONG, bool PK>
__global__ void __launch_bounds__(128, 3)
    k_water_force_it(const SysDev* __restrict__ sys, const WaterParams wp, const WaterScaled pp) {
    constexpr int ROW = W * 3 + 1;  // float4 per lane row (+1 keeps 8 consecutive lanes on distinct banks)
    const SysDev& s = sys[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nclus = s.n_clusters[0];
    long long* __restrict__ FS = LONG ? s.fs_long : s.fs_short;
    const uint32_t* __restrict__ wl = LONG ? s.wl_l : s.wl_s;
    const int* __restrict__ wn = LONG ? s.wn_l : s.wn_s;
    const float4* __restrict__ wrec4 = reinterpret_cast<const float4*>(s.wrec);
    const int* __restrict__ clus_n = s.clus_n;
    const int wcap = s.wcap;
    float limx = wp.lim[0], limy = wp.lim[1], limz = wp.lim[2];
    if (LONG) {
        const float m = 2.f * (*s.max_delta) * 1.0001f + 1e-4f;
        limx -= m;
        limy -= m;
        limz -= m;
    }
    extern __shared__ float4 dyn[];
    float4* __restrict__ fis = dyn + static_cast<size_t>(wid) * 32 * ROW;  // [32][ROW]
    float4* __restrict__ myrow = fis + lane * ROW;
    __shared__ float4 sp_all[kWaterWarps][W * 3];
    __shared__ float4 ibuf[kWaterWarps][2][W * 3];
    __shared__ float4 jbuf[kWaterWarps][2][32 * 3];
    // long range: a chunk's j forces (fixed point, 9 per lane) and j slots,
    // so that the reductions go out with consecutive lanes on consecutive
    // components (fewer L2 sectors per reduction instruction); the short
    // range, with mostly partial chunks, reduces straight from registers
    __shared__ long long jst[LONG ? kWaterWarps : 1][LONG ? 32 * 9 : 1];
    __shared__ int jsl[LONG ? kWaterWarps : 1][32];
    float4* __restrict__ sp = sp_all[wid];
#pragma unroll
    for (int c = 0; c < W * 3; ++c) myrow[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // Clusters are handed out dynamically (one counter per launch), so warps
    // that drew cheap clusters take more and all warps finish together.  The
    // next cluster's list head, i-records and first j-chunk are fetched while
    // the current cluster's last chunk is computed.
    int* __restrict__ ctr = s.n_deferred + (LONG ? 3 : 2);
    auto fetch = [&]() {
        int c = 0;
        if (lane == 0) c = atomicAdd(ctr, 1);
        return __shfl_sync(0xffffffffu, c, 0);
    };
    int ci = fetch();
    int n_cur = ci < nclus ? clus_n[ci] : 0;
    int ib = 0, jb = 0;
    int cnt = 0;
    uint32_t e_cur = 0u, e_nx = 0u;
    if (ci < nclus) {
        cnt = wn[ci];
        const uint32_t* __restrict__ l0 = wl + static_cast<size_t>(ci) * wcap;
        e_cur = lane < cnt ? __ldg(l0 + lane) : 0u;
        e_nx = 32 + lane < cnt ? __ldg(l0 + 32 + lane) : 0u;
        if (lane < W * 3) cp_async16(&ibuf[wid][ib][lane], wrec4 + 3 * (ci * W) + lane);
        if (e_cur & 0xffu) {
            const int js = static_cast<int>(e_cur >> 8);
#pragma unroll
            for (int q = 0; q < 3; ++q) cp_async16(&jbuf[wid][jb][3 * lane + q], wrec4 + 3 * js + q);
        }
    }
    cp_async_commit();

    while (ci < nclus) {
        const int n = n_cur;
        const int base = ci * W;
        const uint32_t* __restrict__ list = wl + static_cast<size_t>(ci) * wcap;
        const int nch = (cnt + 31) >> 5;
        // the next cluster: asked for now, its index, size and list head read
        // at chunk max(nch - 2, 0), one chunk before they are needed
        int cn_raw = 0;
        if (lane == 0) cn_raw = atomicAdd(ctr, 1);
        int cn = nclus, cnt_n = 0, n_next = 0;
        uint32_t raw0 = 0u, raw1 = 0u;
        const int c_take = nch >= 2 ? nch - 2 : 0;
        auto take_next = [&]() {
            cn = __shfl_sync(0xffffffffu, cn_raw, 0);
            if (cn < nclus) {
                cnt_n = wn[cn];
                n_next = clus_n[cn];
                const uint32_t* __restrict__ ln = wl + static_cast<size_t>(cn) * wcap;
                if (lane < wcap) raw0 = __ldg(ln + lane);
                if (32 + lane < wcap) raw1 = __ldg(ln + 32 + lane);
            }
        };
        if (nch == 0) take_next();
        cp_async_wait<0>();
        __syncwarp();
        const double x00 = rec_x(ibuf[wid][ib][0]), y00 = rec_y(ibuf[wid][ib][0]);
        const double z00 = rec_x(ibuf[wid][ib][1]);
        float4 pk_p = make_float4(0.f, 0.f, 0.f, 0.f);
        if (lane < W * 3) {
            const int k = lane / 3, a = lane % 3;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < n) {
                const float4 v0 = ibuf[wid][ib][3 * k], v1 = ibuf[wid][ib][3 * k + 1], v2 = ibuf[wid][ib][3 * k + 2];
                const float dx = a == 0 ? 0.f : (a == 1 ? v1.z : v2.y);
                const float dy = a == 0 ? 0.f : (a == 1 ? v1.w : v2.z);
                const float dz = a == 0 ? 0.f : (a == 1 ? v2.x : v2.w);
                p.x = float(rec_x(v0) - x00) + dx;
                p.y = float(rec_y(v0) - y00) + dy;
                p.z = float(rec_x(v1) - z00) + dz;
            }
            if (!PK) sp[lane] = p;
            pk_p = p;
        }
        if constexpr (PK) {
            // water k's three float4: {p0x, p0x, p0y, p0y}, {p0z, p0z, p1x, p2x},
            // {p1y, p2y, p1z, p2z} (the operand pairs of the packed units)
            const int k3 = (lane / 3) * 3;
            const float a0x = __shfl_sync(0xffffffffu, pk_p.x, k3), a0y = __shfl_sync(0xffffffffu, pk_p.y, k3);
            const float a0z = __shfl_sync(0xffffffffu, pk_p.z, k3);
            const float a1x = __shfl_sync(0xffffffffu, pk_p.x, k3 + 1), a1y = __shfl_sync(0xffffffffu, pk_p.y, k3 + 1);
            const float a1z = __shfl_sync(0xffffffffu, pk_p.z, k3 + 1);
            const float a2x = __shfl_sync(0xffffffffu, pk_p.x, k3 + 2), a2y = __shfl_sync(0xffffffffu, pk_p.y, k3 + 2);
            const float a2z = __shfl_sync(0xffffffffu, pk_p.z, k3 + 2);
            const int r = lane - k3;
            if (lane < W * 3)
                sp[lane] = r == 0 ? make_float4(a0x, a0x, a0y, a0y)
                                  : (r == 1 ? make_float4(a0z, a0z, a1x, a2x) : make_float4(a1y, a2y, a1z, a2z));
        }
        float elj = 0.f, ecrf = 0.f, v0s = 0.f, v1s = 0.f, v2s = 0.f, v3s = 0.f, v4s = 0.f, v5s = 0.f;
        float2 ecrf2 = make_float2(0.f, 0.f), elj2 = make_float2(0.f, 0.f);  // packed units' energies
        int n_wp = 0;  // water pairs evaluated (the CRF constant term is added per pair at the end)
        uint32_t e_cur_n = 0u, e_nx_n = 0u;
        for (int c = 0; c < nch; ++c) {
            if (c == c_take) take_next();
            if (c + 1 < nch) {
                if (e_nx & 0xffu) {
                    const int js = static_cast<int>(e_nx >> 8);
#pragma unroll
                    for (int q = 0; q < 3; ++q) cp_async16(&jbuf[wid][jb ^ 1][3 * lane + q], wrec4 + 3 * js + q);
                }
            } else if (cn < nclus) {
                // last chunk: the next cluster's i-records and first j-chunk
                e_cur_n = lane < cnt_n ? raw0 : 0u;
                e_nx_n = 32 + lane < cnt_n ? raw1 : 0u;
                if (lane < W * 3) cp_async16(&ibuf[wid][ib ^ 1][lane], wrec4 + 3 * (cn * W) + lane);
                if (e_cur_n & 0xffu) {
                    const int js = static_cast<int>(e_cur_n >> 8);
#pragma unroll
                    for (int q = 0; q < 3; ++q) cp_async16(&jbuf[wid][jb ^ 1][3 * lane + q], wrec4 + 3 * js + q);
                }
            }
            cp_async_commit();
            const int e2 = (c + 2) * 32 + lane;
            const uint32_t e_nn = e2 < cnt ? __ldg(list + e2) : 0u;
            cp_async_wait<1>();
            __syncwarp();
            unsigned mask = e_cur & 0xffu;
            const int js = static_cast<int>(e_cur >> 8);
            if (LONG) jsl[wid][lane] = mask ? js : -1;
            if (PK && mask) {
                water_entry_packed<LJ00, LONG>(s, wp, pp, sp, myrow, jbuf[wid][jb] + 3 * lane, x00, y00, z00, limx,
                                               limy, limz, base, js, mask, FS, LONG ? jst[wid] + lane * 9 : nullptr,
                                               ecrf, elj, ecrf2, elj2, v0s, v1s, v2s, v3s, v4s, v5s, n_wp);
            } else if (mask) {
                const float4 r0 = jbuf[wid][jb][3 * lane], r1 = jbuf[wid][jb][3 * lane + 1], r2 = jbuf[wid][jb][3 * lane + 2];
                double dx = x00 - rec_x(r0), dy = y00 - rec_y(r0), dz = z00 - rec_x(r1);
                if (wp.boundary) {
                    dx -= wp.box[0] * rint(dx * wp.inv_box[0]);
                    dy -= wp.box[1] * rint(dy * wp.inv_box[1]);
                    dz -= wp.box[2] * rint(dz * wp.inv_box[2]);
                }
                const float Dx = float(dx), Dy = float(dy), Dz = float(dz);
                const float qx[3] = {-Dx, r1.z - Dx, r2.y - Dx};
                const float qy[3] = {-Dy, r1.w - Dy, r2.z - Dy};
                const float qz[3] = {-Dz, r2.x - Dz, r2.w - Dz};
                float gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
                while (mask) {
                    const int k = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const float4 p0 = sp[k * 3], p1 = sp[k * 3 + 1], p2 = sp[k * 3 + 2];
                    float pxk[3] = {p0.x, p1.x, p2.x}, pyk[3] = {p0.y, p1.y, p2.y}, pzk[3] = {p0.z, p1.z, p2.z};
                    float r0x = pxk[0] - qx[0], r0y = pyk[0] - qy[0], r0z = pzk[0] - qz[0];
                    float shx = 0.f, shy = 0.f, shz = 0.f;
                    bool shifted = false;
                    if (!(fabsf(r0x) < limx && fabsf(r0y) < limy && fabsf(r0z) < limz)) {
                        if (wp.boundary) {
                            shx = -wp.boxf[0] * rintf(r0x * wp.inv_boxf[0]);
                            shy = -wp.boxf[1] * rintf(r0y * wp.inv_boxf[1]);
                            shz = -wp.boxf[2] * rintf(r0z * wp.inv_boxf[2]);
                        }
                        r0x += shx;
                        r0y += shy;
                        r0z += shz;
                        if (!(fabsf(r0x) < limx && fabsf(r0y) < limy && fabsf(r0z) < limz)) {
                            const int d = atomicAdd(&s.n_deferred[LONG ? 1 : 0], 1);
                            if (d < s.defer_cap) {
                                s.deferred[2 * (LONG ? s.defer_cap + d : d)] = base + k;
                                s.deferred[2 * (LONG ? s.defer_cap + d : d) + 1] = js;
                            } else {
                                atomicOr(&s.err[0], ERR_DEFER_OVERFLOW);
                            }
                            continue;
                        }
#pragma unroll
                        for (int a = 0; a < 3; ++a) {  // r0 already carries the shift
                            pxk[a] += shx;
                            pyk[a] += shy;
                            pzk[a] += shz;
                        }
                        shifted = true;
                    }
                    // the i-force row is loaded now and the pair forces accumulate
                    // into it with FMAs; j-forces likewise into g
                    float4 f[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) f[a] = myrow[k * 3 + a];
                    float gs0 = 0.f, gs1 = 0.f, gs2 = 0.f;
                    if (shifted) {
                        gs0 = gx[0] + gx[1] + gx[2];
                        gs1 = gy[0] + gy[1] + gy[2];
                        gs2 = gz[0] + gz[1] + gz[2];
                    }
                    float x[9], y[9], z[9], r2[9];
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            const int t = a * 3 + b;
                            x[t] = (t == 0) ? r0x : pxk[a] - qx[b];
                            y[t] = (t == 0) ? r0y : pyk[a] - qy[b];
                            z[t] = (t == 0) ? r0z : pzk[a] - qz[b];
                            r2[t] = fmaf(x[t], x[t], fmaf(y[t], y[t], z[t] * z[t]));
                        }
                    water_pair_math<LJ00>(x, y, z, r2, f, gx, gy, gz, ecrf, elj, wp, pp);
#pragma unroll
                    for (int a = 0; a < 3; ++a) myrow[k * 3 + a] = f[a];
                    ++n_wp;
                    // virial sum_ab x_ab (x) f_ab = sum_a P_a (x) fi_a + sum_b Q_b (x) g_b
                    // (P, Q: positions relative to the cluster origin): the
                    // i-part is taken once per cluster from the column sums of
                    // the unshifted P; a shifted image adds shift (x) sum_a fi_a,
                    // which is minus the change of the j sums
                    if (shifted) {
                        const float sx = gs0 - (gx[0] + gx[1] + gx[2]);
                        const float sy = gs1 - (gy[0] + gy[1] + gy[2]);
                        const float sz = gs2 - (gz[0] + gz[1] + gz[2]);
                        v0s = fmaf(shx, sx, v0s);
                        v1s = fmaf(shx, sy, v1s);
                        v2s = fmaf(shx, sz, v2s);
                        v3s = fmaf(shy, sy, v3s);
                        v4s = fmaf(shy, sz, v4s);
                        v5s = fmaf(shz, sz, v5s);
                    }
                }
                // the j-part of the virial: Q_b (x) g_b, g_b = -sum_a f_ab
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    v0s = fmaf(qx[b], gx[b], v0s);
                    v1s = fmaf(qx[b], gy[b], v1s);
                    v2s = fmaf(qx[b], gz[b], v2s);
                    v3s = fmaf(qy[b], gy[b], v3s);
                    v4s = fmaf(qy[b], gz[b], v4s);
                    v5s = fmaf(qz[b], gz[b], v5s);
                }
                if (LONG) {
                    long long* __restrict__ st = jst[wid] + lane * 9;
#pragma unroll
                    for (int b = 0; b < 3; ++b) {  // the forces carry the 2^32 scale already
                        st[3 * b] = __float2ll_rn(gx[b]);
                        st[3 * b + 1] = __float2ll_rn(gy[b]);
                        st[3 * b + 2] = __float2ll_rn(gz[b]);
                    }
                } else {
                    long long* __restrict__ fj = FS + static_cast<size_t>(js) * 9;
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        red_add(fj + 3 * b, __float2ll_rn(gx[b]));
                        red_add(fj + 3 * b + 1, __float2ll_rn(gy[b]));
                        red_add(fj + 3 * b + 2, __float2ll_rn(gz[b]));
                    }
                }
            }
            if (LONG) {
                __syncwarp();
                // element e = 32 r + lane is component e % 9 of lane e / 9's j
                // water: the 9 components of a j water are contiguous in FS
#pragma unroll
                for (int r = 0; r < 9; ++r) {
                    const int e = r * 32 + lane;
                    const int src = e / 9;
                    const int jw = jsl[wid][src];
                    if (jw >= 0) red_add(FS + static_cast<size_t>(jw) * 9 + (e - 9 * src), jst[wid][e]);
                }
            }
            e_cur = e_nx;
            e_nx = e_nn;
            jb ^= 1;
            __syncwarp();
        }
        if (nch == 0 && cn < nclus) {  // empty list: fetch the next cluster here
            e_cur_n = lane < cnt_n ? raw0 : 0u;
            e_nx_n = 32 + lane < cnt_n ? raw1 : 0u;
            if (lane < W * 3) cp_async16(&ibuf[wid][ib ^ 1][lane], wrec4 + 3 * (cn * W) + lane);
            if (e_cur_n & 0xffu) {
                const int js = static_cast<int>(e_cur_n >> 8);
#pragma unroll
                for (int q = 0; q < 3; ++q) cp_async16(&jbuf[wid][jb][3 * lane + q], wrec4 + 3 * js + q);
            }
            cp_async_commit();
        }
        __syncwarp();
        // column sums of the lane rows: lane c < 3W owns i atom c (water c / 3)
        if constexpr (PK) {
            packed_column_sums<W>(fis, sp, FS + static_cast<size_t>(base) * 9, lane, n, v0s, v1s, v2s, v3s, v4s,
                                  v5s);
        } else if (lane < W * 3) {
            float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll 8
            for (int r = 0; r < 32; ++r) {
                const float4 f = fis[r * ROW + lane];
                sx += f.x;
                sy += f.y;
                sz += f.z;
            }
            if (lane / 3 < n) {
                long long* __restrict__ fo = FS + static_cast<size_t>(base) * 9 + 3 * lane;
                red_add(fo, __float2ll_rn(sx));
                red_add(fo + 1, __float2ll_rn(sy));
                red_add(fo + 2, __float2ll_rn(sz));
                // the i-part of the virial: P (x) F for this i atom
                const float4 P = sp[lane];
                v0s = fmaf(P.x, sx, v0s);
                v1s = fmaf(P.x, sy, v1s);
                v2s = fmaf(P.x, sz, v2s);
                v3s = fmaf(P.y, sy, v3s);
                v4s = fmaf(P.y, sz, v4s);
                v5s = fmaf(P.z, sz, v5s);
            }
        }
        __syncwarp();
#pragma unroll
        for (int cc = 0; cc < W * 3; ++cc) myrow[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (PK) {
            elj += elj2.x + elj2.y;
            ecrf += ecrf2.x + ecrf2.y;
        }
        acc[0] += to_fixed_f(elj, 16777216.0f);
        acc[1] += to_fixed_f(fmaf(-pp.crfc_sumq, float(n_wp), ecrf), 16777216.0f);
        // the virial sums carry the forces' 2^32; its fixed point is 2^24
        acc[2] += to_fixed_f(v0s, 0.00390625f);
        acc[3] += to_fixed_f(v1s, 0.00390625f);
        acc[4] += to_fixed_f(v2s, 0.00390625f);
        acc[5] += to_fixed_f(v3s, 0.00390625f);
        acc[6] += to_fixed_f(v4s, 0.00390625f);
        acc[7] += to_fixed_f(v5s, 0.00390625f);
        ib ^= 1;
        ci = cn;
        n_cur = n_next;
        cnt = cnt_n;
        e_cur = e_cur_n;
        e_nx = e_nx_n;
        __syncwarp();
    }
    cp_async_wait<0>();
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[v] = warp_sum_ll(acc[v]);
    __shared__ unsigned long long sh[8];
    if (threadIdx.x < 8) sh[threadIdx.x] = 0ull;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < 8; ++v)
            if (acc[v]) atomicAdd(&sh[v], static_cast<unsigned long long>(acc[v]));
    __syncthreads();
    if (threadIdx.x < 8 && sh[threadIdx.x]) {
        long long* dst = LONG ? s.acc_long : s.acc_short;
        const int G = wp.G, vb = 2 * G * G;
        const int v = threadIdx.x;
        const int i0 = v == 0 ? wp.slot : v == 1 ? G * G + wp.slot : vb + (v == 2 ? 0 : v == 3 ? 1 : v == 4 ? 2 : v == 5 ? 4 : v == 6 ? 5 : 8);
        const int i1 = v == 3 ? vb + 3 : v == 4 ? vb + 6 : v == 6 ? vb + 7 : -1;
        atomicAdd(reinterpret_cast<unsigned long long*>(dst + i0), sh[v]);
        if (i1 >= 0) atomicAdd(reinterpret_cast<unsigned long long*>(dst + i1), sh[v]);
    }
    // The last block to finish evaluates the pairs every block deferred (no
    // separate launch): its deferred-list reads follow every block's fence.
    __shared__ int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(s.n_deferred + (LONG ? 5 : 4), 1) == int(gridDim.x) - 1;
    __syncthreads();
    if (last) process_deferred<LJ00, LONG>(s, wp, threadIdx.x, blockDim.x);
}

template <int W>
constexpr size_t water_it_smem() {
    return size_t(kWaterWarps) * 32 * (W * 3 + 1) * sizeof(float4);
}

// The deferred pairs of the shared-bit kernel (the bit-iterating kernel
// evaluates its own in its last block).
template <bool LJ00, bool LONG>
__global__ void __launch_bounds__(128) k_water_deferred(const SysDev* __restrict__ sys, const WaterParams wp) {
    process_deferred<LJ00, LONG>(sys[blockIdx.y], wp, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template __global__ void k_water_deferred<true, false>(const SysDev*, const WaterParams);
template __global__ void k_water_deferred<true, true>(const SysDev*, const WaterParams);
template __global__ void k_water_deferred<false, false>(const SysDev*, const WaterParams);
template __global__ void k_water_deferred<false, true>(const SysDev*, const WaterParams);
template __global__ void k_water_force<true, false>(const SysDev*, const WaterParams);
template __global__ void k_water_force<true, true>(const SysDev*, const WaterParams);
template __global__ void k_water_force<false, false>(const SysDev*, const WaterParams);
template __global__ void k_water_force<false, true>(const SysDev*, const WaterParams);

}  // namespace gnb

namespace gnb {
template __global__ void k_water_force_it<4, true, false, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, true, true, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, false, false, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, false, true, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, true, false, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, true, true, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, false, false, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, false, true, false>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, true, false, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, true, true, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, false, false, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<4, false, true, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, true, false, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, true, true, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, false, false, true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_it<8, false, true, true>(const SysDev*, const WaterParams, const WaterScaled);
}  // namespace gnb
