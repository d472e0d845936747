// water_ps.cu -- short-range water-water forces, pair-stream layout (layout 3).
//
// Physics per atom pair: lj_crf_interaction
// (crates/gromos-forces/src/nonbonded/innerloops.rs:21-55, r^2 < 1e-10 gives
// zeros) over the nine atom pairs of every listed solvent CG pair, with the
// parameter table of the first solvent molecule (innerloops.rs:241-255) and
// one image per CG pair taken from the first atoms (innerloops.rs:264-267).
//
// Work layout.  A warp takes units of two consecutive i-clusters (W = 4
// waters each) from a counter.  The entries of a cluster's j-list (sorted by
// mask popcount, most bits first) are dealt to the 32 lanes in snake order
// (round r: lane l gets entry 32 r + l, or 32 r + 31 - l on odd rounds; the
// second cluster of the unit starts reversed), so that the lanes' shares of
// water pairs are close to equal.  Each lane then streams its own water
// pairs: one water pair (one mask bit) per iteration, moving on to its next
// entry when the current one has no bits left.  No lane waits for another
// lane's bits, only for the unit's longest share.
//
// Per lane: the current j-water (FP32 coordinates relative to its cluster's
// first atom, after an FP64 nearest image), its force accumulated over the
// entry's bits in registers and reduced once per entry into the slot's
// 64-bit fixed-point sum; the records of the next entry arrive by cp.async
// into a lane-private buffer while the current one is computed.  i-forces
// accumulate in a lane-private shared-memory row per unit and are summed over
// the lanes when the unit retires.  The assignment of pairs to lanes depends
// only on the list, so every FP32 partial sum, and hence every fixed-point
// total, is the same run to run.
//
// Force constants carry the fixed-point scale 2^32, so the FP32 sums convert
// to fixed point without a multiply; energies use the unscaled constants.
#include "nb_common.cuh"

namespace gnb {

constexpr int kPsWarps = 4;
constexpr int kPsAtoms = 2 * 4 * 3;    // i atoms of a unit: two clusters of 4 three-site waters
constexpr int kPsRow = kPsAtoms + 1;   // float4 per lane row (+1: consecutive lanes on distinct banks)
constexpr int kPsJRow = 7;             // float4 per lane j buffer: 2 x 3 records + 1 pad

template <int N>
__device__ __forceinline__ void ps_cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ps_red(long long* addr, long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(addr), "l"(v) : "memory");
}

// Entry index of lane `lane` in round r of a cluster whose snake phase is `ph`.
__device__ __forceinline__ int ps_entry(int r, int ph, int lane) { return 32 * r + (((r ^ ph) & 1) ? 31 - lane : lane); }

template <bool LJ00>
__global__ void __launch_bounds__(128, 3)
    k_water_force_ps(const SysDev* __restrict__ sys, const WaterParams wp, const WaterScaled pp) {
    constexpr int W = 4;
    const SysDev& s = sys[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int nclus = s.n_clusters[0];
    const int nunits = (nclus + 1) >> 1;
    long long* __restrict__ FS = s.fs_short;
    const uint32_t* __restrict__ wl = s.wl_s;
    const int* __restrict__ wn = s.wn_s;
    const float4* __restrict__ wrec4 = reinterpret_cast<const float4*>(s.wrec);
    const int* __restrict__ clus_n = s.clus_n;
    const size_t wcap = static_cast<size_t>(s.wcap);
    const float limx = wp.lim[0], limy = wp.lim[1], limz = wp.lim[2];

    extern __shared__ float4 dyn_ps[];
    float4* __restrict__ myrow = dyn_ps + (static_cast<size_t>(wid) * 32 + lane) * kPsRow;
    float4* __restrict__ rows = dyn_ps + static_cast<size_t>(wid) * 32 * kPsRow;
    __shared__ float4 ibuf_all[kPsWarps][2][kPsAtoms];  // raw i-records: current unit, next unit
    __shared__ float4 sp_all[kPsWarps][kPsAtoms];       // i atoms relative to their cluster's first atom
    __shared__ float4 jb_all[kPsWarps][32][kPsJRow];    // lane-private j-record double buffer
    float4* __restrict__ sp = sp_all[wid];
    float4* __restrict__ jb = jb_all[wid][lane];
#pragma unroll
    for (int c = 0; c < kPsAtoms; ++c) myrow[c] = make_float4(0.f, 0.f, 0.f, 0.f);

    int* __restrict__ ctr = s.n_deferred + 2;
    auto fetch = [&]() {
        int c = 0;
        if (lane == 0) c = atomicAdd(ctr, 1);
        return __shfl_sync(0xffffffffu, c, 0);
    };
    // unit header: entry counts and water counts of its two clusters
    auto header = [&](int u, int& c0, int& c1, int& n0, int& n1) {
        c0 = c1 = n0 = n1 = 0;
        if (u < nunits) {
            c0 = wn[2 * u];
            n0 = clus_n[2 * u];
            if (2 * u + 1 < nclus) {
                c1 = wn[2 * u + 1];
                n1 = clus_n[2 * u + 1];
            }
        }
    };
    auto irec_copy = [&](int u, int buf) {
        if (u < nunits && lane < kPsAtoms) {
            const int c = 2 * u + lane / 12;
            if (c < nclus) cp_async16(&ibuf_all[wid][buf][lane], wrec4 + 3 * (static_cast<size_t>(c) * W) + lane % 12);
        }
    };

    // units: current (uc) and next (un); a warp holds at most one unit ahead,
    // so that the last units go to the warps that finish first
    int uc = fetch(), un = fetch();
    int cc0, cc1, nc0, nc1, cn0, cn1, nn0, nn1;
    header(uc, cc0, cc1, nc0, nc1);
    header(un, cn0, cn1, nn0, nn1);
    int ib = 0;
    irec_copy(uc, ib);
    irec_copy(un, ib ^ 1);
    cp_async_commit();

    // ---- per-lane entry stream: a generator over (unit 0 = current, 1 = next; half; round)
    int gu = 0, gh = 0, gr = 0;
    auto gen = [&](int& pu, int& ph, int& pe) -> bool {
        while (gu < 2) {
            const int cnt = gu == 0 ? (gh == 0 ? cc0 : cc1) : (gh == 0 ? cn0 : cn1);
            const bool uvalid = (gu == 0 ? uc : un) < nunits;
            if (uvalid) {
                const int e = ps_entry(gr, gh, lane);
                if (e < cnt) {
                    pu = gu;
                    ph = gh;
                    pe = e;
                    ++gr;
                    return true;
                }
            }
            if (gh == 0 && uvalid) {
                gh = 1;
                gr = 0;
                continue;
            }
            ++gu;
            gh = 0;
            gr = 0;
        }
        return false;
    };
    auto word_at = [&](int pu, int ph, int pe) -> uint32_t {
        const int u = pu == 0 ? uc : un;
        return __ldg(wl + static_cast<size_t>(2 * u + ph) * wcap + pe);
    };
    // queue: cur (in registers), nxt (records in jb[nb]), nq (word loading)
    bool cur_v = false, nxt_v = false, nq_v = false;
    int cur_h = 0, nxt_u = 0, nxt_h = 0, nq_u = 0, nq_h = 0, nb = 0;
    uint32_t cur_mask = 0u, nxt_w = 0u, nq_w = 0u;
    int cur_js = 0;
    float qx[3], qy[3], qz[3], g[9];
    {
        int pu, ph, pe;
        if ((nxt_v = gen(pu, ph, pe))) {
            nxt_u = pu;
            nxt_h = ph;
            nxt_w = word_at(pu, ph, pe);
        }
        if ((nq_v = gen(pu, ph, pe))) {
            nq_u = pu;
            nq_h = ph;
            nq_w = word_at(pu, ph, pe);
        }
        if (nxt_v) {
            const int js = static_cast<int>(nxt_w >> 8);
#pragma unroll
            for (int q = 0; q < 3; ++q) cp_async16(&jb[nb * 3 + q], wrec4 + 3 * static_cast<size_t>(js) + q);
        }
        cp_async_commit();
    }

    float ecrf = 0.f, elj = 0.f, v0s = 0.f, v1s = 0.f, v2s = 0.f, v3s = 0.f, v4s = 0.f, v5s = 0.f;
    int n_wp = 0;
    long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};

    // nxt -> cur (its records have landed: the lane's only copy in flight),
    // nq -> nxt (records copy issued), generator -> nq (word load issued).
    // Only entries of the current unit are promoted.  Within a unit the nxt
    // copy is the lane's most recent group (wait for all); at a unit start the
    // caller has already waited for every group older than the boundary's.
    auto promote = [&](bool wait_all) {
        cur_v = nxt_v && nxt_u == 0;
        if (!cur_v) return;
        if (wait_all) ps_cp_async_wait<0>();
        const float4 r0 = jb[nb * 3], r1 = jb[nb * 3 + 1], r2 = jb[nb * 3 + 2];
        const float4 o0 = ibuf_all[wid][ib][nxt_h * 12], o1 = ibuf_all[wid][ib][nxt_h * 12 + 1];
        double dx = rec_x(o0) - rec_x(r0), dy = rec_y(o0) - rec_y(r0), dz = rec_x(o1) - rec_x(r1);
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
#pragma unroll
        for (int c = 0; c < 9; ++c) g[c] = 0.f;
        cur_h = nxt_h;
        cur_mask = nxt_w & 0xfu;  // width-4 clusters: bits 0..3
        cur_js = static_cast<int>(nxt_w >> 8);
        nb ^= 1;
        nxt_v = nq_v;
        nxt_u = nq_u;
        nxt_h = nq_h;
        nxt_w = nq_w;
        if (nxt_v) {
            const int js = static_cast<int>(nxt_w >> 8);
#pragma unroll
            for (int q = 0; q < 3; ++q) cp_async16(&jb[nb * 3 + q], wrec4 + 3 * static_cast<size_t>(js) + q);
        }
        cp_async_commit();
        int pu, ph, pe;
        if ((nq_v = gen(pu, ph, pe))) {
            nq_u = pu;
            nq_h = ph;
            nq_w = word_at(pu, ph, pe);
        }
    };
    // the finished entry's j forces (fixed point) and the j part of the virial
    auto flush = [&]() {
        long long* __restrict__ fj = FS + static_cast<size_t>(cur_js) * 9;
#pragma unroll
        for (int c = 0; c < 9; ++c) ps_red(fj + c, __float2ll_rn(g[c]));
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            v0s = fmaf(qx[b], g[3 * b], v0s);
            v1s = fmaf(qx[b], g[3 * b + 1], v1s);
            v2s = fmaf(qx[b], g[3 * b + 2], v2s);
            v3s = fmaf(qy[b], g[3 * b + 1], v3s);
            v4s = fmaf(qy[b], g[3 * b + 2], v4s);
            v5s = fmaf(qz[b], g[3 * b + 2], v5s);
        }
    };

    // copy groups this lane committed after the ones the unit start needs
    // (the next unit's i-records, and an entry copy of the next unit)
    int late_groups = 0;
    while (uc < nunits) {
        // i atoms of the current unit relative to their cluster's first atom;
        // the current unit's i-records and first entry records were committed
        // before the last `late_groups` groups
        if (late_groups == 0)
            ps_cp_async_wait<0>();
        else if (late_groups == 1)
            ps_cp_async_wait<1>();
        else
            ps_cp_async_wait<2>();
        __syncwarp();
        if (lane < kPsAtoms) {
            const int h = lane / 12, k = (lane % 12) / 3, a = lane % 3;
            const int n = h == 0 ? nc0 : nc1;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < n) {
                const float4* rb = &ibuf_all[wid][ib][h * 12];
                const double x00 = rec_x(rb[0]), y00 = rec_y(rb[0]), z00 = rec_x(rb[1]);
                const float4 v0 = rb[3 * k], v1 = rb[3 * k + 1], v2 = rb[3 * k + 2];
                const float dx = a == 0 ? 0.f : (a == 1 ? v1.z : v2.y);
                const float dy = a == 0 ? 0.f : (a == 1 ? v1.w : v2.z);
                const float dz = a == 0 ? 0.f : (a == 1 ? v2.x : v2.w);
                p.x = float(rec_x(v0) - x00) + dx;
                p.y = float(rec_y(v0) - y00) + dy;
                p.z = float(rec_x(v1) - z00) + dz;
            }
            sp[lane] = p;
        }
        __syncwarp();
        promote(false);

        while (__any_sync(0xffffffffu, cur_v)) {
            if (cur_v && cur_mask != 0u) {
                const int k = __ffs(cur_mask) - 1;
                cur_mask &= cur_mask - 1;
                const int ia = (cur_h * W + k) * 3;
                const float4 p0 = sp[ia], p1 = sp[ia + 1], p2 = sp[ia + 2];
                float px[3] = {p0.x, p1.x, p2.x}, py[3] = {p0.y, p1.y, p2.y}, pz[3] = {p0.z, p1.z, p2.z};
                // the first-atom vector decides whether the FP32 image is certain;
                // otherwise one FP32 re-image of the CG pair, and if still not
                // certain the pair goes to the exact FP64 path (deferred)
                float r0x = px[0] - qx[0], r0y = py[0] - qy[0], r0z = pz[0] - qz[0];
                bool go = true, shifted = false;
                float shx = 0.f, shy = 0.f, shz = 0.f;
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
                        const int d = atomicAdd(&s.n_deferred[0], 1);
                        if (d < s.defer_cap) {
                            s.deferred[2 * d] = (2 * uc + cur_h) * W + k;
                            s.deferred[2 * d + 1] = cur_js;
                        } else {
                            atomicOr(&s.err[0], ERR_DEFER_OVERFLOW);
                        }
                        go = false;
                    } else {
#pragma unroll
                        for (int a = 0; a < 3; ++a) {  // r0 already carries the shift
                            px[a] += shx;
                            py[a] += shy;
                            pz[a] += shz;
                        }
                        shifted = true;
                    }
                }
                if (go) {
                    float gs0 = 0.f, gs1 = 0.f, gs2 = 0.f;
                    if (shifted) {
                        gs0 = g[0] + g[3] + g[6];
                        gs1 = g[1] + g[4] + g[7];
                        gs2 = g[2] + g[5] + g[8];
                    }
                    float x[9], y[9], z[9], r2[9];
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            const int t = a * 3 + b;
                            x[t] = (t == 0) ? r0x : px[a] - qx[b];
                            y[t] = (t == 0) ? r0y : py[a] - qy[b];
                            z[t] = (t == 0) ? r0z : pz[a] - qz[b];
                            r2[t] = fmaf(x[t], x[t], fmaf(y[t], y[t], z[t] * z[t]));
                        }
                    float4 f[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) f[a] = myrow[ia + a];
                    float gx[3] = {g[0], g[3], g[6]}, gy[3] = {g[1], g[4], g[7]}, gz[3] = {g[2], g[5], g[8]};
                    water_pair_math<LJ00>(x, y, z, r2, f, gx, gy, gz, ecrf, elj, wp, pp);
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        g[3 * b] = gx[b];
                        g[3 * b + 1] = gy[b];
                        g[3 * b + 2] = gz[b];
                    }
#pragma unroll
                    for (int a = 0; a < 3; ++a) myrow[ia + a] = f[a];
                    ++n_wp;
                    if (shifted) {
                        // a re-imaged pair adds shift (x) (sum of its forces on the i atoms)
                        // = -shift (x) (change of the j sums)
                        const float sx = gs0 - (g[0] + g[3] + g[6]);
                        const float sy = gs1 - (g[1] + g[4] + g[7]);
                        const float sz = gs2 - (g[2] + g[5] + g[8]);
                        v0s = fmaf(shx, sx, v0s);
                        v1s = fmaf(shx, sy, v1s);
                        v2s = fmaf(shx, sz, v2s);
                        v3s = fmaf(shy, sy, v3s);
                        v4s = fmaf(shy, sz, v4s);
                        v5s = fmaf(shz, sz, v5s);
                    }
                }
            }
            if (cur_v && cur_mask == 0u) {
                flush();
                promote(true);
            }
        }

        // ---- retire the unit: column sums of the lane rows (lane c < 24 owns i atom c)
        __syncwarp();
        if (lane < kPsAtoms) {
            float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll 8
            for (int r = 0; r < 32; ++r) {
                const float4 f = rows[r * kPsRow + lane];
                sx += f.x;
                sy += f.y;
                sz += f.z;
            }
            const int h = lane / 12, k = (lane % 12) / 3, a = lane % 3;
            if (k < (h == 0 ? nc0 : nc1)) {
                long long* __restrict__ fo = FS + (static_cast<size_t>(2 * uc + h) * W + k) * 9 + 3 * a;
                red_add(fo, __float2ll_rn(sx));
                red_add(fo + 1, __float2ll_rn(sy));
                red_add(fo + 2, __float2ll_rn(sz));
                const float4 P = sp[lane];  // the i part of the virial: P (x) F
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
        for (int c = 0; c < kPsAtoms; ++c) myrow[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        acc[0] += to_fixed_f(elj, 16777216.0f);
        acc[1] += to_fixed_f(fmaf(-pp.crfc_sumq, float(n_wp), ecrf), 16777216.0f);
        // forces carry 2^32; the virial fixed point is 2^24
        acc[2] += to_fixed_f(v0s, 0.00390625f);
        acc[3] += to_fixed_f(v1s, 0.00390625f);
        acc[4] += to_fixed_f(v2s, 0.00390625f);
        acc[5] += to_fixed_f(v3s, 0.00390625f);
        acc[6] += to_fixed_f(v4s, 0.00390625f);
        acc[7] += to_fixed_f(v5s, 0.00390625f);
        ecrf = elj = v0s = v1s = v2s = v3s = v4s = v5s = 0.f;
        n_wp = 0;

        // ---- next unit: the one after it is fetched now
        uc = un;
        cc0 = cn0;
        cc1 = cn1;
        nc0 = nn0;
        nc1 = nn1;
        un = uc < nunits ? fetch() : nunits;
        header(un, cn0, cn1, nn0, nn1);
        ib ^= 1;
        irec_copy(un, ib ^ 1);
        cp_async_commit();
        late_groups = 1;
        // stream positions move down one unit
        if (gu > 0) --gu;
        if (nxt_v) --nxt_u;
        if (nq_v) --nq_u;
        if (!nq_v) {  // a lane whose stream had run out resumes in the new next unit
            int pu, ph, pe;
            if ((nq_v = gen(pu, ph, pe))) {
                nq_u = pu;
                nq_h = ph;
                nq_w = word_at(pu, ph, pe);
            }
        }
        if (!nxt_v && nq_v) {  // promote needs nxt: move nq up and start its copy
            nxt_v = true;
            nxt_u = nq_u;
            nxt_h = nq_h;
            nxt_w = nq_w;
            const int js = static_cast<int>(nxt_w >> 8);
#pragma unroll
            for (int q = 0; q < 3; ++q) cp_async16(&jb[nb * 3 + q], wrec4 + 3 * static_cast<size_t>(js) + q);
            cp_async_commit();
            late_groups = 2;  // this entry belongs to the next unit (its stream had run out)
            int pu, ph, pe;
            if ((nq_v = gen(pu, ph, pe))) {
                nq_u = pu;
                nq_h = ph;
                nq_w = word_at(pu, ph, pe);
            }
        }
    }
    ps_cp_async_wait<0>();
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[v] = warp_sum_ll(acc[v]);
    __shared__ unsigned long long sh_ps[8];
    if (threadIdx.x < 8) sh_ps[threadIdx.x] = 0ull;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < 8; ++v)
            if (acc[v]) atomicAdd(&sh_ps[v], static_cast<unsigned long long>(acc[v]));
    __syncthreads();
    if (threadIdx.x < 8 && sh_ps[threadIdx.x]) {
        long long* dst = s.acc_short;
        const int G = wp.G, vb = 2 * G * G;
        const int v = threadIdx.x;
        const int i0 = v == 0 ? wp.slot : v == 1 ? G * G + wp.slot : vb + (v == 2 ? 0 : v == 3 ? 1 : v == 4 ? 2 : v == 5 ? 4 : v == 6 ? 5 : 8);
        const int i1 = v == 3 ? vb + 3 : v == 4 ? vb + 6 : v == 6 ? vb + 7 : -1;
        atomicAdd(reinterpret_cast<unsigned long long*>(dst + i0), sh_ps[v]);
        if (i1 >= 0) atomicAdd(reinterpret_cast<unsigned long long*>(dst + i1), sh_ps[v]);
    }
    // the last block to finish evaluates the pairs every block deferred
    __shared__ int last_ps;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last_ps = atomicAdd(s.n_deferred + 4, 1) == int(gridDim.x) - 1;
    __syncthreads();
    if (last_ps) process_deferred<LJ00, false>(s, wp, threadIdx.x, blockDim.x);
}

constexpr size_t water_ps_smem() { return size_t(kPsWarps) * 32 * kPsRow * sizeof(float4); }

template __global__ void k_water_force_ps<true>(const SysDev*, const WaterParams, const WaterScaled);
template __global__ void k_water_force_ps<false>(const SysDev*, const WaterParams, const WaterScaled);

}  // namespace gnb
