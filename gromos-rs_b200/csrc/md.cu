// md.cu -- MD steps around the force evaluation, device resident.
//
// One step is the sequence of gromos-md's md binary (md.rs:1144-1230) without
// thermostat: Forcefield::apply (the nonbonded path of this library) at r(t),
// leap-frog velocity v(t+dt/2) = v(t-dt/2) + F/m dt (leap_frog.rs:37-85),
// leap-frog position r(t+dt) = r(t) + v dt (leap_frog.rs:116-148) and SETTLE
// for every 3-site solvent molecule (constraints.rs:815-1010).  Positions,
// velocities and forces never leave the device between steps.
//
// Overflow recovery: list overflows (pairlist capacity, deferred water pairs)
// are detected after the fact from the device error flags.  The runner keeps
// a device snapshot of (positions, velocities) at the start of every block of
// pairlist periods (a period is the steps between two rebuilds), reads the
// flags at the end of the block, and on overflow grows the lists, restores
// the snapshot and runs the block again, so an overflow never leaks into the
// trajectory.
#include <cuda_runtime.h>

namespace gnb {

struct MdDev {
    double* vel;              // n_atoms*3
    const double* inv_mass;   // n_atoms
    const double* mass;       // n_atoms
    double dt, dt_i;
    int settle;               // SETTLE every solvent molecule
    double m_o, m_h, ra, rb, rc;  // canonical SETTLE triangle (constraints.rs:836-840)
    long long* ke;            // [3]: [0] kinetic energy of the velocities entering the step, [1] accumulator
                              // of the velocities leaving it (fixed point 2^24), [2] blocks finished
    int* failures;            // [1] molecules SETTLE could not solve
    const double* t0;         // [1] Berendsen bath temperature (device memory: a replica exchange changes it
                              // without touching recorded graphs)
    double tau, dof;          // Berendsen bath (tau < 0: none)
    int prep_next;            // also write the next step's water records (SETTLE units, no rebuild next)
};

// Berendsen weak coupling (berendsen_thermostat.rs:74-98): lambda from the
// kinetic energy of the velocities entering this step.
__device__ __forceinline__ double berendsen_lambda(const MdDev& md) {
    if (md.tau < 0.0) return 1.0;
    const double kB = 0.00831446261815324;
    const double ekin = double(md.ke[0]) / kEnergyScale;
    const double t0 = *md.t0;
    double t = md.dof > 0.0 ? 2.0 * ekin / (md.dof * kB) : 0.0;
    if (t < 1e-10) t = t0;
    if (t < 1e-10) return 1.0;
    return md.tau == 0.0 ? sqrt(t0 / t) : sqrt(1.0 + md.dt / md.tau * (t0 / t - 1.0));
}

// Velocities scaled by `f` (temperature exchange), kinetic energy with them.
__global__ void k_scale_velocities(double* __restrict__ vel, int n3, double f, long long* ke) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) vel[i] *= f;
    if (blockIdx.x == 0 && threadIdx.x == 0) ke[0] = __double2ll_rn(double(ke[0]) * f * f);
}

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// SETTLE for one molecule (Miyamoto & Kollman 1992, eqs. A3-A17): the frame
// is spanned by the old molecular plane and the new centre of mass; the
// three rotation sines are solved analytically.  Velocities receive the
// displacement / dt.  Returns false (molecule left unconstrained, as the
// reference does) when a sine leaves [-1, 1].
__device__ bool settle_molecule(const D3 old[3], D3 nw[3], D3 v[3], const MdDev& md) {
    D3 b0 = old[1] - old[0], c0 = old[2] - old[0];
    const double mt_i = 1.0 / (md.m_o + 2.0 * md.m_h);
    const D3 d0 = (nw[0] * md.m_o + nw[1] * md.m_h + nw[2] * md.m_h) * mt_i;
    D3 a1 = nw[0] - d0, b1 = nw[1] - d0, c1 = nw[2] - d0;
    D3 n0 = cross3(b0, c0);
    D3 n1 = cross3(a1, n0);
    D3 n2 = cross3(n0, n1);
    n0 = n0 * rsqrt(dot3(n0, n0));
    n1 = n1 * rsqrt(dot3(n1, n1));
    n2 = n2 * rsqrt(dot3(n2, n2));
    b0 = d3(dot3(n1, b0), dot3(n2, b0), dot3(n0, b0));
    c0 = d3(dot3(n1, c0), dot3(n2, c0), dot3(n0, c0));
    a1 = d3(dot3(n1, a1), dot3(n2, a1), dot3(n0, a1));
    b1 = d3(dot3(n1, b1), dot3(n2, b1), dot3(n0, b1));
    c1 = d3(dot3(n1, c1), dot3(n2, c1), dot3(n0, c1));
    const double sinphi = a1.z / md.ra;
    const double omp = 1.0 - sinphi * sinphi;
    if (omp < 0.0) return false;
    const double cosphi = sqrt(omp);
    const double sinpsi = (b1.z - c1.z) / (2.0 * md.rc * cosphi);
    const double omq = 1.0 - sinpsi * sinpsi;
    if (omq < 0.0) return false;
    const double cospsi = sqrt(omq);
    const double y_a2 = md.ra * cosphi, x_b2 = -md.rc * cospsi;
    const double y_b2 = -md.rb * cosphi - md.rc * sinpsi * sinphi;
    const double y_c2 = -md.rb * cosphi + md.rc * sinpsi * sinphi;
    const double alpha = x_b2 * (b0.x - c0.x) + b0.y * y_b2 + c0.y * y_c2;
    const double beta = x_b2 * (c0.y - b0.y) + b0.x * y_b2 + c0.x * y_c2;
    const double gamma = b0.x * b1.y - b1.x * b0.y + c0.x * c1.y - c1.x * c0.y;
    const double ab2 = alpha * alpha + beta * beta;
    const double disc = ab2 - gamma * gamma;
    if (disc < 0.0) return false;
    const double sintheta = (alpha * gamma - beta * sqrt(disc)) / ab2;
    const double omt = 1.0 - sintheta * sintheta;
    if (omt < 0.0) return false;
    const double costheta = sqrt(omt);
    const D3 r3[3] = {d3(-y_a2 * sintheta, y_a2 * costheta, a1.z),
                      d3(x_b2 * costheta - y_b2 * sintheta, x_b2 * sintheta + y_b2 * costheta, b1.z),
                      d3(-x_b2 * costheta - y_c2 * sintheta, -x_b2 * sintheta + y_c2 * costheta, c1.z)};
    // back to the lab frame: rows of the transposed basis
    const D3 m1 = d3(n1.x, n2.x, n0.x), m2 = d3(n1.y, n2.y, n0.y), m0 = d3(n1.z, n2.z, n0.z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const D3 p = d3(dot3(r3[k], m1), dot3(r3[k], m2), dot3(r3[k], m0)) + d0;
        const D3 d = p - nw[k];
        nw[k] = p;
        v[k] = v[k] + d * md.dt_i;
    }
    return true;
}

// One thread per unit: a solute atom (leap-frog only) or a solvent molecule
// (leap-frog of its atoms, then SETTLE).  Forces are the finalized FP64
// forces of this step's evaluation.  With prep_next the kernel also does the
// next evaluation's k_water_prep for each molecule from its new coordinates
// (same record, same cleared force sums, same excluded energies and extent;
// the slots are those of the current lists, so only when the next step keeps
// them): the next evaluation then skips k_water_prep.
__global__ void k_md_step(const SysDev* __restrict__ sys, MdDev md) {
    // descriptor pointers in registers and every load of a unit before its
    // stores (stores through descriptor pointers would otherwise order the
    // later reads behind them)
    const SysDev& s = *sys;
    const int nsa = s.n_solute_atoms, n = s.n_atoms, nscg = s.n_solute_cg;
    const double* __restrict__ f_out = s.f_out;
    double* __restrict__ pos = s.pos;
    const int* __restrict__ cg_slot = s.cg_slot;
    const double* __restrict__ charge = s.charge;
    const bool excl = s.excl_atoms < n;
    const int n_mol = md.settle ? (n - nsa) / 3 : 0;
    const int n_units = md.settle ? nsa + n_mol : n;
    const double lambda = berendsen_lambda(md);
    long long ke = 0;
    double e_excl = 0.0;
    float m_ext = 0.f;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n_units; u += gridDim.x * blockDim.x) {
        const bool mol = md.settle && u >= nsa;
        const int a0 = mol ? nsa + 3 * (u - nsa) : u;
        const int na = mol ? 3 : 1;
        const bool rec = mol && md.prep_next;
        const int slot = rec ? cg_slot[nscg + (u - nsa)] : -1;
        double q3[3] = {0.0, 0.0, 0.0};
        if (rec && excl)
#pragma unroll
            for (int a = 0; a < 3; ++a) q3[a] = charge[a0 + a];
        D3 old[3], nw[3], v[3];
        double mass[3];
        for (int k = 0; k < na; ++k) {
            const int i = a0 + k;
            const D3 f = d3(f_out[3 * i], f_out[3 * i + 1], f_out[3 * i + 2]);
            const double im = md.inv_mass[i];
            mass[k] = md.mass[i];
            v[k] = (d3(md.vel[3 * i], md.vel[3 * i + 1], md.vel[3 * i + 2]) + f * im * md.dt) * lambda;
            old[k] = d3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
            nw[k] = old[k] + v[k] * md.dt;
        }
        if (mol && !settle_molecule(old, nw, v, md)) atomicAdd(md.failures, 1);
        if (rec && slot >= 0) {
            const double p[9] = {nw[0].x, nw[0].y, nw[0].z, nw[1].x, nw[1].y, nw[1].z, nw[2].x, nw[2].y, nw[2].z};
            water_record(s, slot, p, q3, excl, e_excl, m_ext);
        }
        for (int k = 0; k < na; ++k) {
            const int i = a0 + k;
            pos[3 * i] = nw[k].x;
            pos[3 * i + 1] = nw[k].y;
            pos[3 * i + 2] = nw[k].z;
            md.vel[3 * i] = v[k].x;
            md.vel[3 * i + 1] = v[k].y;
            md.vel[3 * i + 2] = v[k].z;
            ke += to_fixed_d(0.5 * mass[k] * dot3(v[k], v[k]), kEnergyScale);
        }
    }
    if (md.prep_next) water_record_flush(s, m_ext, e_excl, excl);  // block-uniform
    ke = warp_sum_ll(ke);
    if ((threadIdx.x & 31) == 0 && ke) atomicAdd(reinterpret_cast<unsigned long long*>(md.ke + 1),
                                                  static_cast<unsigned long long>(ke));
    // The last block to finish makes the accumulated kinetic energy the next
    // step's input (every block read ke[0] for its bath factor before adding).
    __shared__ int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last = atomicAdd(reinterpret_cast<unsigned long long*>(md.ke + 2), 1ull) == gridDim.x - 1;
    __syncthreads();
    if (last && threadIdx.x == 0) {
        md.ke[0] = static_cast<long long>(atomicExch(reinterpret_cast<unsigned long long*>(md.ke + 1), 0ull));
        md.ke[2] = 0;
    }
}

}  // namespace gnb

using namespace gnb;

gr_status NbSystem::md_init(const double* mass, const double* vel, const gr_md_params* p) {
    prepped_next = false;
    if (!uploaded) {
        set_error("gr_md_init before gr_system_upload");
        return GR_ERR_STATE;
    }
    if (!mass || !p) {
        set_error("gr_md_init: null mass or params");
        return GR_ERR_INVALID;
    }
    if (!(p->dt > 0.0)) {
        set_error("gr_md_init: dt must be positive");
        return GR_ERR_INVALID;
    }
    for (int i = 0; i < N; ++i)
        if (!(mass[i] > 0.0)) {
            set_error("gr_md_init: every mass must be positive");
            return GR_ERR_INVALID;
        }
    const bool settle = p->settle != 0 && N > NSA;
    if (settle) {
        if (aps != 3 || (N - NSA) % 3 != 0) {
            set_error("gr_md_init: SETTLE needs 3-site solvent molecules");
            return GR_ERR_UNSUPPORTED;
        }
        for (int i = NSA; i < N; i += 3)
            if (mass[i] != mass[NSA] || mass[i + 1] != mass[NSA + 1] || mass[i + 2] != mass[NSA + 1]) {
                set_error("gr_md_init: SETTLE needs one solvent with equal masses of sites 1 and 2");
                return GR_ERR_UNSUPPORTED;
            }
        if (!(p->dist_oh > 0.0) || !(p->dist_hh > 0.0) || !(p->dist_hh < 2.0 * p->dist_oh)) {
            set_error("gr_md_init: SETTLE lengths must satisfy 0 < dist_hh < 2 dist_oh");
            return GR_ERR_INVALID;
        }
    }
    std::vector<double> inv(N);
    for (int i = 0; i < N; ++i) inv[i] = 1.0 / mass[i];
    std::vector<double> v0(size_t(N) * 3, 0.0);
    if (vel) std::copy(vel, vel + size_t(N) * 3, v0.begin());
    gr_status st;
    if ((st = upload_array(&md_mass, mass, N)) || (st = upload_array(&md_inv_mass, inv.data(), N)) ||
        (st = upload_array(&md_vel, v0.data(), size_t(N) * 3)) || (st = alloc(&md_pos_snap, size_t(N) * 3)) ||
        (st = alloc(&md_vel_snap, size_t(N) * 3)) || (st = alloc(&md_ke, 3)) || (st = alloc(&md_ke_snap, 1)) ||
        (st = alloc(&md_psnap_pos, size_t(N) * 3)) || (st = alloc(&md_psnap_vel, size_t(N) * 3)) ||
        (st = alloc(&md_psnap_ke, 1)) || (st = alloc(&md_fail, 1)) || (st = alloc(&md_t0, 1)))
        return st;
    GR_CUDA(cudaMemcpy(md_t0, &p->temperature, sizeof(double), cudaMemcpyHostToDevice));
    {
        double ke0 = 0.0;
        for (int i = 0; i < N; ++i)
            ke0 += 0.5 * mass[i] * (v0[3 * i] * v0[3 * i] + v0[3 * i + 1] * v0[3 * i + 1] + v0[3 * i + 2] * v0[3 * i + 2]);
        const long long k[3] = {static_cast<long long>(std::llround(ke0 * kEnergyScale)), 0, 0};
        GR_CUDA(cudaMemcpy(md_ke, k, sizeof(k), cudaMemcpyHostToDevice));
    }
    GR_CUDA(cudaMemset(md_fail, 0, sizeof(int)));
    md_steps_total = 0;
    md_rollbacks = 0;
    md_step_idx = 0;
    md_psnap_valid = false;
    // an MD run starts a pairlist period with a build at its first step
    built = false;
    lr_computed = false;
    if (!md_err_host) GR_CUDA(cudaMallocHost(&md_err_host, 8 * sizeof(long long)));
    if (!ev_md) GR_CUDA(cudaEventCreateWithFlags(&ev_md, cudaEventDisableTiming));
    mdp = *p;
    md_settle = settle;
    // degrees of freedom: 3N minus the solvent constraints (md.rs:1158-1172; NDFMIN 0)
    md_dof = 3.0 * N - (settle ? 3.0 * ((N - NSA) / 3) : 0.0);
    if (settle) {  // canonical triangle (constraints.rs:836-840)
        md_m_o = mass[NSA];
        md_m_h = mass[NSA + 1];
        const double half_mo_div_mh = 0.5 * md_m_o / md_m_h;
        md_rc = 0.5 * p->dist_hh;
        md_ra = std::sqrt(p->dist_oh * p->dist_oh - md_rc * md_rc) / (1.0 + half_mo_div_mh);
        md_rb = half_mo_div_mh * md_ra;
    }
    md_ready = true;
    return GR_OK;
}

// Zeroes the kinetic-energy accumulator and launches one MD step kernel.
gr_status NbSystem::md_step_launch(cudaStream_t s, bool fuse_prep) {
    MdDev md;
    md.vel = md_vel;
    md.inv_mass = md_inv_mass;
    md.mass = md_mass;
    md.dt = mdp.dt;
    md.dt_i = 1.0 / mdp.dt;
    md.settle = md_settle ? 1 : 0;
    md.m_o = md_m_o;
    md.m_h = md_m_h;
    md.ra = md_ra;
    md.rb = md_rb;
    md.rc = md_rc;
    md.ke = md_ke;
    md.failures = md_fail;
    md.t0 = md_t0;
    md.tau = mdp.tau;
    md.dof = md_dof;
    // the next evaluation keeps this period's lists (no rebuild): its water
    // records come from this kernel
    md.prep_next = fuse_prep && md_settle && NCG > NSCG && h.wrec && !in_capture && built &&
                   steps_since_update < prm.nsnb;
    prepped_next = md.prep_next != 0;
    const int n_units = md_settle ? NSA + (N - NSA) / 3 : N;
    const unsigned grid = std::max(1u, std::min(unsigned((n_units + 255) / 256), unsigned(sm_count() * 8)));
    (++launches, k_md_step<<<grid, 256, 0, s>>>(d_sys, md));
    return GR_OK;
}

gr_status NbSystem::md_stats(cudaStream_t s, gr_md_stats* out) {
    long long ke = 0;
    int fails = 0;
    std::vector<double> e(acc_size(G));
    GR_CUDA(cudaMemcpyAsync(&ke, md_ke, sizeof(ke), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaMemcpyAsync(&fails, md_fail, sizeof(int), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaMemcpyAsync(e.data(), h.e_out, e.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaStreamSynchronize(s));
    double elj = 0.0, ecrf = 0.0;
    for (int g = 0; g < G * G; ++g) {
        elj += e[g];
        ecrf += e[G * G + g];
    }
    out->steps = md_steps_total;
    out->e_lj = elj;
    out->e_crf = ecrf;
    out->e_kin = double(ke) / kEnergyScale;
    out->settle_failures = fails;
    out->rollbacks = int(md_rollbacks);
    return GR_OK;
}

gr_status NbSystem::md_run(cudaStream_t s, int n_steps, gr_md_stats* out) {
    if (!md_ready) {
        set_error("gr_md_run before gr_md_init");
        return GR_ERR_STATE;
    }
    if (n_steps < 0) {
        set_error("gr_md_run: n_steps must be >= 0");
        return GR_ERR_INVALID;
    }
    const size_t bytes3 = size_t(N) * 3 * sizeof(double);
    // The error flags are sticky in device memory, so they are read once per
    // block of whole pairlist periods (one host synchronisation per block);
    // an overflow anywhere in the block rolls the whole block back.  Kernels
    // are launched one by one: the host runs ahead of the device, and the
    // recorded step graphs would add their per-step flag copy and timing
    // events (measured slower here).
    //
    // The rollback point of a block is its start when the block starts a
    // pairlist period.  A block that starts inside a period (the previous
    // call ended there) rolls back to that period's start, kept in md_psnap,
    // and replays the steps up to the block start: the lists are rebuilt at
    // the period's own first step, so the rebuild and long-range schedule is
    // that of a run without overflow, and (the sums being fixed point) the
    // replayed steps reproduce the block's starting state bit for bit.
    const int kblock = std::max(1, prm.nsnb) * 4;
    int done = 0, attempts = 0, rollbacks = 0;
    gr_status st;
    while (done < n_steps) {
        const int ssu0 = steps_since_update;
        const bool from_period = built && ssu0 < prm.nsnb && md_psnap_valid && md_step_idx - md_psnap_step == ssu0;
        GR_CUDA(cudaMemcpyAsync(md_pos_snap, from_period ? md_psnap_pos : h.pos, bytes3, cudaMemcpyDeviceToDevice, s));
        GR_CUDA(cudaMemcpyAsync(md_vel_snap, from_period ? md_psnap_vel : md_vel, bytes3, cudaMemcpyDeviceToDevice, s));
        GR_CUDA(cudaMemcpyAsync(md_ke_snap, from_period ? md_psnap_ke : md_ke, sizeof(long long),
                                cudaMemcpyDeviceToDevice, s));
        const long long idx0 = from_period ? md_psnap_step : md_step_idx;
        int replay = 0;  // steps re-run before the block's own steps (after a rollback)
        int k = 0;
        for (;;) {  // attempts at this block
            bool overflow = false;
            k = 0;
            for (int r = 0;;) {
                if (pending_check) {  // the flags of this period's rebuild
                    bool of = false;
                    if ((st = resolve_pending(&of))) return st;
                    if (of) {
                        overflow = true;
                        break;
                    }
                }
                if (!built || steps_since_update >= prm.nsnb) {  // this step starts a pairlist period
                    GR_CUDA(cudaMemcpyAsync(md_psnap_pos, h.pos, bytes3, cudaMemcpyDeviceToDevice, s));
                    GR_CUDA(cudaMemcpyAsync(md_psnap_vel, md_vel, bytes3, cudaMemcpyDeviceToDevice, s));
                    GR_CUDA(cudaMemcpyAsync(md_psnap_ke, md_ke, sizeof(long long), cudaMemcpyDeviceToDevice, s));
                    md_psnap_step = md_step_idx;
                    md_psnap_valid = true;
                }
                if ((st = eval(s, 0, false))) return st;
                if ((st = md_step_launch(s, true))) return st;
                ++md_step_idx;
                if (r < replay) {
                    ++r;
                    continue;
                }
                ++k;
                if (done + k >= n_steps || (steps_since_update >= prm.nsnb && k >= kblock)) break;
            }
            if (!overflow) {
                // everything of this block (builds and force kernels) has set its flags
                GR_CUDA(cudaMemcpyAsync(md_err_host, h.err, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
                GR_CUDA(cudaEventRecord(ev_md, s));
                GR_CUDA(cudaEventSynchronize(ev_md));
                const int* e = reinterpret_cast<const int*>(md_err_host);
                pending_check = false;  // a rebuild at the block's last step: its flags are in e[0] too
                if (e[0]) {
                    const int f = e[0];
                    GR_CUDA(cudaMemset(h.err, 0, 4 * sizeof(int)));
                    if (f & (ERR_CELL_TOO_DENSE | ERR_CG_TOO_LARGE)) {
                        set_error(f & ERR_CELL_TOO_DENSE ? "pairlist: a grid cell holds more than 2048 charge groups"
                                                         : "pairlist: solute charge group larger than 8 atoms");
                        return GR_ERR_UNSUPPORTED;
                    }
                    if (f & ERR_WLIST_OVERFLOW) wcap_want = std::max(wcap_want, wcap_alloc) * 2;
                    if (f & ERR_SLIST_OVERFLOW) scap_want = std::max(scap_want, scap_alloc) * 2;
                    if (f & ERR_PERT_OVERFLOW) pcap_want = std::max(pcap_want, pcap_alloc) * 2;
                    if (f & ERR_DEFER_OVERFLOW) {
                        defer_want = std::max(defer_want, h.defer_cap) * 4;
                        clus_alloc = 0;
                    }
                    overflow = true;
                }
            }
            if (!overflow) break;
            if (++attempts > 8) {
                set_error("md: list capacity could not be grown far enough");
                return GR_ERR_OVERFLOW;
            }
            GR_CUDA(cudaMemcpyAsync(h.pos, md_pos_snap, bytes3, cudaMemcpyDeviceToDevice, s));
            GR_CUDA(cudaMemcpyAsync(md_vel, md_vel_snap, bytes3, cudaMemcpyDeviceToDevice, s));
            GR_CUDA(cudaMemcpyAsync(md_ke, md_ke_snap, sizeof(long long), cudaMemcpyDeviceToDevice, s));
            prepped_next = false;
            md_step_idx = idx0;
            steps_since_update = prm.nsnb;
            built = false;  // the rollback point starts a period: rebuilt there with the grown lists
            lr_computed = false;
            replay = from_period ? ssu0 : 0;
            ++rollbacks;
        }
        attempts = 0;
        done += k;
    }
    md_steps_total += done;
    md_rollbacks += rollbacks;
    if (out) {
        if ((st = md_stats(s, out))) return st;
        out->steps = done;
        out->rollbacks = rollbacks;
    }
    return GR_OK;
}

extern "C" {

gr_status gr_md_init(gr_ctx* ctx, const double* mass, const double* vel, const gr_md_params* params) {
    CTX_GUARD(ctx);
    return ctx->sys.md_init(mass, vel, params);
}

gr_status gr_md_run(gr_ctx* ctx, int32_t n_steps, gr_md_stats* out) {
    CTX_GUARD(ctx);
    return ctx->sys.md_run(ctx->stream, n_steps, out);
}

gr_status gr_md_set_temperature(gr_ctx* ctx, double t0, int32_t rescale_velocities) {
    CTX_GUARD(ctx);
    NbSystem& S = ctx->sys;
    if (!S.md_ready) {
        set_error("gr_md_set_temperature before gr_md_init");
        return GR_ERR_STATE;
    }
    if (!(t0 > 0.0)) {
        set_error("gr_md_set_temperature: t0 must be positive");
        return GR_ERR_INVALID;
    }
    // the bath temperature lives in device memory (k_md_step reads it every
    // step): recorded step graphs stay valid, and the write is ordered after
    // the steps already enqueued on this context's stream
    GR_CUDA(cudaMemcpyAsync(S.md_t0, &t0, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (rescale_velocities) {
        // Replica::rescale_velocities (replica.rs:355-371): scale to t0 from the
        // instantaneous temperature over 3N degrees of freedom
        long long ke = 0;
        GR_CUDA(cudaMemcpyAsync(&ke, S.md_ke, sizeof(ke), cudaMemcpyDeviceToHost, ctx->stream));
        GR_CUDA(cudaStreamSynchronize(ctx->stream));
        const double t_now = 2.0 * (double(ke) / gnb::kEnergyScale) / (3.0 * S.N * 0.00831446261815324);
        if (!(t_now > 0.0)) {
            S.mdp.temperature = t0;
            GR_CUDA(cudaStreamSynchronize(ctx->stream));
            return GR_OK;
        }
        const double f = std::sqrt(t0 / t_now);
        const int n3 = 3 * S.N;
        (++S.launches, gnb::k_scale_velocities<<<std::max(1, std::min((n3 + 255) / 256, 1024)), 256, 0, ctx->stream>>>(
            S.md_vel, n3, f, S.md_ke));
        GR_CUDA(cudaGetLastError());
    }
    S.mdp.temperature = t0;
    // complete before returning: a batch launches its members' steps on its own stream
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_md_stats_get(gr_ctx* ctx, gr_md_stats* out) {
    CTX_GUARD(ctx);
    if (!ctx->sys.md_ready || !out) {
        set_error("gr_md_stats_get: MD not initialised or null out");
        return ctx->sys.md_ready ? GR_ERR_INVALID : GR_ERR_STATE;
    }
    return ctx->sys.md_stats(ctx->stream, out);
}

gr_status gr_md_download(gr_ctx* ctx, double* pos, double* vel) {
    CTX_GUARD(ctx);
    NbSystem& S = ctx->sys;
    if (!S.md_ready) {
        set_error("gr_md_download before gr_md_init");
        return GR_ERR_STATE;
    }
    const size_t bytes3 = size_t(S.N) * 3 * sizeof(double);
    if (pos) GR_CUDA(cudaMemcpyAsync(pos, S.h.pos, bytes3, cudaMemcpyDeviceToHost, ctx->stream));
    if (vel) GR_CUDA(cudaMemcpyAsync(vel, S.md_vel, bytes3, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

}  // extern "C"
