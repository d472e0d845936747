// api.cu -- host runtime and C ABI of libgromos_nb (include/gromos_nb.h).
//
// NbSystem owns one system's device state (topology, positions, pairlist,
// accumulators) and runs the per-step launch sequence that replaces
// gromos-rs Forcefield::apply's nonbonded part
// (crates/gromos-integrators/src/algorithms/forcefield.rs:226-1020):
//   rebuild (every NSNB calls) -> short range -> long range at rebuilds
//   (twin-range cache) -> RF excluded/self + 1-4 -> FEP corrections -> sum.
// gr_ctx wraps one NbSystem on its own stream; gr_batch (batch.cu) holds many.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gromos_nb.h"
#include "kernels.cuh"
#include "nb_system.h"

namespace gnb {

thread_local std::string g_last_error;

void set_error(const std::string& m) { g_last_error = m; }

#define GR_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
            return GR_ERR_CUDA;                                                               \
        }                                                                                     \
    } while (0)

// CRFParameters::new (crates/gromos-forces/src/nonbonded/params.rs:78-96).
void crf_params(double cutoff, double epsilon, double rf_epsilon, double rf_kappa, double out[4]) {
    double kappa_cut = rf_kappa * cutoff;
    double kappa_cut2 = kappa_cut * kappa_cut;
    double crf = (2.0 * (epsilon - rf_epsilon) * (1.0 + kappa_cut) - rf_epsilon * kappa_cut2) /
                 ((epsilon + 2.0 * rf_epsilon) * (1.0 + kappa_cut) + rf_epsilon * kappa_cut2);
    double cut3i = 1.0 / (cutoff * cutoff * cutoff);
    double crf_cut3i = crf * cut3i;
    out[0] = (1.0 - crf / 2.0) / cutoff;  // crf_cut
    out[1] = crf_cut3i / 2.0;             // crf_2cut3i
    out[2] = crf_cut3i;                   // crf_cut3i
    out[3] = cutoff * cutoff;             // cutoff_sq
}

// f64::powi by squaring, as Rust expands it.
static double powi(double a, int b) {
    bool recip = b < 0;
    unsigned e = recip ? unsigned(-b) : unsigned(b);
    double r = 1.0;
    while (true) {
        if (e & 1u) r *= a;
        e >>= 1;
        if (e == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// PerturbedLambdaParams::from_lambda(λ, λ, λ, λ, 1, 1, 1, 1, n)
// (perturbed.rs:57-101 called as in forcefield.rs:767-777).
void lambda_params(double lam, int n, double lp[17]) {
    lp[0] = powi(1.0 - lam, n);
    lp[1] = powi(lam, n);
    lp[2] = powi(1.0 - lam, n);
    lp[3] = powi(lam, n);
    lp[4] = powi(1.0 - lam, n - 1);
    lp[5] = powi(lam, n - 1);
    lp[6] = powi(1.0 - lam, n - 1);
    lp[7] = powi(lam, n - 1);
    lp[8] = 1.0 - lam;
    lp[9] = lam;
    lp[10] = (1.0 - lam) * (1.0 - lam);
    lp[11] = lam * lam;
    lp[12] = 1.0 - lam;
    lp[13] = lam;
    lp[14] = (1.0 - lam) * (1.0 - lam);
    lp[15] = lam * lam;
    lp[16] = double(n);
}

// Device memory of every context comes from one stream-ordered pool per GPU
// that keeps freed blocks for reuse: a context created after another was
// released (a serving job after a finished one) reuses that memory, and
// releasing a context synchronises only its own stream -- cudaFree would
// synchronise the whole device, stalling every other context's work.
cudaError_t device_pool(cudaMemPool_t* pool) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if ((e = cudaMemPoolCreate(&pools[dev], &props)) != cudaSuccess) {
            pools[dev] = nullptr;
            return e;
        }
        uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool until the process exits
        if ((e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
            return e;
    }
    *pool = pools[dev];
    return cudaSuccess;
}

// A pool allocation, complete before it returns (so any stream and synchronous
// copies may use it at once), and its release after the work on this
// context's stream.  Buffers are reallocated or released only when no other
// stream has work on them (batch steps synchronise before members change).
cudaError_t NbSystem::dev_malloc(void** p, size_t n) {
    cudaMemPool_t pool = nullptr;
    cudaError_t e = device_pool(&pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, n, pool, mem_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(mem_stream);
    return e;
}

void NbSystem::dev_free(void* p) {
    if (!p) return;
    cudaStreamSynchronize(mem_stream);
    cudaFreeAsync(p, mem_stream);
}

NbSystem::~NbSystem() { release(); }

void NbSystem::release() {
    const bool any = !allocs.empty() || d_sys;
    for (void* p : allocs) dev_free(p);
    allocs.clear();
    if (d_sys) dev_free(d_sys);
    d_sys = nullptr;
    if (any) cudaStreamSynchronize(mem_stream);  // the blocks are back in the pool before the stream goes
    std::memset(&h, 0, sizeof(h));
    d_cg_key = nullptr;
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ev) e = nullptr;
    for (auto& e : evk)
        if (e) cudaEventDestroy(e);
    for (auto& e : evk) e = nullptr;
    if (ev_err) cudaEventDestroy(ev_err);
    ev_err = nullptr;
    if (err_host) cudaFreeHost(err_host);
    err_host = nullptr;
    pending_check = false;
    drop_graphs();
    if (err_step_host) cudaFreeHost(err_step_host);
    err_step_host = nullptr;
    if (err_dl_host) cudaFreeHost(err_dl_host);
    err_dl_host = nullptr;
    if (e_dl_host) cudaFreeHost(e_dl_host);
    e_dl_host = nullptr;
    e_dl_n = 0;
    if (ev_step) cudaEventDestroy(ev_step);
    ev_step = nullptr;
    step_check = false;
    // MD buffers were freed with `allocs`
    md_vel = md_mass = md_inv_mass = md_pos_snap = md_vel_snap = nullptr;
    md_ke = nullptr;
    md_ke_snap = nullptr;
    md_t0 = nullptr;
    md_psnap_pos = md_psnap_vel = nullptr;
    md_psnap_ke = nullptr;
    md_psnap_valid = false;
    md_fail = nullptr;
    if (md_err_host) cudaFreeHost(md_err_host);
    md_err_host = nullptr;
    if (ev_md) cudaEventDestroy(ev_md);
    ev_md = nullptr;
    md_ready = false;
}

// (Re)allocates *p; a previous allocation made through alloc() is freed.
template <class T>
gr_status NbSystem::alloc(T** p, size_t n) {
    if (*p) {
        for (size_t k = 0; k < allocs.size(); ++k)
            if (allocs[k] == static_cast<void*>(*p)) {
                dev_free(*p);
                allocs.erase(allocs.begin() + long(k));
                break;
            }
        *p = nullptr;
    }
    if (n == 0) n = 1;
    cudaError_t e = dev_malloc(reinterpret_cast<void**>(p), n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(std::string("device allocation: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? GR_ERR_OOM : GR_ERR_CUDA;
    }
    allocs.push_back(*p);
    bytes += n * sizeof(T);
    ++alloc_gen;
    acc_clean = false;
    return GR_OK;
}

template <class T>
gr_status NbSystem::upload_array(T** p, const T* host, size_t n) {
    gr_status st = alloc(p, n);
    if (st) return st;
    if (n && host) {
        cudaError_t e = cudaMemcpy(*p, host, n * sizeof(T), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            set_error(std::string("cudaMemcpy: ") + cudaGetErrorString(e));
            return GR_ERR_CUDA;
        }
    }
    return GR_OK;
}

static gr_status validate(const gr_topology* t) {
    if (!t || t->n_atoms <= 0 || t->n_chargegroups <= 0 || !t->cg_offsets || !t->charge || !t->iac || !t->lj ||
        !t->excl_offsets || t->n_types <= 0) {
        set_error("gr_topology: missing arrays or empty system");
        return GR_ERR_INVALID;
    }
    if (t->cg_offsets[0] != 0 || t->cg_offsets[t->n_chargegroups] != t->n_atoms) {
        set_error("gr_topology: cg_offsets must start at 0 and end at n_atoms");
        return GR_ERR_INVALID;
    }
    for (int c = 0; c < t->n_chargegroups; ++c)
        if (t->cg_offsets[c + 1] <= t->cg_offsets[c]) {
            set_error("gr_topology: empty or unordered charge group");
            return GR_ERR_INVALID;
        }
    if (t->n_solute_chargegroups < 0 || t->n_solute_chargegroups > t->n_chargegroups ||
        t->cg_offsets[t->n_solute_chargegroups] != t->n_solute_atoms) {
        set_error("gr_topology: solute atoms must be exactly the solute charge groups");
        return GR_ERR_INVALID;
    }
    for (int a = 0; a < t->n_atoms; ++a)
        if (t->iac[a] < 0 || t->iac[a] >= t->n_types) {
            set_error("gr_topology: iac out of range");
            return GR_ERR_INVALID;
        }
    int G = t->n_energy_groups > 0 ? t->n_energy_groups : 1;
    if (G > kMaxGroups) {
        set_error("gr_topology: at most 16 energy groups");
        return GR_ERR_UNSUPPORTED;
    }
    if (t->energy_group)
        for (int a = 0; a < t->n_atoms; ++a)
            if (t->energy_group[a] < 0 || t->energy_group[a] >= G) {
                set_error("gr_topology: energy group id out of range");
                return GR_ERR_INVALID;
            }
    for (int c = 0; c < t->n_solute_chargegroups; ++c)
        if (t->cg_offsets[c + 1] - t->cg_offsets[c] > kMaxCGAtoms) {
            set_error("gr_topology: solute charge groups of more than 8 atoms are not supported");
            return GR_ERR_UNSUPPORTED;
        }
    int nsolv_cg = t->n_chargegroups - t->n_solute_chargegroups;
    if (nsolv_cg > 0) {
        if (t->atoms_per_solvent != 3) {
            set_error("gr_topology: solvent molecules must have 3 atoms (SPC-type water)");
            return GR_ERR_UNSUPPORTED;
        }
        for (int c = t->n_solute_chargegroups; c < t->n_chargegroups; ++c)
            if (t->cg_offsets[c + 1] - t->cg_offsets[c] != t->atoms_per_solvent) {
                set_error("gr_topology: every solvent charge group must be one molecule");
                return GR_ERR_INVALID;
            }
    }
    for (int k = 0; k < t->n_perturbed; ++k) {
        const gr_perturbed_atom& p = t->perturbed[k];
        if (p.atom < 0 || p.atom >= t->n_solute_atoms || p.a_iac < 0 || p.a_iac >= t->n_types || p.b_iac < 0 ||
            p.b_iac >= t->n_types) {
            set_error("gr_topology: perturbed atom must be a solute atom with valid IACs");
            return GR_ERR_INVALID;
        }
    }
    return GR_OK;
}

gr_status NbSystem::upload(const gr_topology* t) {
    gr_status st = validate(t);
    if (st) return st;
    prepped_next = false;
    release();
    bytes = 0;
    N = t->n_atoms;
    NCG = t->n_chargegroups;
    NSCG = t->n_solute_chargegroups;
    NSA = t->n_solute_atoms;
    NT = t->n_types;
    G = t->n_energy_groups > 0 ? t->n_energy_groups : 1;
    aps = t->atoms_per_solvent;
    fpe = t->four_pi_eps_i;
    h_cg_off.assign(t->cg_offsets, t->cg_offsets + NCG + 1);
    h_excl_off.assign(t->excl_offsets, t->excl_offsets + N + 1);
    h_excl.assign(t->excl, t->excl + h_excl_off[N]);
    if (t->o14_offsets) {
        h_o14_off.assign(t->o14_offsets, t->o14_offsets + N + 1);
        h_o14.assign(t->o14, t->o14 + h_o14_off[N]);
    } else {
        h_o14_off.assign(N + 1, 0);
        h_o14.clear();
    }
    h_egroup.assign(N, 0);
    if (t->energy_group) h_egroup.assign(t->energy_group, t->energy_group + N);
    // solvent energy group (the water kernel attributes to one group pair)
    solvent_group = -1;
    if (NSA < N) {
        solvent_group = h_egroup[NSA];
        for (int a = NSA; a < N; ++a)
            if (h_egroup[a] != solvent_group) {
                set_error("gr_topology: all solvent atoms must be in one energy group");
                return GR_ERR_UNSUPPORTED;
            }
    }
    std::vector<float2> lj32(size_t(NT) * NT);
    for (size_t k = 0; k < lj32.size(); ++k) lj32[k] = make_float2(float(t->lj[4 * k]), float(t->lj[4 * k + 1]));
    std::vector<int> atom_cg(N);
    for (int c = 0; c < NCG; ++c)
        for (int a = h_cg_off[c]; a < h_cg_off[c + 1]; ++a) atom_cg[a] = c;
    // perturbation
    std::vector<int> pidx(N, -1), piac, pp;
    std::vector<double> pq, palpha;
    for (int k = 0; k < t->n_perturbed; ++k) {
        const gr_perturbed_atom& p = t->perturbed[k];
        pidx[p.atom] = k;
        piac.push_back(p.a_iac);
        piac.push_back(p.b_iac);
        pq.push_back(p.a_charge);
        pq.push_back(p.b_charge);
        palpha.push_back(p.alpha_lj);
        palpha.push_back(p.alpha_crf);
    }
    for (int k = 0; k < t->n_perturbed_pairs; ++k) {
        const gr_perturbed_pair& p = t->perturbed_pairs[k];
        pp.insert(pp.end(), {p.i, p.j, p.a_type, p.b_type});
    }
    n_pert = t->n_perturbed;
    std::memset(&h, 0, sizeof(h));
    h.n_atoms = N;
    h.n_cg = NCG;
    h.n_solute_cg = NSCG;
    h.n_solute_atoms = NSA;
    h.aps = aps;
    h.n_types = NT;
    h.n_egroups = G;
    h.fpe = fpe;
    h.solvent_group = solvent_group;
    h.has_pert = n_pert > 0;
    h.n_pert = n_pert;
    h.n_pp = t->n_perturbed_pairs;
    int* cg_off = nullptr;
    double* charge = nullptr;
    int* iac = nullptr;
    double* lj64 = nullptr;
    float2* lj32d = nullptr;
    int *excl_off = nullptr, *excl = nullptr, *o14_off = nullptr, *o14 = nullptr, *eg = nullptr, *acg = nullptr;
    int *pidx_d = nullptr, *piac_d = nullptr, *pp_d = nullptr;
    double *pq_d = nullptr, *pa_d = nullptr;
    if ((st = upload_array(&cg_off, h_cg_off.data(), h_cg_off.size()))) return st;
    if ((st = upload_array(&charge, t->charge, size_t(N)))) return st;
    if ((st = upload_array(&iac, t->iac, size_t(N)))) return st;
    if ((st = upload_array(&lj64, t->lj, size_t(NT) * NT * 4))) return st;
    if ((st = upload_array(&lj32d, lj32.data(), lj32.size()))) return st;
    if ((st = upload_array(&excl_off, h_excl_off.data(), h_excl_off.size()))) return st;
    if ((st = upload_array(&excl, h_excl.data(), h_excl.size()))) return st;
    if ((st = upload_array(&o14_off, h_o14_off.data(), h_o14_off.size()))) return st;
    if ((st = upload_array(&o14, h_o14.data(), h_o14.size()))) return st;
    if ((st = upload_array(&eg, h_egroup.data(), h_egroup.size()))) return st;
    if ((st = upload_array(&acg, atom_cg.data(), atom_cg.size()))) return st;
    if ((st = upload_array(&pidx_d, pidx.data(), pidx.size()))) return st;
    if ((st = upload_array(&piac_d, piac.data(), piac.size()))) return st;
    if ((st = upload_array(&pq_d, pq.data(), pq.size()))) return st;
    if ((st = upload_array(&pa_d, palpha.data(), palpha.size()))) return st;
    if ((st = upload_array(&pp_d, pp.data(), pp.size()))) return st;
    h.cg_off = cg_off;
    h.charge = charge;
    h.iac = iac;
    h.lj64 = lj64;
    h.lj32 = lj32d;
    h.excl_off = excl_off;
    h.excl = excl;
    h.o14_off = o14_off;
    h.o14 = o14;
    h.egroup = eg;
    h.atom_cg = acg;
    h.pert_idx = pidx_d;
    h.pert_iac = piac_d;
    h.pert_q = pq_d;
    h.pert_alpha = pa_d;
    h.pp = pp_d;
    // solvent exclusions exactly the other atoms of the molecule and no 1-4
    // pairs (Topology::solvate, topology.rs:1240-1262): then the energy-only
    // solvent excluded terms are computed with the per-step water data
    solvent_excl_intra = NSA < N;
    for (int c = NSCG; c < NCG && solvent_excl_intra; ++c)
        for (int a = h_cg_off[c]; a < h_cg_off[c + 1] && solvent_excl_intra; ++a) {
            int k = h_excl_off[a];
            for (int b = h_cg_off[c]; b < h_cg_off[c + 1]; ++b) {
                if (b == a) continue;
                if (k >= h_excl_off[a + 1] || h_excl[k] != b) {
                    solvent_excl_intra = false;
                    break;
                }
                ++k;
            }
            if (k != h_excl_off[a + 1] || h_o14_off[a + 1] != h_o14_off[a]) solvent_excl_intra = false;
        }
    h.excl_atoms = solvent_excl_intra ? NSA : N;
    // solvent parameter table from the first solvent molecule (innerloops.rs:241-255)
    h.water_lj00_only = 1;
    if (NSA < N) {
        int f = NSA;
        for (int a = 0; a < aps; ++a)
            for (int b = 0; b < aps; ++b) {
                const double* lj = t->lj + 4 * (size_t(t->iac[f + a]) * NT + t->iac[f + b]);
                h.w_c6[a * 4 + b] = float(lj[0]);
                h.w_c12[a * 4 + b] = float(lj[1]);
                h.w_qq[a * 4 + b] = float(t->charge[f + a] * t->charge[f + b] * fpe);
                if ((a || b) && (lj[0] != 0.0 || lj[1] != 0.0)) h.water_lj00_only = 0;
            }
        double qs = 0.0;  // sum of the charges of one solvent molecule (zero for a neutral one)
        for (int a = 0; a < aps; ++a) qs += t->charge[f + a];
        w_qq_sum = qs * qs * fpe;
    }
    if ((st = alloc(&h.pos, size_t(N) * 3))) return st;
    if ((st = alloc(&h.ref, size_t(NCG) * 3))) return st;
    if ((st = alloc(&h.keys, size_t(NCG)))) return st;
    if ((st = alloc(&d_cg_key, size_t(NCG)))) return st;
    if ((st = alloc(&h.build_ctr, 4))) return st;
    GR_CUDA(cudaMemset(h.build_ctr, 0, 4 * sizeof(int)));  // each last block leaves its counter at zero
    if ((st = alloc(&h.cg_cell, size_t(NCG)))) return st;
    if ((st = alloc(&h.sorted_cg, size_t(NCG)))) return st;
    if ((st = alloc(&h.sref, 3 * (size_t(NCG) + 2)))) return st;
    if ((st = alloc(&h.cg_spos, size_t(NCG)))) return st;
    if ((st = alloc(&h.cg_slot, size_t(NCG)))) return st;
    if ((st = alloc(&h.n_clusters, 1))) return st;
    if ((st = alloc(&h.sn, size_t(std::max(NSCG, 1))))) return st;
    if ((st = alloc(&h.n_pert_pairs, 1))) return st;
    if ((st = alloc(&h.n_cgp, 2))) return st;
    if ((st = alloc(&h.pos32, size_t(N)))) return st;
    if ((st = alloc(&h.f32, size_t(N) * 3))) return st;
    if ((st = alloc(&h.f32_long, size_t(N) * 3))) return st;
    if ((st = alloc(&h.e64, 16))) return st;
    if ((st = alloc(&h.e64_long, 16))) return st;
    if ((st = alloc(&h.f_short, size_t(N) * 3))) return st;
    if ((st = alloc(&h.f_long, size_t(N) * 3))) return st;
    if ((st = alloc(&h.acc_short, size_t(acc_size(G))))) return st;
    if ((st = alloc(&h.acc_long, size_t(acc_size(G))))) return st;
    if ((st = alloc(&h.f_out, size_t(N) * 3))) return st;
    if ((st = alloc(&h.e_out, size_t(acc_size(G))))) return st;
    if ((st = alloc(&h.err, 4))) return st;
    if ((st = alloc(&h.n_deferred, 8))) return st;  // deferred counts [2], water work counters [2], blocks done [2], search counter
    if ((st = alloc(&h.max_delta, 1))) return st;
    GR_CUDA(cudaMemset(h.err, 0, 4 * sizeof(int)));
    GR_CUDA(cudaMemset(h.f_long, 0, size_t(N) * 3 * sizeof(long long)));
    GR_CUDA(cudaMemset(h.acc_long, 0, size_t(acc_size(G)) * sizeof(long long)));
    GR_CUDA(cudaMemset(h.f32_long, 0, size_t(N) * 3 * sizeof(float)));
    GR_CUDA(cudaMemset(h.e64_long, 0, 16 * sizeof(double)));
    GR_CUDA(dev_malloc(reinterpret_cast<void**>(&d_sys), sizeof(SysDev)));
    for (auto& e : ev) GR_CUDA(cudaEventCreate(&e));
    for (auto& e : evk) GR_CUDA(cudaEventCreate(&e));
    GR_CUDA(cudaEventCreateWithFlags(&ev_err, cudaEventDisableTiming));
    if (!err_host) GR_CUDA(cudaMallocHost(reinterpret_cast<void**>(&err_host), 4 * sizeof(int)));
    err_host[0] = 0;
    pending_check = false;
    ever_built = false;
    // list capacities are sized at the first build (need the box)
    cells_alloc = 0;
    clus_alloc = 0;
    wcap_alloc = 0;
    scap_alloc = 0;
    pcap_alloc = 0;
    cgp_alloc = 0;
    uploaded = true;
    built = false;
    lr_computed = false;
    steps_since_update = 0;
    return GR_OK;
}

gr_status NbSystem::set_params(const gr_nb_params* p) {
    prepped_next = false;  // the records' excluded energies depend on the parameters
    if (!p || p->rcutp <= 0 || p->rcutl < p->rcutp || p->skin < 0 || p->nsnb <= 0) {
        set_error("gr_nb_params: need 0 < rcutp <= rcutl, skin >= 0, nsnb >= 1");
        return GR_ERR_INVALID;
    }
    if (p->boundary != 0 && p->boundary != 1) {
        set_error("gr_nb_params: boundary must be 0 (vacuum) or 1 (rectangular)");
        return GR_ERR_UNSUPPORTED;
    }
    if (p->kernel != GR_KERNEL_FIXED && p->kernel != GR_KERNEL_PLAIN) {
        set_error("gr_nb_params: unknown kernel");
        return GR_ERR_INVALID;
    }
    if (p->cluster_size != 0 && p->cluster_size != 4 && p->cluster_size != 8) {
        set_error("gr_nb_params: cluster_size must be 0, 4 or 8");
        return GR_ERR_INVALID;
    }
    if (p->water_layout == 1 && p->cluster_size == 8) {
        set_error("gr_nb_params: the shared-bit layout supports cluster_size 4 only");
        return GR_ERR_INVALID;
    }
    if (p->water_layout == 3 && p->cluster_size == 8) {
        set_error("gr_nb_params: the pair-stream layout supports cluster_size 4 only");
        return GR_ERR_INVALID;
    }
    if (p->water_layout < 0 || p->water_layout > 4) {
        set_error("gr_nb_params: water_layout must be 0, 1, 2, 3 or 4");
        return GR_ERR_INVALID;
    }
    if (p->list_capacity < 0) {
        set_error("gr_nb_params: list_capacity must be >= 0");
        return GR_ERR_INVALID;
    }
    if (params_set) {
        // a change of list_capacity alone only re-sizes the list storage at the
        // next rebuild: the current lists and the rebuild schedule stay
        const gr_nb_params& o = prm;
        const bool same = p->rcutp == o.rcutp && p->rcutl == o.rcutl && p->skin == o.skin &&
                          p->epsilon == o.epsilon && p->epsrf == o.epsrf && p->kappa == o.kappa &&
                          p->nsnb == o.nsnb && p->boundary == o.boundary && p->lambda == o.lambda &&
                          p->nlam == o.nlam && p->kernel == o.kernel && p->cluster_size == o.cluster_size &&
                          p->water_layout == o.water_layout;
        if (same) {
            if (p->list_capacity != prm.list_capacity) relist = true;
            prm.list_capacity = p->list_capacity;
            return GR_OK;
        }
    }
    prm = *p;
    // water kernel layout: 1 = lanes share the mask bits (width 4 only),
    // 2 = each lane iterates over its own bits (width 4 or 8), 3 = each lane
    // streams its own water pairs over units of two clusters (width 4; short
    // range, the long range runs layout 2), 4 = layout 2 with the atom pairs
    // evaluated two at a time in packed FP32x2 arithmetic (width 4 or 8)
    layout = p->water_layout == 1 ? 1 : p->water_layout == 3 ? 3 : p->water_layout == 4 ? 4 : 2;
    W = ((layout == 2 || layout == 4) && p->cluster_size == 8) ? 8 : 4;
    h.W = W;
    clus_alloc = 0;  // cluster arrays depend on W
    wcap_want = 0;   // list capacity from the (new) parameters
    h.boundary = p->boundary;
    h.twin = p->rcutp < p->rcutl - 1e-10 ? 1 : 0;  // forcefield.rs:126
    double rs = p->rcutp + p->skin, rl = p->rcutl + p->skin;
    h.c2s = rs * rs;
    h.c2l = rl * rl;
    double c[4];
    crf_params(p->rcutl, p->epsilon, p->epsrf, p->kappa, c);  // md.rs:815: cutoff = RCUTL
    h.crf_cut = c[0];
    h.crf_2cut3i = c[1];
    h.crf_cut3i = c[2];
    h.cutoff_sq = c[3];
    h.crf_cut_f = float(c[0]);
    h.crf_2cut3i_f = float(c[1]);
    h.crf_cut3i_f = float(c[2]);
    lambda_params(p->lambda, p->nlam, h.lp);
    params_set = true;
    built = false;
    lr_computed = false;
    warm = false;
    if (box_set) {  // the cell grid depends on the cutoffs
        const double b[3] = {h.box[0], h.box[1], h.box[2]};
        return set_box(b);
    }
    return GR_OK;
}

gr_status NbSystem::set_box(const double box[3]) {
    prepped_next = false;
    if (prm.boundary == 1 && (!(box[0] > 0) || !(box[1] > 0) || !(box[2] > 0))) {
        set_error("gr_set_box: rectangular box edges must be positive");
        return GR_ERR_INVALID;
    }
    for (int k = 0; k < 3; ++k) {
        h.box[k] = box[k];
        h.inv_box[k] = prm.boundary == 1 ? 1.0 / box[k] : 0.0;
        h.boxf[k] = float(box[k]);
        h.inv_boxf[k] = float(h.inv_box[k]);
        h.half_boxf[k] = float(box[k] * 0.5);
    }
    // use_cg_grouped_solute (forcefield.rs:267-283)
    if (prm.boundary == 0)
        h.cg_grouped = 1;
    else {
        double half_min = std::min(std::min(box[0], box[1]), box[2]) * 0.5;
        h.cg_grouped = half_min > prm.rcutl + prm.skin + 0.3 ? 1 : 0;
    }
    // cell grid: each cell strictly wider than rcutl + skin, so every pair
    // within the cutoff lies in the same or an adjacent cell
    double minc = (prm.rcutl + prm.skin) * (1.0 + 1e-7) + 1e-12;
    for (int k = 0; k < 3; ++k) {
        double g = 1.0;
        if (prm.boundary == 1) g = std::max(1.0, std::min(std::floor(box[k] / minc), double(1 << 20)));
        h.gdim[k] = int(g);
    }
    // a sparse box far larger than the cutoff: coarser cells (still wider than
    // the cutoff, so the lists are the same) keep the cell count in range
    while (static_cast<long long>(h.gdim[0]) * h.gdim[1] * h.gdim[2] > (1LL << 24)) {
        const int k = (h.gdim[0] >= h.gdim[1] && h.gdim[0] >= h.gdim[2]) ? 0 : (h.gdim[1] >= h.gdim[2] ? 1 : 2);
        h.gdim[k] = (h.gdim[k] + 1) / 2;
    }
    for (int k = 0; k < 3; ++k) h.cell_size[k] = prm.boundary == 1 ? box[k] / double(h.gdim[k]) : 1.0;
    // columns of about 0.5 nm (the edge of the volume of four waters) order
    // the CGs inside a cell, so that W consecutive solvent CGs are compact
    for (int k = 0; k < 2; ++k) h.ncol[k] = std::max(1, std::min(4, int(h.cell_size[k] / 0.5 + 0.5)));
    h.n_cells = h.gdim[0] * h.gdim[1] * h.gdim[2];
    box_set = true;
    return GR_OK;
}

gr_status NbSystem::ensure_capacity() {
    gr_status st;
    if (h.n_cells > cells_alloc) {
        int n = h.n_cells;
        if ((st = alloc(&h.cell_count, size_t(n)))) return st;
        GR_CUDA(cudaMemset(h.cell_count, 0, size_t(n) * sizeof(int)));  // k_refpos clears it after use
        if ((st = alloc(&h.cell_fill, size_t(n)))) return st;
        GR_CUDA(cudaMemset(h.cell_fill, 0, size_t(n) * sizeof(int)));  // likewise
        if ((st = alloc(&h.cell_start, size_t(n) + 1))) return st;
        if ((st = alloc(&h.cell_nsolute, size_t(n)))) return st;
        if ((st = alloc(&h.cell_nclus, size_t(n) + 1))) return st;
        if ((st = alloc(&h.cell_cand, 2 * size_t(n)))) return st;
        if ((st = alloc(&h.cell_ncand, 2 * size_t(n)))) return st;
        cells_alloc = n;
    }
    int nsolv = NCG - NSCG;
    int maxc = nsolv / W + h.n_cells + 1;
    // solvent list entries pack (j slot << 8 | i mask) into 32 bits
    if (static_cast<long long>(maxc) * W > (1LL << 24)) {
        set_error("pairlist: more than 2^24 solvent cluster slots (about 16.7 M solvent molecules)");
        return GR_ERR_UNSUPPORTED;
    }
    if (maxc > clus_alloc) {
        if ((st = alloc(&h.clus_cell, size_t(maxc)))) return st;
        if ((st = alloc(&h.clus_first, size_t(maxc)))) return st;
        if ((st = alloc(&h.clus_n, size_t(maxc)))) return st;
        if ((st = alloc(&h.slot_cg, size_t(maxc) * W))) return st;
        if ((st = alloc(&h.clus_geo, size_t(maxc)))) return st;
        if ((st = alloc(&h.clus_ext, size_t(maxc)))) return st;
        // each cluster is a candidate in both lists of its own cell and in one
        // list of each of its at most 26 neighbour cells
        h.cand_cap = int(std::min<long long>(28LL * maxc, (1LL << 31) - 1));
        if ((st = alloc(&h.cand_geo, size_t(h.cand_cap)))) return st;
        if ((st = alloc(&h.cand_ext, size_t(h.cand_cap)))) return st;
        if ((st = alloc(&h.clus_x64, size_t(maxc) * 4))) return st;
        if ((st = alloc(&h.slot_off, size_t(maxc) * W))) return st;
        if ((st = alloc(&h.wn_s, size_t(maxc)))) return st;
        if ((st = alloc(&h.wn_l, size_t(maxc)))) return st;
        if ((st = alloc(&h.wrec, size_t(maxc) * W))) return st;
        // pairs near half a box edge are few unless the box is small for the cutoff
        {
            double half_min = std::min(std::min(h.box[0], h.box[1]), h.box[2]) * 0.5;
            int per = (prm.rcutl + prm.skin + 0.3 > half_min) ? 64 : 4;
            h.defer_cap = std::max(4096, std::max(defer_want, (NCG - NSCG) * per));
        }
        if ((st = alloc(&h.deferred, size_t(4) * h.defer_cap))) return st;
        if ((st = alloc(&h.fs_short, size_t(maxc) * W * 9))) return st;
        if ((st = alloc(&h.fs_long, size_t(maxc) * W * 9))) return st;
        fs_long_zeroed = false;
        clus_alloc = maxc;
        wcap_alloc = 0;  // lists must be re-sized with the cluster count
    }
    h.max_clusters = clus_alloc;
    // entries per cluster: at most every solvent CG of the 27 neighbour cells
    double per_cell = double(NCG) / double(h.n_cells);
    int want_w = wcap_want ? wcap_want
                           : (prm.list_capacity > 0 ? prm.list_capacity
                                                    : int(std::min<double>(nsolv, per_cell * 27.0 * 1.25 + 64.0)));
    want_w = std::max(want_w, 32);
    if (want_w > wcap_alloc) {
        if ((st = alloc(&h.wl_s, size_t(clus_alloc) * want_w))) return st;
        if ((st = alloc(&h.wl_l, size_t(clus_alloc) * want_w))) return st;
        wcap_alloc = want_w;
    }
    h.wcap = wcap_alloc;
    int want_s = scap_want ? scap_want : int(std::min<double>(NCG + 1, per_cell * 27.0 * 1.25 + 64.0));
    if (NSCG > 0 && want_s > scap_alloc) {
        if ((st = alloc(&h.sl, size_t(NSCG) * want_s))) return st;
        if ((st = alloc(&h.sl_excl, size_t(NSCG) * want_s))) return st;
        scap_alloc = want_s;
    }
    h.scap = std::max(scap_alloc, 1);
    if (n_pert > 0) {
        int want_p = pcap_want ? pcap_want : n_pert * 8 * 2048 + 1024;
        if (want_p > pcap_alloc) {
            if ((st = alloc(&h.pert_pairs, size_t(want_p) * 3))) return st;
            pcap_alloc = want_p;
        }
    }
    h.pcap = pcap_alloc;
    return GR_OK;
}

gr_status NbSystem::ensure_cgp_capacity() {
    gr_status st;
    // CG pairs within rcutl + skin: half the CGs of a sphere per CG, plus slack
    double rl = prm.rcutl + prm.skin;
    double per_cg = double(NCG);
    if (prm.boundary == 1) {
        double vol = h.box[0] * h.box[1] * h.box[2];
        per_cg = std::min(double(NCG), NCG / vol * 4.18879 * rl * rl * rl * 0.75 + 64.0);
    }
    long long want = cgp_want ? cgp_want : (long long)(double(NCG) * per_cg) + 1024;
    want = std::min<long long>(want, (long long)2000000000);
    if (want > cgp_alloc) {
        if ((st = alloc(&h.cgp, size_t(want) * 3))) return st;
        if ((st = alloc(&h.cgp_excl, size_t(want)))) return st;
        cgp_alloc = int(want);
    }
    h.cgp_cap = cgp_alloc;
    return GR_OK;
}

// Events the host waits on or times: while a graph is being recorded they
// become event-record nodes of the graph (external records), so replays
// record them like a plain launch sequence would.
cudaError_t NbSystem::record_event(cudaEvent_t e, cudaStream_t s) {
    return in_capture ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
}

gr_status NbSystem::push_descriptor(cudaStream_t s) {
    if (in_capture) return GR_OK;
    GR_CUDA(cudaMemcpyAsync(d_sys, &h, sizeof(SysDev), cudaMemcpyHostToDevice, s));
    return GR_OK;
}

static inline unsigned blocks_for(long long n, int t) { return unsigned((n + t - 1) / t); }

gr_status NbSystem::check_errors(cudaStream_t s, bool* retry) {
    int err[4];
    GR_CUDA(cudaMemcpyAsync(err, h.err, sizeof(err), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaStreamSynchronize(s));
    *retry = false;
    if (err[0] == 0) return GR_OK;
    GR_CUDA(cudaMemset(h.err, 0, 4 * sizeof(int)));
    if (err[0] & ERR_CELL_TOO_DENSE) {
        set_error("pairlist: a grid cell holds more than 2048 charge groups");
        return GR_ERR_UNSUPPORTED;
    }
    if (err[0] & ERR_CG_TOO_LARGE) {
        set_error("pairlist: solute charge group larger than 8 atoms");
        return GR_ERR_UNSUPPORTED;
    }
    if (++regrow_count > 8) {
        set_error("pairlist: list capacity could not be grown far enough");
        return GR_ERR_OVERFLOW;
    }
    if (err[0] & ERR_WLIST_OVERFLOW) wcap_want = std::max(wcap_want, wcap_alloc) * 2;
    if (err[0] & ERR_SLIST_OVERFLOW) scap_want = std::max(scap_want, scap_alloc) * 2;
    if (err[0] & ERR_PERT_OVERFLOW) pcap_want = std::max(pcap_want, pcap_alloc) * 2;
    if (err[0] & ERR_CGPAIR_OVERFLOW) cgp_want = (long long)std::max<long long>(cgp_want, cgp_alloc) * 2;
    *retry = true;
    return GR_OK;
}

// Reads the overflow flags of the last asynchronous rebuild.  On overflow the
// list capacities are grown and the next evaluation rebuilds; *overflowed
// tells the caller that the evaluation based on that rebuild is invalid.
gr_status NbSystem::resolve_pending(bool* overflowed) {
    *overflowed = false;
    if (!pending_check) return GR_OK;
    GR_CUDA(cudaEventSynchronize(ev_err));
    pending_check = false;
    if (err_host[0] == 0) return GR_OK;
    const int e = err_host[0];
    GR_CUDA(cudaMemset(h.err, 0, 4 * sizeof(int)));
    if (e & ERR_CELL_TOO_DENSE) {
        set_error("pairlist: a grid cell holds more than 2048 charge groups");
        return GR_ERR_UNSUPPORTED;
    }
    if (e & ERR_CG_TOO_LARGE) {
        set_error("pairlist: solute charge group larger than 8 atoms");
        return GR_ERR_UNSUPPORTED;
    }
    if (e & ERR_WLIST_OVERFLOW) wcap_want = std::max(wcap_want, wcap_alloc) * 2;
    if (e & ERR_SLIST_OVERFLOW) scap_want = std::max(scap_want, scap_alloc) * 2;
    if (e & ERR_PERT_OVERFLOW) pcap_want = std::max(pcap_want, pcap_alloc) * 2;
    built = false;  // the next evaluation rebuilds with the grown capacities
    *overflowed = true;
    return GR_OK;
}

// PairlistAlgorithm::update (pairlist.rs:828-839) on the device.
gr_status NbSystem::build_pairlist(cudaStream_t s, bool sync) {
    if (!uploaded || !params_set || !box_set) {
        set_error("pairlist build before gr_system_upload / gr_set_params / gr_set_box");
        return GR_ERR_STATE;
    }
    regrow_count = 0;
    if (relist) {  // list storage sized afresh from the requested capacity
        wcap_alloc = 0;
        wcap_want = 0;
        relist = false;
    }
    for (;;) {
        gr_status st = ensure_capacity();
        if (st) return st;
        if ((st = push_descriptor(s))) return st;
        (++launches, k_refpos<<<blocks_for(NCG, 256), 256, 0, s>>>(d_sys, d_cg_key));
        (++launches, k_scatter<<<blocks_for(NCG, 256), 256, 0, s>>>(d_sys, d_cg_key));
        (++launches, k_cell_sort<<<h.n_cells, 256, 0, s>>>(d_sys));
        (++launches, k_cluster_setup<<<h.n_cells, 128, 0, s>>>(d_sys));
        if (NCG > NSCG) {
            (++launches, k_cell_candidates<<<dim3(h.n_cells, 2), 256, 0, s>>>(d_sys));
            SearchParams P;
            for (int k = 0; k < 3; ++k) {
                P.box[k] = h.box[k];
                P.inv_box[k] = h.inv_box[k];
                P.boxf[k] = h.boxf[k];
                P.inv_boxf[k] = h.inv_boxf[k];
                P.half_boxf[k] = h.half_boxf[k];
            }
            P.c2s = h.c2s;
            P.c2l = h.c2l;
            P.boundary = h.boundary;
            P.wcap = h.wcap;
            // persistent: one wave of blocks (SMs x resident blocks per SM),
            // fewer for a small system; warps draw clusters from a counter
            const long long need = (static_cast<long long>(h.max_clusters) + kSearchWarps - 1) / kSearchWarps;
            auto search_grid = [&](int occ) {
                return unsigned(std::max<long long>(1, std::min<long long>(static_cast<long long>(sm_count()) * occ, need)));
            };
#define GR_WATER_SEARCH(WW, POP)                                                                            \
    do {                                                                                                    \
        int occ = 1;                                                                                        \
        GR_CUDA(occupancy(k_water_search<WW, POP>, kSearchWarps * 32, 0, &occ));                            \
        (++launches, k_water_search<WW, POP><<<search_grid(occ), kSearchWarps * 32, 0, s>>>(d_sys, P));     \
    } while (0)
            if (layout == 1)
                GR_WATER_SEARCH(4, false);
            else if (W == 4)
                GR_WATER_SEARCH(4, true);
            else
                GR_WATER_SEARCH(8, true);
#undef GR_WATER_SEARCH
        }
        if (NSCG > 0) (++launches, k_solute_search<<<blocks_for(NSCG, 4), 128, 0, s>>>(d_sys));
        if (n_pert > 0 && NSCG > 0) {
            GR_CUDA(cudaMemsetAsync(h.n_pert_pairs, 0, sizeof(int), s));
            (++launches, k_pert_pairs<<<blocks_for((long long)NSCG * h.scap, 256), 256, 0, s>>>(d_sys));
        }
        GR_CUDA(cudaGetLastError());
        if (!sync) {
            // overflow flags are read back asynchronously and resolved by the next
            // call that synchronises (resolve_pending)
            GR_CUDA(cudaMemcpyAsync(err_host, h.err, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
            GR_CUDA(record_event(ev_err, s));
            pending_check = true;
            break;
        }
        bool retry = false;
        if ((st = check_errors(s, &retry))) return st;
        if (!retry) break;
    }
    built = true;
    cgp_valid = false;
    steps_since_update = 0;
    return GR_OK;
}

gr_status NbSystem::expand_cg_pairs(cudaStream_t s) {
    regrow_count = 0;
    for (;;) {
        gr_status st = ensure_cgp_capacity();
        if (st) return st;
        if ((st = push_descriptor(s))) return st;
        GR_CUDA(cudaMemsetAsync(h.n_cgp, 0, 2 * sizeof(int), s));
        long long nthreads = (long long)h.max_clusters * h.wcap + (long long)std::max(NSCG, 0) * h.scap;
        for (int lr = 0; lr < 2; ++lr) (++launches, k_expand_cgpairs<<<blocks_for(nthreads, 256), 256, 0, s>>>(d_sys, lr));
        GR_CUDA(cudaGetLastError());
        bool retry = false;
        if ((st = check_errors(s, &retry))) return st;
        if (!retry) break;
    }
    int n[2];
    GR_CUDA(cudaMemcpyAsync(n, h.n_cgp, sizeof(n), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaStreamSynchronize(s));
    if ((long long)n[0] + n[1] > cgp_alloc) {
        cgp_want = (long long)(n[0] + n[1]) * 2;
        return expand_cg_pairs(s);
    }
    n_cgp_host[0] = n[0];
    n_cgp_host[1] = n[1];
    cgp_valid = true;
    return GR_OK;
}

// One Forcefield::apply, nonbonded part.
gr_status NbSystem::eval(cudaStream_t s, int flags, bool record_events) {
    if (!uploaded || !params_set || !box_set || !pos_set) {
        set_error("gr_forces_eval before topology, parameters, box and positions are set");
        return GR_ERR_STATE;
    }
    gr_status st;
    bool overflowed = false;
    if ((st = resolve_pending(&overflowed))) return st;
    if (overflowed) lr_computed = false;
    bool rebuild = !built || steps_since_update >= prm.nsnb || (flags & GR_EVAL_FORCE_REBUILD);
    // the previous MD step wrote the water records of these positions (the
    // lists, and so the slots, are kept); a recorded graph always holds the prep
    const bool prepped = prepped_next && !rebuild && !in_capture;
    prepped_next = false;
    // stage timing events are recorded kernel by kernel only: inside a recorded
    // graph each event node adds its own latency to the step, so a graph holds
    // just the first and last (the step's total device time)
    const bool stage = record_events && !in_capture;
    if (stage) last_staged = true;
    if (stage) {
        evk_valid = prm.kernel == GR_KERNEL_FIXED && NCG > NSCG;
        evk_long = false;
    }
    if (record_events) GR_CUDA(record_event(ev[0], s));
    if (rebuild) {
        // the first build of a system synchronises to size the list capacities
        if ((st = build_pairlist(s, !ever_built))) return st;
        ever_built = true;
        if (prm.kernel == GR_KERNEL_PLAIN)
            if ((st = expand_cg_pairs(s))) return st;
    } else if ((st = push_descriptor(s))) {
        return st;
    }
    last_rebuilt = rebuild;
    steps_since_update += 1;
    if (stage) GR_CUDA(record_event(ev[1], s));
    const int NA = acc_size(G);
    // The per-atom short-range accumulators (and the per-step counters) are
    // zeroed by the previous evaluation's k_finalize as it reads them; only
    // after a (re)allocation or an interrupted evaluation are they cleared here.
    const bool clean = acc_clean;
    acc_clean = false;  // until this evaluation's finalize is enqueued
    if (!clean) {
        GR_CUDA(cudaMemsetAsync(h.f_short, 0, size_t(N) * 3 * sizeof(long long), s));
        GR_CUDA(cudaMemsetAsync(h.acc_short, 0, size_t(NA) * sizeof(long long), s));
        if (NCG > NSCG) {
            GR_CUDA(cudaMemsetAsync(h.max_delta, 0, sizeof(float), s));
            GR_CUDA(cudaMemsetAsync(h.n_deferred, 0, 8 * sizeof(int), s));
        }
    }
    if (NCG > NSCG && !fs_long_zeroed) {
        // the slot layout changes at rebuilds; keep the long cache consistent
        GR_CUDA(cudaMemsetAsync(h.fs_long, 0, size_t(h.max_clusters) * W * 9 * sizeof(long long), s));
        fs_long_zeroed = true;
    }
    bool do_long = h.twin && (rebuild || !lr_computed);
    const int sm = sm_count();
    const size_t shg = size_t(2 * G * G) * sizeof(unsigned long long);
    if (prm.kernel == GR_KERNEL_FIXED) {
        WaterParams wp;
        if (NCG > NSCG) {
            wp = water_params();
            if (!prepped) (++launches, k_water_prep<<<blocks_for(NCG - NSCG, 128), 128, 0, s>>>(d_sys));
            if (stage) GR_CUDA(record_event(evk[0], s));
            if ((st = launch_water(s, wp, false))) return st;
            if (stage) GR_CUDA(record_event(evk[1], s));
        }
        // solute work items: (CG, chunk of list entries), 4 warps per block
        const unsigned sgrid = std::max(1u, std::min(blocks_for((long long)NSCG * ((h.scap + kSoluteChunk - 1) / kSoluteChunk), 4),
                                                     unsigned(sm * 8)));
        if (NSCG > 0) (++launches, k_solute_force<false><<<sgrid, 128, shg, s>>>(d_sys));
        if (stage) GR_CUDA(record_event(ev[2], s));
        if (do_long) {
            GR_CUDA(cudaMemsetAsync(h.f_long, 0, size_t(N) * 3 * sizeof(long long), s));
            GR_CUDA(cudaMemsetAsync(h.acc_long, 0, size_t(NA) * sizeof(long long), s));
            if (NCG > NSCG)
                GR_CUDA(cudaMemsetAsync(h.fs_long, 0, size_t(h.max_clusters) * W * 9 * sizeof(long long), s));
            if (NCG > NSCG) {
                if (stage) GR_CUDA(record_event(evk[2], s));
                if ((st = launch_water(s, wp, true))) return st;
                if (stage) GR_CUDA(record_event(evk[3], s));
            }
            if (NSCG > 0) (++launches, k_solute_force<true><<<sgrid, 128, shg, s>>>(d_sys));
            lr_computed = true;
            if (stage && NCG > NSCG) evk_long = true;
        }
    } else {
        if (NCG > NSCG && !prepped)  // per-step water data incl. the solvent excluded energies
            (++launches, k_water_prep<<<blocks_for(NCG - NSCG, 128), 128, 0, s>>>(d_sys));
        (++launches, k_pos32<<<blocks_for(N, 256), 256, 0, s>>>(d_sys));
        GR_CUDA(cudaMemsetAsync(h.f32, 0, size_t(N) * 3 * sizeof(float), s));
        GR_CUDA(cudaMemsetAsync(h.e64, 0, 16 * sizeof(double), s));
        unsigned grid = std::max(1u, std::min(blocks_for(n_cgp_host[0], 256), unsigned(sm * 16)));
        (++launches, k_plain_force<<<grid, 256, 0, s>>>(d_sys, 0));
        if (stage) GR_CUDA(record_event(ev[2], s));
        if (do_long) {
            GR_CUDA(cudaMemsetAsync(h.f32_long, 0, size_t(N) * 3 * sizeof(float), s));
            GR_CUDA(cudaMemsetAsync(h.e64_long, 0, 16 * sizeof(double), s));
            unsigned gl = std::max(1u, std::min(blocks_for(n_cgp_host[1], 256), unsigned(sm * 16)));
            (++launches, k_plain_force<<<gl, 256, 0, s>>>(d_sys, 1));
            lr_computed = true;
        }
    }
    if (stage) GR_CUDA(record_event(ev[3], s));
    const size_t sha = size_t(NA) * sizeof(unsigned long long);
    if (h.excl_atoms > 0) (++launches, k_excluded_14<<<blocks_for(h.excl_atoms, 128), 128, sha, s>>>(d_sys));
    if (n_pert > 0) {
        if (NSCG > 0)
            (++launches, k_pert_pairs_force<<<blocks_for((std::max(pcap_alloc, 1) + kPertRun - 1) / kPertRun, 128), 128, sha,
                                              s>>>(d_sys));
        (++launches, k_pert_terms<<<blocks_for(std::max(N, h.n_pp), 128), 128, sha, s>>>(d_sys));
    }
    (++launches, k_finalize<<<blocks_for(std::max<long long>(3LL * N, NA), 256), 256, 0, s>>>(d_sys, prm.kernel == GR_KERNEL_PLAIN));
    acc_clean = true;  // k_finalize leaves the short-range accumulators zero
    if (prm.kernel == GR_KERNEL_PLAIN) (++launches, k_finalize_plain_energies<<<1, 32, 0, s>>>(d_sys));
    if (record_events) GR_CUDA(record_event(ev[4], s));
    GR_CUDA(cudaGetLastError());
    last_long = do_long;
    return GR_OK;
}

void NbSystem::drop_graphs() {
    for (auto& g : g_step) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    g_gen = -1;
}

// One evaluation replayed from a recorded CUDA graph: the whole step (memsets,
// kernels, timing events, error-flag copies) is submitted with one launch, so
// the kernels run back to back instead of waiting for the host's launches.
// Two graphs are recorded on first use: the short-range step and the rebuild
// step (pairlist build + long-range refresh); they are recorded again after
// any device reallocation.  The host-side cadence (steps since the rebuild)
// is kept exactly as eval() keeps it.  Cases the graphs do not cover (first
// evaluation, plain kernel, a long-range refresh outside a rebuild step after
// an overflow) run through eval().
gr_status NbSystem::eval_graph(cudaStream_t s, int flags) {
    gr_status st;
    if (!err_step_host) GR_CUDA(cudaMallocHost(&err_step_host, 4 * sizeof(int)));
    if (!ev_step) GR_CUDA(cudaEventCreateWithFlags(&ev_step, cudaEventDisableTiming));
    if (step_check) {  // flags of the previous graph step (deferred-pair overflow)
        GR_CUDA(cudaEventSynchronize(ev_step));
        step_check = false;
        if (err_step_host[0] & ERR_DEFER_OVERFLOW) {
            GR_CUDA(cudaMemset(h.err, 0, 4 * sizeof(int)));
            defer_want = std::max(defer_want, h.defer_cap) * 4;
            clus_alloc = 0;
            built = false;
            lr_computed = false;
            pending_check = false;
            set_error("the previous evaluation overflowed the deferred-pair list; the list was grown, evaluate again");
            return GR_ERR_OVERFLOW;
        }
    }
    bool overflowed = false;
    if ((st = resolve_pending(&overflowed))) return st;
    if (overflowed) lr_computed = false;
    const bool rebuild = !built || steps_since_update >= prm.nsnb || (flags & GR_EVAL_FORCE_REBUILD);
    const bool do_long = h.twin && (rebuild || !lr_computed);
    if (!ever_built || !warm || prm.kernel != GR_KERNEL_FIXED || (!rebuild && do_long)) {
        st = eval(s, flags, true);
        if (!st) warm = true;
        return st;
    }
    // capacities grown after an overflow are allocated before the rebuild
    // graph runs; a reallocation records the graphs again
    if (rebuild && relist) {  // a list_capacity change: the lists are re-sized (graphs recorded again)
        wcap_alloc = 0;
        wcap_want = 0;
        relist = false;
    }
    if (rebuild && (st = ensure_capacity())) return st;
    if (g_gen != alloc_gen) {
        drop_graphs();
        if ((st = ensure_capacity())) return st;
        if ((st = push_descriptor(s))) return st;
        GR_CUDA(cudaStreamSynchronize(s));
        const int ssu0 = steps_since_update;
        const bool built0 = built, lr0 = lr_computed;
        const long long l0 = launches;
        in_capture = true;
        for (int v = 0; v < 2 && !st; ++v) {
            steps_since_update = v ? prm.nsnb : 1;
            built = true;
            lr_computed = true;
            pending_check = false;
            const long long lv = launches;
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                st = eval(s, v ? GR_EVAL_FORCE_REBUILD : 0, true);
                if (!st) e = cudaMemcpyAsync(err_step_host, h.err, 4 * sizeof(int), cudaMemcpyDeviceToHost, s);
                cudaError_t e2 = cudaStreamEndCapture(s, &graph);
                if (e == cudaSuccess) e = e2;
            }
            if (!st && e == cudaSuccess) e = cudaGraphInstantiate(&g_step[v], graph, 0);
            if (graph) cudaGraphDestroy(graph);
            g_step_launches[v] = launches - lv;
            if (!st && e != cudaSuccess) {
                set_error(std::string("evaluation graph: ") + cudaGetErrorString(e));
                st = GR_ERR_CUDA;
            }
        }
        in_capture = false;
        launches = l0;
        steps_since_update = ssu0;
        built = built0;
        lr_computed = lr0;
        pending_check = false;
        if (st) {
            drop_graphs();
            return st;
        }
        g_gen = alloc_gen;
    }
    prepped_next = false;  // the graphs hold their own prep
    GR_CUDA(cudaGraphLaunch(g_step[rebuild ? 1 : 0], s));
    last_staged = false;
    GR_CUDA(cudaEventRecord(ev_step, s));
    step_check = true;
    launches += g_step_launches[rebuild ? 1 : 0];
    // the cadence eval() keeps
    if (rebuild) {
        built = true;
        cgp_valid = false;
        steps_since_update = 0;
        pending_check = true;  // the rebuild's flags were copied to err_host inside the graph
    }
    last_rebuilt = rebuild;
    steps_since_update += 1;
    if (do_long) lr_computed = true;
    last_long = do_long;
    return GR_OK;
}

// Per-launch constants of the water kernels (both ranges).  `lim` keeps the
// FP32 image decision away from half a box edge: 1e-4 nm covers the FP32
// rounding of the first-atom vector (short list); the long-range kernel also
// subtracts twice the largest molecule extent measured this step, since it
// images every atom pair.
WaterParams NbSystem::water_params() const {
    WaterParams wp;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            wp.qq[a * 3 + b] = h.w_qq[a * 4 + b];
            wp.c6[a * 3 + b] = h.w_c6[a * 4 + b];
            wp.c12[a * 3 + b] = h.w_c12[a * 4 + b];
        }
    wp.crf2 = h.crf_2cut3i_f;
    wp.crfc = h.crf_cut_f;
    wp.crf3 = h.crf_cut3i_f;
    const float margin = 1e-4f;  // the long list adds the measured molecule extent in the kernel
    for (int k = 0; k < 3; ++k) {
        wp.lim[k] = h.boundary ? h.half_boxf[k] - margin : 3.0e38f;
        wp.box[k] = h.box[k];
        wp.inv_box[k] = h.inv_box[k];
        wp.boxf[k] = h.boxf[k];
        wp.inv_boxf[k] = h.inv_boxf[k];
    }
    wp.boundary = h.boundary;
    wp.G = G;
    const int gs = solvent_group < 0 ? 0 : solvent_group;
    wp.slot = gs * G + gs;
    return wp;
}

// Force constants of the pair-stream kernel: the solvent table with the
// fixed-point scale 2^32 folded in (a power of two: the scaling is exact).
WaterScaled NbSystem::water_scaled(const WaterParams& wp) const {
    WaterScaled pp;
    const double sc = kForceScale;
    for (int t = 0; t < 9; ++t) {
        pp.qf[t] = float(double(wp.qq[t]) * sc);
        pp.qcf[t] = float(double(wp.qq[t]) * double(h.crf_cut3i_f) * sc);
        pp.c6f[t] = float(6.0 * double(wp.c6[t]) * sc);
        pp.c12f[t] = float(12.0 * double(wp.c12[t]) * sc);
    }
    pp.crfc_sumq = float(h.crf_cut * w_qq_sum);
    for (int u = 0; u < 4; ++u) {
        const int t0 = unit_t(u, 0), t1 = unit_t(u, 1);
        pp.pqf[u] = make_float2(pp.qf[t0], pp.qf[t1]);
        pp.pqcf[u] = make_float2(pp.qcf[t0], pp.qcf[t1]);
        pp.pqq[u] = make_float2(wp.qq[t0], wp.qq[t1]);
        pp.pc12[u] = make_float2(wp.c12[t0], wp.c12[t1]);
        pp.pnc6[u] = make_float2(-wp.c6[t0], -wp.c6[t1]);
        pp.pc12f[u] = make_float2(pp.c12f[t0], pp.c12f[t1]);
        pp.pnc6f[u] = make_float2(-pp.c6f[t0], -pp.c6f[t1]);
    }
    pp.ncrf2 = make_float2(-wp.crf2, -wp.crf2);
    return pp;
}

// The water force kernel of the selected layout and width, then the
// deferred-pair kernel.
gr_status NbSystem::launch_water(cudaStream_t s, const WaterParams& wp, bool lr) {
    const int sm = sm_count();
    const bool lj00 = h.water_lj00_only != 0;
    // The water kernels are persistent (grid-stride over i-clusters): the grid
    // is exactly one wave, SMs x resident blocks per SM, so that no block
    // starts after the first ones have finished their share -- or fewer
    // blocks for a small system, which leaves SMs to the other members of a
    // batch.
    auto water_grid = [&](int wave) {
        const long long need = (static_cast<long long>(h.max_clusters) + kWaterWarps - 1) / kWaterWarps;
        return unsigned(std::max<long long>(1, std::min<long long>(wave, need)));
    };
#define GR_WATER_IT(WW, LJ, LL)                                                                          \
    do {                                                                                                 \
        const size_t smem = water_it_smem<WW>();                                                         \
        int occ = 1;                                                                                     \
        if (layout == 4) {                                                                               \
            GR_CUDA(occupancy(k_water_force_it<WW, LJ, LL, true>, 128, smem, &occ));                     \
            (++launches,                                                                                 \
             k_water_force_it<WW, LJ, LL, true><<<water_grid(sm * occ), 128, smem, s>>>(d_sys, wp, ws));   \
        } else {                                                                                         \
            GR_CUDA(occupancy(k_water_force_it<WW, LJ, LL, false>, 128, smem, &occ));                    \
            (++launches,                                                                                 \
             k_water_force_it<WW, LJ, LL, false><<<water_grid(sm * occ), 128, smem, s>>>(d_sys, wp, ws));  \
        }                                                                                                \
    } while (0)
#define GR_WATER_SHARED(LJ, LL)                                                                          \
    do {                                                                                                 \
        int occ = 1;                                                                                     \
        GR_CUDA(occupancy(k_water_force<LJ, LL>, 128, 0, &occ));                                         \
        (++launches, k_water_force<LJ, LL><<<water_grid(sm * occ), 128, 0, s>>>(d_sys, wp));            \
    } while (0)
    const WaterScaled ws = water_scaled(wp);
    if (layout == 3 && !lr) {
        const WaterScaled& pp = ws;
        const size_t smem = water_ps_smem();
        int occ = 1;
        if (lj00) {
            GR_CUDA(occupancy(k_water_force_ps<true>, kPsWarps * 32, smem, &occ));
            const long long need = (static_cast<long long>(h.max_clusters + 1) / 2 + kPsWarps - 1) / kPsWarps;
            const unsigned grid = unsigned(std::max<long long>(1, std::min<long long>(sm * occ, need)));
            (++launches, k_water_force_ps<true><<<grid, kPsWarps * 32, smem, s>>>(d_sys, wp, pp));
        } else {
            GR_CUDA(occupancy(k_water_force_ps<false>, kPsWarps * 32, smem, &occ));
            const long long need = (static_cast<long long>(h.max_clusters + 1) / 2 + kPsWarps - 1) / kPsWarps;
            const unsigned grid = unsigned(std::max<long long>(1, std::min<long long>(sm * occ, need)));
            (++launches, k_water_force_ps<false><<<grid, kPsWarps * 32, smem, s>>>(d_sys, wp, pp));
        }
    } else if (layout == 1) {
        if (lj00) {
            if (lr) GR_WATER_SHARED(true, true); else GR_WATER_SHARED(true, false);
        } else {
            if (lr) GR_WATER_SHARED(false, true); else GR_WATER_SHARED(false, false);
        }
    } else if (W == 4) {
        if (lj00) {
            if (lr) GR_WATER_IT(4, true, true); else GR_WATER_IT(4, true, false);
        } else {
            if (lr) GR_WATER_IT(4, false, true); else GR_WATER_IT(4, false, false);
        }
    } else {
        if (lj00) {
            if (lr) GR_WATER_IT(8, true, true); else GR_WATER_IT(8, true, false);
        } else {
            if (lr) GR_WATER_IT(8, false, true); else GR_WATER_IT(8, false, false);
        }
    }
#undef GR_WATER_IT
#undef GR_WATER_SHARED
    if (layout == 1) {  // the bit-iterating kernel handles its deferred pairs itself
        if (lj00) {
            if (lr) (++launches, k_water_deferred<true, true><<<sm, 128, 0, s>>>(d_sys, wp));
            else (++launches, k_water_deferred<true, false><<<sm, 128, 0, s>>>(d_sys, wp));
        } else {
            if (lr) (++launches, k_water_deferred<false, true><<<sm, 128, 0, s>>>(d_sys, wp));
            else (++launches, k_water_deferred<false, false><<<sm, 128, 0, s>>>(d_sys, wp));
        }
    }
    GR_CUDA(cudaGetLastError());
    return GR_OK;
}

template <class K>
cudaError_t NbSystem::occupancy(K* kernel, int threads, size_t smem, int* occ) {
    const void* key = reinterpret_cast<const void*>(kernel);
    for (const auto& e : occ_cache)
        if (e.first == key) {
            *occ = e.second;
            return cudaSuccess;
        }
    cudaError_t e;
    if (smem > 0 && (e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))))
        return e;
    int o = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, threads, smem))) return e;
    if (o < 1) o = 1;
    occ_cache.emplace_back(key, o);
    *occ = o;
    return cudaSuccess;
}

int NbSystem::sm_count() {
    if (sms_cached == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms_cached, cudaDevAttrMultiProcessorCount, dev);
        if (sms_cached <= 0) sms_cached = 1;
    }
    return sms_cached;
}

gr_status NbSystem::pair_counts(cudaStream_t s, long long* n_short, long long* n_long) {
    // atom-pair interactions per evaluation: sum over listed CG pairs of
    // (atoms_i * atoms_j) minus excluded pairs; computed from the CG pair set.
    gr_status st;
    if (!cgp_valid)
        if ((st = expand_cg_pairs(s))) return st;
    if (pair_count_valid) {
        *n_short = pairs_short;
        *n_long = pairs_long;
        return GR_OK;
    }
    std::vector<int> cgp(static_cast<size_t>(cgp_alloc) * 3, 0);
    std::vector<unsigned long long> xm(static_cast<size_t>(cgp_alloc), 0ull);
    GR_CUDA(cudaMemcpy(cgp.data(), h.cgp, cgp.size() * sizeof(int), cudaMemcpyDeviceToHost));
    GR_CUDA(cudaMemcpy(xm.data(), h.cgp_excl, xm.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    long long ns = 0, nl = 0;
    auto count = [&](int idx) {
        int ci = cgp[3 * idx], cj = cgp[3 * idx + 1];
        int ni = h_cg_off[ci + 1] - h_cg_off[ci], nj = h_cg_off[cj + 1] - h_cg_off[cj];
        long long n = (long long)ni * nj;
        n -= __builtin_popcountll(xm[idx]);
        return n;
    };
    for (int p = 0; p < n_cgp_host[0]; ++p) ns += count(p);
    for (int p = 0; p < n_cgp_host[1]; ++p) nl += count(cgp_alloc - 1 - p);
    pairs_short = ns;
    pairs_long = nl;
    pair_count_valid = true;
    *n_short = ns;
    *n_long = nl;
    return GR_OK;
}

// Energies, the error flags and (if requested) the forces are copied in
// stream order -- the flags and energies into pinned buffers -- and read
// after one synchronisation.
gr_status NbSystem::download(cudaStream_t s, gr_result* out) {
    if (!out) return GR_OK;
    const int NA = acc_size(G);
    if (e_dl_n < NA) {
        if (e_dl_host) cudaFreeHost(e_dl_host);
        e_dl_host = nullptr;
        e_dl_n = 0;
        GR_CUDA(cudaMallocHost(&e_dl_host, size_t(NA) * sizeof(double)));
        e_dl_n = NA;
    }
    if (!err_dl_host) GR_CUDA(cudaMallocHost(&err_dl_host, 4 * sizeof(int)));
    const double* e = e_dl_host;
    GR_CUDA(cudaMemcpyAsync(e_dl_host, h.e_out, NA * sizeof(double), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaMemcpyAsync(err_dl_host, h.err, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (out->forces)
        GR_CUDA(cudaMemcpyAsync(out->forces, h.f_out, size_t(N) * 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaStreamSynchronize(s));
    double lj = 0, crf = 0;
    for (int a = 0; a < G; ++a)
        for (int b = a; b < G; ++b) {
            lj += e[a * G + b];
            crf += e[G * G + a * G + b];
        }
    out->e_lj = lj;
    out->e_crf = crf;
    for (int v = 0; v < 9; ++v) out->virial[v] = e[2 * G * G + v];
    out->dhdl = e[NA - 1];
    if (out->egroup_lj)
        for (int k = 0; k < G * G; ++k) out->egroup_lj[k] = e[k];
    if (out->egroup_crf)
        for (int k = 0; k < G * G; ++k) out->egroup_crf[k] = e[G * G + k];
    out->rebuilt = last_rebuilt ? 1 : 0;
    return GR_OK;
}

}  // namespace gnb

using gnb::NbSystem;
using gnb::set_error;

struct gr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    NbSystem sys;
};

#define CTX_GUARD(ctx)                                  \
    do {                                                \
        if (!(ctx)) {                                   \
            set_error("null gr_ctx");                   \
            return GR_ERR_INVALID;                      \
        }                                               \
        cudaError_t e_ = cudaSetDevice((ctx)->device);  \
        if (e_ != cudaSuccess) {                        \
            set_error(cudaGetErrorString(e_));          \
            return GR_ERR_CUDA;                         \
        }                                               \
    } while (0)

extern "C" {

const char* gr_last_error(void) { return gnb::g_last_error.c_str(); }

gr_status gr_ctx_create(int device, gr_ctx** out) {
    if (!out) {
        set_error("gr_ctx_create: null out");
        return GR_ERR_INVALID;
    }
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        set_error("gr_ctx_create: no CUDA device");
        return GR_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        set_error("gr_ctx_create: device index out of range");
        return GR_ERR_INVALID;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        set_error("gr_ctx_create: cudaSetDevice failed");
        return GR_ERR_CUDA;
    }
    auto* c = new gr_ctx;
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        set_error("gr_ctx_create: stream creation failed");
        return GR_ERR_CUDA;
    }
    c->sys.mem_stream = c->stream;
    *out = c;
    return GR_OK;
}

gr_status gr_ctx_destroy(gr_ctx* ctx) {
    if (!ctx) return GR_OK;
    if (ctx->sys.batch_member) {
        set_error("gr_ctx_destroy: the context is a batch member; gr_batch_remove it first");
        return GR_ERR_STATE;
    }
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->sys.release();
    cudaStreamDestroy(ctx->stream);
    ctx->sys.mem_stream = nullptr;
    delete ctx;
    return GR_OK;
}

void* gr_ctx_stream(gr_ctx* ctx) { return ctx ? reinterpret_cast<void*>(ctx->stream) : nullptr; }

gr_status gr_system_upload(gr_ctx* ctx, const gr_topology* topo) {
    CTX_GUARD(ctx);
    return ctx->sys.upload(topo);
}

gr_status gr_set_params(gr_ctx* ctx, const gr_nb_params* params) {
    CTX_GUARD(ctx);
    if (!ctx->sys.uploaded) {
        set_error("gr_set_params before gr_system_upload");
        return GR_ERR_STATE;
    }
    return ctx->sys.set_params(params);
}

gr_status gr_set_box(gr_ctx* ctx, const double box[3]) {
    CTX_GUARD(ctx);
    if (!box) {
        set_error("gr_set_box: null box");
        return GR_ERR_INVALID;
    }
    if (!ctx->sys.params_set) {
        set_error("gr_set_box before gr_set_params");
        return GR_ERR_STATE;
    }
    return ctx->sys.set_box(box);
}

gr_status gr_positions_upload(gr_ctx* ctx, const double* xyz) {
    CTX_GUARD(ctx);
    if (!ctx->sys.uploaded || !xyz) {
        set_error("gr_positions_upload: no system or null positions");
        return GR_ERR_STATE;
    }
    ctx->sys.prepped_next = false;
    cudaError_t e = cudaMemcpyAsync(ctx->sys.h.pos, xyz, size_t(ctx->sys.N) * 3 * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        return GR_ERR_CUDA;
    }
    ctx->sys.pos_set = true;
    return GR_OK;
}

gr_status gr_positions_device(gr_ctx* ctx, double** dev_xyz) {
    CTX_GUARD(ctx);
    if (!ctx->sys.uploaded || !dev_xyz) {
        set_error("gr_positions_device: no system");
        return GR_ERR_STATE;
    }
    *dev_xyz = ctx->sys.h.pos;
    ctx->sys.prepped_next = false;  // the caller may write the coordinates
    ctx->sys.pos_set = true;
    return GR_OK;
}

gr_status gr_pairlist_build(gr_ctx* ctx) {
    CTX_GUARD(ctx);
    if (!ctx->sys.pos_set) {
        set_error("gr_pairlist_build before positions are set");
        return GR_ERR_STATE;
    }
    gr_status st = ctx->sys.build_pairlist(ctx->stream, true);
    if (st) return st;
    ctx->sys.ever_built = true;
    ctx->sys.pair_count_valid = false;
    return GR_OK;  // the explicit CG-pair lists are expanded when first asked for
}

// The four reference lists from the device CG pair set (pairlist.rs:59-70):
// solute_short (intra-CG + non-excluded solute-solute + all solute-solvent
// atom pairs), solute_long, solvent_short (first-atom sentinels),
// solvent_long (all atom pairs), each sorted.
static gr_status build_reference_lists(gr_ctx* ctx, std::vector<std::pair<int, int>> lists[4]) {
    NbSystem& S = ctx->sys;
    if (!S.built) {
        set_error("pairlist not built");
        return GR_ERR_STATE;
    }
    gr_status st;
    if (!S.cgp_valid)
        if ((st = S.expand_cg_pairs(ctx->stream))) return st;
    size_t cap = size_t(S.cgp_alloc);
    std::vector<int> cgp(cap * 3);
    std::vector<unsigned long long> xm(cap);
    if (cudaMemcpy(cgp.data(), S.h.cgp, cgp.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(xm.data(), S.h.cgp_excl, xm.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
        set_error("pairlist download copy failed");
        return GR_ERR_CUDA;
    }
    const auto& off = S.h_cg_off;
    auto emit = [&](int idx) {
        int c1 = cgp[3 * idx], c2 = cgp[3 * idx + 1], lr = cgp[3 * idx + 2];
        unsigned long long m = xm[idx];
        bool s1 = c1 < S.NSCG, s2 = c2 < S.NSCG;
        if (!s1 && !s2) {
            if (!lr) {
                lists[2].push_back({off[c1], off[c2]});
            } else {
                for (int a = off[c1]; a < off[c1 + 1]; ++a)
                    for (int b = off[c2]; b < off[c2 + 1]; ++b) lists[3].push_back({a, b});
            }
            return;
        }
        auto& dst = lr ? lists[1] : lists[0];
        for (int a = off[c1]; a < off[c1 + 1]; ++a)
            for (int b = off[c2]; b < off[c2 + 1]; ++b) {
                int ia = a - off[c1], ib = b - off[c2];
                if (m & (1ull << (ia * 8 + ib))) continue;
                dst.push_back({a, b});
            }
    };
    for (int p = 0; p < S.n_cgp_host[0]; ++p) emit(p);
    for (int p = 0; p < S.n_cgp_host[1]; ++p) emit(int(cap) - 1 - p);
    for (int k = 0; k < 4; ++k) std::sort(lists[k].begin(), lists[k].end());
    return GR_OK;
}

gr_status gr_pairlist_counts(gr_ctx* ctx, int64_t counts[4]) {
    CTX_GUARD(ctx);
    if (!counts) {
        set_error("gr_pairlist_counts: null counts");
        return GR_ERR_INVALID;
    }
    std::vector<std::pair<int, int>> L[4];
    gr_status st = build_reference_lists(ctx, L);
    if (st) return st;
    for (int k = 0; k < 4; ++k) counts[k] = int64_t(L[k].size());
    return GR_OK;
}

gr_status gr_pairlist_download(gr_ctx* ctx, int32_t* ss, int32_t* sl, int32_t* vs, int32_t* vl) {
    CTX_GUARD(ctx);
    std::vector<std::pair<int, int>> L[4];
    gr_status st = build_reference_lists(ctx, L);
    if (st) return st;
    int32_t* dst[4] = {ss, sl, vs, vl};
    for (int k = 0; k < 4; ++k)
        if (dst[k])
            for (size_t p = 0; p < L[k].size(); ++p) {
                dst[k][2 * p] = L[k][p].first;
                dst[k][2 * p + 1] = L[k][p].second;
            }
    return GR_OK;
}

gr_status gr_pairlist_cg_pairs(gr_ctx* ctx, int32_t* out, int64_t* n_pairs) {
    CTX_GUARD(ctx);
    NbSystem& S = ctx->sys;
    if (!n_pairs) {
        set_error("gr_pairlist_cg_pairs: null n_pairs");
        return GR_ERR_INVALID;
    }
    if (!S.built) {
        set_error("pairlist not built");
        return GR_ERR_STATE;
    }
    gr_status st;
    if (!S.cgp_valid)
        if ((st = S.expand_cg_pairs(ctx->stream))) return st;
    size_t cap = size_t(S.cgp_alloc);
    std::vector<int> cgp(cap * 3);
    if (cudaMemcpy(cgp.data(), S.h.cgp, cgp.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("copy failed");
        return GR_ERR_CUDA;
    }
    std::vector<std::array<int, 3>> v;
    for (int p = 0; p < S.n_cgp_host[0]; ++p) {
        int i = cgp[3 * p], j = cgp[3 * p + 1];
        if (i != j) v.push_back({i, j, 0});
    }
    for (int p = 0; p < S.n_cgp_host[1]; ++p) {
        int q = int(cap) - 1 - p;
        v.push_back({cgp[3 * q], cgp[3 * q + 1], 1});
    }
    std::sort(v.begin(), v.end());
    int64_t capn = *n_pairs;
    *n_pairs = int64_t(v.size());
    if (out) {
        if (capn < int64_t(v.size())) {
            set_error("gr_pairlist_cg_pairs: buffer too small");
            return GR_ERR_INVALID;
        }
        for (size_t k = 0; k < v.size(); ++k)
            for (int c = 0; c < 3; ++c) out[3 * k + c] = v[k][c];
    }
    return GR_OK;
}

gr_status gr_forces_eval(gr_ctx* ctx, int32_t flags, gr_result* out) {
    CTX_GUARD(ctx);
    NbSystem& S = ctx->sys;
    const bool download = out && !(flags & GR_EVAL_NO_DOWNLOAD);
    gr_status st;
    for (int attempt = 0;; ++attempt) {
        st = (flags & GR_EVAL_GRAPH) ? S.eval_graph(ctx->stream, flags) : S.eval(ctx->stream, flags, true);
        if (st) return st;
        if (!download) return GR_OK;  // overflow (if any) is reported by the next call
        if ((st = S.download(ctx->stream, out))) return st;
        S.step_check = false;  // the flags are checked here, read with the download
        if (S.err_dl_host[0] & gnb::ERR_DEFER_OVERFLOW) {
            // grow the deferred-pair list and redo this evaluation (long range too)
            cudaMemset(S.h.err, 0, 4 * sizeof(int));
            if (attempt >= 8) {
                set_error("water kernel: deferred-pair list could not be grown far enough");
                return GR_ERR_OVERFLOW;
            }
            S.defer_want = std::max(S.defer_want, S.h.defer_cap) * 4;
            S.clus_alloc = 0;  // re-run the cluster allocation with the larger list
            S.built = false;
            S.lr_computed = false;
            continue;
        }
        bool overflowed = false;
        if ((st = S.resolve_pending(&overflowed))) return st;
        if (!overflowed) break;
        if (attempt >= 8) {
            set_error("pairlist: list capacity could not be grown far enough");
            return GR_ERR_OVERFLOW;
        }
        // re-run this evaluation with the grown lists
    }
    if (S.last_rebuilt) S.pair_count_valid = false;
    long long ns = 0, nl = 0;
    if (out->n_pairs_short >= 0) {  // caller may pass -1 to skip the count
        if ((st = S.pair_counts(ctx->stream, &ns, &nl))) return st;
    }
    out->n_pairs_short = ns;
    out->n_pairs_long = S.last_long ? nl : 0;
    return GR_OK;
}

gr_status gr_forces_device(gr_ctx* ctx, const double** dev_forces) {
    CTX_GUARD(ctx);
    if (!dev_forces) return GR_ERR_INVALID;
    *dev_forces = ctx->sys.h.f_out;
    return GR_OK;
}

gr_status gr_result_download(gr_ctx* ctx, gr_result* out) {
    CTX_GUARD(ctx);
    return ctx->sys.download(ctx->stream, out);
}

gr_status gr_ctx_launches(gr_ctx* ctx, int64_t* n) {
    CTX_GUARD(ctx);
    if (!n) return GR_ERR_INVALID;
    *n = ctx->sys.launches;
    return GR_OK;
}

gr_status gr_ffma_peak(int device, double* ops_per_s) {
    if (!ops_per_s) return GR_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        set_error("gr_ffma_peak: no such CUDA device");
        return GR_ERR_NO_DEVICE;
    }
    GR_CUDA(cudaSetDevice(device));
    int sms = 0;
    GR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float* out = nullptr;
    GR_CUDA(cudaMalloc(&out, sizeof(float)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int threads = 256, blocks = sms * 8, iters = 2048;
    gnb::k_ffma_peak<<<blocks, threads>>>(out, 64, 0.999f, 1e-7f);  // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a);
        gnb::k_ffma_peak<<<blocks, threads>>>(out, iters, 0.999f, 1e-7f);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        double ops = double(blocks) * threads * iters * 16.0 * 8.0;
        if (ms > 0) best = std::max(best, ops / (ms * 1e-3));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    GR_CUDA(cudaGetLastError());
    *ops_per_s = best;
    return GR_OK;
}

gr_status gr_last_timings(gr_ctx* ctx, float ms[5]) {
    CTX_GUARD(ctx);
    if (!ms) {
        set_error("gr_last_timings: null ms");
        return GR_ERR_INVALID;
    }
    NbSystem& S = ctx->sys;
    if (cudaEventSynchronize(S.ev[4]) != cudaSuccess) {
        set_error("no timed evaluation");
        return GR_ERR_STATE;
    }
    if (S.last_staged) {
        cudaEventElapsedTime(&ms[0], S.ev[0], S.ev[1]);
        cudaEventElapsedTime(&ms[1], S.ev[1], S.ev[2]);
        cudaEventElapsedTime(&ms[2], S.ev[2], S.ev[3]);
        cudaEventElapsedTime(&ms[3], S.ev[3], S.ev[4]);
    } else {
        ms[0] = ms[1] = ms[2] = ms[3] = -1.f;  // a graph step: its total only
    }
    cudaEventElapsedTime(&ms[4], S.ev[0], S.ev[4]);
    return GR_OK;
}

gr_status gr_last_kernel_timings(gr_ctx* ctx, float ms[3]) {
    CTX_GUARD(ctx);
    if (!ms) {
        set_error("gr_last_kernel_timings: null ms");
        return GR_ERR_INVALID;
    }
    NbSystem& S = ctx->sys;
    if (cudaEventSynchronize(S.ev[4]) != cudaSuccess) {
        set_error("no timed evaluation");
        return GR_ERR_STATE;
    }
    ms[0] = ms[1] = ms[2] = -1.f;
    if (S.last_staged && S.evk_valid) {
        cudaEventElapsedTime(&ms[0], S.ev[1], S.evk[0]);
        cudaEventElapsedTime(&ms[1], S.evk[0], S.evk[1]);
        if (S.evk_long) cudaEventElapsedTime(&ms[2], S.evk[2], S.evk[3]);
    }
    return GR_OK;
}

}  // extern "C"

extern "C" gr_status gr_lj_crf_innerloop(const float* positions, const float* charges, const uint32_t* iac,
                                         uint32_t n_atoms, const uint32_t* pairlist, uint32_t n_pairs,
                                         const double* lj_params, uint32_t n_types, const double* box_data,
                                         uint32_t boundary_type, double crf_cut, double crf_2cut3i,
                                         double crf_cut3i, float* forces, double* energies, double* virial) {
    using namespace gnb;
    if (!forces || !energies || !virial) {
        set_error("gr_lj_crf_innerloop: null output");
        return GR_ERR_INVALID;
    }
    std::memset(forces, 0, sizeof(float) * 3 * n_atoms);
    energies[0] = energies[1] = 0.0;
    for (int k = 0; k < 9; ++k) virial[k] = 0.0;
    if (boundary_type > 1) {
        set_error("gr_lj_crf_innerloop: triclinic boundaries are not supported");
        return GR_ERR_UNSUPPORTED;
    }
    if (n_atoms == 0 || n_pairs == 0) return GR_OK;
    if (!positions || !charges || !iac || !pairlist || !lj_params || (boundary_type == 1 && !box_data)) {
        set_error("gr_lj_crf_innerloop: null input");
        return GR_ERR_INVALID;
    }
    for (uint32_t p = 0; p < 2 * n_pairs; ++p)
        if (pairlist[p] >= n_atoms) {
            set_error("gr_lj_crf_innerloop: pair index out of range");
            return GR_ERR_INVALID;
        }
    for (uint32_t a = 0; a < n_atoms; ++a)
        if (iac[a] >= n_types) {
            set_error("gr_lj_crf_innerloop: iac out of range");
            return GR_ERR_INVALID;
        }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("gr_lj_crf_innerloop: no CUDA device");
        return GR_ERR_NO_DEVICE;
    }
    std::vector<float2> lj(size_t(n_types) * n_types);
    for (size_t k = 0; k < lj.size(); ++k) lj[k] = make_float2(float(lj_params[2 * k]), float(lj_params[2 * k + 1]));
    float *dpos = nullptr, *dq = nullptr, *dF = nullptr;
    uint32_t *diac = nullptr, *dpairs = nullptr;
    float2* dlj = nullptr;
    double* dE = nullptr;
    gr_status st = GR_OK;
    auto fail = [&](cudaError_t e) {
        set_error(std::string("gr_lj_crf_innerloop: ") + cudaGetErrorString(e));
        st = GR_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&dpos, sizeof(float) * 3 * n_atoms)) || (e = cudaMalloc(&dq, sizeof(float) * n_atoms)) ||
        (e = cudaMalloc(&dF, sizeof(float) * 3 * n_atoms)) || (e = cudaMalloc(&diac, sizeof(uint32_t) * n_atoms)) ||
        (e = cudaMalloc(&dpairs, sizeof(uint32_t) * 2 * n_pairs)) || (e = cudaMalloc(&dlj, sizeof(float2) * lj.size())) ||
        (e = cudaMalloc(&dE, sizeof(double) * 11))) {
        fail(e);
    } else if ((e = cudaMemcpy(dpos, positions, sizeof(float) * 3 * n_atoms, cudaMemcpyHostToDevice)) ||
               (e = cudaMemcpy(dq, charges, sizeof(float) * n_atoms, cudaMemcpyHostToDevice)) ||
               (e = cudaMemcpy(diac, iac, sizeof(uint32_t) * n_atoms, cudaMemcpyHostToDevice)) ||
               (e = cudaMemcpy(dpairs, pairlist, sizeof(uint32_t) * 2 * n_pairs, cudaMemcpyHostToDevice)) ||
               (e = cudaMemcpy(dlj, lj.data(), sizeof(float2) * lj.size(), cudaMemcpyHostToDevice)) ||
               (e = cudaMemset(dF, 0, sizeof(float) * 3 * n_atoms)) || (e = cudaMemset(dE, 0, sizeof(double) * 11))) {
        fail(e);
    } else {
        float bx = boundary_type ? float(box_data[0]) : 1.f, by = boundary_type ? float(box_data[1]) : 1.f;
        float bz = boundary_type ? float(box_data[2]) : 1.f;
        unsigned grid = std::min(4096u, (n_pairs + 255) / 256);
        k_innerloop_pairs<<<grid, 256>>>(dpos, dq, diac, dpairs, n_pairs, dlj, n_types, bx, by, bz,
                                         int(boundary_type), float(crf_cut), float(crf_2cut3i), float(crf_cut3i),
                                         138.9354f, dF, dE);
        double h[11];
        if ((e = cudaGetLastError()) || (e = cudaMemcpy(forces, dF, sizeof(float) * 3 * n_atoms, cudaMemcpyDeviceToHost)) ||
            (e = cudaMemcpy(h, dE, sizeof(h), cudaMemcpyDeviceToHost))) {
            fail(e);
        } else {
            energies[0] = h[0];
            energies[1] = h[1];
            for (int k = 0; k < 9; ++k) virial[k] = h[2 + k];
        }
    }
    cudaFree(dpos);
    cudaFree(dq);
    cudaFree(dF);
    cudaFree(diac);
    cudaFree(dpairs);
    cudaFree(dlj);
    cudaFree(dE);
    return st;
}

// rust_lj_crf_innerloop_parallel (crates/gromos-core/src/ffi.rs:105-145)
// delegates to the serial stub in gromos-rs; here both names run the same
// device evaluation.
extern "C" gr_status gr_lj_crf_innerloop_parallel(const float* positions, const float* charges, const uint32_t* iac,
                                                  uint32_t n_atoms, const uint32_t* pairlist, uint32_t n_pairs,
                                                  const double* lj_params, uint32_t n_types, const double* box_data,
                                                  uint32_t boundary_type, double crf_cut, double crf_2cut3i,
                                                  double crf_cut3i, float* forces, double* energies, double* virial) {
    return gr_lj_crf_innerloop(positions, charges, iac, n_atoms, pairlist, n_pairs, lj_params, n_types, box_data,
                               boundary_type, crf_cut, crf_2cut3i, crf_cut3i, forces, energies, virial);
}
