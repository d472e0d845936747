// nb_system.h -- host-side owner of one system's device state.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gromos_nb.h"
#include "nb_common.cuh"

namespace gnb {

struct WaterParams;
struct WaterScaled;
void set_error(const std::string& m);
void crf_params(double cutoff, double epsilon, double rf_epsilon, double rf_kappa, double out[4]);
void lambda_params(double lam, int n, double lp[17]);

class NbSystem {
   public:
    ~NbSystem();
    void release();
    gr_status upload(const gr_topology* t);
    gr_status set_params(const gr_nb_params* p);
    gr_status set_box(const double box[3]);
    gr_status build_pairlist(cudaStream_t s, bool sync);
    gr_status resolve_pending(bool* overflowed);
    gr_status expand_cg_pairs(cudaStream_t s);
    gr_status eval(cudaStream_t s, int flags, bool record_events);
    gr_status eval_graph(cudaStream_t s, int flags);
    void drop_graphs();
    gr_status download(cudaStream_t s, gr_result* out);
    gr_status pair_counts(cudaStream_t s, long long* n_short, long long* n_long);
    gr_status push_descriptor(cudaStream_t s);
    cudaError_t dev_malloc(void** p, size_t n);
    void dev_free(void* p);
    cudaStream_t mem_stream = nullptr;  // the context's stream: pool allocations and releases are ordered on it
    cudaError_t record_event(cudaEvent_t e, cudaStream_t s);
    int sm_count();
    // Resident blocks per SM of `kernel` at this launch shape, looked up once
    // per context: function attributes (the dynamic shared-memory opt-in) and
    // occupancy belong to the device, and a process may hold contexts on
    // several GPUs.
    template <class K>
    cudaError_t occupancy(K* kernel, int threads, size_t smem, int* occ);
    WaterParams water_params() const;
    WaterScaled water_scaled(const WaterParams& wp) const;
    gr_status launch_water(cudaStream_t s, const WaterParams& wp, bool lr);
    gr_status md_init(const double* mass, const double* vel, const gr_md_params* p);
    gr_status md_run(cudaStream_t s, int n_steps, gr_md_stats* out);
    gr_status md_step_launch(cudaStream_t s, bool fuse_prep = false);
    gr_status md_stats(cudaStream_t s, gr_md_stats* out);
    gr_status ensure_capacity();

    // sizes
    int N = 0, NCG = 0, NSCG = 0, NSA = 0, NT = 0, G = 1, aps = 3, W = 4, layout = 2;
    int n_pert = 0, solvent_group = -1;
    double fpe = 138.9354;
    double w_qq_sum = 0.0;  // sum over a solvent molecule's atom pairs of q_a q_b fpe
    gr_nb_params prm{};
    // host copies needed for list expansion
    std::vector<int> h_cg_off, h_excl_off, h_excl, h_o14_off, h_o14, h_egroup;
    // device descriptor (host mirror + device copy)
    SysDev h{};
    SysDev* d_sys = nullptr;
    unsigned long long* d_cg_key = nullptr;
    // state
    bool uploaded = false, params_set = false, box_set = false, pos_set = false;
    bool built = false, lr_computed = false, last_rebuilt = false, last_long = false;
    bool cgp_valid = false, pair_count_valid = false;
    int steps_since_update = 0;
    int n_cgp_host[2] = {0, 0};
    long long pairs_short = 0, pairs_long = 0;
    long long launches = 0;  // kernels launched by this system
    // capacities
    int cells_alloc = 0, clus_alloc = 0, wcap_alloc = 0, scap_alloc = 0, pcap_alloc = 0, cgp_alloc = 0;
    int wcap_want = 0, scap_want = 0, pcap_want = 0, defer_want = 0;
    long long cgp_want = 0;
    int regrow_count = 0;
    size_t bytes = 0;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // kernel-level events of a staged evaluation: after the water prep, after the
    // short-range water kernel, around the long-range water kernel
    cudaEvent_t evk[4] = {nullptr, nullptr, nullptr, nullptr};
    bool evk_valid = false;  // the last staged evaluation recorded evk (a solvent, fixed-point kernel)
    bool evk_long = false;   // ... and ran the long-range water kernel
    cudaEvent_t ev_err = nullptr;
    int* err_host = nullptr;  // pinned copy of the device error flags
    bool pending_check = false, ever_built = false;
    bool solvent_excl_intra = false;
    bool fs_long_zeroed = false;  // solvent exclusions are exactly the molecule's other atoms
    // MD state (md.cu)
    bool md_ready = false, md_settle = false;
    gr_md_params mdp{};
    double md_m_o = 0, md_m_h = 0, md_ra = 0, md_rb = 0, md_rc = 0;
    double *md_vel = nullptr, *md_mass = nullptr, *md_inv_mass = nullptr;
    double *md_pos_snap = nullptr, *md_vel_snap = nullptr;
    long long* md_ke = nullptr;      // [2]: kinetic energy entering the next step, accumulator
    long long* md_ke_snap = nullptr;
    double* md_t0 = nullptr;         // [1] Berendsen bath temperature, read by k_md_step every step
    double md_dof = 0.0;
    int* md_fail = nullptr;
    long long* md_err_host = nullptr;  // pinned
    cudaEvent_t ev_md = nullptr;
    long long md_steps_total = 0, md_rollbacks = 0;
    // state at the start of the current pairlist period (a rollback point for
    // a block that starts inside the period) and its MD step index
    double *md_psnap_pos = nullptr, *md_psnap_vel = nullptr;
    long long* md_psnap_ke = nullptr;
    long long md_step_idx = 0, md_psnap_step = 0;
    bool md_psnap_valid = false;
    bool relist = false;  // list storage re-sized at the next rebuild (a list_capacity change)
    bool warm = false;        // evaluated at least once with the current parameters
    bool acc_clean = false;   // short-range accumulators and per-step counters are zero
    bool batch_member = false;  // held by a gr_batch (its graphs point at this system)
    long long alloc_gen = 0;  // bumped by every device (re)allocation: recorded graphs are stale
    // recorded evaluation graphs (GR_EVAL_GRAPH): [0] short-range step, [1] rebuild step
    cudaGraphExec_t g_step[2] = {nullptr, nullptr};
    long long g_step_launches[2] = {0, 0};
    long long g_gen = -1;
    int* err_step_host = nullptr;  // pinned: device error flags after the last graph step
    int* err_dl_host = nullptr;    // pinned: device error flags read with the last download
    double* e_dl_host = nullptr;   // pinned: energies / virial of the last download
    int e_dl_n = 0;
    cudaEvent_t ev_step = nullptr;
    bool step_check = false;
    bool in_capture = false;  // recording a CUDA graph: the device descriptor is already current
    bool last_staged = false; // the last timed evaluation recorded its stage events (kernel by kernel)
    bool prepped_next = false; // the last MD step wrote this evaluation's water records (k_water_prep skipped)

   private:
    template <class T>
    gr_status alloc(T** p, size_t n);
    template <class T>
    gr_status upload_array(T** p, const T* host, size_t n);
    gr_status ensure_cgp_capacity();
    gr_status check_errors(cudaStream_t s, bool* retry);
    std::vector<void*> allocs;
    std::vector<std::pair<const void*, int>> occ_cache;
    int sms_cached = 0;
};

}  // namespace gnb
