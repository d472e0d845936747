// batch.cu -- many systems (REMD replicas, FEP lambda windows, serving jobs)
// stepped together on one GPU.
//
// A batch holds member contexts of uneven size.  One MD step of the whole
// batch is ONE CUDA graph launch: the graph forks one branch per member
// (force evaluation + leap-frog/SETTLE kernel on the member's own stream) and
// joins them, so the kernels of different members overlap on the GPU and
// small members fill the SMs that large ones leave idle.  Each member keeps
// its own rebuild phase (members may join at any step), so the graph of batch
// step t depends only on t mod NSNB: NSNB graphs are captured and replayed.
// Inside a recorded step a member's work depends only on whether it starts a
// pairlist period there, so phases with the same set of rebuilding members
// share one recorded graph (members on a common phase need two recordings,
// not NSNB).
// After every step a gather kernel collects the members' error flags into
// pinned host memory; a member whose lists overflowed is rolled back to the
// snapshot taken at the start of its pairlist period (inside its rebuild
// step's graph branch), its lists are grown, and its steps are re-run on its
// own, so an overflow never reaches its trajectory and never disturbs the
// other members.  Every member's arithmetic is exactly that of a standalone
// run (fixed-point sums, same kernels, same order of launches per member), so
// results are bit-identical alone and in the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <memory>

namespace gnb {

// err[0] of every member -> flags[i]
__global__ void k_gather_flags(int* const* __restrict__ err, int n, int* __restrict__ flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flags[i] = err[i][0];
}

}  // namespace gnb

struct gr_batch {
    struct Member {
        gr_ctx* ctx = nullptr;
        int offset = 0;                // member phase at batch step t = (t + offset) mod NSNB
        cudaEvent_t join = nullptr;
    };
    int device = 0;
    cudaStream_t s0 = nullptr;
    std::vector<Member> m;
    int nsnb = 0;
    long long t = 0;                   // batch MD steps done
    std::vector<cudaGraphExec_t> g;    // one graph per step phase (t mod NSNB)
    std::vector<long long> g_launches; // kernels per graph launch
    std::vector<long long> gens;       // members' allocation generations the graphs were recorded with
    bool valid = false;
    cudaEvent_t fork = nullptr, done = nullptr, t0 = nullptr, t1 = nullptr;
    int** d_errp = nullptr;            // device array of the members' err pointers
    int* d_flags = nullptr;
    int* h_flags = nullptr;            // pinned
    int cap = 0;
    long long launches = 0;
    float last_ms = 0.f;               // device time of the last gr_batch_md_run / gr_batch_eval
    long long records = 0;             // step graphs recorded (distinct graphs, every membership)
    double record_s = 0.0;             // host time spent recording and instantiating them

    void drop_graphs() {
        for (size_t i = 0; i < g.size(); ++i) {  // phases may share one graph: destroy it once
            if (!g[i]) continue;
            bool seen = false;
            for (size_t k = 0; k < i; ++k) seen = seen || g[k] == g[i];
            if (!seen) cudaGraphExecDestroy(g[i]);
        }
        g.clear();
        g_launches.clear();
        valid = false;
    }
};

namespace {

using gnb::NbSystem;

int member_phase(const gr_batch& b, const gr_batch::Member& mb) {
    return int((b.t + mb.offset) % b.nsnb);
}

gr_status batch_capacity(gr_batch* b) {
    const int n = int(b->m.size());
    if (n <= b->cap) return GR_OK;
    const int c = std::max(n, 2 * b->cap + 8);
    if (b->d_errp) cudaFree(b->d_errp);
    if (b->d_flags) cudaFree(b->d_flags);
    if (b->h_flags) cudaFreeHost(b->h_flags);
    b->d_errp = nullptr;
    b->d_flags = nullptr;
    b->h_flags = nullptr;
    GR_CUDA(cudaMalloc(&b->d_errp, sizeof(int*) * c));
    GR_CUDA(cudaMalloc(&b->d_flags, sizeof(int) * c));
    GR_CUDA(cudaMallocHost(&b->h_flags, sizeof(int) * c));
    b->cap = c;
    return GR_OK;
}

// Members that never ran get one synchronous rebuild + evaluation: it sizes
// their list capacities and performs the one-time kernel attribute set-up,
// neither of which may happen while a graph is being recorded.
gr_status batch_prepare(gr_batch* b, bool need_md) {
    gr_status st;
    for (auto& mb : b->m) {
        NbSystem& S = mb.ctx->sys;
        if (need_md && !S.md_ready) {
            set_error("gr_batch_md_run: every member needs gr_md_init first");
            return GR_ERR_STATE;
        }
        if (!S.ever_built || !S.warm) {
            if ((st = S.eval(mb.ctx->stream, GR_EVAL_FORCE_REBUILD, false))) return st;
            GR_CUDA(cudaStreamSynchronize(mb.ctx->stream));
            bool of = false;
            if ((st = S.resolve_pending(&of))) return st;
            S.warm = true;
            b->valid = false;
        }
    }
    return GR_OK;
}

gr_status batch_capture_graphs(gr_batch* b);

// Records the NSNB step graphs (host time and count kept for gr_batch_record_stats).
gr_status batch_capture(gr_batch* b) {
    const auto t0 = std::chrono::steady_clock::now();
    const gr_status st = batch_capture_graphs(b);
    b->record_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

gr_status batch_capture_graphs(gr_batch* b) {
    b->drop_graphs();
    gr_status st;
    const int n = int(b->m.size());
    if ((st = batch_capacity(b))) return st;
    std::vector<int*> errp(n);
    for (int i = 0; i < n; ++i) {
        NbSystem& S = b->m[i].ctx->sys;
        // settle every capacity now: nothing may be allocated during capture
        if ((st = S.ensure_capacity())) return st;
        if ((st = S.push_descriptor(b->m[i].ctx->stream))) return st;
        errp[i] = S.h.err;
    }
    GR_CUDA(cudaMemcpy(b->d_errp, errp.data(), sizeof(int*) * n, cudaMemcpyHostToDevice));
    for (auto& mb : b->m) GR_CUDA(cudaStreamSynchronize(mb.ctx->stream));
    for (auto& mb : b->m) mb.ctx->sys.in_capture = true;
    std::vector<long long> launches0(n);  // recording is not launching: restored below
    for (int i = 0; i < n; ++i) launches0[i] = b->m[i].ctx->sys.launches;
    b->g.assign(b->nsnb, nullptr);
    b->g_launches.assign(b->nsnb, 0);
    std::vector<std::vector<char>> rebuilds(b->nsnb, std::vector<char>(n, 0));
    for (int p = 0; p < b->nsnb; ++p)
        for (int i = 0; i < n; ++i) rebuilds[p][i] = (p + b->m[i].offset) % b->nsnb == 0;
    for (int p = 0; p < b->nsnb; ++p) {
        int same = -1;  // an earlier phase with the same rebuilding members
        for (int q = 0; q < p && same < 0; ++q)
            if (rebuilds[q] == rebuilds[p]) same = q;
        if (same >= 0) {
            b->g[p] = b->g[same];
            b->g_launches[p] = b->g_launches[same];
            continue;
        }
        long long l0 = 0;
        for (auto& mb : b->m) l0 += mb.ctx->sys.launches;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(b->s0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->s0);
        st = GR_OK;
        for (int i = 0; i < n && e == cudaSuccess && !st; ++i) {
            auto& mb = b->m[i];
            NbSystem& S = mb.ctx->sys;
            cudaStream_t si = mb.ctx->stream;
            const int ph = int((p + mb.offset) % b->nsnb);
            e = cudaStreamWaitEvent(si, b->fork, 0);
            if (e != cudaSuccess) break;
            const size_t bytes3 = size_t(S.N) * 3 * sizeof(double);
            if (ph == 0) {  // pairlist period starts: snapshot for rollback, then rebuild
                e = cudaMemcpyAsync(S.md_pos_snap, S.h.pos, bytes3, cudaMemcpyDeviceToDevice, si);
                if (e == cudaSuccess) e = cudaMemcpyAsync(S.md_vel_snap, S.md_vel, bytes3, cudaMemcpyDeviceToDevice, si);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(S.md_ke_snap, S.md_ke, sizeof(long long), cudaMemcpyDeviceToDevice, si);
                if (e != cudaSuccess) break;
                S.steps_since_update = S.prm.nsnb;
            } else {
                S.steps_since_update = 1;
            }
            S.built = true;
            S.lr_computed = true;
            S.pending_check = false;
            st = S.eval(si, 0, false);
            if (!st) st = S.md_step_launch(si);
            if (!st) e = cudaEventRecord(mb.join, si);
            if (!st && e == cudaSuccess) e = cudaStreamWaitEvent(b->s0, mb.join, 0);
        }
        if (e == cudaSuccess && !st) {
            gnb::k_gather_flags<<<(n + 255) / 256, 256, 0, b->s0>>>(b->d_errp, n, b->d_flags);
            e = cudaMemcpyAsync(b->h_flags, b->d_flags, sizeof(int) * n, cudaMemcpyDeviceToHost, b->s0);
        }
        cudaError_t e2 = cudaStreamEndCapture(b->s0, &graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess && !st) e = cudaGraphInstantiate(&b->g[p], graph, 0);
        if (e == cudaSuccess && !st) b->records += 1;
        if (graph) cudaGraphDestroy(graph);
        long long l1 = 0;
        for (auto& mb : b->m) l1 += mb.ctx->sys.launches;
        b->g_launches[p] = l1 - l0 + 1;  // + the flag gather
        if (st || e != cudaSuccess) {
            for (int i = 0; i < n; ++i) b->m[i].ctx->sys.launches = launches0[i];
            for (auto& mb : b->m) mb.ctx->sys.in_capture = false;
            b->drop_graphs();
            if (!st) {
                set_error(std::string("gr_batch: graph capture failed: ") + cudaGetErrorString(e));
                st = GR_ERR_CUDA;
            }
            return st;
        }
    }
    b->gens.resize(n);
    for (int i = 0; i < n; ++i) {
        NbSystem& S = b->m[i].ctx->sys;
        S.in_capture = false;
        S.pending_check = false;
        S.launches = launches0[i];
        b->gens[i] = S.alloc_gen;
    }
    b->valid = true;
    return GR_OK;
}

// A member whose lists overflowed during its current pairlist period: grow,
// restore its period-start snapshot and re-run its `steps` steps on its own.
gr_status batch_recover(gr_batch* b, gr_batch::Member& mb, int flags, int steps) {
    NbSystem& S = mb.ctx->sys;
    cudaStream_t si = mb.ctx->stream;
    GR_CUDA(cudaMemsetAsync(S.h.err, 0, 4 * sizeof(int), si));
    if (flags & (gnb::ERR_CELL_TOO_DENSE | gnb::ERR_CG_TOO_LARGE)) {
        set_error(flags & gnb::ERR_CELL_TOO_DENSE ? "pairlist: a grid cell holds more than 2048 charge groups"
                                                  : "pairlist: solute charge group larger than 8 atoms");
        return GR_ERR_UNSUPPORTED;
    }
    if (flags & gnb::ERR_WLIST_OVERFLOW) S.wcap_want = std::max(S.wcap_want, S.wcap_alloc) * 2;
    if (flags & gnb::ERR_SLIST_OVERFLOW) S.scap_want = std::max(S.scap_want, S.scap_alloc) * 2;
    if (flags & gnb::ERR_PERT_OVERFLOW) S.pcap_want = std::max(S.pcap_want, S.pcap_alloc) * 2;
    if (flags & gnb::ERR_DEFER_OVERFLOW) {
        S.defer_want = std::max(S.defer_want, S.h.defer_cap) * 4;
        S.clus_alloc = 0;
    }
    const size_t bytes3 = size_t(S.N) * 3 * sizeof(double);
    GR_CUDA(cudaMemcpyAsync(S.h.pos, S.md_pos_snap, bytes3, cudaMemcpyDeviceToDevice, si));
    S.prepped_next = false;
    GR_CUDA(cudaMemcpyAsync(S.md_vel, S.md_vel_snap, bytes3, cudaMemcpyDeviceToDevice, si));
    GR_CUDA(cudaMemcpyAsync(S.md_ke, S.md_ke_snap, sizeof(long long), cudaMemcpyDeviceToDevice, si));
    S.steps_since_update = S.prm.nsnb;
    S.built = false;
    S.lr_computed = false;
    S.pending_check = false;
    gr_status st = S.md_run(si, steps, nullptr);
    S.prepped_next = false;  // the batch's step graphs write their own water records
    if (st) return st;
    S.md_steps_total -= steps;  // counted once, by the batch step that failed
    S.md_rollbacks += 1;
    GR_CUDA(cudaStreamSynchronize(si));
    b->valid = false;  // capacities changed: re-record the graphs
    return GR_OK;
}

gr_batch::Member* find_member(gr_batch* b, gr_ctx* ctx) {
    for (auto& mb : b->m)
        if (mb.ctx == ctx) return &mb;
    return nullptr;
}

}  // namespace

#define BATCH_GUARD(b)                                  \
    do {                                                \
        if (!(b)) {                                     \
            set_error("null gr_batch");                 \
            return GR_ERR_INVALID;                      \
        }                                               \
        cudaError_t e_ = cudaSetDevice((b)->device);    \
        if (e_ != cudaSuccess) {                        \
            set_error(cudaGetErrorString(e_));          \
            return GR_ERR_CUDA;                         \
        }                                               \
    } while (0)

extern "C" {

gr_status gr_batch_create(int device, gr_batch** out) {
    if (!out) {
        set_error("gr_batch_create: null out");
        return GR_ERR_INVALID;
    }
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        set_error("gr_batch_create: no CUDA device");
        return GR_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        set_error("gr_batch_create: device index out of range");
        return GR_ERR_INVALID;
    }
    GR_CUDA(cudaSetDevice(device));
    auto b = std::make_unique<gr_batch>();
    b->device = device;
    GR_CUDA(cudaStreamCreateWithFlags(&b->s0, cudaStreamNonBlocking));
    GR_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    GR_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    GR_CUDA(cudaEventCreate(&b->t0));
    GR_CUDA(cudaEventCreate(&b->t1));
    *out = b.release();
    return GR_OK;
}

gr_status gr_batch_destroy(gr_batch* b) {
    if (!b) return GR_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->s0);
    b->drop_graphs();
    for (auto& mb : b->m) {
        if (mb.join) cudaEventDestroy(mb.join);
        mb.ctx->sys.batch_member = false;
    }
    if (b->d_errp) cudaFree(b->d_errp);
    if (b->d_flags) cudaFree(b->d_flags);
    if (b->h_flags) cudaFreeHost(b->h_flags);
    for (cudaEvent_t e : {b->fork, b->done, b->t0, b->t1})
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(b->s0);
    delete b;
    return GR_OK;
}

gr_status gr_batch_add(gr_batch* b, gr_ctx* ctx) {
    BATCH_GUARD(b);
    if (!ctx) {
        set_error("gr_batch_add: null ctx");
        return GR_ERR_INVALID;
    }
    NbSystem& S = ctx->sys;
    if (ctx->device != b->device) {
        set_error("gr_batch_add: member lives on another device");
        return GR_ERR_INVALID;
    }
    if (!S.uploaded || !S.params_set || !S.box_set || !S.pos_set) {
        set_error("gr_batch_add: member needs topology, parameters, box and positions");
        return GR_ERR_STATE;
    }
    if (S.prm.kernel != GR_KERNEL_FIXED) {
        set_error("gr_batch_add: batches run the fixed-point kernel");
        return GR_ERR_UNSUPPORTED;
    }
    if (find_member(b, ctx) || S.batch_member) {
        set_error("gr_batch_add: already a member of a batch");
        return GR_ERR_INVALID;
    }
    if (b->m.empty()) b->nsnb = std::max(1, S.prm.nsnb);
    if (std::max(1, S.prm.nsnb) != b->nsnb) {
        set_error("gr_batch_add: every member of a batch needs the same NSNB");
        return GR_ERR_INVALID;
    }
    gr_batch::Member mb;
    mb.ctx = ctx;
    mb.offset = int((b->nsnb - b->t % b->nsnb) % b->nsnb);  // its first batch step rebuilds
    GR_CUDA(cudaEventCreateWithFlags(&mb.join, cudaEventDisableTiming));
    S.steps_since_update = S.prm.nsnb;
    S.built = false;
    S.batch_member = true;
    b->m.push_back(mb);
    b->valid = false;
    return GR_OK;
}

gr_status gr_batch_remove(gr_batch* b, gr_ctx* ctx) {
    BATCH_GUARD(b);
    for (size_t i = 0; i < b->m.size(); ++i)
        if (b->m[i].ctx == ctx) {
            GR_CUDA(cudaStreamSynchronize(b->s0));
            NbSystem& S = ctx->sys;
            const int ph = member_phase(*b, b->m[i]);
            S.steps_since_update = ph == 0 ? S.prm.nsnb : ph;  // standalone use continues the cadence
            if (b->m[i].join) cudaEventDestroy(b->m[i].join);
            S.batch_member = false;
            b->m.erase(b->m.begin() + long(i));
            b->valid = false;
            return GR_OK;
        }
    set_error("gr_batch_remove: not a member");
    return GR_ERR_INVALID;
}

gr_status gr_batch_size(gr_batch* b, int32_t* n) {
    BATCH_GUARD(b);
    if (!n) return GR_ERR_INVALID;
    *n = int32_t(b->m.size());
    return GR_OK;
}

// n MD steps of every member: one graph launch per step.
gr_status gr_batch_md_run(gr_batch* b, int32_t n_steps) {
    BATCH_GUARD(b);
    if (n_steps < 0) {
        set_error("gr_batch_md_run: n_steps must be >= 0");
        return GR_ERR_INVALID;
    }
    b->last_ms = 0.f;
    if (b->m.empty() || n_steps == 0) return GR_OK;
    gr_status st;
    if ((st = batch_prepare(b, true))) return st;
    float total_ms = 0.f;
    for (int k = 0; k < n_steps; ++k) {
        // a member reallocated since the graphs were recorded (parameters,
        // list growth): record them again
        if (b->valid)
            for (size_t i = 0; i < b->m.size(); ++i)
                if (b->gens[i] != b->m[i].ctx->sys.alloc_gen) b->valid = false;
        if (!b->valid && (st = batch_capture(b))) return st;
        const int p = int(b->t % b->nsnb);
        GR_CUDA(cudaEventRecord(b->t0, b->s0));
        GR_CUDA(cudaGraphLaunch(b->g[p], b->s0));
        GR_CUDA(cudaEventRecord(b->t1, b->s0));
        b->launches += b->g_launches[p];
        GR_CUDA(cudaEventSynchronize(b->t1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->t0, b->t1);
        total_ms += ms;
        for (auto& mb : b->m) mb.ctx->sys.md_steps_total += 1;
        for (size_t i = 0; i < b->m.size(); ++i) {
            const int f = b->h_flags[i];
            if (!f) continue;
            auto& mb = b->m[i];
            const int ph = member_phase(*b, mb);  // phase of the step just run
            if ((st = batch_recover(b, mb, f, ph + 1))) return st;
        }
        b->t += 1;
    }
    b->last_ms = total_ms;
    return GR_OK;
}

// One force evaluation of every member (no MD); results per member through
// gr_result_download.  Members are evaluated concurrently on their streams.
gr_status gr_batch_eval(gr_batch* b, int32_t flags) {
    BATCH_GUARD(b);
    gr_status st;
    if ((st = batch_prepare(b, false))) return st;
    GR_CUDA(cudaEventRecord(b->t0, b->s0));
    GR_CUDA(cudaEventRecord(b->fork, b->s0));
    for (auto& mb : b->m) {
        GR_CUDA(cudaStreamWaitEvent(mb.ctx->stream, b->fork, 0));
        if ((st = mb.ctx->sys.eval(mb.ctx->stream, flags & ~GR_EVAL_NO_DOWNLOAD, false))) return st;
        GR_CUDA(cudaEventRecord(mb.join, mb.ctx->stream));
        GR_CUDA(cudaStreamWaitEvent(b->s0, mb.join, 0));
    }
    GR_CUDA(cudaEventRecord(b->t1, b->s0));
    GR_CUDA(cudaEventSynchronize(b->t1));
    cudaEventElapsedTime(&b->last_ms, b->t0, b->t1);
    // overflow check per member; a member that overflowed is evaluated again
    // through the retrying single-system path
    for (auto& mb : b->m) {
        NbSystem& S = mb.ctx->sys;
        int e[4] = {0, 0, 0, 0};
        GR_CUDA(cudaMemcpy(e, S.h.err, sizeof(e), cudaMemcpyDeviceToHost));
        bool of = false;
        if ((st = S.resolve_pending(&of))) return st;
        if (e[0] & gnb::ERR_DEFER_OVERFLOW) {
            GR_CUDA(cudaMemset(S.h.err, 0, sizeof(e)));
            S.defer_want = std::max(S.defer_want, S.h.defer_cap) * 4;
            S.clus_alloc = 0;
            S.built = false;
            S.lr_computed = false;
            of = true;
        }
        if (of) {
            gr_result r{};
            r.n_pairs_short = -1;
            S.steps_since_update = S.prm.nsnb;  // the failed evaluation's rebuild is redone
            if ((st = gr_forces_eval(mb.ctx, flags & ~GR_EVAL_NO_DOWNLOAD, &r))) return st;
        }
    }
    b->valid = false;  // member cadences moved outside the graphs
    return GR_OK;
}

gr_status gr_batch_last_ms(gr_batch* b, float* ms) {
    BATCH_GUARD(b);
    if (!ms) return GR_ERR_INVALID;
    *ms = b->last_ms;
    return GR_OK;
}

gr_status gr_batch_record_stats(gr_batch* b, int64_t* graphs, double* seconds) {
    BATCH_GUARD(b);
    if (!graphs || !seconds) return GR_ERR_INVALID;
    *graphs = b->records;
    *seconds = b->record_s;
    return GR_OK;
}

gr_status gr_batch_phase(gr_batch* b, int32_t* phase, int32_t* period) {
    BATCH_GUARD(b);
    if (!phase || !period) return GR_ERR_INVALID;
    *period = b->nsnb > 0 ? b->nsnb : 1;
    *phase = -1;
    for (size_t i = 0; i < b->m.size(); ++i) {
        const int ph = member_phase(*b, b->m[i]);
        if (i == 0) *phase = ph;
        else if (ph != *phase) {
            *phase = -1;
            break;
        }
    }
    return GR_OK;
}

gr_status gr_batch_launches(gr_batch* b, int64_t* n) {
    BATCH_GUARD(b);
    if (!n) return GR_ERR_INVALID;
    *n = b->launches;
    return GR_OK;
}

gr_status gr_ctx_device_bytes(gr_ctx* ctx, int64_t* bytes) {
    CTX_GUARD(ctx);
    if (!bytes) return GR_ERR_INVALID;
    *bytes = int64_t(ctx->sys.bytes);
    return GR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner: picks the solvent kernel variant (lane layout and i-cluster
// width) by timing full pairlist periods (one rebuild + long-range refresh +
// NSNB short-range steps) of the systems themselves.  The rebuild interval is
// not tuned: with the reference's twin-range scheme (no skin) NSNB decides
// which pairs are evaluated, so changing it would change the results.
namespace {

struct Variant {
    int layout, width;
};
constexpr Variant kVariants[] = {{2, 4}, {2, 8}, {1, 4}, {3, 4}};
constexpr int kNumVariants = int(sizeof(kVariants) / sizeof(kVariants[0]));

// `periods` timed pairlist periods of every member, concurrently on their
// streams; returns device ms per step.
gr_status time_periods(std::vector<gr_ctx*>& ms, cudaStream_t s0, cudaEvent_t fork,
                       std::vector<cudaEvent_t>& joins, cudaEvent_t t0, cudaEvent_t t1, int nsnb, int periods,
                       float* ms_per_step) {
    gr_status st;
    GR_CUDA(cudaEventRecord(t0, s0));
    for (int p = 0; p < periods; ++p)
        for (int k = 0; k < nsnb; ++k) {
            GR_CUDA(cudaEventRecord(fork, s0));
            for (size_t i = 0; i < ms.size(); ++i) {
                NbSystem& S = ms[i]->sys;
                GR_CUDA(cudaStreamWaitEvent(ms[i]->stream, fork, 0));
                if ((st = S.eval(ms[i]->stream, k == 0 ? GR_EVAL_FORCE_REBUILD : 0, false))) return st;
                GR_CUDA(cudaEventRecord(joins[i], ms[i]->stream));
                GR_CUDA(cudaStreamWaitEvent(s0, joins[i], 0));
            }
        }
    GR_CUDA(cudaEventRecord(t1, s0));
    GR_CUDA(cudaEventSynchronize(t1));
    float t = 0.f;
    GR_CUDA(cudaEventElapsedTime(&t, t0, t1));
    *ms_per_step = t / float(periods * nsnb);
    return GR_OK;
}

gr_status autotune(std::vector<gr_ctx*>& ms, cudaStream_t s0, cudaEvent_t fork, std::vector<cudaEvent_t>& joins,
                   cudaEvent_t t0, cudaEvent_t t1, int periods, gr_autotune_result* out) {
    if (ms.empty()) {
        set_error("autotune: nothing to tune");
        return GR_ERR_STATE;
    }
    const int nsnb = std::max(1, ms[0]->sys.prm.nsnb);
    periods = std::max(1, periods);
    gr_autotune_result r{};
    float best = 3.0e38f;
    int best_k = -1;
    gr_status st;
    for (int k = 0; k < kNumVariants; ++k) {
        r.cand_layout[k] = kVariants[k].layout;
        r.cand_cluster_size[k] = kVariants[k].width;
        r.cand_ms_per_step[k] = -1.f;
        bool ok = true;
        for (gr_ctx* c : ms) {
            gr_nb_params p = c->sys.prm;
            p.water_layout = kVariants[k].layout;
            p.cluster_size = kVariants[k].width;
            if (c->sys.set_params(&p) != GR_OK) ok = false;
        }
        if (!ok) continue;
        float t = 0.f;
        // one untimed period: list growth and one-time kernel set-up happen here
        if ((st = time_periods(ms, s0, fork, joins, t0, t1, nsnb, 1, &t))) return st;
        if ((st = time_periods(ms, s0, fork, joins, t0, t1, nsnb, periods, &t))) return st;
        r.cand_ms_per_step[k] = t;
        if (t < best) {
            best = t;
            best_k = k;
        }
    }
    r.n_candidates = kNumVariants;
    if (best_k < 0) {
        set_error("autotune: no variant applies");
        return GR_ERR_UNSUPPORTED;
    }
    for (gr_ctx* c : ms) {
        gr_nb_params p = c->sys.prm;
        p.water_layout = kVariants[best_k].layout;
        p.cluster_size = kVariants[best_k].width;
        if ((st = c->sys.set_params(&p))) return st;
        bool of = false;
        GR_CUDA(cudaStreamSynchronize(c->stream));
        if ((st = c->sys.resolve_pending(&of))) return st;
        GR_CUDA(cudaMemset(c->sys.h.err, 0, 4 * sizeof(int)));  // trial overflows were absorbed by re-runs
        c->sys.steps_since_update = c->sys.prm.nsnb;           // the next step rebuilds
    }
    r.water_layout = kVariants[best_k].layout;
    r.cluster_size = kVariants[best_k].width;
    if (out) *out = r;
    return GR_OK;
}

}  // namespace

extern "C" {

gr_status gr_autotune(gr_ctx* ctx, int32_t periods, gr_autotune_result* out) {
    CTX_GUARD(ctx);
    if (!ctx->sys.uploaded || !ctx->sys.params_set || !ctx->sys.box_set || !ctx->sys.pos_set) {
        set_error("gr_autotune: needs topology, parameters, box and positions");
        return GR_ERR_STATE;
    }
    if (ctx->sys.prm.kernel != GR_KERNEL_FIXED) {
        set_error("gr_autotune: tunes the fixed-point kernel");
        return GR_ERR_UNSUPPORTED;
    }
    std::vector<gr_ctx*> ms{ctx};
    cudaEvent_t fork = nullptr, join = nullptr, t0 = nullptr, t1 = nullptr;
    GR_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    GR_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    GR_CUDA(cudaEventCreate(&t0));
    GR_CUDA(cudaEventCreate(&t1));
    std::vector<cudaEvent_t> joins{join};
    cudaStream_t s0 = nullptr;
    GR_CUDA(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
    gr_status st = autotune(ms, s0, fork, joins, t0, t1, periods, out);
    cudaStreamSynchronize(s0);
    cudaStreamDestroy(s0);
    for (cudaEvent_t e : {fork, join, t0, t1}) cudaEventDestroy(e);
    return st;
}

gr_status gr_batch_set_variant(gr_batch* b, int32_t water_layout, int32_t cluster_size) {
    BATCH_GUARD(b);
    gr_status st;
    for (auto& mb : b->m) {
        NbSystem& S = mb.ctx->sys;
        gr_nb_params p = S.prm;
        p.water_layout = water_layout;
        p.cluster_size = cluster_size;
        if ((st = S.set_params(&p))) return st;
        S.steps_since_update = S.prm.nsnb;  // the next step rebuilds
    }
    for (auto& mb : b->m) mb.offset = int((b->nsnb - b->t % b->nsnb) % b->nsnb);  // every member rebuilds next
    b->valid = false;
    return GR_OK;
}

gr_status gr_batch_autotune(gr_batch* b, int32_t periods, gr_autotune_result* out) {
    BATCH_GUARD(b);
    std::vector<gr_ctx*> ms;
    std::vector<cudaEvent_t> joins;
    for (auto& mb : b->m) {
        ms.push_back(mb.ctx);
        joins.push_back(mb.join);
    }
    gr_status st = autotune(ms, b->s0, b->fork, joins, b->t0, b->t1, periods, out);
    if (st) return st;
    for (auto& mb : b->m) mb.offset = int((b->nsnb - b->t % b->nsnb) % b->nsnb);  // every member rebuilds next
    b->valid = false;
    return GR_OK;
}

}  // extern "C"
