// server.cu -- native MD job server: continuous batching on one GPU.
//
// Jobs are submitted with their topology, parameters, coordinates and MD
// settings (copied, so the caller's buffers are free after the call) and wait
// in a queue on the host.  Each gr_server_step admits queued jobs while the
// device bytes of the resident jobs plus the next job stay within the HBM
// budget, runs one chunk of MD steps for every resident job through one
// gr_batch (one CUDA graph launch per step for all of them), and retires the
// jobs that have finished: their final state is copied out and their device
// memory freed at once.  A job submitted while others run joins them at the
// next step call.  Admission estimates a job's bytes from the largest
// bytes-per-atom seen so far, then builds its pairlist (which sizes the lists)
// and checks the measured bytes; a job that does not fit after all is released
// and waits.  Every job's trajectory is bit-identical to a standalone run.
// A job whose setup fails (bad topology or parameters, a footprint above the
// whole budget, or no device memory with nothing else resident to wait for)
// is marked failed with its status and message and leaves the queue, so one
// bad submission never blocks the jobs behind it.
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <string>

namespace {

// Deep copy of a gr_topology (the caller's arrays may go away after submit).
struct HostTopology {
    gr_topology t{};
    std::vector<int32_t> cg_off, iac, excl_off, excl, o14_off, o14, egroup;
    std::vector<double> charge, lj;
    std::vector<gr_perturbed_atom> pert;
    std::vector<gr_perturbed_pair> pp;

    template <class T>
    static void take(std::vector<T>& v, const T* p, size_t n) {
        v.assign(p ? p : nullptr, p ? p + n : nullptr);
    }
    void copy_from(const gr_topology& s) {
        t = s;
        const size_t n = size_t(std::max(0, s.n_atoms)), ncg = size_t(std::max(0, s.n_chargegroups));
        take(cg_off, s.cg_offsets, ncg + 1);
        take(charge, s.charge, n);
        take(iac, s.iac, n);
        take(lj, s.lj, size_t(std::max(0, s.n_types)) * size_t(std::max(0, s.n_types)) * 4);
        take(excl_off, s.excl_offsets, n + 1);
        take(excl, s.excl, s.excl_offsets ? size_t(s.excl_offsets[n]) : 0);
        take(o14_off, s.o14_offsets, s.o14_offsets ? n + 1 : 0);
        take(o14, s.o14, s.o14_offsets ? size_t(s.o14_offsets[n]) : 0);
        take(egroup, s.energy_group, s.energy_group ? n : 0);
        take(pert, s.perturbed, size_t(std::max(0, s.n_perturbed)));
        take(pp, s.perturbed_pairs, size_t(std::max(0, s.n_perturbed_pairs)));
        t.cg_offsets = cg_off.data();
        t.charge = charge.data();
        t.iac = iac.data();
        t.lj = lj.data();
        t.excl_offsets = excl_off.data();
        t.excl = excl.empty() ? nullptr : excl.data();
        t.o14_offsets = o14_off.empty() ? nullptr : o14_off.data();
        t.o14 = o14.empty() ? nullptr : o14.data();
        t.energy_group = egroup.empty() ? nullptr : egroup.data();
        t.perturbed = pert.empty() ? nullptr : pert.data();
        t.perturbed_pairs = pp.empty() ? nullptr : pp.data();
    }
};

struct Job {
    int64_t id = 0;
    HostTopology topo;
    gr_nb_params params{};
    gr_md_params md{};
    double box[3] = {0, 0, 0};
    std::vector<double> pos, vel, mass;
    int64_t n_steps = 0, steps_done = 0;
    int32_t state = GR_JOB_QUEUED;
    double t_submit = 0, t_admit = -1, t_done = -1;
    int64_t bytes = 0;
    gr_ctx* ctx = nullptr;
    gr_md_stats stats{};
    gr_status error = GR_OK;
    std::string message;
};

}  // namespace

struct gr_server {
    int device = 0;
    int64_t budget = 0;
    int chunk = 5;
    gr_batch* batch = nullptr;
    std::deque<int64_t> queue;
    std::map<int64_t, Job> jobs;
    std::vector<int64_t> resident;
    int64_t next_id = 1, resident_bytes = 0, max_resident_bytes = 0, steps_run = 0;
    int32_t max_resident_jobs = 0;
    int64_t joined_running = 0;  // admitted while resident jobs had already stepped
    double bytes_per_atom = 8192.0;
    bool measured = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

void destroy_job_ctx(Job& j) {
    if (j.ctx) {
        gr_ctx_destroy(j.ctx);
        j.ctx = nullptr;
    }
}

// A context for the job with its pairlist built (lists sized): its device
// bytes are then the job's resident footprint.
gr_status make_job_ctx(gr_server* srv, Job& j) {
    gr_status st;
    gr_ctx* c = nullptr;
    if ((st = gr_ctx_create(srv->device, &c))) return st;
    if ((st = gr_system_upload(c, &j.topo.t)) || (st = gr_set_params(c, &j.params)) || (st = gr_set_box(c, j.box)) ||
        (st = gr_positions_upload(c, j.pos.data())) || (st = gr_pairlist_build(c)) ||
        (st = gr_md_init(c, j.mass.data(), j.vel.data(), &j.md))) {
        gr_ctx_destroy(c);
        return st;
    }
    j.ctx = c;
    j.bytes = int64_t(c->sys.bytes);
    return GR_OK;
}

void fail_job(gr_server* srv, Job& j, gr_status st, const char* msg) {
    destroy_job_ctx(j);
    j.state = GR_JOB_FAILED;
    j.error = st;
    j.message = msg ? msg : "";
    j.t_done = srv->now();
}

gr_status admit(gr_server* srv) {
    while (!srv->queue.empty()) {
        Job& j = srv->jobs[srv->queue.front()];
        const int64_t est = int64_t(double(j.topo.t.n_atoms) * srv->bytes_per_atom);
        if (!srv->resident.empty() && srv->resident_bytes + est > srv->budget) return GR_OK;
        gr_status st = make_job_ctx(srv, j);
        if (st == GR_ERR_OOM && !srv->resident.empty()) return GR_OK;  // wait for resident jobs to finish
        if (st) {
            fail_job(srv, j, st, gr_last_error());
            srv->queue.pop_front();
            continue;
        }
        const double per_atom = double(j.bytes) / double(std::max(1, j.topo.t.n_atoms));
        srv->bytes_per_atom = srv->measured ? std::max(srv->bytes_per_atom, per_atom) : per_atom;
        srv->measured = true;
        if (j.bytes > srv->budget) {
            fail_job(srv, j, GR_ERR_OOM, "job's device footprint exceeds the server's HBM budget");
            srv->queue.pop_front();
            continue;
        }
        if (srv->resident_bytes + j.bytes > srv->budget) {
            destroy_job_ctx(j);  // does not fit after all: wait for memory
            return GR_OK;
        }
        bool running = false;
        for (int64_t id : srv->resident) running = running || srv->jobs[id].steps_done > 0;
        if ((st = gr_batch_add(srv->batch, j.ctx))) {
            destroy_job_ctx(j);
            return st;
        }
        srv->joined_running += running ? 1 : 0;
        srv->queue.pop_front();
        j.state = GR_JOB_RUNNING;
        j.t_admit = srv->now();
        srv->resident.push_back(j.id);
        srv->resident_bytes += j.bytes;
        srv->max_resident_bytes = std::max(srv->max_resident_bytes, srv->resident_bytes);
        srv->max_resident_jobs = std::max(srv->max_resident_jobs, int32_t(srv->resident.size()));
    }
    return GR_OK;
}

gr_status retire(gr_server* srv) {
    gr_status st;
    for (size_t i = 0; i < srv->resident.size();) {
        Job& j = srv->jobs[srv->resident[i]];
        if (j.steps_done < j.n_steps) {
            ++i;
            continue;
        }
        if ((st = gr_batch_remove(srv->batch, j.ctx))) return st;
        const size_t n3 = size_t(j.topo.t.n_atoms) * 3;
        j.pos.assign(n3, 0.0);
        j.vel.assign(n3, 0.0);
        if ((st = gr_md_download(j.ctx, j.pos.data(), j.vel.data()))) return st;
        if ((st = gr_md_stats_get(j.ctx, &j.stats))) return st;
        destroy_job_ctx(j);
        srv->resident_bytes -= j.bytes;
        j.state = GR_JOB_DONE;
        j.t_done = srv->now();
        srv->resident.erase(srv->resident.begin() + long(i));
    }
    return GR_OK;
}

}  // namespace

#define SERVER_GUARD(srv)                               \
    do {                                                \
        if (!(srv)) {                                   \
            set_error("null gr_server");                \
            return GR_ERR_INVALID;                      \
        }                                               \
        cudaError_t e_ = cudaSetDevice((srv)->device);  \
        if (e_ != cudaSuccess) {                        \
            set_error(cudaGetErrorString(e_));          \
            return GR_ERR_CUDA;                         \
        }                                               \
    } while (0)

extern "C" {

gr_status gr_server_create(int device, int64_t hbm_budget_bytes, int32_t chunk_steps, gr_server** out) {
    if (!out || hbm_budget_bytes <= 0 || chunk_steps <= 0) {
        set_error("gr_server_create: need out, a positive budget and chunk_steps");
        return GR_ERR_INVALID;
    }
    *out = nullptr;
    gr_batch* b = nullptr;
    gr_status st = gr_batch_create(device, &b);
    if (st) return st;
    auto* s = new gr_server;
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->chunk = chunk_steps;
    s->batch = b;
    *out = s;
    return GR_OK;
}

gr_status gr_server_destroy(gr_server* srv) {
    if (!srv) return GR_OK;
    cudaSetDevice(srv->device);
    for (int64_t id : srv->resident) {
        Job& j = srv->jobs[id];
        gr_batch_remove(srv->batch, j.ctx);
        destroy_job_ctx(j);
    }
    gr_batch_destroy(srv->batch);
    delete srv;
    return GR_OK;
}

gr_status gr_server_submit(gr_server* srv, const gr_job_desc* job, int64_t* job_id) {
    SERVER_GUARD(srv);
    if (!job || !job->topo || !job->params || !job->box || !job->pos || !job->mass || !job->md || job->n_steps < 0) {
        set_error("gr_server_submit: incomplete job description");
        return GR_ERR_INVALID;
    }
    const int n = job->topo->n_atoms;
    if (n <= 0 || job->params->kernel != GR_KERNEL_FIXED) {
        set_error("gr_server_submit: jobs need atoms and the fixed-point kernel");
        return GR_ERR_INVALID;
    }
    Job j;
    j.id = srv->next_id++;
    j.topo.copy_from(*job->topo);
    j.params = *job->params;
    j.md = *job->md;
    for (int k = 0; k < 3; ++k) j.box[k] = job->box[k];
    j.pos.assign(job->pos, job->pos + size_t(n) * 3);
    j.mass.assign(job->mass, job->mass + size_t(n));
    if (job->vel)
        j.vel.assign(job->vel, job->vel + size_t(n) * 3);
    else
        j.vel.assign(size_t(n) * 3, 0.0);
    j.n_steps = job->n_steps;
    j.t_submit = srv->now();
    const int64_t id = j.id;
    srv->jobs.emplace(id, std::move(j));  // moving the vectors keeps the topology's pointers valid
    srv->queue.push_back(id);
    if (job_id) *job_id = id;
    return GR_OK;
}

gr_status gr_server_step(gr_server* srv, int32_t* n_running) {
    SERVER_GUARD(srv);
    gr_status st;
    if ((st = admit(srv))) return st;
    if (!srv->resident.empty()) {
        int64_t n = srv->chunk;
        for (int64_t id : srv->resident) n = std::min(n, srv->jobs[id].n_steps - srv->jobs[id].steps_done);
        if (n > 0) {
            if ((st = gr_batch_md_run(srv->batch, int32_t(n)))) return st;
            srv->steps_run += n;
        }
        for (int64_t id : srv->resident) srv->jobs[id].steps_done += n;
        if ((st = retire(srv))) return st;
    }
    if (n_running) *n_running = int32_t(srv->resident.size());
    return GR_OK;
}

gr_status gr_server_job(gr_server* srv, int64_t job_id, gr_job_status* out, double* pos, double* vel) {
    SERVER_GUARD(srv);
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end()) {
        set_error("gr_server_job: unknown job");
        return GR_ERR_INVALID;
    }
    const Job& j = it->second;
    if (out) {
        out->state = j.state;
        out->steps_done = j.steps_done;
        out->t_submit = j.t_submit;
        out->t_admit = j.t_admit;
        out->t_done = j.t_done;
        out->device_bytes = j.bytes;
        out->stats = j.stats;
        out->error = j.error;
        std::memset(out->message, 0, sizeof(out->message));
        std::strncpy(out->message, j.message.c_str(), sizeof(out->message) - 1);
    }
    if ((pos || vel) && j.state != GR_JOB_DONE) {
        set_error("gr_server_job: coordinates are available once the job is done");
        return GR_ERR_STATE;
    }
    const size_t n3 = size_t(j.topo.t.n_atoms) * 3;
    if (pos) std::copy(j.pos.begin(), j.pos.begin() + long(n3), pos);
    if (vel) std::copy(j.vel.begin(), j.vel.begin() + long(n3), vel);
    return GR_OK;
}

gr_status gr_server_cancel(gr_server* srv, int64_t job_id) {
    SERVER_GUARD(srv);
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end()) {
        set_error("gr_server_cancel: unknown job");
        return GR_ERR_INVALID;
    }
    Job& j = it->second;
    if (j.state == GR_JOB_QUEUED) {
        srv->queue.erase(std::find(srv->queue.begin(), srv->queue.end(), job_id));
    } else if (j.state == GR_JOB_RUNNING) {
        gr_status st = gr_batch_remove(srv->batch, j.ctx);
        if (st) return st;
        destroy_job_ctx(j);
        srv->resident_bytes -= j.bytes;
        srv->resident.erase(std::find(srv->resident.begin(), srv->resident.end(), job_id));
    } else {
        set_error("gr_server_cancel: the job has already ended");
        return GR_ERR_STATE;
    }
    j.state = GR_JOB_CANCELLED;
    j.t_done = srv->now();
    return GR_OK;
}

gr_status gr_server_release(gr_server* srv, int64_t job_id) {
    SERVER_GUARD(srv);
    auto it = srv->jobs.find(job_id);
    if (it == srv->jobs.end() || it->second.state < GR_JOB_DONE) {
        set_error("gr_server_release: not an ended job");
        return GR_ERR_STATE;
    }
    srv->jobs.erase(it);
    return GR_OK;
}

gr_status gr_server_stats(gr_server* srv, gr_server_stats_t* out) {
    SERVER_GUARD(srv);
    if (!out) return GR_ERR_INVALID;
    std::vector<double> lat;
    out->jobs_failed = out->jobs_cancelled = 0;
    for (const auto& kv : srv->jobs) {
        if (kv.second.state == GR_JOB_DONE) lat.push_back(kv.second.t_done - kv.second.t_submit);
        out->jobs_failed += kv.second.state == GR_JOB_FAILED;
        out->jobs_cancelled += kv.second.state == GR_JOB_CANCELLED;
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
        if (lat.empty()) return 0.0;
        const double r = q * double(lat.size() - 1);
        const size_t lo = size_t(r), hi = std::min(lat.size() - 1, lo + 1);
        return lat[lo] + (lat[hi] - lat[lo]) * (r - double(lo));
    };
    out->jobs_done = int64_t(lat.size());
    out->jobs_queued = int64_t(srv->queue.size());
    out->jobs_running = int64_t(srv->resident.size());
    out->latency_p50_s = pct(0.50);
    out->latency_p99_s = pct(0.99);
    out->resident_bytes = srv->resident_bytes;
    out->max_resident_bytes = srv->max_resident_bytes;
    out->max_resident_jobs = srv->max_resident_jobs;
    out->batch_steps = srv->steps_run;
    out->jobs_joined_running = srv->joined_running;
    return GR_OK;
}

}  // extern "C"
