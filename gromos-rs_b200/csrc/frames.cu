// frames.cu -- nonbonded energies of many configurations (trajectory frames).
//
// single_point_energy (crates/gromos-forces/src/energy.rs:96-239), nonbonded
// part, for a whole trajectory in one call (the loop of the ener analysis,
// crates/gromos-analysis/src/bin/energy/ener.rs:106-124): each frame's
// positions (and box) are copied in stream order, the pairlist is built from
// scratch and the LJ and CRF energies (incl. the RF-excluded and 1-4 terms)
// per energy group are gathered in device memory.  single_point_energy uses
// one cutoff for both ranges and no skin; the caller sets rcutp = rcutl =
// cutoff and skin 0 in the context's parameters (with a twin-range setting
// every frame is evaluated with both ranges, as a first MD step is).
//
// One frame is in flight while the host checks the one before it: its
// pairlist overflow flags (read asynchronously by the build) and its
// deferred-pair flag (copied to pinned memory after the frame); a frame that
// overflowed is computed again once the capacities have grown.
#include <deque>

extern "C" gr_status gr_energy_frames(gr_ctx* ctx, int32_t n_frames, const double* frames, const double* boxes,
                                      double* e_lj, double* e_crf, double* egroup_lj, double* egroup_crf) {
    CTX_GUARD(ctx);
    NbSystem& S = ctx->sys;
    if (n_frames < 0 || (n_frames > 0 && (!frames || !e_lj || !e_crf))) {
        set_error("gr_energy_frames: need n_frames >= 0, frames and the energy outputs");
        return GR_ERR_INVALID;
    }
    if (!S.uploaded || !S.params_set || (!boxes && !S.box_set)) {
        set_error("gr_energy_frames before gr_system_upload / gr_set_params (and gr_set_box without boxes)");
        return GR_ERR_STATE;
    }
    if (n_frames == 0) return GR_OK;
    cudaStream_t st = ctx->stream;
    const int G = S.G, NA = acc_size(G);
    const size_t n3 = size_t(S.N) * 3;
    double* dE = nullptr;
    int* pin_err = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    gr_status r = GR_OK;
    auto cleanup = [&]() {
        if (dE) cudaFree(dE);
        if (pin_err) cudaFreeHost(pin_err);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    };
    if (cudaMalloc(&dE, size_t(n_frames) * NA * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        dE = nullptr;
        set_error("gr_energy_frames: device allocation of the per-frame energies failed");
        return GR_ERR_OOM;
    }
    if (cudaMallocHost(&pin_err, 8 * sizeof(int)) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        set_error("gr_energy_frames: could not create pinned flags / events");
        return GR_ERR_CUDA;
    }
#define FR_CUDA(call)                            \
    do {                                         \
        cudaError_t e_ = (call);                 \
        if (e_ != cudaSuccess) {                 \
            set_error(cudaGetErrorString(e_));   \
            return GR_ERR_CUDA;                  \
        }                                        \
    } while (0)
    // frame f into flag slot `slot`: box, positions, rebuild + evaluation,
    // energies to dE[f], flags to pinned memory, flags cleared
    auto enqueue = [&](int f, int slot) -> gr_status {
        gr_status q;
        if (boxes && (q = S.set_box(boxes + 3 * size_t(f)))) return q;
        FR_CUDA(cudaMemcpyAsync(S.h.pos, frames + n3 * size_t(f), n3 * sizeof(double), cudaMemcpyHostToDevice, st));
        S.pos_set = true;
        S.prepped_next = false;
        if ((q = S.eval(st, GR_EVAL_FORCE_REBUILD, false))) return q;
        FR_CUDA(cudaMemcpyAsync(dE + size_t(f) * NA, S.h.e_out, NA * sizeof(double), cudaMemcpyDeviceToDevice, st));
        FR_CUDA(cudaMemcpyAsync(pin_err + 4 * slot, S.h.err, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
        FR_CUDA(cudaMemsetAsync(S.h.err, 0, 4 * sizeof(int), st));
        FR_CUDA(cudaEventRecord(ev[slot], st));
        return GR_OK;
    };
    // the deferred-pair flag of the frame in `slot` (after its event); a set
    // flag grows the list as gr_forces_eval does
    auto deferred_overflow = [&](int slot, bool* bad) -> gr_status {
        FR_CUDA(cudaEventSynchronize(ev[slot]));
        if (pin_err[4 * slot] & gnb::ERR_DEFER_OVERFLOW) {
            S.defer_want = std::max(S.defer_want, S.h.defer_cap) * 4;
            S.clus_alloc = 0;
            S.built = false;
            *bad = true;
        }
        return GR_OK;
    };
#undef FR_CUDA
    std::deque<int> todo;
    for (int f = 0; f < n_frames; ++f) todo.push_back(f);
    int inflight = -1, in_slot = 0, next_slot = 0, redo = 0;
    while (!todo.empty() || inflight >= 0) {
        bool bad = false;
        // the in-flight frame's pairlist flags: waits for its build only
        if (inflight >= 0 && (r = S.resolve_pending(&bad))) break;
        int f = -1, slot = next_slot;
        if (!todo.empty()) {
            f = todo.front();
            todo.pop_front();
            if ((r = enqueue(f, slot))) break;
            next_slot ^= 1;
        }
        if (inflight >= 0) {
            if ((r = deferred_overflow(in_slot, &bad))) break;
            if (bad) {
                if (++redo > 16 + n_frames) {
                    set_error("gr_energy_frames: list capacities could not be grown far enough");
                    r = GR_ERR_OVERFLOW;
                    break;
                }
                todo.push_front(inflight);
            }
        }
        inflight = f;
        in_slot = slot;
    }
    if (r) {
        cudaStreamSynchronize(st);
        cleanup();
        return r;
    }
    std::vector<double> e(size_t(n_frames) * NA);
    if (cudaMemcpyAsync(e.data(), dE, e.size() * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        set_error(cudaGetErrorString(cudaGetLastError()));
        cleanup();
        return GR_ERR_CUDA;
    }
    cleanup();
    for (int f = 0; f < n_frames; ++f) {
        const double* ef = e.data() + size_t(f) * NA;
        double lj = 0, crf = 0;
        for (int a = 0; a < G; ++a)
            for (int b = a; b < G; ++b) {
                lj += ef[a * G + b];
                crf += ef[G * G + a * G + b];
            }
        e_lj[f] = lj;
        e_crf[f] = crf;
        if (egroup_lj)
            for (int k = 0; k < G * G; ++k) egroup_lj[size_t(f) * G * G + k] = ef[k];
        if (egroup_crf)
            for (int k = 0; k < G * G; ++k) egroup_crf[size_t(f) * G * G + k] = ef[G * G + k];
    }
    return GR_OK;
}
