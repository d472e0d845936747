/*
 * gromos_nb.h -- C ABI of the B200 nonbonded library (libgromos_nb.so).
 *
 * This is the drop-in boundary for gromos-rs's nonbonded hot path: the
 * charge-group twin-range pairlist and the Lennard-Jones + reaction-field
 * (LJ/CRF) force / energy / virial evaluation, with the soft-core FEP
 * corrections.  Every entry point names the gromos-rs interface it replaces
 * (paths relative to the gromos-rs repository).  A Rust `-sys` crate binds
 * these declarations one to one; ctypes does the same from Python.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Host pointers unless a name says
 *    "device".  The library owns all device memory; the caller owns host
 *    buffers.
 *  - Every call returns gr_status (0 = GR_OK).  gr_last_error() returns a
 *    thread-local message for the last failing call on this thread.
 *  - One context per host thread (or an external lock).  All work of a
 *    context runs on its own CUDA stream.
 *  - Positions are FP64 xyz triples (the layout of gromos-rs `Vec3 = DVec3`),
 *    forces are returned as FP64 xyz triples.
 *  - Charge groups are contiguous atom ranges given by offsets; solute CGs
 *    first, then one CG per solvent molecule (gromos-rs Topology order).
 */
#ifndef GROMOS_NB_H
#define GROMOS_NB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gr_status;
enum {
    GR_OK = 0,
    GR_ERR_INVALID = 1,      /* bad argument or inconsistent topology */
    GR_ERR_CUDA = 2,         /* CUDA runtime error */
    GR_ERR_OOM = 3,          /* device allocation failed / over budget */
    GR_ERR_STATE = 4,        /* call order violated (e.g. eval before upload) */
    GR_ERR_UNSUPPORTED = 5,  /* feature outside this library's scope */
    GR_ERR_OVERFLOW = 6,     /* a device list overflowed and could not be regrown */
    GR_ERR_TIMEOUT = 7,      /* a bounded device wait gave up */
    GR_ERR_NO_DEVICE = 8     /* no CUDA device / library built without it */
};

/* Which force kernel evaluates the pair lists. */
enum {
    GR_KERNEL_FIXED = 0,  /* CG-relative FP32 pair math, 64-bit fixed-point accumulation (default) */
    GR_KERNEL_PLAIN = 1   /* absolute FP32 coordinates, FP32 atomics (baseline) */
};

/* gr_forces_eval flags */
enum {
    GR_EVAL_VIRIAL = 1,           /* compute the virial tensor */
    GR_EVAL_FORCE_REBUILD = 2,    /* rebuild the pairlist now regardless of NSNB */
    GR_EVAL_NO_DOWNLOAD = 4,      /* keep results on the device (read them later) */
    GR_EVAL_GRAPH = 8             /* replay the step from a recorded CUDA graph (recorded on first
                                     use, again after reallocation); with GR_EVAL_NO_DOWNLOAD a
                                     deferred-pair overflow is reported by the next call */
};

/* Perturbed atom: PertAtomInfo (crates/gromos-forces/src/nonbonded/perturbed.rs:271-279);
 * alpha_lj / alpha_crf are the per-atom soft-core alphas ALREADY multiplied
 * by ALPHLJ / ALPHC (forcefield.rs:146-170). */
typedef struct {
    int32_t atom;
    int32_t a_iac, b_iac;
    double a_charge, b_charge;
    double alpha_lj, alpha_crf;
} gr_perturbed_atom;

/* PERTATOMPAIR entry (crates/gromos-core/src/topology.rs:227-236); b_type -1 = None. */
typedef struct {
    int32_t i, j, a_type, b_type;
} gr_perturbed_pair;

/* Topology subset read by the nonbonded path (topology.rs:619-712). */
typedef struct {
    int32_t n_atoms;
    int32_t n_solute_atoms;
    int32_t n_chargegroups;
    int32_t n_solute_chargegroups;
    const int32_t* cg_offsets;   /* n_chargegroups+1 */
    const double* charge;        /* n_atoms */
    const int32_t* iac;          /* n_atoms, 0-based */
    int32_t n_types;
    const double* lj;            /* n_types*n_types*4: c6, c12, cs6, cs12 (LJParamMatrix, params.rs:30-58) */
    const int32_t* excl_offsets; /* n_atoms+1, symmetric sorted exclusions */
    const int32_t* excl;
    const int32_t* o14_offsets;  /* n_atoms+1, 1-4 partners (INE14) */
    const int32_t* o14;
    const int32_t* energy_group; /* n_atoms or NULL (one group) */
    int32_t n_energy_groups;
    int32_t atoms_per_solvent;   /* 3 for SPC */
    int32_t n_perturbed;
    const gr_perturbed_atom* perturbed;
    int32_t n_perturbed_pairs;
    const gr_perturbed_pair* perturbed_pairs;
    double four_pi_eps_i;        /* PHYSICALCONSTANTS FPEPSI (md.rs:1108) */
} gr_topology;

/* IMD PAIRLIST / NONBONDED / PERTURBATION fields (imd.rs:81-92, 168-176). */
typedef struct {
    double rcutp, rcutl, skin;   /* PairlistContainer::new (pairlist.rs:90-102) */
    double epsilon, epsrf, kappa;/* CRFParameters::new(rcutl, epsilon, epsrf, kappa) (params.rs:78-96) */
    int32_t nsnb;                /* rebuild interval (pairlist.rs:105-107) */
    int32_t boundary;            /* 0 vacuum, 1 rectangular */
    double lambda;               /* RLAM */
    int32_t nlam;                /* NLAM */
    int32_t kernel;              /* GR_KERNEL_* */
    int32_t cluster_size;        /* solvent i-cluster width 4 or 8 (0 = 4) */
    int32_t water_layout;        /* 0 default, 1 lanes share mask bits (width 4), 2 lanes iterate own bits,
                                    3 lanes stream their own water pairs (width 4, short range), 4 as 2 with
                                    the atom pairs evaluated two at a time in packed FP32x2 arithmetic */
    int32_t list_capacity;       /* entries per solvent i-cluster list, 0 = sized from the density; a list
                                    that overflows is grown (doubling) and its step evaluated again.  A
                                    gr_set_params call that changes only this field keeps the current
                                    lists and rebuild schedule; the new size applies from the next rebuild */
} gr_nb_params;

/* Results of one evaluation (ForceStorage + Energy, params.rs:100-138). */
typedef struct {
    double* forces;       /* host n_atoms*3 or NULL */
    double e_lj, e_crf;   /* totals */
    double dhdl;          /* nonbonded dH/dlambda */
    double virial[9];     /* virial[a*3+b] = sum r_a F_b (forcefield.rs:976-1000) */
    double* egroup_lj;    /* host G*G or NULL; [min(g_i,g_j)][max] */
    double* egroup_crf;   /* host G*G or NULL */
    int64_t n_pairs_short;/* atom-pair interactions evaluated this call, short range */
    int64_t n_pairs_long; /* long-range atom pairs evaluated this call (rebuild steps) */
    int32_t rebuilt;      /* 1 if the pairlist was rebuilt in this call */
} gr_result;

typedef struct gr_ctx gr_ctx;

/* ---- context lifecycle -------------------------------------------------- */
/* Replaces constructing gromos-rs `Forcefield::new` (forcefield.rs:119-167). */
gr_status gr_ctx_create(int device, gr_ctx** out);
/* GR_ERR_STATE while the context is a batch member (gr_batch_remove it first). */
gr_status gr_ctx_destroy(gr_ctx* ctx);
const char* gr_last_error(void);
/* CUDA stream used by the context (cudaStream_t as void*), for graph capture / interop. */
void* gr_ctx_stream(gr_ctx* ctx);

/* ---- system set-up ------------------------------------------------------ */
/* Topology upload: `Forcefield::init` (forcefield.rs:210-223) + LJ matrix
 * conversion (forcefield.rs:173-178) + build_pert_info (:146-170). */
gr_status gr_system_upload(gr_ctx* ctx, const gr_topology* topo);
/* CRFParameters::new + PairlistContainer::new + NSNB (md.rs:326-330, 815, 836-841).
 * The next evaluation rebuilds the pairlist, unless no field other than
 * list_capacity changed (then the lists and their schedule stay). */
gr_status gr_set_params(gr_ctx* ctx, const gr_nb_params* params);
/* Periodicity refresh from the box (forcefield.rs:243-265); box = 3 edge lengths. */
gr_status gr_set_box(gr_ctx* ctx, const double box[3]);
/* conf.current().pos -> device (host buffer, n_atoms*3 FP64). */
gr_status gr_positions_upload(gr_ctx* ctx, const double* xyz);
/* Device pointer to the FP64 positions (n_atoms*3), for device-resident MD. */
gr_status gr_positions_device(gr_ctx* ctx, double** dev_xyz);

/* ---- pairlist ----------------------------------------------------------- */
/* PairlistAlgorithm::update (pairlist.rs:828-839): rebuild now, reset counter. */
gr_status gr_pairlist_build(gr_ctx* ctx);
/* Sizes of the four lists in the reference's atom-pair form:
 * counts[0] solute_short, [1] solute_long, [2] solvent_short (first-atom
 * sentinel pairs), [3] solvent_long (PairlistContainer, pairlist.rs:59-70). */
gr_status gr_pairlist_counts(gr_ctx* ctx, int64_t counts[4]);
/* The four lists, each as (i, j) int32 pairs sorted ascending; the caller
 * passes buffers of 2*counts[k] int32 (any may be NULL). */
gr_status gr_pairlist_download(gr_ctx* ctx, int32_t* solute_short, int32_t* solute_long,
                               int32_t* solvent_short, int32_t* solvent_long);
/* Charge-group pair set: (cg1 < cg2, range) with range 0 short / 1 long,
 * sorted; *n_pairs in/out (capacity in, count out). */
gr_status gr_pairlist_cg_pairs(gr_ctx* ctx, int32_t* cg_pairs_3xn, int64_t* n_pairs);

/* ---- evaluation --------------------------------------------------------- */
/* One `Forcefield::apply` nonbonded evaluation (forcefield.rs:226-1020):
 * rebuild when NSNB says so, short range every call, twin-range long range
 * refreshed at rebuilds and reused in between, RF excluded + self terms,
 * 1-4 pairs, soft-core FEP corrections.  Positions must be current. */
gr_status gr_forces_eval(gr_ctx* ctx, int32_t flags, gr_result* out);
/* Device pointer to the last evaluation's FP64 forces (n_atoms*3). */
gr_status gr_forces_device(gr_ctx* ctx, const double** dev_forces);
/* Read back the last evaluation (for GR_EVAL_NO_DOWNLOAD). */
gr_status gr_result_download(gr_ctx* ctx, gr_result* out);
/* Device-event timing of the last evaluation's stages in ms:
 * [0] pairlist build, [1] short-range force kernels, [2] long-range force
 * kernels, [3] excluded/1-4/FEP terms, [4] total.  A step replayed from a
 * recorded graph (GR_EVAL_GRAPH) records only its first and last event (the
 * step's device time, [4]); [0]-[3] read -1 for it. */
gr_status gr_last_timings(gr_ctx* ctx, float ms[5]);
/* Device-event timing of single kernels of the last evaluation, in ms, when it
 * was launched kernel by kernel (not from a graph) with solvent and the
 * fixed-point kernel: [0] the per-step water records (k_water_prep; ~0 when
 * the MD step wrote them), [1] the short-range water force kernel, [2] the
 * long-range water force kernel (-1 when that step kept the twin-range
 * cache).  Entries that do not apply read -1.  Part of the same stage timing
 * as gr_last_timings (Forcefield::apply has no kernel-level timers). */
gr_status gr_last_kernel_timings(gr_ctx* ctx, float ms[3]);

/* ---- measurement utilities (no counterpart in gromos-rs) ---------------- */
/* Kernels launched by this context since creation (for launch accounting). */
gr_status gr_ctx_launches(gr_ctx* ctx, int64_t* n);
/* FP32 FMA issue rate of `device`, measured with an FFMA-chain kernel; one
 * FFMA counts as one operation (the force kernel's operation convention). */
gr_status gr_ffma_peak(int device, double* ops_per_s);

/* ---- MD steps around the force call ------------------------------------- */
/* The step sequence of gromos-md's md binary without thermostat
 * (crates/gromos-md/src/bin/md.rs:1144-1230): Forcefield::apply at r(t),
 * LeapFrogVelocity (crates/gromos-integrators/src/algorithms/leap_frog.rs:37-85),
 * LeapFrogPosition (:116-148) and SETTLE of every solvent molecule
 * (crates/gromos-integrators/src/constraints.rs:815-1010), all on the
 * device; positions and velocities stay resident between calls. */
typedef struct {
    double dt;        /* time step, ps */
    int32_t settle;   /* 1: SETTLE every 3-site solvent molecule */
    double dist_oh;   /* SETTLE constraint lengths, nm (solvent_constraint_template 0 and 2) */
    double dist_hh;
    double temperature; /* Berendsen reference temperature T0, K */
    double tau;         /* Berendsen coupling time, ps (berendsen_thermostat.rs:58-118); < 0 = none (NVE) */
} gr_md_params;

typedef struct {
    int64_t steps;            /* steps done by the call (gr_md_stats_get: since gr_md_init) */
    double e_lj, e_crf;       /* nonbonded energies of the last force evaluation */
    double e_kin;             /* sum 0.5 m v^2 of the last half-step velocities */
    int32_t settle_failures;  /* SETTLE failures since gr_md_init (molecule left as moved, as the reference) */
    int32_t rollbacks;        /* pairlist periods re-run after a list overflow (by the call / since init) */
} gr_md_stats;

/* masses: n_atoms (all > 0); vel: n_atoms*3 initial v(-dt/2) or NULL (zero).
 * Positions are those of the last gr_positions_upload.  The run starts a
 * pairlist period: its first step builds the lists (as the md binary's first
 * step does). */
gr_status gr_md_init(gr_ctx* ctx, const double* mass, const double* vel, const gr_md_params* params);
/* Runs n_steps MD steps on the context's stream; out may be NULL.  A list
 * overflow rolls the steps back to the start of the affected pairlist period
 * and re-runs them with grown lists, so the rebuild and long-range schedule
 * (every NSNB steps from gr_md_init) and the results are those of a run
 * without overflow, also when a call starts inside a period. */
gr_status gr_md_run(gr_ctx* ctx, int32_t n_steps, gr_md_stats* out);
/* New Berendsen reference temperature (an accepted replica exchange); with
 * rescale_velocities the velocities are scaled to t0 from the instantaneous
 * temperature over 3N degrees of freedom (replica.rs:355-371, called by
 * remd.rs perform_exchange).  Takes effect for the next step. */
gr_status gr_md_set_temperature(gr_ctx* ctx, double t0, int32_t rescale_velocities);
/* Statistics of the last step and totals since gr_md_init. */
gr_status gr_md_stats_get(gr_ctx* ctx, gr_md_stats* out);
/* Current positions and velocities (either may be NULL). */
gr_status gr_md_download(gr_ctx* ctx, double* pos, double* vel);

/* ---- batches: many systems stepped together on one GPU ------------------- */
/* No single gromos-rs counterpart: replaces stepping REMD replicas
 * (crates/gromos-integrators/src/replica.rs:163 calculate_forces, :315
 * run_md_steps, driven by remd.rs:168 run_md_parallel) or FEP lambda windows
 * one after the other.  Members are ordinary contexts (topology, params, box,
 * positions and gr_md_init done) of uneven size on the batch's device; they
 * must use GR_KERNEL_FIXED and share NSNB.  One batch MD step is one CUDA
 * graph launch whose branches (one per member) overlap on the GPU; each
 * member's results are bit-identical to a standalone run.  A member may be
 * added or removed between calls (continuous batching); it stays owned by
 * the caller. */
typedef struct gr_batch gr_batch;
gr_status gr_batch_create(int device, gr_batch** out);
gr_status gr_batch_destroy(gr_batch* b);            /* members are not destroyed */
gr_status gr_batch_add(gr_batch* b, gr_ctx* ctx);   /* the member's next step rebuilds its pairlist */
gr_status gr_batch_remove(gr_batch* b, gr_ctx* ctx);
gr_status gr_batch_size(gr_batch* b, int32_t* n);
/* n_steps MD steps of every member (results: gr_md_stats_get / gr_md_download per member). */
gr_status gr_batch_md_run(gr_batch* b, int32_t n_steps);
/* One force evaluation of every member (results: gr_result_download per member). */
gr_status gr_batch_eval(gr_batch* b, int32_t flags);
/* Device time (CUDA events) of the last gr_batch_md_run / gr_batch_eval, ms. */
gr_status gr_batch_last_ms(gr_batch* b, float* ms);
/* Kernels launched by the batch's graphs so far. */
gr_status gr_batch_launches(gr_batch* b, int64_t* n);
/* Where the members stand in their pairlist periods (no counterpart in
 * gromos-rs): *period = NSNB, *phase = the step of the period the next batch
 * step is (0: every member rebuilds its lists there), or -1 when the batch is
 * empty or its members are at different steps of their periods.  A member
 * added to the batch starts a period at its first batch step, so adding
 * members only at phase 0 keeps every member on one phase, which the batch
 * records with two step graphs instead of NSNB. */
gr_status gr_batch_phase(gr_batch* b, int32_t* phase, int32_t* period);
/* Step graphs the batch has recorded so far (after membership and capacity
 * changes; phases sharing a graph count once) and the host time spent
 * recording and instantiating them, in seconds (no counterpart in gromos-rs). */
gr_status gr_batch_record_stats(gr_batch* b, int64_t* graphs, double* seconds);
/* Autotuner (no counterpart in gromos-rs): times full pairlist periods
 * (rebuild + long-range refresh + NSNB short-range steps) of the system(s)
 * for every solvent kernel variant -- lane layout x i-cluster width: (2, 4),
 * (2, 8), (1, 4), (3, 4) -- and keeps the fastest.  NSNB is not tuned: in the reference's twin-range
 * scheme it decides which pairs are evaluated.  Tuning evaluates forces only
 * (positions and velocities are untouched); the next step rebuilds. */
typedef struct {
    int32_t water_layout, cluster_size;   /* chosen variant (gr_nb_params fields) */
    int32_t n_candidates;
    int32_t cand_layout[4], cand_cluster_size[4];
    float cand_ms_per_step[4];            /* device ms per step; -1 = not applicable */
} gr_autotune_result;
gr_status gr_autotune(gr_ctx* ctx, int32_t periods, gr_autotune_result* out);
gr_status gr_batch_autotune(gr_batch* b, int32_t periods, gr_autotune_result* out);
/* Applies a solvent kernel variant (e.g. an earlier gr_batch_autotune result kept by the
 * caller) to every member without timing; every member rebuilds at the next step. */
gr_status gr_batch_set_variant(gr_batch* b, int32_t water_layout, int32_t cluster_size);
/* Device bytes held by a context (topology, lists, accumulators, MD state). */
gr_status gr_ctx_device_bytes(gr_ctx* ctx, int64_t* bytes);

/* ---- energies of many configurations (trajectory analysis) ---------------- */
/* single_point_energy (crates/gromos-forces/src/energy.rs:96-239), nonbonded
 * part, over n_frames configurations in one call (the frame loop of the ener
 * tool, crates/gromos-analysis/src/bin/energy/ener.rs:106-124).  frames holds
 * n_frames x n_atoms x 3 positions; boxes n_frames x 3 edge lengths, or NULL
 * to keep the context's box.  Each frame gets a fresh pairlist built with the
 * context's parameters (single_point_energy: rcutp = rcutl = cutoff, skin 0)
 * and LJ + CRF energies including the RF-excluded and 1-4 terms: e_lj[f],
 * e_crf[f] and, if non-NULL, egroup_lj / egroup_crf (n_frames x G x G).
 * Bonded terms are not computed here.  Afterwards the context holds the last
 * frame's positions. */
gr_status gr_energy_frames(gr_ctx* ctx, int32_t n_frames, const double* frames, const double* boxes,
                           double* e_lj, double* e_crf, double* egroup_lj, double* egroup_crf);

/* ---- job server: continuous batching of MD jobs on one GPU ---------------- */
/* No gromos-rs counterpart (the reference runs one simulation per process).
 * Jobs are submitted with all their inputs (copied: the caller's buffers are
 * free after the call) and queue on the host.  Each gr_server_step admits
 * queued jobs while the resident jobs' device bytes plus the next job's stay
 * within the HBM budget, runs one chunk of MD steps (at most chunk_steps, and
 * no job beyond its n_steps) for every resident job through one batch, and
 * retires finished jobs (their state is copied out and their device memory
 * freed).  Jobs submitted while others run join them at the next step call.
 * Each job's trajectory is bit-identical to a standalone run.
 * A job that cannot be set up (invalid topology or parameters, or a measured
 * footprint above the whole budget) ends in GR_JOB_FAILED with its status code
 * and message; the other jobs carry on.  gr_server_cancel ends a queued or
 * running job (GR_JOB_CANCELLED) and frees its device memory at once. */
enum { GR_JOB_QUEUED = 0, GR_JOB_RUNNING = 1, GR_JOB_DONE = 2, GR_JOB_FAILED = 3, GR_JOB_CANCELLED = 4 };

typedef struct {
    const gr_topology* topo;
    const gr_nb_params* params;   /* kernel must be GR_KERNEL_FIXED */
    const double* box;            /* 3 edge lengths */
    const double* pos;            /* n_atoms*3 */
    const double* mass;           /* n_atoms */
    const double* vel;            /* n_atoms*3 or NULL (zero) */
    const gr_md_params* md;
    int64_t n_steps;
} gr_job_desc;

typedef struct {
    int32_t state;                /* GR_JOB_* */
    int64_t steps_done;
    double t_submit, t_admit, t_done;  /* seconds since the server was created; -1 = not yet */
    int64_t device_bytes;         /* measured footprint while resident */
    gr_md_stats stats;            /* final statistics (done jobs) */
    int32_t error;                /* gr_status of a failed job, else GR_OK */
    char message[160];            /* its error message, NUL-terminated */
} gr_job_status;

typedef struct {
    int64_t jobs_done, jobs_queued, jobs_running;
    double latency_p50_s, latency_p99_s;   /* submit -> done, over the done jobs */
    int64_t resident_bytes, max_resident_bytes;
    int32_t max_resident_jobs;
    int64_t batch_steps;
    int64_t jobs_failed, jobs_cancelled;
    int64_t jobs_joined_running;  /* admitted while resident jobs had already stepped */
} gr_server_stats_t;

typedef struct gr_server gr_server;
gr_status gr_server_create(int device, int64_t hbm_budget_bytes, int32_t chunk_steps, gr_server** out);
gr_status gr_server_destroy(gr_server* srv);
gr_status gr_server_submit(gr_server* srv, const gr_job_desc* job, int64_t* job_id);
/* Admit, run one chunk, retire; *n_running = resident jobs afterwards (may be NULL). */
gr_status gr_server_step(gr_server* srv, int32_t* n_running);
/* Status of a job; pos/vel (n_atoms*3, may be NULL) receive the final state of a done job. */
gr_status gr_server_job(gr_server* srv, int64_t job_id, gr_job_status* out, double* pos, double* vel);
/* End a queued or running job; GR_ERR_STATE if it has already ended. */
gr_status gr_server_cancel(gr_server* srv, int64_t job_id);
/* Forget an ended (done, failed or cancelled) job. */
gr_status gr_server_release(gr_server* srv, int64_t job_id);
gr_status gr_server_stats(gr_server* srv, gr_server_stats_t* out);

/* ---- reference FFI stub replacement ------------------------------------ */
/* Replaces `rust_lj_crf_innerloop` (crates/gromos-core/src/ffi.rs:55-103):
 * lj_crf_innerloop over an explicit atom-pair list with per-atom nearest
 * image (innerloops.rs:169-210), evaluated on the calling thread's current
 * CUDA device (cudaSetDevice before the call selects another GPU).  lj_params
 * holds (c6, c12) per type pair; q_i*q_j is scaled by four_pi_eps_i = 138.9354
 * (crates/gromos-core/src/units.rs:53); boundary_type 0 vacuum, 1
 * rectangular (2 = triclinic is rejected).  Outputs are overwritten.
 * Returns GR_OK or an error (the stub returned void). */
gr_status gr_lj_crf_innerloop(const float* positions, const float* charges, const uint32_t* iac,
                              uint32_t n_atoms, const uint32_t* pairlist, uint32_t n_pairs,
                              const double* lj_params, uint32_t n_types, const double* box_data,
                              uint32_t boundary_type, double crf_cut, double crf_2cut3i,
                              double crf_cut3i, float* forces, double* energies, double* virial);
/* Replaces `rust_lj_crf_innerloop_parallel` (crates/gromos-core/src/ffi.rs:105-145),
 * which delegates to the serial stub: the same call as gr_lj_crf_innerloop
 * (the GPU evaluation is parallel either way), same arguments and results. */
gr_status gr_lj_crf_innerloop_parallel(const float* positions, const float* charges, const uint32_t* iac,
                                       uint32_t n_atoms, const uint32_t* pairlist, uint32_t n_pairs,
                                       const double* lj_params, uint32_t n_types, const double* box_data,
                                       uint32_t boundary_type, double crf_cut, double crf_2cut3i,
                                       double crf_cut3i, float* forces, double* energies, double* virial);

/* ---- allocation-free variant (no counterpart in gromos-rs) -------------- */
/* gr_lj_crf_innerloop on DEVICE buffers, enqueued on `stream` (a
 * cudaStream_t; NULL = legacy default stream) of the calling thread's current
 * device, without allocating device memory: for callers that cannot call
 * cudaMalloc while forces are computed (a loop that must not wait on the
 * allocator's implicit device synchronisation, a host program whose device
 * memory belongs to another allocator that has reserved the GPU's free
 * memory).  All inputs and outputs are
 * device pointers with the meaning of gr_lj_crf_innerloop (lj_params is the
 * double (c6, c12) table), except box_data: 3 doubles of host memory, read
 * during the call and passed to the kernel by value.  Its scratch (the FP32 table and the energy /
 * virial accumulators) is one static device array per GPU, sized for at most
 * 64 atom types: n_types > 64 returns GR_ERR_INVALID.  The first call on a
 * device looks the array's address up (cudaGetSymbolAddress) and must come
 * before any stream capture on that device.  The address is kept for the
 * life of the process: do not use this entry point on a device after
 * cudaDeviceReset (or any other destruction of its primary context).  The box
 * and the CRF constants are taken by value at each call, so a caller whose box
 * changes passes the new box on every call.  forces are cleared by the call;
 * energies[2] and virial[9] are overwritten.  Pair indices (< n_atoms) and
 * iac values (< n_types) are the caller's to guarantee: they stay on the
 * device and are not checked.  Calls whose work may overlap on the GPU share
 * the scratch and race: order them on one stream. */
gr_status gr_lj_crf_innerloop_noalloc(const float* positions, const float* charges, const uint32_t* iac,
                                      uint32_t n_atoms, const uint32_t* pairlist, uint32_t n_pairs,
                                      const double* lj_params, uint32_t n_types, const double* box_data,
                                      uint32_t boundary_type, double crf_cut, double crf_2cut3i,
                                      double crf_cut3i, float* forces, double* energies, double* virial,
                                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GROMOS_NB_H */
