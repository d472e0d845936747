/*
 * gromos_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the gromos-rs nonbonded hot path (charge-group
 * pairlist, LJ + reaction-field inner loops, RF excluded/self terms, 1-4
 * loop, soft-core FEP corrections, twin-range cache).  It is the checker for
 * the CUDA library: only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py may load it.  The product path never calls it.
 *
 * Each function cites the reference file:line it restates (paths relative to
 * the gromos-rs repository root).  Arithmetic follows the reference's
 * operation order so that the oracle is bit-reproducible against it when
 * compiled with -ffp-contract=off (Rust never contracts a*b+c into an FMA).
 */
#ifndef GROMOS_ORACLE_H
#define GROMOS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Topology subset used by the nonbonded path
 * (crates/gromos-core/src/topology.rs:619-712). */
typedef struct {
    int32_t n_atoms;
    int32_t n_solute_atoms;          /* atoms [0, n_solute_atoms) are solute */
    int32_t n_cg;
    int32_t n_solute_cg;             /* CGs [0, n_solute_cg) are solute */
    const int32_t* cg_offsets;       /* n_cg+1; CG c = atoms [off[c], off[c+1]) */
    const double* charge;            /* n_atoms */
    const int32_t* iac;              /* n_atoms, 0-based */
    int32_t n_types;
    const double* lj;                /* n_types*n_types*4: c6, c12, cs6, cs12 */
    const int32_t* excl_off;         /* n_atoms+1; symmetric, sorted, deduped */
    const int32_t* excl;
    const int32_t* o14_off;          /* n_atoms+1; 1-4 partners as stored */
    const int32_t* o14;
    const int32_t* egroup;           /* n_atoms energy group or NULL (1 group) */
    int32_t n_egroups;
    /* perturbation (PertAtomInfo, forcefield.rs:146-170); pert_idx[a] = -1
     * for unperturbed atoms, else an index into the per-perturbed arrays.
     * alpha values are already multiplied by ALPHLJ / ALPHC. */
    const int32_t* pert_idx;         /* n_atoms or NULL */
    const int32_t* pert_a_iac;
    const int32_t* pert_b_iac;
    const double* pert_a_q;
    const double* pert_b_q;
    const double* pert_alpha_lj;
    const double* pert_alpha_crf;
    int32_t n_pert;
    int32_t n_pert_pairs;            /* PERTATOMPAIR (topology.rs:227-236) */
    const int32_t* pp_i;
    const int32_t* pp_j;
    const int32_t* pp_a_type;
    const int32_t* pp_b_type;        /* -1 = pair disappears in state B */
    int32_t atoms_per_solvent;
} orc_topology;

typedef struct {
    double rcutp, rcutl, skin;       /* PairlistContainer::new (pairlist.rs:90) */
    double epsilon, epsrf, kappa;    /* CRFParameters::new(rcutl, eps, epsrf, kappa) */
    double four_pi_eps_i;
    int32_t nsnb;
    int32_t boundary;                /* 0 vacuum, 1 rectangular */
    double box[3];
    int32_t algorithm;               /* 0 standard, 2 cell list (pairlist.rs:815) */
    int32_t virial;                  /* compute the virial tensor */
    double lambda;                   /* FEP RLAM */
    int32_t nlam;                    /* FEP NLAM */
    int32_t nthreads;                /* 0/1: serial reference order; >1: threaded fold/reduce */
} orc_params;

typedef struct {
    double e_lj, e_crf;              /* totals (Energy.lj_total/crf_total) */
    double dhdl;                     /* nonbonded dH/dlambda */
    double virial[9];                /* virial[a*3+b] = sum r_a F_b */
    double* forces;                  /* caller buffer n_atoms*3 */
    double* egroup_lj;               /* caller buffer G*G or NULL ([min][max]) */
    double* egroup_crf;              /* caller buffer G*G or NULL */
} orc_result;

typedef struct orc_pairlist orc_pairlist;
typedef struct orc_ff orc_ff;

/* CRFParameters::new (crates/gromos-forces/src/nonbonded/params.rs:78-96).
 * out = {crf_cut, crf_2cut3i, crf_cut3i, cutoff_sq} */
void orc_crf_params(double cutoff, double eps, double epsrf, double kappa, double out[4]);

/* Pairlist build (pairlist.rs:155-442 standard, :509-777 cell list).
 * Lists: 0 solute_short, 1 solute_long, 2 solvent_short, 3 solvent_long. */
orc_pairlist* orc_pairlist_build(const orc_topology* t, const orc_params* p, const double* pos);
int64_t orc_pairlist_size(const orc_pairlist* pl, int which);
void orc_pairlist_get(const orc_pairlist* pl, int which, int32_t* out_pairs /* 2*size */);
void orc_pairlist_free(orc_pairlist* pl);

/* Forcefield (crates/gromos-integrators/src/algorithms/forcefield.rs:37-1060),
 * nonbonded part only.  create() performs the initial pairlist build
 * (gromos-md/src/bin/md.rs:864-867); apply() is one Forcefield::apply. */
orc_ff* orc_ff_create(const orc_topology* t, const orc_params* p, const double* pos);
int orc_ff_apply(orc_ff* ff, const double* pos, orc_result* out);
void orc_ff_set_box(orc_ff* ff, const double box[3]);
void orc_ff_destroy(orc_ff* ff);

/* PerturbedLambdaParams::from_lambda (perturbed.rs:57-101); out[17] in
 * struct order a_lj_n, b_lj_n, a_crf_n, b_crf_n, a_lj_n1, b_lj_n1, a_crf_n1,
 * b_crf_n1, a_ljs, b_ljs, a_ljs2, b_ljs2, a_crfs, b_crfs, a_crfs2, b_crfs2, n */
void orc_lambda_params(double lj, double ljs, double crf, double crfs,
                       double dlj, double dljs, double dcrf, double dcrfs,
                       int n, double out[17]);

/* perturbed_lj_crf_interaction (perturbed.rs:124-266) for one pair.
 * out = {force, e_lj, e_crf, de_lj, de_crf} */
void orc_perturbed_pair(const double r[3], double a_c6, double a_c12, double b_c6, double b_c12,
                        double a_q, double b_q, double alpha_lj, double alpha_crf,
                        const double lp[17], const double crf[4], double four_pi_eps_i,
                        double out[5]);

/* MD steps around orc_ff_apply, the sequence of gromos-md/src/bin/md.rs
 * (:1144-1230) without thermostat: leap-frog velocity (leap_frog.rs:37-85),
 * Berendsen velocity scaling from the kinetic energy entering the step
 * (berendsen_thermostat.rs:74-98, between the two leap-frog updates),
 * leap-frog position (:116-148), SETTLE of every solvent molecule
 * (crates/gromos-integrators/src/constraints.rs:815-1010).  pos/vel are
 * updated in place; returns the number of molecules SETTLE could not solve.
 * e_kin = sum 0.5 m v^2 of the final half-step velocities; energies = the
 * last step's {e_lj, e_crf}. */
typedef struct {
    double dt;
    int32_t settle;
    double dist_oh, dist_hh;
    double temperature, tau;   /* Berendsen bath (berendsen_thermostat.rs:58-118); tau < 0 = none */
} orc_md_params;
int orc_md_run(orc_ff* ff, double* pos, double* vel, const double* mass, const orc_md_params* p,
               int n_steps, double* e_kin, double energies[2]);

#ifdef __cplusplus
}
#endif
#endif
