/*
 * oracle.h -- C ABI of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Two shared libraries export exactly these symbols:
 *   oracle/_build/liboracle_port.so  -- the restatement: plain C++ written for
 *                                       this project, every step citing the
 *                                       reference file:line it follows;
 *   oracle/_ref/libkaram_ref.so      -- the same driver linked against the
 *                                       reference's own sources (tensorize,
 *                                       generic kernels, stampSoABlock, CSR
 *                                       assembly, dense/sparse LU, Min-Fill),
 *                                       compiled from the reference tree by
 *                                       oracle/Makefile.
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark load
 * them. The product library never links or calls anything in oracle/.
 */
#ifndef KARAM_ORACLE_H
#define KARAM_ORACLE_H
#include <stdint.h>
#include "../include/karam.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_LS_DENSE 0  /* solveLU_Pivoted           math/linalg.h:742-854      */
#define ORACLE_LS_SPARSE 1 /* solveSparse_LU + symbolic math/sparse_lu.cpp:14-330  */

typedef struct oracle_opts {
  int32_t max_nr_iter;   /* 50 */
  int32_t gmin_steps;    /* 19 */
  double reltol, vntol;  /* 1e-3, 1e-6 */
  double kcl_shortcut;   /* 1e-9 */
  double kcl_tol;        /* 1e-12 */
  int32_t polish_max;    /* 0 = reference stopping rule */
  double polish_rel, polish_abs;
  int32_t linear_solver; /* ORACLE_LS_* */
  int32_t seeded;        /* start from v0 at the final GMIN step */
  int32_t seed_max_iter; /* fall back to full GMIN stepping after this many */
  int32_t max_halvings;  /* transient step halvings after NR failure (3 = the
                            reference's 4 attempts, circuitsim_solver.cpp:583) */
  double lte_rel, lte_abs; /* LTE step control of the product's transient (the
                            linear-extrapolation test of karam_solver_opts
                            lte_reltol / lte_abstol); lte_rel 0 = off */
} oracle_opts;

typedef struct oracle_stats {
  int32_t converged;
  int32_t iterations;    /* counted as circuitsim_solver.cpp:447-466 counts */
  int32_t polish_iters;
  int32_t damped;        /* damping re-evaluations (circuitsim_solver.cpp:391-406) */
  int32_t gmin_step;     /* last GMIN step entered */
  int32_t singular;
  int32_t seeded_ok;
  int32_t max_step_iters; /* transient: most NR iterations of one step */
  double residual;       /* final max |KCL| [A] */
  /* DC convergence diagnostics of CircuitSim::solveDC (circuitsim_solver.cpp:408-443, 516) */
  int32_t failure_type;  /* ConvergenceEngine::classifyFailure over the whole DC history */
  int32_t stagnation;
  int32_t divergence;
  int32_t history_len;
  int32_t halvings;      /* transient sub-steps redone with half the step */
  int32_t lte_rejects;   /* ... of those, by the LTE test */
} oracle_stats;

/* Fills o with the reference constants; polish off, dense solver. */
void oracle_default_opts(oracle_opts *o);

/* SoA order of tensorizeNetlist (tensors/physics_tensors.cpp:305-493):
 * mos_order[soa] = netlist index, dio_order[soa] = netlist index. */
int oracle_tensorize(const karam_netlist *nl, int32_t *mos_order, int32_t *dio_order);

/* CSR pattern built from the stamp triplets (physics/circuitsim.h:2413-2751
 * + addDiagonalConditioning :2857) by MatrixConstructor::buildPattern
 * (math/linalg.h:421). transient=0: DC stamps (no capacitor companions);
 * transient=1: with capacitor companions. Returns nnz; arrays may be NULL to
 * query sizes. */
int oracle_pattern(const karam_netlist *nl, int32_t transient, int32_t *row_ptr,
                   int32_t *col, int32_t cap);

/* Stamp-slot -> CSR index map (CachedCsrPattern::indexOf of every triplet in
 * insertion order), for the transient pattern. Returns the triplet count. */
int oracle_stamp_map(const karam_netlist *nl, int32_t *slot_csr, int32_t cap);

/* One stamping pass at v for instance inst on the transient pattern:
 * vals[nnz] = assembleFast values without the gmin diagonal, rhs[n].
 * h = 0 -> DC (no companions); otherwise method KARAM_TRAN_* with capacitor
 * history cap_vprev/cap_iprev[n_cap] in SoA (= netlist) order, and sources
 * evaluated at time t. */
int oracle_stamp(const karam_netlist *nl, const karam_instances *inst, int32_t idx,
                 const double *v, double h, int32_t method, const double *cap_vprev,
                 const double *cap_iprev, double t, double *vals, double *rhs);

/* The same stamping pass as oracle_stamp, reporting per CSR value the sum of
 * the magnitudes of its triplets (abs_vals[nnz]) and their count
 * (n_terms[nnz]): the scale of the summation error of a value whose terms are
 * added in another order. */
int oracle_stamp_abs(const karam_netlist *nl, const karam_instances *inst, int32_t idx,
                     const double *v, double h, int32_t method, const double *cap_vprev,
                     const double *cap_iprev, double t, double *abs_vals, int32_t *n_terms);

/* Min-Fill ordering of FactorGraph::fromTensorizedBlock
 * (infrastructure/factor_graph.cpp:9-162, treewidth_analyzer.cpp:14-141).
 * raw[*raw_len] = eliminationOrdering as produced (branch ids included);
 * perm[n] = translation to a 0-based permutation of the n unknowns (ids in
 * 1..n kept, repeats dropped, minus one). Returns the treewidth. */
int oracle_ordering(const karam_netlist *nl, uint32_t *raw, int32_t *raw_len,
                    int32_t *perm);

/* symbolicFactorize (math/sparse_lu.cpp:14-128) on the transient pattern with
 * the translated ordering. Returns nnz of the filled pattern; *fill_in gets
 * estimatedFillIn. Arrays may be NULL to query the size. */
int oracle_symbolic(const karam_netlist *nl, int32_t *perm, int32_t *iperm,
                    int32_t *f_row_ptr, int32_t *f_col, int32_t *fill_in, int32_t cap);

/* Linear solve of (vals + gmin*I) x = rhs on the transient pattern with the
 * selected solver. Returns 0, or 1 when the solver reports a singular matrix. */
int oracle_linsolve(const karam_netlist *nl, const double *vals, double gmin,
                    const double *rhs, int32_t solver, double *x);

/* DC operating point (circuitsim_solver.cpp:176-555 with the residual
 * F(v) = J(v) v - rhs(v) from the same stamps). v0: initial guess when
 * opts->seeded, else NULL. */
int oracle_solve_dc(const karam_netlist *nl, const karam_instances *inst, int32_t idx,
                    const oracle_opts *opts, const double *v0, double *v_out,
                    oracle_stats *st);

/* Fixed-step transient from v_start (a DC solution): companions of
 * math/integration_method.h:47-115, PULSE of physics/circuitsim.h:2155-2170,
 * history update of circuitsim_solver.cpp:669-699. wave_out[n_steps][n_wave]. */
int oracle_transient(const karam_netlist *nl, const karam_instances *inst, int32_t idx,
                     const oracle_opts *opts, const double *v_start, double dt,
                     int32_t n_steps, int32_t method, const int32_t *wave_nodes,
                     int32_t n_wave, double *wave_out, double *v_out, oracle_stats *st);

/* DC + transient for instances [i0, i1) on n_threads host threads (one
 * instance per thread at a time). v_out[(i1-i0)][n]; st[(i1-i0)] (DC stats
 * with transient iterations added). n_steps = 0 runs DC only. */
int oracle_run_batch(const karam_netlist *nl, const karam_instances *inst, int32_t i0,
                     int32_t i1, const oracle_opts *opts, double dt, int32_t n_steps,
                     int32_t method, int32_t n_threads, double *v_out, oracle_stats *st);

/* Small-signal AC sweep at the DC point v_dc[n] of instance idx
 * (ACSolver::solveAC_Sparse, solvers/ac_solver.h:711-773): n_points
 * log-spaced frequencies from f_start to f_stop (its formula), and at each
 * Y(jw) x = b solved by LU with partial pivoting on the complex magnitude
 * (solveComplexLU_Sparse, math/linalg.h:993-1078), with the input node
 * driven through 1e6 S at amplitude volts. rule 1: Y = the NR Jacobian at
 * v_dc (the stamps of physics/circuitsim.h:2413-2751, device conductances of
 * the instance's own models) + jwC + 1e-12 on every diagonal. rule 0
 * (reference build only): the reference's own admittance build
 * (buildAdmittanceMatrixSparse, ac_solver.h:618-704). out_re / out_im
 * [n_points][n]. Returns the number of points whose matrix was singular. */
int oracle_ac(const karam_netlist *nl, const karam_instances *inst, int32_t idx,
              const double *v_dc, double f_start, double f_stop, int32_t n_points,
              int32_t input_node, double amplitude, int32_t rule, double *out_re,
              double *out_im);

#ifdef __cplusplus
}
#endif
#endif
