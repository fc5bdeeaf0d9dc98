/*
 * karam.h -- C ABI of the B200 Newton-Raphson inner loop (device evaluation,
 * MNA stamping, sparse LU refactorisation + triangular solves, convergence test).
 *
 * The reference engine has no extern "C" surface: its solver entry points are
 * C++ member functions hidden behind the ENGINE_API visibility macros
 * (engine_export.h:19-39). This header is the flat boundary that replaces them:
 *
 *   CircuitSim::solveDC(TensorNetlist&)        physics/circuitsim.h:1110,
 *                                              solvers/circuitsim_solver.cpp:176-555
 *   CircuitSim::solveDC(const CompiledTensorBlock&)      circuitsim_solver.cpp:790-807
 *   CircuitSim::stepTransient(TensorNetlist&, dt, t)     circuitsim_solver.cpp:559-780
 *   SessionImpl::runMonteCarlo (sequential DC loop)      engine_impl.cpp:259-281
 *
 * Conventions
 *   - Plain pointers and sizes only; the caller owns every host buffer and the
 *     library never keeps a caller pointer after a call returns.
 *   - Node ids are 1-based, 0 is ground (netlist/circuit.h:1056-1216).
 *   - Every function returns KARAM_OK (0) or a negative KARAM_E_* code; the text
 *     of the last error of a context is available from karam_last_error().
 *   - No exceptions cross this boundary. Per-instance solver outcomes are
 *     reported as KARAM_ST_* codes in the caller's status array.
 *   - A context owns one CUDA device and one stream; a context and the problems
 *     made from it must not be used from two threads at once.
 */
#ifndef KARAM_H
#define KARAM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define KARAM_API __attribute__((visibility("default")))
#else
#define KARAM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------ */
#define KARAM_OK 0
#define KARAM_E_INVALID (-1)     /* bad argument or malformed netlist        */
#define KARAM_E_CUDA (-2)        /* CUDA runtime error or no usable device    */
#define KARAM_E_NOMEM (-3)       /* host or device allocation failed          */
#define KARAM_E_UNSUPPORTED (-4) /* netlist uses something this path lacks   */
#define KARAM_E_STATE (-5)       /* call out of order (e.g. no DC solution)   */

/* ---- per-instance solver status (the reference reports converged=false +
 *      error_detail, rankDeficient, and falls back to the CPU; this path has
 *      no fallback and reports one of these instead) ------------------------ */
#define KARAM_ST_CONVERGED 0
#define KARAM_ST_NOCONV 1   /* NR did not converge within its iteration budget */
#define KARAM_ST_SINGULAR 2 /* a pivot fell below the singularity threshold     */
#define KARAM_ST_NAN 3      /* non-finite values met in the residual            */
#define KARAM_ST_TIMEOUT 4  /* round budget of the launch exhausted             */

/* ---- precision / schedule / method selectors ---------------------------- */
#define KARAM_PREC_FP64 0  /* FP64 evaluation, FP64 LU                        */
#define KARAM_PREC_MIXED 1 /* FP32 Jacobian + FP32 LU, FP64 residual + refinement */

#define KARAM_TRAN_BE 0    /* backward Euler (Gear1, math/integration_method.h:83-115) */
#define KARAM_TRAN_TRAP 1  /* trapezoidal (math/integration_method.h:47-81)           */

#define KARAM_SEED_NONE 0   /* plain NR from the reference seed (seedInitialGuess)     */
#define KARAM_SEED_CALLER 1 /* the caller's guesses (karam_solve_dc seed_v)            */
#define KARAM_SEED_EMA 2    /* batch statistical seeder, NeuralSeeder::predictSeed
                               (solvers/neural_seeder.h:100-137): the first
                               KARAM_SEED_HISTORY instances run plain NR; their
                               converged DC solutions, each weighted 0.8 per later
                               one, seed every instance when the mean per-node
                               confidence 1 / (1 + variance) is at least 0.3       */
#define KARAM_SEED_HISTORY 8
#define KARAM_SEED_MLP 3    /* the learned seeder attached by karam_problem_set_seeder */

#define KARAM_SRC_DC 0
#define KARAM_SRC_PULSE 1  /* PULSE(v1 v2 td tr tf pw per), physics/circuitsim.h:2155-2170 */

#define KARAM_MODEL_NMOS 0
#define KARAM_MODEL_PMOS 1
#define KARAM_MODEL_DIODE 2

/*
 * Flat netlist in netlist (insertion) order: the global block of a
 * TensorNetlist (netlist/circuit.h:1056-1216) without hierarchy. The library
 * performs the reference's tensorisation itself (device regrouping by model
 * name, tensors/physics_tensors.cpp:305-493). Optional arrays may be NULL.
 */
typedef struct karam_netlist {
  int32_t n_nodes; /* highest node id; unknowns are nodes 1..n_nodes            */
  double temp_k;   /* ambient temperature [K]; reference default 300.15         */

  /* independent voltage sources, Norton model G = 1e3 S (physics/circuitsim.h:2441-2467) */
  int32_t n_vsrc;
  const int32_t *vs_pos, *vs_neg;
  const double *vs_dc;   /* DC value (also the DC operating-point value)        */
  const int32_t *vs_kind; /* KARAM_SRC_*; NULL = all DC                          */
  const double *vs_pulse; /* [n_vsrc][7] v1 v2 td tr tf pw per; NULL if none     */

  /* independent current sources (physics/circuitsim.h:2470-2477) */
  int32_t n_isrc;
  const int32_t *is_pos, *is_neg;
  const double *is_amp;

  /* resistors (physics/circuitsim.h:2417-2438) */
  int32_t n_res;
  const int32_t *r_n1, *r_n2;
  const double *r_ohm;

  /* capacitors (companions in transient only) */
  int32_t n_cap;
  const int32_t *c_n1, *c_n2;
  const double *c_farad;

  /* diodes: Is, N, Vt as in TensorBlock::addDiode (netlist/circuit.h:815-826) */
  int32_t n_dio;
  const int32_t *d_anode, *d_cathode;
  const double *d_is, *d_n, *d_vt;
  const int32_t *d_model; /* model index, -1 = "diode_generic"; NULL = all -1     */

  /* level-1 MOSFETs (netlist/circuit.h:832-843); model index required */
  int32_t n_mos;
  const int32_t *m_d, *m_g, *m_s, *m_b;
  const double *m_w, *m_l;
  const int32_t *m_model;

  /* model cards (netlist/circuit.h:31-42); a NaN parameter means "not given",
   * so the reference default of tensors/physics_tensors.cpp:424-441 applies */
  int32_t n_models;
  const char *const *model_name;
  const int32_t *model_type; /* KARAM_MODEL_* */
  const double *model_kp, *model_vto, *model_lambda;
} karam_netlist;

/*
 * Per-instance parameters of a Monte-Carlo / corner batch. Every instance shares
 * the netlist's topology. Arrays are instance-major; NULL means "use the
 * netlist value for every instance". MOSFET KP/VTO are FP32-representable by
 * contract (the sampler quantises them), so FP32 device storage is exact.
 */
typedef struct karam_instances {
  int32_t n_instances;
  const float *mos_kp;  /* [n_instances][n_mos], netlist MOSFET order          */
  const float *mos_vto; /* [n_instances][n_mos]                                */
  const double *vs_dc;  /* [n_instances][n_vsrc]: DC value; for PULSE sources the
                           value scales v1 and v2 by vs_dc/netlist vs_dc when the
                           netlist value is non-zero                           */
} karam_instances;

/* Solver options; karam_default_opts() fills the reference's constants
 * (physics/physics_constants.h:62-85, physics/circuitsim.h:1206-1207). */
typedef struct karam_solver_opts {
  int32_t precision;     /* KARAM_PREC_*                                        */
  int32_t max_nr_iter;   /* per GMIN step / per time step (reference: 50)       */
  int32_t gmin_steps;    /* half-decade GMIN schedule length (reference: 19)    */
  double reltol, vntol;  /* 1e-3, 1e-6                                          */
  double kcl_shortcut;   /* converged outright below this KCL residual (1e-9 A)  */
  double kcl_tol;        /* KCL tolerance at the final GMIN step / transient (1e-12 A) */
  int32_t polish_max;    /* extra NR iterations after the reference criterion;
                            0 keeps the reference stopping rule                  */
  double polish_rel;     /* polishing stops once |dv_i| <= polish_rel*|v_i| + polish_abs */
  double polish_abs;     /*   for every node, or when |dv| stops shrinking        */
  double lu_growth_limit; /* a static-pivot solve whose multipliers exceed this goes
                            to the rescue path (FP64 static pivots, then
                            partial pivoting); 0 = 1e4 in FP32 / 1e10 in FP64;
                            < 0 = no growth test (tiny or non-finite pivots and
                            non-finite solutions still go to the rescue)       */
  int32_t seeded;        /* KARAM_SEED_*: a seeded instance starts from its seed at
                            the final GMIN step and falls back to full GMIN
                            stepping if it has not converged after seed_max_iter
                            iterations. KARAM_SEED_CALLER needs karam_solve_dc's
                            seed_v; KARAM_SEED_EMA applies to batches of more than
                            KARAM_SEED_HISTORY instances (smaller ones run plain);
                            KARAM_SEED_MLP needs an attached, trained seeder     */
  int32_t seed_max_iter; /* K of the seeded fallback                              */
  int32_t schedule;      /* factor/solve schedule: instances per CTA (1..32; a warp each
                            on the level schedule, or a lane each on the pivot
                            program), -1 one CTA per instance with its slots in
                            shared memory, -2 the same with them in global
                            memory, -3 one CTA per instance with its slots and
                            the packed level program in shared memory, -4 the
                            persistent kernel: one CTA per instance running all
                            of its rounds in one launch (the code of -3), -5 one
                            CTA per instance with its slots and its solve vector
                            in global memory (taken by 0 only where -2 does not
                            fit shared memory); 0 =
                            chosen from shared memory, occupancy and batch size
                            (-4 for batches no larger than the SM count where it
                            fits). Batches larger than the SM count switch to
                            -4 for their last rounds, once no more instances
                            are live than SMs, unless kernel_timing is set     */
  int32_t max_rounds;    /* device round budget per launch (0 = unlimited)        */
  int32_t max_halvings;  /* transient: a step whose NR exhausts max_nr_iter restarts
                            from the last time point with half the step, at most
                            this many times (reference attempt loop: 3)          */
  int32_t kernel_timing; /* 1: CUDA events around every kernel of every round, summed
                            into karam_timing's eval_ms / lu_ms / rescue_ms. The
                            event records slow a round down (B200, config 2:
                            ~24 us of a ~160 us round), so 0 (the default) leaves
                            them out and those three fields at 0               */
  double lte_reltol;     /* transient step control by local truncation error: a
                            converged sub-step of size h whose accepted point x
                            leaves, at some node, the linear extrapolation
                            p = v1 + (h / h1) (v1 - v2) from the two previous
                            accepted points (v1 after a sub-step of size h1) by
                            more than lte_reltol * max(|x|, |v1|) + lte_abstol
                            is redone from v1 with half the step, as an NR
                            failure is, while max_halvings allows (then it is
                            accepted). The first sub-step of a transient has no
                            predictor and is not tested. 0 (the default): off,
                            the reference's fixed-step behaviour              */
  double lte_abstol;     /* [V], with lte_reltol                                  */
} karam_solver_opts;

/* Sizes of the symbolic analysis of a problem. */
typedef struct karam_problem_info {
  int32_t n;           /* unknowns (node voltages)                              */
  int32_t nnz;         /* CSR non-zeros of the Jacobian pattern                  */
  int32_t nnz_filled;  /* non-zeros of L+U on the translated Min-Fill ordering   */
  int32_t fill_in;     /* symbolicFactorize's estimatedFillIn                     */
  int32_t treewidth;   /* TreewidthAnalyzer's estimatedTreewidth                  */
  int32_t n_triplets;  /* stamp slots (triplets) per iteration incl. gmin         */
  int32_t n_instances;
  int32_t n_mos, n_dio, n_res, n_cap, n_vsrc, n_isrc;
  int32_t lu_ops;      /* scaled + update operations of the LU program           */
  int32_t n_slots;     /* value slots: filled positions the static-pivot LU can
                          make non-zero (what the device stores and factors)     */
  int32_t es_blocks;   /* evaluation + stamping blocks (one CTA each per 32 instances) */
  int32_t es_device_evals; /* device evaluations per instance and round, counting
                          devices shared by two blocks twice                     */
} karam_problem_info;

/* Per-instance counters returned by the solves. */
typedef struct karam_instance_stats {
  int32_t status;       /* KARAM_ST_*                                            */
  int32_t iterations;   /* NR iterations counted as the reference counts them    */
  int32_t polish_iters; /* extra iterations spent polishing                       */
  int32_t damped;       /* damping re-evaluations                                 */
  int32_t gmin_step;    /* GMIN step reached (DC)                                 */
  int32_t seeded_ok;    /* 1 if the seeded start converged without fallback       */
  int32_t rescued;      /* linear solves redone by the rescue path (FP64 static
                           pivots, then partial pivoting) because the
                           static pivots of the working precision were unusable */
  int32_t halvings;     /* transient step halvings after NR failures              */
  int32_t max_step_iters; /* most NR iterations spent on one transient attempt    */
  double residual;      /* final max KCL residual [A]                             */
  /* DC convergence diagnostics (SolverStats, infrastructure/simtrace.h:86-104;
   * filled as CircuitSim::solveDC fills them, solvers/circuitsim_solver.cpp:408-443, 516) */
  int32_t failure_type; /* KARAM_FAIL_*: ConvergenceEngine::classifyFailure on the
                           DC history (solvers/convergence_engine.h:26-87); set
                           for converged solves too, as the reference does       */
  int32_t stagnation;   /* SolverStats::stagnationDetected                        */
  int32_t divergence;   /* SolverStats::divergenceDetected                        */
  int32_t history_len;  /* DC NR iterations recorded (convergenceHistory.size())  */
  int32_t lte_rejects;  /* transient sub-steps redone by the LTE test (opts.lte_reltol;
                           counted in halvings too)                              */
  int32_t reserved_;
} karam_instance_stats;

/* ConvergenceFailureType (infrastructure/simtrace.h:39-47), same order. */
#define KARAM_FAIL_NONE 0
#define KARAM_FAIL_SINGULAR_MATRIX 1
#define KARAM_FAIL_DIVERGENCE 2
#define KARAM_FAIL_LIMIT_CYCLE 3
#define KARAM_FAIL_SLOW_CONVERGENCE 4
#define KARAM_FAIL_FLOATING_NODE_INDUCED 5
#define KARAM_FAIL_EXPONENTIAL_OVERFLOW 6
/* Length of the per-instance ring of DC convergence history records. */
#define KARAM_HISTORY_MAX 16

typedef struct karam_ctx karam_ctx;
typedef struct karam_problem karam_problem;

/* ---- context ------------------------------------------------------------ */
KARAM_API int karam_ctx_create(int device, karam_ctx **out);
KARAM_API void karam_ctx_destroy(karam_ctx *ctx);
/* Text of the last error recorded on ctx (or of a failed karam_ctx_create when ctx is NULL). */
KARAM_API const char *karam_last_error(const karam_ctx *ctx);
KARAM_API void karam_default_opts(karam_solver_opts *opts);

/* ---- problems ------------------------------------------------------------
 * karam_problem_create runs the host symbolic analysis once per topology
 * (the reference's NetlistCompiler::compile, infrastructure/netlist_compiler.cpp:17-90):
 * tensorisation, stamp-slot -> CSR map, Min-Fill ordering, symbolic fill, LU
 * program; it uploads the shared topology and sizes device state for
 * max_instances instances. */
KARAM_API int karam_problem_create(karam_ctx *ctx, const karam_netlist *nl,
                                   int32_t max_instances, karam_problem **out);
KARAM_API void karam_problem_destroy(karam_problem *p);
/* Symbolic-analysis cache: karam_problem_create keeps the last 32 analyses
 * (at most 8 GiB of their fill-sized tables together; a larger one is not
 * kept) by netlist content (every count, index, value, model name and the
 * temperature), process-wide, and reuses one for an identical netlist -- the
 * role of the reference's compiled block / pattern cache keyed by
 * topologyHash (infrastructure/compiled_block.h:45-88,
 * solvers/circuitsim_solver.cpp:262-268), which keys on structure alone
 * because its values are stamped per solve. karam_netlist_hash is a 64-bit
 * fingerprint of that content. */
KARAM_API int karam_netlist_hash(const karam_netlist *nl, uint64_t *out);
KARAM_API int karam_symbolic_cache_info(int32_t *entries, int64_t *hits, int64_t *misses);
KARAM_API void karam_symbolic_cache_clear(void);
KARAM_API int karam_problem_info_get(const karam_problem *p, karam_problem_info *out);
/* Copies per-instance parameters host -> device (the batch to solve next). */
KARAM_API int karam_set_instances(karam_problem *p, const karam_instances *inst);

/* ---- solves (host buffers; copies are part of the call) ------------------
 * DC operating point of every instance (circuitsim_solver.cpp:176-555).
 * seed_v: [n_instances][n] initial guesses when opts->seeded, else NULL.
 * out_v:  [n_instances][n]; stats: [n_instances] (either may be NULL). */
KARAM_API int karam_solve_dc(karam_problem *p, const karam_solver_opts *opts,
                             const double *seed_v, double *out_v,
                             karam_instance_stats *stats);

/* Fixed-step transient from the current DC (or previous transient) solution:
 * n_steps steps of dt with the chosen companion (KARAM_TRAN_*).
 * wave_nodes/n_wave: optional node ids recorded after every step into
 * wave_out[n_instances][n_steps][n_wave]. out_v receives the final voltages. */
KARAM_API int karam_step_transient(karam_problem *p, const karam_solver_opts *opts,
                                   double dt, int32_t n_steps, int32_t method,
                                   const int32_t *wave_nodes, int32_t n_wave,
                                   double *wave_out, double *out_v,
                                   karam_instance_stats *stats);

/* One Monte-Carlo job: set the instances, DC, then the transient, with results
 * copied back. It is the call a SessionImpl::runMonteCarlo caller replaces its
 * sequential loop with. out_v: [n_instances][n] final voltages. */
KARAM_API int karam_run_mc(karam_problem *p, const karam_instances *inst,
                           const karam_solver_opts *opts, double dt, int32_t n_steps,
                           int32_t method, double *out_v, karam_instance_stats *stats);

/* ---- device-resident variants (inputs already in HBM; results stay there) --
 * Same work as karam_run_mc after karam_set_instances, with no host copies;
 * karam_read_results copies the device results back afterwards. */
KARAM_API int karam_run_mc_device(karam_problem *p, const karam_solver_opts *opts,
                                  double dt, int32_t n_steps, int32_t method);
/* One launch over problems of different circuits and sizes (an uneven batch;
 * the reference runs such jobs one after another, MonteCarloRunner::run,
 * infrastructure/monte_carlo.h:18-127): karam_run_mc_device of every problem
 * (same context, unseeded, same opts / dt / n_steps / method) as ONE launch of
 * the persistent per-instance kernel, one CTA per instance of every problem
 * (the problems with the most LU work per instance on the first CTAs), each
 * problem on the first factor/solve layout that fits a CTA (packed level
 * program and slots in shared memory; slots in shared memory; slots in a
 * global workspace). Results per problem through karam_read_results; each
 * problem's karam_timing holds the whole launch (job_ms, rounds = the most
 * rounds any instance ran, level_schedule 5). A problem's rescues share its
 * rescue workspace slots (a CTA takes a free one for each rescue, waiting up
 * to about 8 s of GPU clock; a solve that finds none is singular and the call
 * returns KARAM_E_CUDA after the job, results still readable). KARAM_E_INVALID
 * with a message naming the problem when one does not fit (evaluation or
 * factor data beyond a CTA's shared memory), and for a problem listed twice or
 * problems of different contexts. */
KARAM_API int karam_run_mc_multi(karam_problem *const *probs, int32_t n_probs,
                                 const karam_solver_opts *opts, double dt, int32_t n_steps,
                                 int32_t method);
/* Small-signal AC sweep of every instance at its DC operating point, after a
 * DC-only solve (karam_solve_dc): the analysis of ACSolver::solveAC_Sparse
 * (solvers/ac_solver.h:711-773), which the reference runs per netlist with a
 * dense complex LU (math/linalg.h:993-1078). Y(jw) = the NR Jacobian at the
 * DC point (every device conductance from the instance's own models) + jwC +
 * 1e-12 on every diagonal, with input_node (1-based; 0 = none) driven through
 * 1e6 S at `amplitude` volts; n_points log-spaced frequencies from f_start to
 * f_stop by the reference's formula (freqs_out[n_points] when non-NULL). One
 * CTA per (instance, frequency) factors Y on the problem's static pivots and
 * level schedule in complex FP64 and solves it. out_re / out_im:
 * [n_instances][n_points][n] node voltages (node i at index i - 1). status
 * [n_instances][n_points] (may be NULL): KARAM_ST_CONVERGED, KARAM_ST_SINGULAR
 * when a static pivot failed, or the instance's DC status when its DC did not
 * converge. Unlike the reference's admittance build, MOSFETs are linearised
 * with their own KP / VTO / LAMBDA and PMOS sign (ac_solver.h:688-696 uses
 * fixed NMOS values) and diode conductance keeps the DC floor of 1e-12 S (the
 * reference's AC build floors at 1e-15). KARAM_E_UNSUPPORTED when the problem
 * has no packed level program or its complex slots exceed one CTA's shared
 * memory; KARAM_E_STATE without a DC-only solve. */
KARAM_API int karam_ac_sweep(karam_problem *p, double f_start, double f_stop, int32_t n_points,
                             int32_t input_node, double amplitude, double *freqs_out,
                             double *out_re, double *out_im, int32_t *status);
/* SPICE netlist front-end (SPICEParser::parse, netlist/spice_parser.cpp:148-262)
 * for the subset the engine solves: R, C, V (DC, PULSE), I (DC), D, M with
 * .MODEL NMOS / PMOS (KP, VTO, LAMBDA) and D (IS, N), .TEMP, .OP, .TRAN, .END.
 * The reference parser's defects are fixed: MOSFET W= / L= are read, diodes
 * take IS / N from their .MODEL card, model names match case-insensitively,
 * SIN / SINE are both recognised (and rejected: DC and PULSE sources only),
 * and the first physical line is the title even when it starts with '*'. Elements the engine cannot solve are errors, not skipped.
 * karam_spice_parse returns KARAM_E_INVALID with the message (and line) in
 * err on failure. The netlist stays valid until karam_spice_free. Node names
 * map to indices 1.. in order of first appearance (ground: 0 / GND / VSS /
 * GROUND); karam_spice_node returns -1 for an unknown name. */
typedef struct karam_spice karam_spice;
KARAM_API int karam_spice_parse(const char *text, karam_spice **out, char *err, int32_t err_len);
KARAM_API const karam_netlist *karam_spice_netlist(const karam_spice *s);
KARAM_API int32_t karam_spice_node(const karam_spice *s, const char *name);
KARAM_API int karam_spice_analysis(const karam_spice *s, int32_t *has_op, int32_t *has_tran,
                                   double *tran_step, double *tran_stop, double *tran_start);
KARAM_API void karam_spice_free(karam_spice *s);

/* Measured choice of the factor/solve schedule (the warp-per-instance vs
 * block-per-instance autotuner; no reference counterpart: the reference
 * solves one instance at a time). Runs the first `rounds` NR rounds of a DC
 * job from the reference seed once per feasible schedule (the planner's
 * choice, a CTA per instance with its slots and the packed program in shared
 * memory, with its slots alone there, with them in global memory, the
 * persistent kernel), timed on the device, and keeps the fastest for this
 * problem and, process-wide, for problems made from an identical netlist with
 * the same batch size and precision on the same device; solves with
 * opts.schedule == 0 then use it. *schedule receives it as an opts.schedule value and *best_ms (either may
 * be null) its trial time. The problem's state afterwards is a trial's: run
 * the solve again. */
KARAM_API int karam_tune_schedule(karam_problem *p, const karam_solver_opts *opts, int32_t rounds,
                                  int32_t *schedule, double *best_ms);
KARAM_API int karam_read_results(karam_problem *p, double *out_v,
                                 karam_instance_stats *stats);
/* The DC convergence history of one instance after a solve: the last
 * KARAM_HISTORY_MAX (or fewer) records, oldest first -- per NR iteration its
 * max KCL residual [A] and max |v_new - v_old| [V], the residualNorm and
 * maxVoltageDelta of the reference's ConvergenceStep (infrastructure/
 * simtrace.h:30-37, filled at solvers/circuitsim_solver.cpp:408-425). *len
 * receives the count; residual and max_dv (both null, or both KARAM_HISTORY_MAX
 * long) receive the records. */
KARAM_API int karam_get_history(karam_problem *p, int32_t instance, double *residual,
                                double *max_dv, int32_t *len);
/* Blocks until the problem's stream is idle. */
KARAM_API int karam_sync(karam_problem *p);

/* ---- symbolic queries (for bit-exact checks against the reference) -------- */
/* CSR pattern of the Jacobian: row_ptr[n+1], col[nnz]. */
KARAM_API int karam_get_pattern(const karam_problem *p, int32_t *row_ptr, int32_t *col);
/* Stamp slot -> CSR index, in stampSoABlock triplet order (transient pattern,
 * gmin diagonal last): slot_csr[n_triplets]. */
KARAM_API int karam_get_stamp_map(const karam_problem *p, int32_t *slot_csr);
/* Raw Min-Fill ordering (with the reference's branch ids) and its translation
 * to a 0-based permutation of the n unknowns: raw[*raw_len], perm[n]. */
KARAM_API int karam_get_ordering(const karam_problem *p, uint32_t *raw, int32_t *raw_len,
                                 int32_t *perm);
/* Filled L+U pattern in permuted order: f_row_ptr[n+1], f_col[nnz_filled]. */
KARAM_API int karam_get_filled_pattern(const karam_problem *p, int32_t *f_row_ptr,
                                       int32_t *f_col);
/* SoA order of the tensorised devices: soa index -> netlist index. */
KARAM_API int karam_get_device_order(const karam_problem *p, int32_t *mos_order,
                                     int32_t *dio_order);
/* The static-pivot LU program on the value slots (permuted space), as the
 * device runs it: hdr[4 n] = (offset, nL, nU, diagonal slot) per pivot; data
 * at offset = Lrow[nL] Lslot[nL] Ucol[nU] Uslot[nU] T[nL * nU] (update target
 * slots); slot_rc[2 n_slots] = (row, col) of every value slot. With data NULL
 * only *data_len is written. */
KARAM_API int karam_get_lu_program(const karam_problem *p, int32_t *hdr, int32_t *data,
                                   int32_t *data_len, int32_t *slot_rc);
/* The same program packed as the device's pivot records, for programs whose
 * pivots all have nL <= 1 and nU <= 2 (else KARAM_E_UNSUPPORTED): rec[8 n] =
 * (meta, diagonal slot, L slot, L row, U slot 0, U slot 1, target 0, target 1)
 * with meta = nL | nU << 4 | chain << 8 | back-forwarding << 9;
 * rec2[2 n] = (U column 0, U column 1). No counterpart in the reference. */
KARAM_API int karam_get_lu_records(const karam_problem *p, int32_t *rec, int32_t *rec2);
/* The level schedule of the factor/solve kernel's LU (nested-dissection order
 * of the Min-Fill unknowns, its own value slots), as one int32 array:
 * n, n_slots, levels, long-list threshold, then 24 arrays, each as its length
 * followed by its values: nd_perm, nd_src, nd_diag, lv_piv, lv_piv_ptr,
 * lv_l_ptr, l_slot, l_piv, lv_ts_ptr, lv_tl_ptr, t_slot, t_off, pr_l, pr_u,
 * lv_ys_ptr, lv_yl_ptr, y_row, y_off, yp_l, yp_k, bs_off, bs_u, bs_c, and the
 * same schedule packed as the kernel stages it (empty if it does not fit
 * 16-bit fields).
 * With buf NULL (or cap too small) only *len is written; returns
 * KARAM_E_UNSUPPORTED when the problem has no schedule. No counterpart in the
 * reference. */
KARAM_API int karam_get_lu_schedule(const karam_problem *p, int32_t *buf, int64_t cap,
                                    int64_t *len);

/* ---- learned seeder ---------------------------------------------------------
 * The role of solvers/neural_seeder.h, whose learned model is future work in
 * the reference. A multilayer perceptron (hidden layers of `width` GELU units,
 * one linear output layer) maps an instance's device parameters (VTO and KP
 * of every MOSFET) and source DC values to an initial guess of its node
 * voltages. It is trained, on the problem's device, on DC solutions that
 * plain NR produced for the instances of a problem, and serves
 * opts->seeded = KARAM_SEED_MLP solves of problems with the same topology.
 * The GEMMs use BF16 weights and activations with FP32 accumulation; master
 * weights and Adam moments are FP32. Plain NR still decides convergence: a seeded
 * instance that has not converged after seed_max_iter iterations falls back
 * to full GMIN stepping. No counterpart in the reference. */
typedef struct karam_seeder karam_seeder;
KARAM_API int karam_seeder_create(karam_problem *p, int32_t width, int32_t hidden_layers,
                                  uint64_t init_seed, karam_seeder **out);
KARAM_API void karam_seeder_destroy(karam_seeder *s);
/* Adds the DC solutions of the problem's converged instances as training
 * samples; the problem's last solve must be a DC one (karam_solve_dc, or
 * karam_run_mc_device with n_steps = 0). *added = samples added. */
KARAM_API int karam_seeder_add_dc(karam_seeder *s, karam_problem *p, int32_t *added);
/* Adam on the mean squared error of the normalised voltages (feature and
 * voltage normalisations taken from the samples at the first call).
 * *final_loss = mean loss of the last epoch. */
KARAM_API int karam_seeder_train(karam_seeder *s, int32_t epochs, int32_t batch, float lr,
                                 uint64_t shuffle_seed, float *final_loss);
/* Attaches s (NULL detaches) for KARAM_SEED_MLP solves of p; p must have the
 * topology sizes the seeder was created for, and s must outlive that use. */
KARAM_API int karam_problem_set_seeder(karam_problem *p, karam_seeder *s);
/* The seeder's guesses for p's current instances: out_v[n_instances][n],
 * node order (index 0 = node 1). */
KARAM_API int karam_seeder_predict(karam_seeder *s, karam_problem *p, double *out_v);
/* The seeder's GEMM on host buffers, for tests: C[M][N] = op(A) op(B) with
 * op(A)[m][k] = transA ? A[k * lda + m] : A[m * lda + k] (B likewise),
 * operands rounded to BF16, FP32 accumulation, on the current device. */
KARAM_API int karam_seeder_gemm(int32_t M, int32_t N, int32_t K, const float *A, int32_t lda,
                                int32_t transA, const float *B, int32_t ldb, int32_t transB,
                                float *C);

/* ---- single-kernel access for measurement and parity ----------------------
 * Runs the evaluation + stamping kernel once for every instance at the given
 * voltages v[n_instances][n] and returns the Jacobian values without the gmin
 * diagonal (jac[n_instances][nnz], FP64 or FP32 cast up per precision) and the
 * device part of the KCL residual (f[n_instances][n]). h > 0 adds the
 * capacitor companions of the chosen method with history v_prev = i_prev = 0. */
KARAM_API int karam_eval_stamp(karam_problem *p, int32_t precision, const double *v,
                               double *jac, double *f);
/* karam_eval_stamp for callers that cannot allocate device memory at the time
 * of the call -- code whose GPU memory belongs to its own pool allocator, or
 * latency-critical loops where cudaMalloc / cudaFree would synchronise the
 * device. No counterpart in the reference (its evaluation allocates freely).
 * d_v ([n_instances][n], node order), d_jac ([n_instances][nnz], CSR order,
 * without the gmin diagonal) and d_f ([n_instances][n]) are DEVICE pointers the
 * caller owns; the instance parameters are the problem's (karam_set_instances).
 * Intermediates live in one fixed 16 MiB device array of the library, shared
 * by every call on a GPU and held until the process exits: a problem whose
 * batch capacity needs more is rejected with KARAM_E_INVALID and a message.
 * The array keeps the last call's contents; each call clears what it needs
 * cleared. Calls that overlap on the GPU (other threads or streams) race on the
 * array. Every call looks up the array's address on the problem's device (no
 * allocation; the first lookup on a device also loads the library's kernels
 * there), so make the first call on a device before any stream capture. Runs
 * on the problem's stream and synchronises it before returning, when the
 * outputs are written. */
KARAM_API int karam_eval_stamp_noalloc(karam_problem *p, int32_t precision, const double *d_v,
                                       double *d_jac, double *d_f);
/* Device-side accounting of the last solve or evaluation call (CUDA events on
 * the problem's stream; counters kept by the kernels). */
typedef struct karam_timing {
  double job_ms;            /* first kernel of the call to its last one             */
  double eval_ms;           /* summed duration of the device evaluation + stamping
                               launches (one per round; solves: 0 unless
                               opts.kernel_timing)                                   */
  double lu_ms;             /* summed duration of the control flow + factor/solve
                               launches (one per round; 0 unless opts.kernel_timing) */
  double rescue_ms;         /* summed duration of the rescue launches (one per round;
                               0 unless opts.kernel_timing)                          */
  int32_t rounds;           /* NR rounds                                             */
  int32_t eval_launches, lu_launches, rescue_launches, other_launches;
  int32_t lanes;            /* instances per CTA of the factor/solve kernel          */
  int32_t level_schedule;   /* factor/solve kernel that ran: 0 pivot-record LU (k_lu),
                               1 level schedule with a warp per instance (k_lu_nd),
                               2 level schedule with a CTA per instance and the
                               instance's slots in shared memory (k_lu_big), 3 the
                               same with the slots in global memory, 4 a CTA per
                               instance with slots and packed program in shared
                               memory, 5 the persistent kernel (all rounds of an
                               instance in one launch, the code of 4), 6 a CTA per
                               instance with slots and solve vector in global
                               memory                                                 */
  int64_t evals_dc;         /* instance evaluations in DC mode (live instances summed over rounds) */
  int64_t evals_tran;       /* instance evaluations in transient mode                */
  int64_t solves;           /* linear solves by the static-pivot LU                  */
  int64_t rescues;          /* linear solves redone by the rescue path               */
  int64_t rescues_dense;    /* of those, the ones that needed partial pivoting       */
  int32_t tail_rounds;      /* rounds run with a CTA per live instance over the list of
                               live instances (once no more are live than SMs)       */
  int32_t persistent_rounds; /* rounds run inside the persistent per-instance kernel
                               (every remaining round of an instance in one launch) */
  double seed_ms;           /* the learned seeder's inference inside the job (features,
                               the MLP's tcgen05 GEMMs and activations), 0 without it */
  int32_t resident_instances; /* instances whose state the persistent kernel kept in
                               shared memory for its whole launch                   */
  int32_t reserved_;
} karam_timing;
KARAM_API int karam_last_timing(const karam_problem *p, karam_timing *out);

#ifdef __cplusplus
}
#endif
#endif /* KARAM_H */
