// nr_types.h -- data layout shared by the host driver and the kernels.
//
// All vectors live in the permuted index space of the Min-Fill ordering
// (position p holds unknown perm[p]). Matrix values live in "value slots":
// the positions of the filled L+U pattern that the static-pivot elimination
// can make non-zero (the unsymmetric structure of the stamps plus its fill),
// numbered row-major.
//
// Per-instance data is instance-interleaved: item k of instance i sits at
// [k * ld + i], ld = instance count rounded up to 32, so a warp that works on
// one item (a node, a device, a slot) for consecutive instances reads and
// writes whole 32-byte sectors, and every index load is a broadcast.
#ifndef KARAM_NR_TYPES_H
#define KARAM_NR_TYPES_H

#include <vector_types.h>

// Per-instance status codes and selectors (mirror include/karam.h).
#define KST_CONVERGED 0
#define KST_NOCONV 1
#define KST_SINGULAR 2
#define KST_NAN 3
#define KPREC_MIXED 1
#define KTRAN_TRAP 1
#define KSRC_PULSE 1

// Evaluation + stamping blocks: devices held in shared memory at a time, and
// items per block.
#ifndef KES_MAX_DEV
#define KES_MAX_DEV 48
#endif
#ifndef KES_MAX_ITEMS
#define KES_MAX_ITEMS 96
#endif
// Hub items (more devices than one block holds) sharing one group of device chunks.
#define KES_MAX_HUBS 4

enum { MODE_DC = 0, MODE_TRAN = 1, MODE_DONE = 2 };
enum { SUB_NR = 0, SUB_POLISH = 1 };

// Per-instance solver state (one record per instance, instance-major).
struct InstState {
  int mode;       // MODE_*
  int sub;        // SUB_*
  int g;          // GMIN step
  int it;         // NR iterations in the current GMIN step / time step
  int damp;       // damping count of the pending trial point
  int first;      // 1: x == v, nothing to compare yet
  int step;       // transient output step (1-based)
  int status;     // KST_*
  int iters;      // DC iterations, counted as the reference counts them
  int tran_iters; // transient NR iterations
  int polish;     // polishing iterations (DC + transient)
  int damped;     // damping re-evaluations
  int seeded;     // 1 while in a seeded start
  int seeded_ok;
  int pol_cnt;    // polishing iterations of the current solve
  int max_step_it;
  double prevF;   // previous accepted KCL residual (damping test)
  double prev_dv; // previous polishing update (stall test)
  double resid;   // last KCL residual seen
  int rescued;    // linear solves redone by the rescue path
  int depth;      // transient step halvings in effect (sub-step = h / 2^depth)
  int frac;       // part of the current step done, in units of h / 2^max_halvings
  int halvings;   // transient restarts with a halved step
  // convergence history of the DC NR iterations (ConvergenceStep records of
  // CircuitSim::solveDC, circuitsim_solver.cpp:408-443): the last
  // KHIST_LEN (residual, max |dv|) pairs sit in DevInst::hist; these are the
  // running quantities classifyFailure and the stagnation / divergence flags
  // need over the whole history
  int hist_n;       // iterations recorded
  int dir_changes;  // residual direction changes between consecutive iterations
  int hflags;       // KHF_* bits
  int lte_rejects;  // transient sub-steps redone because the LTE test failed
  double h1, h2;    // the last two recorded residuals (h1 most recent)
  double hprev;     // size of the last accepted transient sub-step (0: none yet)
};

// InstState::hflags
#define KHF_STAGNATION 1  // residual plateaued without converging
#define KHF_DIVERGENCE 2  // three consecutive increases of the residual
#define KHF_SINGULAR 4    // a DC linear solve failed for good
#define KHF_OVERFLOW 8    // some iteration moved a node by more than 100 V
#define KHIST_LEN 16

// One linear solve handed to the rescue path.
struct RescueItem {
  int inst;
  int act;
  double gmin;
};

// Shared topology tables (device pointers).
struct DevTopo {
  int n, nv, n_mos, n_dio, n_res, n_cap, n_vs, n_is;
  double temp_k;
  const int4* mos_term;     // d g s b (permuted, -1 = ground)
  const double2* mos_geo;   // {W/L, lambda}
  const int* mos_pmos;
  const double2* mos_card;  // {KP, VTO} of the model card (without per-instance values)
  const int2* dio_term;
  const double4* dio_par;   // {Is, N, Vt, 0}
  const double2* dio_lim;   // {Vt*T/Tnom, vcrit} for junction limiting
  const int* dio_level;     // limiting order levels (diodes of one level share no node)
  int n_dio_levels;
  const int2* res_term;
  const double* res_g;      // 1/R
  const int2* cap_term;
  const double* cap_c;
  const int2* vs_term;
  const int* vs_kind;
  const double* vs_pulse;   // [n_vs][7] (td tr tf pw per used; v1 v2 per instance)
  const int2* is_term;
  const double* is_amp;
  // Jacobian linear part per value slot: R + V stamps pre-summed (jlin) and
  // capacitor companions (jcap: conductance 2C/h_eff)
  const double* jlin_dc;
  const int* jcap_off;
  const int* jcap_code;
  // Evaluation + stamping blocks (see es_blocks in topology.cpp):
  //   es_block[b] = {item offset, items (-h: chunk block of a group of h hub
  //                  items), device offset, devices}
  //   es_hubc[b]  = hub chunk blocks: {chunk, chunks of the group, group, first
  //                 partial row of the group}
  //   es_item[k]  = {item (slot s < nv, node nv + i), term offset, terms,
  //                  hub items: offset of the item's chunk bounds in es_hub}
  //   es_dev      = global device ids (MOSFETs, then n_mos + diode index)
  //   es_jt       = slot device terms: sign bit | offset of the term's value
  //                 in the block's (or chunk's) device values for lane 0
  //   es_ft       = node terms {code, terminal a, terminal b, value offset of
  //                 a device term}, device codes carrying the local device;
  //                 es_fc their coefficients (1/R, source amplitude, 2C, or 0)
  int n_es_blocks;
  const int4* es_block;
  const int4* es_item;
  const int* es_dev;
  const int* es_jt;
  const int4* es_ft;
  const double* es_fc;
  const int* es_hub;        // hub items: term index where each device chunk starts, then the end
  const int4* es_hubc;
  int n_hub_groups, n_hub_rows;
  // the stamp terms in global device numbering, for the per-instance
  // evaluation of tail rounds (k_es_one): slot terms (jt_off [nv + 1],
  // jt_code), node terms (ft_off [n + 1], ft_code, terminals ft_a / ft_b,
  // coefficients ft_coef), and the hub items {item, es_hub offset, chunks, 0}
  const int *jt_off, *jt_code, *ft_off, *ft_code, *ft_a, *ft_b;
  const double* ft_coef;
  const int4* hub_items;    // {item, es_hub offset, chunks, offset of a hub slot's terms}
  int n_hub_items;
  int n_ft_terms, n_hub_slot_terms;  // node terms in all; terms of the hub slots
  int n_jt_terms, pad_jt_;           // slot terms in all
  // LU program per pivot k: hdr = (off, nL, nU, diagonal slot); data at off =
  // Lrow[nL] Lslot[nL] Ucol[nU] Uslot[nU] T[nL*nU] (update target slots)
  const int4* lu_hdr;
  const int* lu_data;
  int lu_small;             // 1: every pivot has nL <= 1 and nU <= 2
  const int4* lu_rec;       // pivot records when lu_small (2 int4 per pivot: meta, diagonal,
                            // Lslot, Lrow | Uslot0, Uslot1, T0, T1; see topology.cpp), else 0
  const int2* lu_rec2;      // back-substitution columns (Ucol0, Ucol1) per pivot
  // level-scheduled LU of the factor/solve kernel (nd_levels > 0): the same
  // static pivots on a nested-dissection order with its own value slots; one
  // warp per instance, pivots of a level side by side (tables as in
  // Topology::nd_*). Per instance in shared memory: nd_S slots, nd_SY
  // right-hand-side entries (odd strides).
  int nd_levels, nd_nv, nd_S, nd_SY;
  const int* nd_pos;        // Min-Fill index -> ND position
  const int* nd_src;        // ND slot -> Min-Fill value slot (-1: 0)
  const int* nd_diag;       // ND pivot -> ND slot of its diagonal
  const int *lv_piv, *lv_piv_ptr, *lv_l_ptr, *l_slot, *l_piv;
  const int *lv_ts_ptr, *lv_tl_ptr, *t_slot, *t_off, *pr_l, *pr_u;
  const int *lv_ys_ptr, *lv_yl_ptr, *y_row, *y_off, *yp_l, *yp_k;
  const int *bs_off, *bs_u, *bs_c;
  const int* nd_prog;       // the schedule packed for shared memory (nd_program)
  int nd_prog_len;          // ints (0: the level-scheduled kernel is not used)
  const int2* slot_rc;      // (row, col) of every value slot (permuted)
  const int* slot_ptr;      // [n + 1] first slot of each row (columns ascending within a row)
  const int* csc_ptr;       // [n + 1] value slots by column: (row, slot) in csc_ent
  const int2* csc_ent;
  const int* seed_vs;       // permuted positive node per source (-1 = ground)
  const int* seed_anode;    // permuted anode per netlist diode (-1 = ground)
  int n_seed_anode;
};

// Per-instance device buffers ([item][ld] unless noted).
struct DevInst {
  int ni;                   // instances in the batch
  int ld;                   // lane stride: ni rounded up to 32
  const float* kp;          // [n_mos][ld] SoA order, or 0 = model card
  const float* vth;         // [n_mos][ld], or 0 = model card
  const double* vs_dc;      // [n_vs][ld]
  const double* vs_v1;      // [n_vs][ld]
  const double* vs_v2;      // [n_vs][ld]
  double* v;                // [n][ld] accepted point
  double* x;                // [n][ld] point under evaluation
  double* F;                // [n][ld] KCL residual at x (device currents, no gmin)
  void* J;                  // [nv][ld] Jacobian value slots at x without gmin (float or double)
  unsigned long long* red_f;   // [ld] max |F| over nodes (bit pattern of a non-negative double)
  unsigned long long* red_dv;  // [ld] max |x - v| over nodes (bit pattern)
  int* red_flags;           // [ld] AND over nodes: bit 0 NR-converged, bit 1 polish-converged
  double* ev_t;             // [ld] time of the point the next round evaluates
  double* ev_heff;          // [ld] its companion step: < 0 not live, 0 DC, > 0 transient
  double* cap_vp;           // [n_cap][ld]
  double* cap_ip;           // [n_cap][ld]
  double* v_tp;             // [n][ld] voltages at the last accepted time point
  double* v_tpp;            // [n][ld] ... and at the accepted point before it (LTE predictor)
  double* ev_lte;           // [ld] LTE predictor ratio of the point the next round evaluates:
                            // sub-step / previous sub-step, < 0 when no LTE test applies
  InstState* st;            // [ni]
  const double* seed;       // [n][ld] caller guesses (permuted) or 0
  double* rescue_ws;        // [rescue_slots][2][n][n]: U and dense row buffers per rescue warp
  RescueItem* rescue_list;  // [ni]
  int* rescue_count;
  int rescue_slots;         // rescue warps (one workspace each)
  const int* live_in;       // tail rounds: the instances live at the start of the round (the
  const int* live_in_count; // block-per-instance kernel takes CTA b -> live_in[b]), else 0
  int* live_out;            // ... and the ones still live after it (filled by that kernel;
  int* live_out_count;      // the count is cleared by the round's k_es)
  void* lu_ws;              // [ni][nd_S] ND slots of the block-per-instance kernel when they
                            // live in global memory (float or double), else 0
  double* hub_part;         // [n_hub_rows][ld] hub items' sums per device chunk
  int* hub_cnt;             // [n_hub_groups][ld / 32] chunk blocks done (0 between launches)
  unsigned long long* counters;  // [5]: evaluations DC, evaluations transient, solves,
                                 // rescues, rescues that needed partial pivoting
  double* hist;             // [KHIST_LEN][2][ld] ring of (residual, max |dv|) per DC iteration
  double* wave;             // [ni][wave_steps][n_wave] node voltages after each step
  const int* wave_pos;      // permuted positions of the recorded nodes (-1 = ground)
  int n_wave, wave_steps;
};

struct JobParams {
  int precision;
  int max_nr_iter, gmin_steps;
  double reltol, vntol, kcl_shortcut, kcl_tol;
  int polish_max;
  double polish_rel, polish_abs;
  int n_steps;
  double h;
  double t0;  // time of step 0 (transient jobs continue from t0)
  int method;
  int seeded, seed_max_iter;
  int seed_bcast;    // 1: one seed for every instance, in lane 0 of DevInst::seed
  int max_halvings;  // transient restarts with a halved step (reference: 3)
  double growth32, growth64;  // static-pivot multiplier limits (FP32 / FP64 solves)
  double lte_rel, lte_abs;    // transient LTE test tolerances (lte_rel 0: no test)
};

// One problem of a multi-problem persistent launch (k_persist_multi): CTAs
// cta0 .. cta0 + I.ni - 1 of the launch run this problem's instances 0 ..
// I.ni - 1. variant: where the factor/solve keeps its ND slots and program --
// 0 packed program and slots in shared memory, 1 slots in shared memory and
// the schedule tables in global memory, 2 slots in I.lu_ws (global memory).
// K: the rescue workspace's column stride. resident_at: > 0 when each
// instance's state lives in the CTA's dynamic shared memory from that byte
// offset on. slot_lock: one word per rescue workspace slot (I.rescue_slots of
// them, 0 = free), the pool this problem's rescues take their slots from.
struct PersistJob {
  DevTopo T;
  DevInst I;
  JobParams P;
  int K;
  int cta0;
  int variant;
  int resident_at;
  int slot_values;  // 1: the evaluation keeps every slot term's value in shared memory
  int pad_;
  int* slot_lock;
};

// One small-signal AC sweep (k_ac): CTA (k, g) solves Y(j omega[k]) x = b for
// instance g. in_slot: value slot of the input node's diagonal, which gets
// g_in; in_pos: the input node's Min-Fill index, whose right-hand side is
// rhs_in (both -1 without excitation). Results go to out_re / out_im
// [ni][n_points][n] in node order (perm: Min-Fill index -> node index) and
// status [ni][n_points]. stage_prog: the packed level program is copied into
// shared memory after the slots (else read from global memory).
struct AcParams {
  const double* omega;
  int n_points;
  int in_slot, in_pos;
  int stage_prog;
  double g_in, rhs_in, gmin, tiny, growth;
  const int* perm;
  double* out_re;
  double* out_im;
  int* status;
};

#endif
