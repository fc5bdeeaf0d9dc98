// nr_types.h -- data layout shared by the host driver, the statically compiled
// kernels and the kernels compiled at run time for a topology (NVRTC).
// No standard-library includes: the run-time compiler sees this text as is.
//
// All vectors live in the permuted index space of the Min-Fill ordering
// (position p holds unknown perm[p]); matrices live in the filled L+U pattern
// of that ordering, row-major. Instance data is instance-major.
#ifndef KARAM_NR_TYPES_H
#define KARAM_NR_TYPES_H

#if !defined(__CUDACC_RTC__)
#include <vector_types.h>
#endif

// Per-instance status codes and selectors (mirror include/karam.h).
#define KST_CONVERGED 0
#define KST_NOCONV 1
#define KST_SINGULAR 2
#define KST_NAN 3
#define KPREC_MIXED 1
#define KTRAN_TRAP 1
#define KSRC_PULSE 1

enum { MODE_DC = 0, MODE_TRAN = 1, MODE_DONE = 2 };
enum { SUB_NR = 0, SUB_POLISH = 1 };

// Per-instance solver state (one 104-byte record).
struct InstState {
  int mode;       // MODE_*
  int sub;        // SUB_*
  int g;          // GMIN step
  int it;         // NR iterations in the current GMIN step / time step
  int damp;       // damping count of the pending trial point
  int first;      // 1: x == v, nothing to judge
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
  int rescued;    // linear solves redone by the partial-pivoting rescue
  int depth;      // transient step halvings in effect (sub-step = h / 2^depth)
  int frac;       // part of the current step done, in units of h / 2^max_halvings
  int halvings;   // transient restarts with a halved step
};

// One linear solve handed to the partial-pivoting rescue.
struct RescueItem {
  int inst;
  int act;
  double gmin;
};

// Shared topology tables (device pointers).
struct DevTopo {
  int n, nf, n_mos, n_dio, n_res, n_cap, n_vs, n_is;
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
  const int* jt_off;
  const int* jt_code;
  const double* jlin_dc;
  const int* jcap_off;
  const int* jcap_code;
  const int* ft_off;
  const int* ft_code;
  const int4* lu_hdr;       // off, nL, nU, dpos
  const int* lu_data;       // Lrow[nL] Lpos[nL] Ucol[nU] Upos[nU] T[nL*nU]
  const int* f_row;         // row of every filled position (permuted)
  const int* f_colp;        // column of every filled position (permuted)
  const int* seed_vs;       // permuted positive node per source (-1 = ground)
  const int* seed_anode;    // permuted anode per netlist diode (-1 = ground)
  int n_seed_anode;
};

// Per-instance device buffers.
struct DevInst {
  int ni;
  const float* kp;          // [ni][n_mos] SoA order, or 0 = model card
  const float* vth;         // [ni][n_mos], or 0 = model card
  const double* vs_dc;      // [ni][n_vs]
  const double* vs_v1;      // [ni][n_vs]
  const double* vs_v2;      // [ni][n_vs]
  double* v;                // [ni][n] accepted point
  double* x;                // [ni][n] point under evaluation
  double* F;                // [ni][n] KCL residual at x (device currents, no gmin)
  double* Fmax;             // [ni]
  void* J;                  // [ni][nf] Jacobian at x without gmin (float or double)
  double* cap_vp;           // [ni][n_cap]
  double* cap_ip;           // [ni][n_cap]
  double* v_tp;             // [ni][n] voltages at the last accepted time point
  InstState* st;            // [ni]
  const double* seed;       // [ni][n] caller guesses (permuted) or 0
  double* rescue_ws;        // [rescue_slots][n][n] dense workspaces
  RescueItem* rescue_list;  // [ni]
  int* rescue_count;
  int rescue_slots;
  unsigned long long* counters;  // [4]: evaluations DC, evaluations transient, solves, rescues
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
  int max_halvings;  // transient restarts with a halved step (reference: 3)
};

#endif
