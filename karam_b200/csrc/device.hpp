// device.hpp -- device-side data layout shared by the kernels and the host driver.
//
// All vectors live in the permuted index space of the Min-Fill ordering
// (position p holds unknown perm[p]); matrices live in the filled L+U pattern
// of that ordering, row-major. Instance data is instance-major.
#pragma once
#include <cstdint>

namespace karam {

enum Mode : int32_t { MODE_DC = 0, MODE_TRAN = 1, MODE_DONE = 2 };
enum Sub : int32_t { SUB_NR = 0, SUB_POLISH = 1 };

// Per-instance solver state (one 104-byte record).
struct InstState {
  int32_t mode;       // Mode
  int32_t sub;        // Sub
  int32_t g;          // GMIN step
  int32_t it;         // NR iterations in the current GMIN step / time step
  int32_t damp;       // damping count of the pending trial point
  int32_t first;      // 1: x == v, nothing to judge
  int32_t step;       // transient step (t = step * h)
  int32_t status;     // KARAM_ST_*
  int32_t iters;      // DC iterations, counted as the reference counts them
  int32_t tran_iters; // transient NR iterations
  int32_t polish;     // polishing iterations (DC + transient)
  int32_t damped;     // damping re-evaluations
  int32_t seeded;     // 1 while in a seeded start
  int32_t seeded_ok;
  int32_t pol_cnt;    // polishing iterations of the current solve
  int32_t max_step_it;
  double prevF;       // previous accepted KCL residual (damping test)
  double prev_dv;     // previous polishing update (stall test)
  double resid;       // last KCL residual seen
  int32_t rescued;    // linear solves redone by the partial-pivoting rescue
  int32_t depth;      // transient step halvings in effect (sub-step = h / 2^depth)
  int32_t frac;       // part of the current step done, in units of h / 2^max_halvings
  int32_t halvings;   // transient restarts with a halved step
};
static_assert(sizeof(InstState) == 104, "InstState layout");

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
  const int4* mos_term;    // d g s b (permuted, -1 = ground)
  const double2* mos_geo;  // {W/L, lambda}
  const int* mos_pmos;
  const double2* mos_card; // {KP, VTO} of the model card (used without per-instance values)
  const int2* dio_term;
  const double4* dio_par;  // {Is, N, Vt, 0}
  const int2* res_term;
  const double* res_g;     // 1/R
  const int2* cap_term;
  const double* cap_c;
  const int2* vs_term;
  const int* vs_kind;
  const double* vs_pulse;  // [n_vs][7] (td tr tf pw per used; v1 v2 per instance)
  const int2* is_term;
  const double* is_amp;
  const int* jt_off;
  const int* jt_code;
  const double* jlin_dc;
  const int* jcap_off;
  const int* jcap_code;
  const int* ft_off;
  const int* ft_code;
  const int4* lu_hdr;      // off, d, dpos, 0
  const int* lu_data;
  const int* f_row;        // row of every filled position (permuted)
  const int* f_colp;       // column of every filled position (permuted)
  const int* seed_vs;      // permuted positive node per source (-1 = ground)
  const int* seed_anode;   // permuted anode per netlist diode (-1 = ground)
  int n_seed_anode;
};

// Per-instance device buffers.
struct DevInst {
  int ni;
  const float* kp;      // [ni][n_mos] SoA order, or nullptr = model card
  const float* vth;     // [ni][n_mos], or nullptr = model card
  const double* vs_dc;  // [ni][n_vs]
  const double* vs_v1;  // [ni][n_vs]
  const double* vs_v2;  // [ni][n_vs]
  double* v;            // [ni][n] accepted point
  double* x;            // [ni][n] point under evaluation
  double* F;            // [ni][n] KCL residual at x (device currents, no gmin)
  double* Fmax;         // [ni]
  void* J;              // [ni][nf] Jacobian at x without gmin (float or double)
  double* cap_vp;       // [ni][n_cap]
  double* cap_ip;       // [ni][n_cap]
  double* v_tp;         // [ni][n] voltages at the last accepted time point
  InstState* st;        // [ni]
  const double* seed;   // [ni][n] caller guesses (permuted) or nullptr
  // rescue of solves the static-pivot LU flags (growth / tiny pivot)
  double* rescue_ws;        // [rescue_slots][n][n] dense workspaces
  struct RescueItem* rescue_list;  // [ni]
  int* rescue_count;
  int rescue_slots;
  unsigned long long* counters;  // [4]: evaluations DC, evaluations transient, solves, rescues
  double* wave;         // [ni][wave_steps][n_wave] node voltages after each step
  const int* wave_pos;  // permuted positions of the recorded nodes (-1 = ground)
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

// Launch wrappers (kernels.cu).
struct LuLaunch {
  int ni_per_cta;  // instances per CTA (one lane each)
  int S;           // odd stride of the value rows
  int Sv;          // odd stride of the vector rows
  size_t smem;     // dynamic shared memory bytes
  int grid;
};
void launch_init(const DevTopo& T, const DevInst& I, const JobParams& P, cudaStream_t s);
// Moves every converged instance into the transient at step 1 (capacitor
// history from the accepted point when init_caps).
void launch_tran_start(const DevTopo& T, const DevInst& I, int init_caps, cudaStream_t s);
void launch_eval(const DevTopo& T, const DevInst& I, const JobParams& P, int prec,
                 cudaStream_t s);
void launch_lu(const DevTopo& T, const DevInst& I, const JobParams& P, const LuLaunch& L,
               int prec, int* active, cudaStream_t s);
size_t eval_smem_bytes(const DevTopo& T);
// Sets the dynamic shared-memory limits of the kernels (call outside stream capture).
void configure_kernels(const DevTopo& T, const LuLaunch& L);
LuLaunch plan_lu(const DevTopo& T, int ni, int prec, int max_smem, int num_sms);
void unpermute(const double* v_perm, const int* perm, double* out, int ni, int n, cudaStream_t s);
// Dense FP64 partial-pivoting solves for the instances the LU kernel flagged.
void launch_rescue(const DevTopo& T, const DevInst& I, const JobParams& P, int prec, int grid,
                   cudaStream_t s);
size_t rescue_smem_bytes(const DevTopo& T);

}  // namespace karam
