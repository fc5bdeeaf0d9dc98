// nr_device.cuh -- device code of the batched Newton-Raphson inner loop.
//
// One NR round over the batch is two kernels:
//   k_es  device evaluation at the trial point x (level-1 MOSFET, diode) into
//         shared memory and stamping: the Jacobian value slots (FP32 or FP64)
//         and the KCL residual F (FP64) with its per-instance reductions;
//   k_lu  per tile of L instances: the control flow (CircuitSim::solveDC's
//         GMIN / damping / convergence logic, circuitsim_solver.cpp:237-485,
//         and the transient NR loop with its attempt loop, :587-660), one
//         decision per round; static-pivot LU of each instance's matrix in
//         shared memory with the forward substitution fused into the
//         elimination, back substitution, x = v + dx, and junction limiting
//         (pnjlim) for DC NR iterations.
// Solves whose static pivots fail go to k_rescue (FP64 static pivots, then
// LU with partial pivoting, one warp per solve), launched after every round.
#ifndef KARAM_NR_DEVICE_CUH
#define KARAM_NR_DEVICE_CUH
#include <cstdint>

#include "nr_types.h"

namespace knr {

constexpr int kRoundThreads = 512;
constexpr int kMaxLanes = 32;
constexpr int kBigThreads = 1024;  // CTA size of the block-per-instance factor/solve kernel
constexpr unsigned kFull = 0xffffffffu;
#define KARAM_SEED_HISTORY_MAX 8  // NeuralSeeder::Config::maxHistory

enum Act : int {
  ACT_SOLVE = 1,
  ACT_DAMP = 2,
  ACT_ACCEPT = 4,
  ACT_TRAN_INIT = 8,
  ACT_STEP = 16,
  ACT_LIMIT = 32,    // sanitize + pnjlim after the solve (DC NR iterations)
  ACT_RESEED = 64,   // seeded start failed: restart from the reference seed
  ACT_RESTART = 128, // transient NR failed: retry from the last time point, halved step
  ACT_WAVE = 256     // a full output step completed: record the waveform
};

__device__ __forceinline__ int code_kind(int c) { return (c >> 24) & 0x7f; }
__device__ __forceinline__ int code_idx(int c) { return c & 0xffffff; }

// PULSE waveform, physics/circuitsim.h:2155-2170.
__device__ double pulse_at(const double* p7, double v1, double v2, double time) {
  const double td = p7[2], tr = p7[3], tf = p7[4], pw = p7[5], per = p7[6];
  double t = time - td;
  if (!(t > 0)) return v1;
  const double period = per > 0 ? per : 1e99;
  t = fmod(t, period);
  if (t < tr) return v1 + (v2 - v1) * (t / tr);
  if (t < tr + pw) return v2;
  if (t < tr + pw + tf) return v2 + (v1 - v2) * ((t - tr - pw) / tf);
  return v1;
}

__device__ __forceinline__ double source_value(const DevTopo& T, const DevInst& I, int g, int s,
                                               bool tran, double t) {
  const size_t k = (size_t)s * I.ld + g;
  if (!tran || T.vs_kind[s] != KSRC_PULSE) return I.vs_dc[k];
  return pulse_at(T.vs_pulse + 7 * s, I.vs_v1[k], I.vs_v2[k], t);
}

// seedInitialGuess (circuitsim_solver.cpp:32-116) for instance g into v, in
// the permuted space; one thread.
__device__ void reference_seed(const DevTopo& T, const DevInst& I, int g, double* v) {
  const int ld = I.ld;
  for (int i = 0; i < T.n; ++i) v[(size_t)i * ld + g] = 0.0;
  double vsup = 5.0;
  for (int s = 0; s < T.n_vs; ++s) {
    const double val = I.vs_dc[(size_t)s * ld + g];
    const int p = T.seed_vs[s];
    if (p >= 0) v[(size_t)p * ld + g] = val;
    if (val > vsup) vsup = val;
  }
  for (int d = 0; d < T.n_seed_anode; ++d) {
    const int p = T.seed_anode[d];
    if (p >= 0) v[(size_t)p * ld + g] = fmax(v[(size_t)p * ld + g], 0.6);
  }
  for (int s = 0; s < T.n_is; ++s) {
    const int p = T.is_term[s].x;
    if (p >= 0 && v[(size_t)p * ld + g] == 0.0) v[(size_t)p * ld + g] = vsup * 0.5;
  }
}

// ---------------------------------------------------------------------------
// init: seed, state (thread per instance; item loops are coalesced across lanes)
// ---------------------------------------------------------------------------
__global__ void k_init(DevTopo T, DevInst I, JobParams P) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= I.ni) return;
  const size_t ld = I.ld;
  const bool seeded = P.seeded && I.seed != nullptr;
  if (seeded) {
    const int sg = P.seed_bcast ? 0 : g;
    for (int i = 0; i < T.n; ++i) I.v[i * ld + g] = I.seed[i * ld + sg];
  } else {
    reference_seed(T, I, g, I.v);
  }
  for (int i = 0; i < T.n; ++i) I.x[i * ld + g] = I.v[i * ld + g];
  InstState s = {};
  s.mode = MODE_DC;
  s.sub = SUB_NR;
  s.g = seeded ? P.gmin_steps - 1 : 0;
  s.first = 1;
  s.status = KST_NOCONV;
  s.seeded = seeded ? 1 : 0;
  s.prevF = 0.0;
  s.prev_dv = -1.0;
  I.st[g] = s;
  I.ev_t[g] = 0.0;
  I.ev_heff[g] = 0.0;
  if (I.ev_lte) I.ev_lte[g] = -1.0;
  I.red_f[g] = 0ull;
  I.red_dv[g] = 0ull;
  I.red_flags[g] = 7;
}

// NeuralSeeder::predictSeed (solvers/neural_seeder.h:100-137, confidence
// :194-219) over the DC solutions of instances 0..W-1 recorded in order, the
// converged ones only (recordSolution follows a successful solve): snapshot j
// of m weighs 0.8^(m-1-j); one snapshot is returned as it is; otherwise the
// weighted mean, kept when the mean over nodes of 1 / (1 + weighted variance)
// is at least 0.3. Writes the seed to lane 0 of `seed` and *ok. One CTA.
__global__ void k_ema_seed(DevTopo T, DevInst I, int W, double* seed, int* ok) {
  __shared__ double wt[KARAM_SEED_HISTORY_MAX];
  __shared__ int idx[KARAM_SEED_HISTORY_MAX];
  __shared__ int s_m;
  __shared__ double s_conf[32];
  if (threadIdx.x == 0) {
    int m = 0;
    for (int j = 0; j < W && j < KARAM_SEED_HISTORY_MAX; ++j) {
      if (I.st[j].status != KST_CONVERGED) continue;
      for (int r = 0; r < m; ++r) wt[r] *= 0.8;  // recordSolution ages the history
      wt[m] = 1.0;
      idx[m++] = j;
    }
    s_m = m;
  }
  __syncthreads();
  const int m = s_m;
  const size_t ld = I.ld;
  double conf = 0.0;
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
    if (m == 0) break;
    if (m == 1) {
      seed[i * ld] = I.v[i * ld + idx[0]];
      continue;
    }
    double sum = 0.0, tw = 0.0;
    for (int r = 0; r < m; ++r) {  // unfused, as the reference's expressions
      tw += wt[r];
      sum = __dadd_rn(sum, __dmul_rn(I.v[i * ld + idx[r]], wt[r]));
    }
    const double si = sum / tw;
    double var = 0.0, tw2 = 0.0;
    for (int r = 0; r < m; ++r) {
      const double d = I.v[i * ld + idx[r]] - si;
      var = __dadd_rn(var, __dmul_rn(__dmul_rn(wt[r], d), d));
      tw2 += wt[r];
    }
    conf += 1.0 / (1.0 + (var / tw2) / (1.0 * 1.0));
    seed[i * ld] = si;
  }
  for (int o = 16; o > 0; o >>= 1) conf += __shfl_xor_sync(kFull, conf, o);
  if ((threadIdx.x & 31) == 0) s_conf[threadIdx.x >> 5] = conf;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) c += s_conf[w];
    *ok = m == 1 || (m >= 2 && c / T.n >= 0.3);
  }
}

// ---------------------------------------------------------------------------
// device physics
// ---------------------------------------------------------------------------
// Level-1 MOSFET of batchMosfetPhysics_generic (tensors/physics_tensors.cpp:53-104).
// Products are kept unfused (__dmul_rn / __dadd_rn) where the reference's
// expression would otherwise be contracted into an FMA, so conductances match
// the CPU bit for bit.
__device__ __forceinline__ void mosfet_eval(double vd, double vg, double vs, double sign,
                                            double kpm, double vthm, double wl, double lam,
                                            double& ids, double& gm, double& gds) {
  const double vgs = vg - vs, vds = vd - vs;
  const double lvgs = sign * vgs, lvds = sign * vds, lvth = sign * vthm;
  const double K = __dmul_rn(__dmul_rn(0.5, kpm), wl);
  const double vov = lvgs - lvth;
  if (vov <= 0.0) {
    ids = 0.0;
    gm = 0.0;
    gds = 1e-12;
  } else if (lvds < vov) {
    const double q = __dadd_rn(__dmul_rn(__dmul_rn(2.0, vov), lvds), -__dmul_rn(lvds, lvds));
    ids = __dmul_rn(__dmul_rn(sign, K), q);
    gm = __dmul_rn(__dmul_rn(2.0, K), lvds);
    gds = __dmul_rn(__dmul_rn(2.0, K), vov - lvds);
  } else {
    const double clm = __dadd_rn(1.0, __dmul_rn(lam, lvds));
    ids = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sign, K), vov), vov), clm);
    gm = __dmul_rn(__dmul_rn(__dmul_rn(2.0, K), vov), clm);
    gds = __dmul_rn(__dmul_rn(__dmul_rn(K, vov), vov), lam);
  }
  if (gds < 1e-12) gds = 1e-12;
}

// Diode of batchDiodePhysics_generic (tensors/physics_tensors.cpp:19-51).
__device__ __forceinline__ void diode_eval(double vdd, double4 par, double& id, double& gd) {
  const double nvt = __dmul_rn(par.y, par.z);
  const double vcrit = __dmul_rn(30.0, nvt);
  const double arg = vdd / nvt;
  const double ex = exp(fmin(arg, 30.0));
  const double ibase = __dmul_rn(par.x, ex - 1.0);
  const double gbase = __dmul_rn(par.x / nvt, ex);
  const double delta = fmax(0.0, vdd - vcrit);
  id = __dadd_rn(ibase, __dmul_rn(delta, gbase));
  gd = fmax(1e-12, gbase);
}

// Inputs of one device evaluation: terminal voltages and parameters
// (MOSFET: vd, vg, vs, KP, VTO, W/L, lambda, sign; diode: v_a - v_c in va,
// Is, N, Vt in p0..p2).
struct DevIn {
  bool mos;
  double va, vb, vc, p0, p1, p2, p3, sign;
};

// A load of an instance buffer: through the read-only data cache when the
// buffer is known to be in global memory (G), else a plain load (the
// persistent kernels may keep the instance's state in shared memory).
template <bool G, typename V>
__device__ __forceinline__ V ld_in(const V* p) {
  if constexpr (G)
    return __ldg(p);
  else
    return *p;
}

// The LTE test of one node at the candidate point x of a transient sub-step:
// the linear extrapolation p = v_tp + r (v_tp - v_tpp) from the two previous
// accepted points (r = sub-step / previous sub-step) must lie within
// lte_rel * max(|x|, |v_tp|) + lte_abs of x.
__device__ __forceinline__ bool lte_node_ok(double x, double vt, double vq, double r,
                                            const JobParams& P) {
  const double p = vt + r * (vt - vq);
  return !(fabs(x - p) > P.lte_rel * fmax(fabs(x), fabs(vt)) + P.lte_abs);
}

// Loads the inputs of device d (MOSFETs first, then diodes) for instance g.
// Nothing here depends on an earlier evaluation, so the loads of several
// devices can be in flight together.
template <bool G = true>
__device__ __forceinline__ DevIn load_device(const DevTopo& T, const DevInst& I, int d, int g) {
  const size_t ld = I.ld;
  const int nm = T.n_mos;
  const double* __restrict__ x = I.x;
  DevIn in;
  in.mos = d < nm;
  if (in.mos) {
    const int4 tm = __ldg(&T.mos_term[d]);
    const double2 geo = __ldg(&T.mos_geo[d]);
    in.sign = __ldg(&T.mos_pmos[d]) ? -1.0 : 1.0;
    if (I.kp) {
      in.p0 = (double)ld_in<G>(&I.kp[d * ld + g]);
      in.p1 = (double)ld_in<G>(&I.vth[d * ld + g]);
    } else {
      const double2 card = __ldg(&T.mos_card[d]);
      in.p0 = card.x;
      in.p1 = card.y;
    }
    in.p2 = geo.x;
    in.p3 = geo.y;
    in.va = tm.x >= 0 ? ld_in<G>(&x[tm.x * ld + g]) : 0.0;
    in.vb = tm.y >= 0 ? ld_in<G>(&x[tm.y * ld + g]) : 0.0;
    in.vc = tm.z >= 0 ? ld_in<G>(&x[tm.z * ld + g]) : 0.0;
  } else {
    const int k = d - nm;
    const int2 tt = __ldg(&T.dio_term[k]);
    const double4 par = T.dio_par[k];
    in.p0 = par.x;
    in.p1 = par.y;
    in.p2 = par.z;
    in.p3 = par.w;
    in.sign = 0.0;
    in.va = (tt.x >= 0 ? ld_in<G>(&x[tt.x * ld + g]) : 0.0) - (tt.y >= 0 ? ld_in<G>(&x[tt.y * ld + g]) : 0.0);
    in.vb = in.vc = 0.0;
  }
  return in;
}

// Evaluates loaded inputs into out[0..2] (stride 32 doubles): MOSFET gm,
// gds, ids; diode g, i.
__device__ __forceinline__ void eval_loaded(const DevIn& in, double* out) {
  if (in.mos) {
    double ids, gm, gds;
    mosfet_eval(in.va, in.vb, in.vc, in.sign, in.p0, in.p1, in.p2, in.p3, ids, gm, gds);
    out[0] = gm;
    out[32] = gds;
    out[64] = ids;
  } else {
    double id, gd;
    diode_eval(in.va, make_double4(in.p0, in.p1, in.p2, in.p3), id, gd);
    out[0] = gd;
    out[32] = id;
  }
}

__device__ __forceinline__ void eval_device(const DevTopo& T, const DevInst& I, int d, int g,
                                            double* out) {
  eval_loaded(load_device(T, I, d, g), out);
}

// Devices k0 and k0 + 8 of a block's device list for instance g (k < n): both
// devices' loads are issued before either computes.
__device__ __forceinline__ void eval_device_pair(const DevTopo& T, const DevInst& I,
                                                 const int* devs, int k0, int n, int g,
                                                 double* s_dev, int lane) {
  const int k1 = k0 + 8;
  const DevIn a = load_device(T, I, __ldg(&devs[k0]), g);
  if (k1 < n) {
    const DevIn b = load_device(T, I, __ldg(&devs[k1]), g);
    eval_loaded(a, s_dev + k0 * 96 + lane);
    eval_loaded(b, s_dev + k1 * 96 + lane);
  } else {
    eval_loaded(a, s_dev + k0 * 96 + lane);
  }
}

// ---------------------------------------------------------------------------
// per-instance control flow
// ---------------------------------------------------------------------------
__device__ __forceinline__ double gmin_of(int g) {
  double gm = pow(10.0, -(3.0 + g * 0.5));
  return gm < 1e-12 ? 1e-12 : gm;
}

__device__ int dc_done(InstState& s, const JobParams& P) {
  if (P.n_steps > 0) {
    s.mode = MODE_TRAN;
    s.sub = SUB_NR;
    s.step = 1;
    s.first = 1;
    s.it = 0;
    s.hprev = 0.0;
    return ACT_TRAN_INIT;
  }
  s.mode = MODE_DONE;
  s.status = KST_CONVERGED;
  return 0;
}

// A transient sub-step converged: advance within the output step; hsub
// receives the completed sub-step's size for the capacitor history update.
__device__ int step_done(InstState& s, const JobParams& P, double& hsub) {
  const int units = 1 << P.max_halvings;
  const int size = units >> s.depth;
  hsub = P.h * size / units;
  s.hprev = P.lte_rel > 0.0 ? hsub : 0.0;  // with the LTE test off no predictor is kept
  s.frac += size;
  s.sub = SUB_NR;
  s.first = 1;
  s.it = 0;
  int a = ACT_STEP;
  if (s.frac >= units) {
    a |= ACT_WAVE;
    s.step++;
    s.frac = 0;
    s.depth = 0;
    if (s.step > P.n_steps) {
      s.mode = MODE_DONE;
      s.status = KST_CONVERGED;
    }
  }
  return a;
}

// A converged transient sub-step passes the LTE test (lte_ok: every node of
// the accepted point lies within lte_rel * max(|x|, |v_tp|) + lte_abs of the
// linear extrapolation from the two previous accepted points) or is redone
// from the last accepted point with half the step while halvings remain; at
// the last halving it is accepted as it is.
__device__ int accept_substep(InstState& s, const JobParams& P, bool lte_ok, double& hsub) {
  if (!lte_ok && P.lte_rel > 0.0 && s.depth < P.max_halvings) {
    s.depth++;
    s.halvings++;
    s.lte_rejects++;
    s.sub = SUB_NR;
    s.it = 0;
    s.first = 1;
    return ACT_RESTART;
  }
  return ACT_ACCEPT | step_done(s, P, hsub);
}

__device__ int start_polish(InstState& s, double& gmin_out) {
  s.sub = SUB_POLISH;
  s.pol_cnt = 0;
  s.prev_dv = -1.0;
  gmin_out = 1e-12;
  return ACT_SOLVE;
}

// Convergence history of a DC NR iteration whose final trial point has KCL
// residual F and moved the nodes by at most dv (before s.prevF, the previous
// iteration's residual, is replaced): the stagnation and divergence flags of
// circuitsim_solver.cpp:427-443 and the running counts classifyFailure
// (solvers/convergence_engine.h:26-87) needs. The (F, dv) pair itself goes
// to the instance's history ring (instance_decide).
__device__ __forceinline__ void record_iteration(InstState& s, double F, double dv,
                                                 const JobParams& P) {
  if (s.it > 0 && fabs(s.prevF - F) < 1e-15 && F > P.kcl_tol) s.hflags |= KHF_STAGNATION;
  if (s.hist_n >= 2 && F > s.h1 && s.h1 > s.h2) s.hflags |= KHF_DIVERGENCE;
  if (s.hist_n >= 2) {
    const double pd = s.h1 - s.h2, cd = F - s.h1;
    if ((pd > 0.0 && cd < 0.0) || (pd < 0.0 && cd > 0.0)) s.dir_changes++;
  }
  if (dv > 100.0) s.hflags |= KHF_OVERFLOW;
  s.h2 = s.h1;
  s.h1 = F;
  s.hist_n++;
}

// One decision of the NR control flow for the trial point x whose KCL
// residual is F (vconv / pok / dv compare x against the accepted point v).
__device__ int decide(InstState& s, double F, bool vconv, bool pok, bool lte_ok, double dv,
                      const JobParams& P, double& gmin_out, double& hsub) {
  const int G = P.gmin_steps;
  if (s.mode == MODE_DONE) return 0;
  s.resid = F;
  if (!isfinite(F)) {
    s.status = KST_NAN;
    s.mode = MODE_DONE;
    return 0;
  }
  if (s.mode == MODE_DC) {
    if (s.sub == SUB_NR) {
      if (s.first) {
        s.first = 0;
        gmin_out = gmin_of(s.g);
        return ACT_SOLVE | ACT_LIMIT;
      }
      // limit-cycle breaker, circuitsim_solver.cpp:391-406
      if (s.it > 0 && F >= s.prevF && s.damp < 2) {
        s.damp++;
        s.damped++;
        return ACT_DAMP;
      }
      s.damp = 0;
      record_iteration(s, F, dv, P);
      s.prevF = F;
      const double tol = (s.g == G - 1) ? P.kcl_tol : 1.0;
      const bool conv = (F < P.kcl_shortcut) || (vconv && !(F > tol));
      s.it++;
      if (conv) {
        s.iters += s.it;
        if (s.g == G - 1) {
          if (s.seeded) s.seeded_ok = 1;
          s.seeded = 0;
          if (P.polish_max > 0) return ACT_ACCEPT | start_polish(s, gmin_out);
          return ACT_ACCEPT | dc_done(s, P);
        }
        s.g++;
        s.it = 0;
        gmin_out = gmin_of(s.g);
        return ACT_ACCEPT | ACT_SOLVE | ACT_LIMIT;
      }
      const int cap = s.seeded ? P.seed_max_iter : P.max_nr_iter;
      if (s.it >= cap) {
        s.iters += s.it + 1;
        if (s.seeded) return ACT_RESEED;
        if (s.g == G - 1 || !(s.prevF < 1.0)) {
          s.status = KST_NOCONV;
          s.mode = MODE_DONE;
          return ACT_ACCEPT;
        }
        s.g++;
        s.it = 0;
      }
      gmin_out = gmin_of(s.g);
      return ACT_ACCEPT | ACT_SOLVE | ACT_LIMIT;
    }
    // polishing: x is the Newton step from v at the final gmin
    s.polish++;
    s.pol_cnt++;
    const bool stalled = s.prev_dv >= 0.0 && dv > 0.5 * s.prev_dv;
    if (pok || dv == 0.0 || stalled || s.pol_cnt >= P.polish_max) return ACT_ACCEPT | dc_done(s, P);
    s.prev_dv = dv;
    gmin_out = 1e-12;
    return ACT_ACCEPT | ACT_SOLVE;
  }
  // transient
  if (s.sub == SUB_NR) {
    if (s.first) {
      s.first = 0;
      s.it = 0;
      gmin_out = 1e-12;
      return ACT_SOLVE;
    }
    const bool conv = (F < P.kcl_shortcut) || (vconv && !(F > P.kcl_tol));
    s.it++;
    if (conv) {
      s.tran_iters += s.it;
      if (s.it > s.max_step_it) s.max_step_it = s.it;
      if (P.polish_max > 0) return ACT_ACCEPT | start_polish(s, gmin_out);
      return accept_substep(s, P, lte_ok, hsub);
    }
    if (s.it >= P.max_nr_iter) {
      // attempt loop of CircuitSim::stepTransient (circuitsim_solver.cpp:587-660)
      s.tran_iters += s.it + 1;
      if (s.it + 1 > s.max_step_it) s.max_step_it = s.it + 1;
      if (s.depth < P.max_halvings) {
        s.depth++;
        s.halvings++;
        s.it = 0;
        s.first = 1;
        return ACT_RESTART;
      }
      s.status = KST_NOCONV;
      s.mode = MODE_DONE;
      return ACT_ACCEPT;
    }
    gmin_out = 1e-12;
    return ACT_ACCEPT | ACT_SOLVE;
  }
  s.polish++;
  s.pol_cnt++;
  const bool stalled = s.prev_dv >= 0.0 && dv > 0.5 * s.prev_dv;
  if (pok || dv == 0.0 || stalled || s.pol_cnt >= P.polish_max) return accept_substep(s, P, lte_ok, hsub);
  s.prev_dv = dv;
  gmin_out = 1e-12;
  return ACT_ACCEPT | ACT_SOLVE;
}

// Time and capacitor-companion step of the point an instance evaluates: DC
// (heff = 0), or the end of the current transient sub-step of size h/2^depth,
// ((step - 1) * units + frac + size) * h / units; heff is the trapezoidal
// companion's step (backward Euler = trapezoidal stamp at 2 h).
__device__ __forceinline__ void eval_point(const InstState& st, const JobParams& P, double& t,
                                           double& heff) {
  if (st.mode != MODE_TRAN) {
    t = 0.0;
    heff = 0.0;
    return;
  }
  const int units = 1 << P.max_halvings;
  const int size = units >> st.depth;
  const double hsub = P.h * size / units;
  t = P.t0 + (double)((st.step - 1) * units + st.frac + size) * (P.h / units);
  heff = P.method == KTRAN_TRAP ? hsub : 2.0 * hsub;
}

// applyPnJunctionLimits (circuitsim_solver.cpp:118-169) for diode d of
// instance g on x against v. The temperature-scaled Vt and vcrit (pnjlim's
// compute_vcrit, physics/device_physics.h:175-179) are per-diode constants the
// host computes with the reference's expressions once per topology.
__device__ __forceinline__ void limit_one(const DevTopo& T, int d, double* x, const double* v,
                                          size_t ld, int g) {
  const int2 tt = __ldg(&T.dio_term[d]);
  const int p = tt.x, q = tt.y;
  if (p < 0 && q < 0) return;
  const double2 lim = __ldg(&T.dio_lim[d]);
  const double vt = lim.x, vcrit = lim.y;
  const size_t pp = (size_t)p * ld + g, qq = (size_t)q * ld + g;
  const double vjo = (p >= 0 ? v[pp] : 0.0) - (q >= 0 ? v[qq] : 0.0);
  const double vjn = (p >= 0 ? x[pp] : 0.0) - (q >= 0 ? x[qq] : 0.0);
  double vl = vjn;
  if (vjo > 30.0 * vt && vjn > 30.0 * vt) {
    vl = vjn;
  } else if (vjo < -5.0 * vt && vjn < -5.0 * vt) {
    vl = vjn;
  } else if (vjn > vcrit && fabs(vjn - vjo) > 2.0 * vt) {
    if (vjo > 0.0) {
      const double arg = 1.0 + (vjn - vjo) / vt;
      vl = arg > 0.0 ? vjo + vt * log(arg) : vcrit;
    } else {
      vl = vt * log(vjn / vt);
    }
  } else if (vjn < -5.0 * vt) {
    vl = fmax(vjn, vjo - 5.0 * vt);
  }
  const double corr = vjn - vl;
  if (fabs(corr) > 1e-12) {
    if (p >= 0 && q >= 0) {
      x[pp] -= corr * 0.5;
      x[qq] += corr * 0.5;
    } else if (p >= 0) {
      x[pp] -= corr;
    } else {
      x[qq] += corr;
    }
  }
}

// Static-pivot LU + solve of one instance on the value slots. A: the slot
// values (gmin already on the diagonal), y: right-hand side in, solution out;
// element k of either sits at [k * L] (L = lanes of the tile). Pivot k of the
// program lists Lrow/Lslot (rows i > k with A[i][k] != 0), Ucol/Uslot (columns
// j > k of row k) and the update target of every (i, j) pair. The forward
// substitution runs inside the elimination (y[k] is final when pivot k is
// reached), which leaves the back substitution as the only second pass.
// Returns false when the static pivots are unusable: a tiny or non-finite
// pivot, a multiplier above growth_limit, or a non-finite solution.
//
// Two schedules with identical arithmetic: when every pivot has nL <= 2 and
// nU <= 2 (chain-like circuits) the program arrives as packed records in
// shared memory (rec), the record of pivot k + 1 is decoded while pivot k
// computes, and all value loads of a pivot are issued before its stores (its
// L, U, diagonal and target slots are distinct), so a pivot costs about one
// shared-memory round trip plus the reciprocal; otherwise (rec == 0) a
// generic loop walks the program in global memory.
// Stages the pivot records into shared memory with every slot / row offset
// multiplied by the lane count L (so the factorisation indexes A and y with
// them directly): rec[2k], rec[2k+1] per pivot, then rec2[k]. Whole CTA.
__device__ __forceinline__ void stage_pivots(const DevTopo& T, int4* rec, int L) {
  int2* rec2 = reinterpret_cast<int2*>(rec + 2 * T.n);
  for (int k = threadIdx.x; k < T.n; k += blockDim.x) {
    const int4 a = __ldg(&T.lu_rec[2 * k]), b = __ldg(&T.lu_rec[2 * k + 1]);
    const int2 c = __ldg(&T.lu_rec2[k]);
    rec[2 * k] = make_int4(a.x, a.y * L, a.z * L, a.w * L);
    rec[2 * k + 1] = make_int4(b.x * L, b.y * L, b.z * L, b.w * L);
    rec2[k] = make_int2(c.x * L, c.y * L);
  }
}

// Correctly rounded reciprocal (the value of 1 / x).
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }

template <typename T>
__device__ bool lu_solve(T* __restrict__ A, T* __restrict__ y, int L, const DevTopo& Tp,
                         const int4* __restrict__ rec, T tiny, T growth_limit) {
  const int n = Tp.n;
  bool ok = true;
  T lmax = T(0);
  if (rec) {
    // w00, w01, wy0: what the previous pivot wrote to its two targets and to
    // its L row's right-hand side; a chain pivot (meta bit 8) takes its L
    // value, second target and L row's right-hand side from them. L values
    // are not stored: the forward substitution runs inside the elimination
    // and the back substitution reads only U, so nothing reads them again.
    const int2* rec2 = reinterpret_cast<const int2*>(rec + 2 * n);
    T w00 = T(0), w01 = T(0), wy0 = T(0);
    int4 ra = rec[0], rb = rec[1];
    for (int k = 0; k < n; ++k) {
      const int kn = k + 1 < n ? k + 1 : k;
      const int4 na = rec[2 * kn], nb = rec[2 * kn + 1];
      const bool chain = (ra.x >> 8) & 1;
      const int nl = ra.x & 15, nu = (ra.x >> 4) & 15;
      const T piv = A[ra.y];
      const T yk = y[k * L];
      const T u0 = nu > 0 ? A[rb.x] : T(0), u1 = nu > 1 ? A[rb.y] : T(0);
      const T b00 = (nl > 0 && nu > 0) ? A[rb.z] : T(0);
      const T a0 = chain ? w00 : (nl > 0 ? A[ra.z] : T(0));
      const T y0 = chain ? wy0 : (nl > 0 ? y[ra.w] : T(0));
      const T b01 = chain ? w01 : ((nl > 0 && nu > 1) ? A[rb.w] : T(0));
      ok = ok && isfinite(piv) && !(fabs(piv) < tiny);
      const T r = recip(piv);
      A[ra.y] = r;
      if (nl > 0) {
        const T l = a0 * r;
        lmax = fmax(lmax, fabs(l));
        wy0 = y0 - l * yk;
        if (nu > 0) w00 = b00 - l * u0;
        if (nu > 1) w01 = b01 - l * u1;
        y[ra.w] = wy0;
        if (nu > 0) A[rb.z] = w00;
        if (nu > 1) A[rb.w] = w01;
      }
      ra = na;
      rb = nb;
    }
    bool finite = true;
    T yprev = T(0);  // the unknown the previous back-substitution step solved
    for (int k = n - 1; k >= 0; --k) {
      const int4 a = rec[2 * k], b = rec[2 * k + 1];
      const int2 c = rec2[k];
      const int nu = (a.x >> 4) & 15;
      const unsigned fb = ((unsigned)a.x >> 9) & 3u;
      T sv = y[k * L];
      if (nu > 0) sv -= A[b.x] * ((fb & 1u) ? yprev : y[c.x]);
      if (nu > 1) sv -= A[b.y] * ((fb & 2u) ? yprev : y[c.y]);
      sv *= A[a.y];
      y[k * L] = sv;
      yprev = sv;
      finite = finite && isfinite(sv);
    }
    return ok && finite && !(lmax > growth_limit);
  }
  const int4* __restrict__ hdr = Tp.lu_hdr;
  const int* __restrict__ data = Tp.lu_data;
  int4 h = __ldg(hdr);
  for (int k = 0; k < n; ++k) {
    const int4 hn = __ldg(hdr + (k + 1 < n ? k + 1 : k));
    const int nl = h.y, nu = h.z;
    const int* lr = data + h.x;
    const int* ls = lr + nl;
    const int* us = ls + nl + nu;
    const int* ts = us + nu;
    const T piv = A[h.w * L];
    ok = ok && isfinite(piv) && !(fabs(piv) < tiny);
    const T r = recip(piv);
    A[h.w * L] = r;
    const T yk = y[k * L];
    for (int a = 0; a < nl; ++a) {
      const int sl = __ldg(ls + a);
      const T l = A[sl * L] * r;
      lmax = fmax(lmax, fabs(l));
      A[sl * L] = l;
      y[__ldg(lr + a) * L] -= l * yk;
      const int* trow = ts + a * nu;
      for (int b = 0; b < nu; ++b) A[__ldg(trow + b) * L] -= l * A[__ldg(us + b) * L];
    }
    h = hn;
  }
  bool finite = true;
  for (int k = n - 1; k >= 0; --k) {
    const int4 hk = __ldg(hdr + k);
    const int nl = hk.y, nu = hk.z;
    const int* uc = data + hk.x + 2 * nl;
    const int* us = uc + nu;
    T s = y[k * L];
    for (int b = 0; b < nu; ++b) s -= A[__ldg(us + b) * L] * y[__ldg(uc + b) * L];
    s *= A[hk.w * L];
    y[k * L] = s;
    finite = finite && isfinite(s);
  }
  return ok && finite && !(lmax > growth_limit);
}

// What the control flow does when a linear solve of a DC NR iteration fails
// for good (the reference's singular-matrix branch, circuitsim_solver.cpp:358-366):
// a seeded start falls back to the reference seed, anything else stops.
// Returns false when the instance stopped.
__device__ bool on_singular(const DevTopo& Tp, const DevInst& I, int g) {
  InstState s = I.st[g];
  if (s.mode == MODE_DC && s.sub == SUB_NR) {
    s.iters += 2 * (s.it + 1);
    s.hflags |= KHF_SINGULAR;
  }
  bool alive = false;
  if (s.mode == MODE_DC && s.sub == SUB_NR && s.seeded) {
    reference_seed(Tp, I, g, I.v);
    for (int i = 0; i < Tp.n; ++i) I.x[(size_t)i * I.ld + g] = I.v[(size_t)i * I.ld + g];
    s.g = 0;
    s.it = 0;
    s.first = 1;
    s.damp = 0;
    s.prevF = 0.0;
    s.seeded = 0;
    alive = true;
  } else {
    s.status = KST_SINGULAR;
    s.mode = MODE_DONE;
  }
  I.st[g] = s;
  return alive;
}

// ---------------------------------------------------------------------------
// the NR round: k_es -> k_lu (-> k_rescue)
// ---------------------------------------------------------------------------
// One KCL term of record q (es_ft / es_fc) for instance g; device terms read
// the CTA's device values sd ([local][3][32] doubles, lane offset applied).
template <bool G = true>
__device__ __forceinline__ double node_term(const DevTopo& T, const DevInst& I, const JobParams& P,
                                            int4 tm, double coef, int g, bool tran, double t,
                                            double heff, const double* sd) {
  const size_t ld = I.ld;
  const int idx = code_idx(tm.x), kind = code_kind(tm.x);
  if (kind >= 4) return sd[tm.w];  // diode i / MOSFET ids, at the offset the table carries
  if (kind == 2) return coef;                                                // current source
  const double va = tm.y >= 0 ? ld_in<G>(&I.x[tm.y * ld + g]) : 0.0;
  const double vb = tm.z >= 0 ? ld_in<G>(&I.x[tm.z * ld + g]) : 0.0;
  if (kind == 0) return coef * (va - vb);                                    // resistor
  if (kind == 1) return 1.0e3 * ((va - vb) - source_value(T, I, g, idx, tran, t));  // Norton V source
  if (!tran) return 0.0;                                                     // capacitor companion
  const size_t ci = (size_t)idx * ld + g;
  double cur = (coef / heff) * ((va - vb) - ld_in<G>(&I.cap_vp[ci]));
  if (P.method == KTRAN_TRAP) cur -= ld_in<G>(&I.cap_ip[ci]);
  return cur;
}

// Device evaluation + stamping at x: blockIdx.x picks 32 consecutive
// instances (one per lane; every warp of the CTA holds the same 32),
// blockIdx.y a block of stamp items. The CTA evaluates the block's devices
// into shared memory, then writes the Jacobian value of each of its slots
// (linear stamps, capacitor companions, device terms, in stamp order) and the
// KCL residual of each of its nodes (terms in node order), and folds max |F|,
// max |x - v| and the convergence flags of its nodes into the instance's
// reductions with one atomic each. Hub items (more devices than shared memory
// holds: the supply node and its diagonal) have their devices split into
// chunks of KES_MAX_DEV, one block per chunk; the last chunk block of a tile
// to finish adds the chunks' sums.
// kLte: the transient LTE test is on (P.lte_rel > 0); the kernel without it
// carries none of its code.
template <typename TJ, bool kLte>
__global__ void __launch_bounds__(256, 4) k_es(DevTopo T, DevInst I, JobParams P) {
  __shared__ double s_dev[KES_MAX_DEV * 3 * 32];
  __shared__ unsigned long long s_f[8][32], s_dv[8][32];
  __shared__ int s_fl[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = blockIdx.x * 32 + lane;
  const size_t ld = I.ld;
  const int nv = T.nv;
  // this round's rescue list (and, in tail rounds, its list of instances
  // still live after it) starts empty: the previous round's k_rescue has
  // finished, and this round's k_lu appends to them
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    if (I.rescue_count) *I.rescue_count = 0;
    if (I.live_out_count) *I.live_out_count = 0;
  }
  const double heff = g < I.ni ? I.ev_heff[g] : -1.0;
  const bool live = heff >= 0.0;
  if (!__syncthreads_or(live)) return;
  const int4 blk = __ldg(&T.es_block[blockIdx.y]);  // item off, items, device off, devices
  const bool tran = heff > 0.0;
  const double t = live ? I.ev_t[g] : 0.0;
  const double lr = kLte && live && I.ev_lte ? I.ev_lte[g] : -1.0;
  const double* sd = s_dev + lane;
  double fmx = 0.0, dvm = 0.0;
  bool bad = false;
  int flags = 7, node_seen = 0;
  auto node_done = [&](int i, double f) {
    const size_t o = (size_t)i * ld + g;
    I.F[o] = f;
    if (!isfinite(f)) bad = true;
    fmx = fmax(fmx, fabs(f));
    const double xi = I.x[o], vi = I.v[o];
    const double dd = fabs(xi - vi), m = fmax(fabs(xi), fabs(vi));
    if (dd > P.reltol * m + P.vntol) flags &= ~1;
    if (dd > P.polish_rel * m + P.polish_abs) flags &= ~2;
    if (kLte && lr >= 0.0 && !lte_node_ok(xi, I.v_tp[o], I.v_tpp[o], lr, P)) flags &= ~4;
    dvm = fmax(dvm, dd);
    node_seen = 1;
  };
  if (blk.y > 0) {
    if (live)
      for (int k = warp; k < blk.w; k += 16)
        eval_device_pair(T, I, T.es_dev + blk.z, k, blk.w, g, s_dev, lane);
    __syncthreads();
    if (live)
#pragma unroll 2
      for (int k = warp; k < blk.y; k += 8) {
        const int4 it = __ldg(&T.es_item[blk.x + k]);
        if (it.x < nv) {
          const int s = it.x;
          double acc = __ldg(&T.jlin_dc[s]);
          if (tran) {
            const int q1 = __ldg(&T.jcap_off[s + 1]);
            for (int q = __ldg(&T.jcap_off[s]); q < q1; ++q) {
              const int c = __ldg(&T.jcap_code[q]);
              const double gq = (2.0 * __ldg(&T.cap_c[code_idx(c)])) / heff;
              acc = c < 0 ? acc - gq : acc + gq;
            }
          }
#pragma unroll 4
          for (int q = it.y; q < it.y + it.z; ++q) {
            const int c = __ldg(&T.es_jt[q]);  // sign | offset of the value (gds, gm, diode g)
            const double val = sd[c & 0x7fffffff];
            acc = c < 0 ? acc - val : acc + val;
          }
          reinterpret_cast<TJ*>(I.J)[(size_t)s * ld + g] = (TJ)acc;
        } else {
          double acc = 0.0;
          int q = it.y;
          const int qe = it.y + it.z;
          for (; q + 1 < qe; q += 2) {  // two terms' loads in flight, sum in order
            const int4 t0 = __ldg(&T.es_ft[q]), t1 = __ldg(&T.es_ft[q + 1]);
            const double c0 = node_term(T, I, P, t0, __ldg(&T.es_fc[q]), g, tran, t, heff, sd);
            const double c1 = node_term(T, I, P, t1, __ldg(&T.es_fc[q + 1]), g, tran, t, heff, sd);
            acc = t0.x < 0 ? acc - c0 : acc + c0;
            acc = t1.x < 0 ? acc - c1 : acc + c1;
          }
          if (q < qe) {
            const int4 t0 = __ldg(&T.es_ft[q]);
            const double c0 = node_term(T, I, P, t0, __ldg(&T.es_fc[q]), g, tran, t, heff, sd);
            acc = t0.x < 0 ? acc - c0 : acc + c0;
          }
          node_done(it.x - nv, acc);
        }
      }
  } else {
    // hub chunk block: chunk hc.x of a group of -blk.y hub items. The eight
    // warps sum consecutive slices of each item's terms of this chunk, and the
    // warp partials are added in warp order into the chunk's partial row. The
    // group's chunk block of this tile that finishes last adds the rows in
    // chunk order to the item's linear part (a fixed order, so results do not
    // vary from run to run).
    const int nh = -blk.y;
    const int4 hc = __ldg(&T.es_hubc[blockIdx.y]);
    const int c = hc.x, nch = hc.y;
    double acc[KES_MAX_HUBS];
#pragma unroll
    for (int m = 0; m < KES_MAX_HUBS; ++m) acc[m] = 0.0;
    if (live)
      for (int k = warp; k < blk.w; k += 16)
        eval_device_pair(T, I, T.es_dev + blk.z, k, blk.w, g, s_dev, lane);
    __syncthreads();
    if (live)
#pragma unroll
      for (int m = 0; m < KES_MAX_HUBS; ++m) {
        if (m >= nh) break;
        const int4 it = __ldg(&T.es_item[blk.x + m]);
        const int lo = __ldg(&T.es_hub[it.w + c]), hi = __ldg(&T.es_hub[it.w + c + 1]);
        const int q0 = lo + (int)(((long long)(hi - lo) * warp) / 8);
        const int q1 = lo + (int)(((long long)(hi - lo) * (warp + 1)) / 8);
        if (it.x < nv) {
          for (int q = it.y + q0; q < it.y + q1; ++q) {  // every slot term is a device term
            const int cc = __ldg(&T.es_jt[q]);  // sign | chunk-local offset
            const double val = sd[cc & 0x7fffffff];
            acc[m] = cc < 0 ? acc[m] - val : acc[m] + val;
          }
        } else {
          for (int q = it.y + q0; q < it.y + q1; ++q) {
            const int4 tm = __ldg(&T.es_ft[q]);
            const double cur = node_term(T, I, P, tm, __ldg(&T.es_fc[q]), g, tran, t, heff, sd);
            acc[m] = tm.x < 0 ? acc[m] - cur : acc[m] + cur;
          }
        }
      }
    __syncthreads();
    // warp partials through shared memory (the device values are no longer needed)
    double* part = s_dev;  // [m][warp][32]
#pragma unroll
    for (int m = 0; m < KES_MAX_HUBS; ++m)
      if (m < nh) part[(m * 8 + warp) * 32 + lane] = acc[m];
    __syncthreads();
    if (warp < nh && live) {
      double sum = 0.0;
      for (int w = 0; w < 8; ++w) sum += part[(warp * 8 + w) * 32 + lane];
      I.hub_part[(size_t)(hc.w + warp * nch + c) * ld + g] = sum;
      __threadfence();  // the row is visible before this block counts itself done
    }
    __syncthreads();
    __shared__ int s_last;
    if (threadIdx.x == 0) {
      int* ctr = I.hub_cnt + (size_t)hc.z * (ld / 32) + blockIdx.x;
      const int done = atomicAdd(ctr, 1);
      s_last = done == nch - 1;
      if (done == nch - 1) *ctr = 0;  // every chunk block has counted: ready for the next launch
    }
    __syncthreads();
    if (s_last && warp < nh && live) {
      __threadfence();
      const int4 it = __ldg(&T.es_item[blk.x + warp]);
      double sum = 0.0;
      if (it.x < nv) {
        sum = __ldg(&T.jlin_dc[it.x]);
        if (tran) {
          const int q1 = __ldg(&T.jcap_off[it.x + 1]);
          for (int q = __ldg(&T.jcap_off[it.x]); q < q1; ++q) {
            const int cc = __ldg(&T.jcap_code[q]);
            const double gq = (2.0 * __ldg(&T.cap_c[code_idx(cc)])) / heff;
            sum = cc < 0 ? sum - gq : sum + gq;
          }
        }
      }
      for (int q = 0; q < nch; ++q) sum += __ldcg(&I.hub_part[(size_t)(hc.w + warp * nch + q) * ld + g]);
      if (it.x < nv)
        reinterpret_cast<TJ*>(I.J)[(size_t)it.x * ld + g] = (TJ)sum;
      else
        node_done(it.x - nv, sum);
    }
  }
  // non-negative doubles order like their bit patterns; NaN sorts above +inf
  s_f[warp][lane] = bad ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(fmx);
  s_dv[warp][lane] = (unsigned long long)__double_as_longlong(dvm);
  s_fl[warp][lane] = flags;
  const bool has_nodes = __syncthreads_or(node_seen);
  if (warp == 0 && live && has_nodes) {
    unsigned long long f = s_f[0][lane], d = s_dv[0][lane];
    int fl = s_fl[0][lane];
    for (int w = 1; w < 8; ++w) {
      f = max(f, s_f[w][lane]);
      d = max(d, s_dv[w][lane]);
      fl &= s_fl[w][lane];
    }
    atomicMax(&I.red_f[g], f);
    atomicMax(&I.red_dv[g], d);
    if (fl != 7) atomicAnd(&I.red_flags[g], fl);
  }
}

// Device evaluation + stamping of one listed live instance per CTA, for the
// tail rounds (few live instances; I.live_in lists them): the CTA's threads
// take the instance's devices, then its stamp items, instead of 32 instances
// in the lanes of every CTA. Slots and nodes sum their terms in the order of
// k_es, and hub items in k_es's order too (chunk by chunk, the eight warp
// slices of each chunk in turn, the chunk sums added to the linear part in
// chunk order), so the results are k_es's. Dynamic shared memory: the
// device values [3][devices] (gm or diode g, gds or diode i, ids), then every
// node term's signed value and every hub slot term's signed value, computed
// side by side before the sums (a - c and a + (-c) round alike); with
// slot_values also every slot term's signed value, so the slot sums read
// consecutive values instead of gathering them term by term.
// The body of k_es_one for instance g, by the whole CTA (s_val: the dynamic
// shared memory described above; s_f, s_dv, s_fl: one entry per warp).
template <typename TJ, bool G = true>
__device__ void es_one_instance(const DevTopo& T, const DevInst& I, const JobParams& P, int g,
                                double* s_val, unsigned long long* s_f, unsigned long long* s_dv,
                                int* s_fl, bool slot_values = false) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const size_t ld = I.ld;
  const int nv = T.nv, n = T.n, nm = T.n_mos, nd = T.n_mos + T.n_dio;
  const double heff = I.ev_heff[g];
  if (heff < 0.0) return;
  const bool tran = heff > 0.0;
  const double t = I.ev_t[g];
  const double lr = P.lte_rel > 0.0 && I.ev_lte ? I.ev_lte[g] : -1.0;
  double* v0 = s_val;           // gm | diode g
  double* v1 = s_val + nd;      // gds | diode i
  double* v2 = s_val + 2 * nd;  // ids
  double* tv = s_val + 3 * nd;  // node terms, signed
  double* hv = tv + T.n_ft_terms;  // hub slot terms, signed
  double* jv = hv + T.n_hub_slot_terms;  // with slot_values: every slot term, signed
  for (int d = tid; d < nd; d += blockDim.x) {
    const DevIn in = load_device<G>(T, I, d, g);
    if (in.mos) {
      double ids, gm, gds;
      mosfet_eval(in.va, in.vb, in.vc, in.sign, in.p0, in.p1, in.p2, in.p3, ids, gm, gds);
      v0[d] = gm;
      v1[d] = gds;
      v2[d] = ids;
    } else {
      double id, gd;
      diode_eval(in.va, make_double4(in.p0, in.p1, in.p2, in.p3), id, gd);
      v0[d] = gd;
      v1[d] = id;
    }
  }
  __syncthreads();
  // a slot term's device value (codes in global numbering: MOSFET or diode index)
  auto slot_val = [&](int c) {  // one load from a selected address: loads of several terms overlap
    const int kind = code_kind(c), idx = code_idx(c);
    const double* src = kind == 0 ? v1 + idx : kind == 2 ? v0 + nm + idx : v0 + idx;  // gds | diode g | gm
    return *src;
  };
  auto node_val = [&](int q) {
    const int c = __ldg(&T.ft_code[q]), kind = code_kind(c), idx = code_idx(c);
    if (kind == 4) return v1[nm + idx];  // diode current
    if (kind == 5) return v2[idx];       // MOSFET ids
    const int4 tm = make_int4(c, __ldg(&T.ft_a[q]), __ldg(&T.ft_b[q]), 0);
    return node_term<G>(T, I, P, tm, __ldg(&T.ft_coef[q]), g, tran, t, heff, s_val);
  };
  auto slot_base = [&](int s) {  // linear part + capacitor companions
    double acc = __ldg(&T.jlin_dc[s]);
    if (tran) {
      const int q1 = __ldg(&T.jcap_off[s + 1]);
      for (int q = __ldg(&T.jcap_off[s]); q < q1; ++q) {
        const int cc = __ldg(&T.jcap_code[q]);
        const double gq = (2.0 * __ldg(&T.cap_c[code_idx(cc)])) / heff;
        acc = cc < 0 ? acc - gq : acc + gq;
      }
    }
    return acc;
  };
  auto is_hub = [&](int it) {
    for (int h = 0; h < T.n_hub_items; ++h)
      if (__ldg(&T.hub_items[h]).x == it) return true;
    return false;
  };
  for (int q = tid; q < T.n_ft_terms; q += blockDim.x) {
    const double c0 = node_val(q);
    tv[q] = __ldg(&T.ft_code[q]) < 0 ? -c0 : c0;
  }
  if (slot_values)
    for (int q = tid; q < T.n_jt_terms; q += blockDim.x) {
      const int c = __ldg(&T.jt_code[q]);
      const double val = slot_val(c);
      jv[q] = c < 0 ? -val : val;
    }
  for (int h = 0; h < T.n_hub_items; ++h) {
    const int4 hb = __ldg(&T.hub_items[h]);
    if (hb.x >= nv) continue;
    const int qs = __ldg(&T.jt_off[hb.x]), nt = __ldg(&T.jt_off[hb.x + 1]) - qs;
    for (int q = tid; q < nt; q += blockDim.x) {
      const int c = __ldg(&T.jt_code[qs + q]);
      const double val = slot_val(c);
      hv[hb.w + q] = c < 0 ? -val : val;
    }
  }
  __syncthreads();
  double fmx = 0.0, dvm = 0.0;
  bool bad = false;
  int flags = 7;
  auto node_done = [&](int i, double f) {
    const size_t o = (size_t)i * ld + g;
    I.F[o] = f;
    if (!isfinite(f)) bad = true;
    fmx = fmax(fmx, fabs(f));
    const double xi = I.x[o], vi = I.v[o];
    const double dd = fabs(xi - vi), m = fmax(fabs(xi), fabs(vi));
    if (dd > P.reltol * m + P.vntol) flags &= ~1;
    if (dd > P.polish_rel * m + P.polish_abs) flags &= ~2;
    if (lr >= 0.0 && !lte_node_ok(xi, I.v_tp[o], I.v_tpp[o], lr, P)) flags &= ~4;
    dvm = fmax(dvm, dd);
  };
  for (int it = tid; it < nv + n; it += blockDim.x) {
    if (is_hub(it)) continue;
    if (it < nv) {
      double acc = slot_base(it);
      const int q1 = __ldg(&T.jt_off[it + 1]);
      int q = __ldg(&T.jt_off[it]);
      if (slot_values)  // the signed values side by side: a - v and a + (-v) round alike
        for (; q < q1; ++q) acc += jv[q];
      // eight terms' codes and values fetched together, then added in term
      // order (a - v and a + (-v) round alike): the loads overlap, the sum
      // is the sequential one
      for (; q + 8 <= q1; q += 8) {
        double sv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int c = __ldg(&T.jt_code[q + k]);
          const double val = slot_val(c);
          sv[k] = c < 0 ? -val : val;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) acc += sv[k];
      }
      for (; q < q1; ++q) {
        const int c = __ldg(&T.jt_code[q]);
        const double val = slot_val(c);
        acc = c < 0 ? acc - val : acc + val;
      }
      reinterpret_cast<TJ*>(I.J)[(size_t)it * ld + g] = (TJ)acc;
    } else {
      const int i = it - nv;
      double acc = 0.0;
      const int q1 = __ldg(&T.ft_off[i + 1]);
      for (int q = __ldg(&T.ft_off[i]); q < q1; ++q) acc += tv[q];
      node_done(i, acc);
    }
  }
  // hub items, one warp each: lane c * 8 + w sums slice w of chunk c (as the
  // warps of k_es's chunk blocks do), lane 0 then combines in k_es's order
  for (int h = warp; h < T.n_hub_items; h += nw) {
    const int4 hb = __ldg(&T.hub_items[h]);
    const int it = hb.x, nch = hb.z;
    const bool slot = it < nv;
    const int qs = slot ? __ldg(&T.jt_off[it]) : __ldg(&T.ft_off[it - nv]);
    double part[2] = {0.0, 0.0};  // up to 64 slices per warp: lanes take two
    for (int r = 0; r < 2; ++r) {
      const int sl = lane + 32 * r, c = sl >> 3, w = sl & 7;
      if (c >= nch) continue;
      const int lo = __ldg(&T.es_hub[hb.y + c]), hi = __ldg(&T.es_hub[hb.y + c + 1]);
      const int q0 = lo + (int)(((long long)(hi - lo) * w) / 8);
      const int q1 = lo + (int)(((long long)(hi - lo) * (w + 1)) / 8);
      const double* src = slot ? hv + hb.w : tv + qs;
      double acc = 0.0;
      for (int q = q0; q < q1; ++q) acc += src[q];
      part[r] = acc;
    }
    double sum = slot ? slot_base(it) : 0.0;
    for (int c = 0; c < nch; ++c) {
      double pc = 0.0;
      for (int w = 0; w < 8; ++w) {
        const int sl = c * 8 + w;
        pc += __shfl_sync(kFull, part[sl >> 5], sl & 31);
      }
      sum += pc;
    }
    if (lane == 0) {
      if (slot)
        reinterpret_cast<TJ*>(I.J)[(size_t)it * ld + g] = (TJ)sum;
      else
        node_done(it - nv, sum);
    }
  }
  // the instance's reductions (one CTA per instance: no other CTA adds to them)
  for (int o = 16; o > 0; o >>= 1) {
    fmx = fmax(fmx, __shfl_xor_sync(kFull, fmx, o));
    dvm = fmax(dvm, __shfl_xor_sync(kFull, dvm, o));
    flags &= __shfl_xor_sync(kFull, flags, o);
  }
  const bool any_bad = __any_sync(kFull, bad);
  if (lane == 0) {
    s_f[warp] = any_bad ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(fmx);
    s_dv[warp] = (unsigned long long)__double_as_longlong(dvm);
    s_fl[warp] = flags;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long f = s_f[0], dv = s_dv[0];
    int fl = s_fl[0];
    for (int w = 1; w < nw; ++w) {
      f = max(f, s_f[w]);
      dv = max(dv, s_dv[w]);
      fl &= s_fl[w];
    }
    atomicMax(&I.red_f[g], f);
    atomicMax(&I.red_dv[g], dv);
    if (fl != 7) atomicAnd(&I.red_flags[g], fl);
  }
}

template <typename TJ>
__global__ void __launch_bounds__(kBigThreads) k_es_one(DevTopo T, DevInst I, JobParams P) {
  extern __shared__ __align__(16) double s_val[];
  __shared__ unsigned long long s_f[kBigThreads / 32], s_dv[kBigThreads / 32];
  __shared__ int s_fl[kBigThreads / 32];
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // the round's lists start empty, as in k_es
    if (I.rescue_count) *I.rescue_count = 0;
    if (I.live_out_count) *I.live_out_count = 0;
  }
  if ((int)blockIdx.x >= *I.live_in_count) return;
  es_one_instance<TJ>(T, I, P, I.live_in[blockIdx.x], s_val, s_f, s_dv, s_fl);
}

// Reductions of an instance back to their neutral values.
__device__ __forceinline__ void reset_reductions(const DevInst& I, int g) {
  I.red_f[g] = 0ull;
  I.red_dv[g] = 0ull;
  I.red_flags[g] = 7;
}

// Evaluation point of the next round from the instance's state.
__device__ __forceinline__ void set_eval_point(const DevInst& I, const JobParams& P, int g,
                                               const InstState& st) {
  if (st.mode == MODE_DONE) {
    I.ev_heff[g] = -1.0;
    I.ev_t[g] = 0.0;
    if (I.ev_lte && P.lte_rel > 0.0) I.ev_lte[g] = -1.0;
    return;
  }
  double t, heff;
  eval_point(st, P, t, heff);
  I.ev_t[g] = t;
  I.ev_heff[g] = heff;
  // the LTE predictor's step ratio, when the test applies to this point (with
  // the test off the ratio is never read: it stays as k_init set it)
  if (I.ev_lte && P.lte_rel > 0.0) {
    if (st.mode == MODE_TRAN && st.hprev > 0.0) {
      const int units = 1 << P.max_halvings;
      const double hsub = P.h * (units >> st.depth) / units;
      I.ev_lte[g] = hsub / st.hprev;
    } else {
      I.ev_lte[g] = -1.0;
    }
  }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// Asynchronous copy of one 4- or 8-byte element; with valid = false nothing
// is read and the destination is zero-filled.
template <int B>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gmem), "n"(B),
               "r"(valid ? B : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// 16-bit field i of the packed half-word array at prog[base].
__device__ __forceinline__ int nd_half(const int* prog, int base, int i) {
  return (prog[base + (i >> 1)] >> (16 * (i & 1))) & 0xFFFF;
}

// The static-pivot LU of one instance by one warp on the packed level
// schedule in shared memory (layout: nd_program in topology.cpp): per level,
// the pivots' reciprocals, then their L values, then the update targets and
// right-hand-side rows (lists longer than Topology::kNdLong summed by the
// whole warp, partials combined in a fixed tree); then the back substitution
// from the last level down. A and y are this instance's ND slots (without
// the gmin diagonal, added to each pivot as it is taken) and right-hand side
// (ND order); y returns the solution. Same failure tests as
// lu_solve: tiny or non-finite pivots, non-finite solutions, multipliers
// above growth_limit.
template <typename T>
__device__ bool nd_solve(T* __restrict__ A, T* __restrict__ y, const int* __restrict__ prog,
                         T gmin, T tiny, T growth_limit, int lane) {
  const int NL = prog[0], lvt = prog[1], tpb = prog[2], ypb = prog[3], bpb = prog[4];
  bool ok = true;
  T lmax = T(0);
  // the gmin diagonal joins before the elimination, as the reference's
  // addDiagonalConditioning (physics/circuitsim.h:2857) precedes its LU
  for (int lv = 0; lv < NL; ++lv) {
    const int* Lt = prog + lvt + 12 * lv;
    for (int q = lane; q < Lt[1]; q += 32) A[prog[Lt[0] + q]] += gmin;
  }
  __syncwarp();
  for (int lv = 0; lv < NL; ++lv) {
    const int* Lt = prog + lvt + 12 * lv;
    const int po = Lt[0], pc = Lt[1], lo = Lt[2], lc = Lt[3];
    for (int q = lane; q < pc; q += 32) {
      const int d = prog[po + q];
      const T piv = A[d];
      ok = ok && isfinite(piv) && !(fabs(piv) < tiny);
      A[d] = recip(piv);
    }
    __syncwarp();
    for (int e = lane; e < lc; e += 32) {
      const int v = prog[lo + e];
      const int sl = v & 0xFFFF;
      const T l = A[sl] * A[(v >> 16) & 0xFFFF];
      A[sl] = l;
      lmax = fmax(lmax, fabs(l));
    }
    __syncwarp();
    const int to = Lt[4], tsc = Lt[5], tlc = Lt[6];
    for (int t = lane; t < tsc; t += 32) {
      const int h = prog[to + 2 * t], off = tpb + prog[to + 2 * t + 1];
      const int sl = h & 0xFFFF, c = (h >> 16) & 0xFFFF;
      T acc = A[sl];
#pragma unroll 4
      for (int q = 0; q < c; ++q) {
        const int pr = prog[off + q];
        acc -= A[pr & 0xFFFF] * A[(pr >> 16) & 0xFFFF];
      }
      A[sl] = acc;
    }
    const int yo = Lt[7], ysc = Lt[8], ylc = Lt[9];
    for (int r = lane; r < ysc; r += 32) {
      const int h = prog[yo + 2 * r], off = ypb + prog[yo + 2 * r + 1];
      const int row = h & 0xFFFF, c = (h >> 16) & 0xFFFF;
      T acc = y[row];
#pragma unroll 4
      for (int q = 0; q < c; ++q) {
        const int pr = prog[off + q];
        acc -= A[pr & 0xFFFF] * y[(pr >> 16) & 0xFFFF];
      }
      y[row] = acc;
    }
    for (int t = tsc; t < tsc + tlc; ++t) {  // long target lists: the warp sums
      const int h = prog[to + 2 * t], off = tpb + prog[to + 2 * t + 1];
      const int c = (h >> 16) & 0xFFFF;
      T part = T(0);
      for (int q = lane; q < c; q += 32) {
        const int pr = prog[off + q];
        part += A[pr & 0xFFFF] * A[(pr >> 16) & 0xFFFF];
      }
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) A[h & 0xFFFF] -= part;
    }
    for (int r = ysc; r < ysc + ylc; ++r) {  // long right-hand-side rows
      const int h = prog[yo + 2 * r], off = ypb + prog[yo + 2 * r + 1];
      const int c = (h >> 16) & 0xFFFF;
      T part = T(0);
      for (int q = lane; q < c; q += 32) {
        const int pr = prog[off + q];
        part += A[pr & 0xFFFF] * y[(pr >> 16) & 0xFFFF];
      }
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) y[h & 0xFFFF] -= part;
    }
    __syncwarp();
  }
  bool finite = true;
  for (int lv = NL - 1; lv >= 0; --lv) {
    const int* Lt = prog + lvt + 12 * lv;
    const int bo = Lt[10], bc = Lt[11];
    for (int q = lane; q < bc; q += 32) {
      const int a = prog[bo + 2 * q], b = prog[bo + 2 * q + 1];
      const int k = a & 0xFFFF, d = (a >> 16) & 0xFFFF;
      const int c = b & 0xFFFF, off = bpb + ((b >> 16) & 0xFFFF);
      T sv = y[k];
#pragma unroll 4
      for (int j = 0; j < c; ++j) {
        const int pr = prog[off + j];
        sv -= A[pr & 0xFFFF] * y[(pr >> 16) & 0xFFFF];
      }
      sv *= A[d];
      y[k] = sv;
      finite = finite && isfinite(sv);
    }
    __syncwarp();
  }
  for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(kFull, lmax, o));
  ok = __all_sync(kFull, ok);
  finite = __all_sync(kFull, finite);
  return ok && finite && !(lmax > growth_limit);
}

// The decision of instance g for this round from the reductions of k_es (the
// reference control flow as a state machine, `decide`): the state advances,
// the reductions return to neutral, and a reseed restarts GMIN stepping from
// the reference seed. Returns the action bits; live = 0 for a finished
// instance; trev = 1 when this round evaluated a transient point.
__device__ __forceinline__ int instance_decide(const DevTopo& Tp, const DevInst& I, const JobParams& P,
                                               int g, int& live, int& trev, double& gm, double& hs) {
  InstState s = I.st[g];
  trev = s.mode == MODE_TRAN;
  live = 0;
  if (s.mode == MODE_DONE) return 0;
  live = 1;
  const unsigned long long fb = I.red_f[g];
  const double Fm = __longlong_as_double((long long)fb);
  const double dvm = __longlong_as_double((long long)I.red_dv[g]);
  const int fl = I.red_flags[g];
  reset_reductions(I, g);
  gm = 1e-12;
  hs = P.h;
  const int h0 = s.hist_n;
  const int a = decide(s, Fm, fl & 1, (fl & 2) != 0, (fl & 4) != 0, dvm, P, gm, hs);
  if (s.hist_n != h0 && I.hist) {
    const size_t k = (size_t)(h0 % KHIST_LEN) * 2;
    I.hist[k * I.ld + g] = Fm;
    I.hist[(k + 1) * I.ld + g] = dvm;
  }
  if (a & ACT_RESEED) {
    s.g = 0;
    s.it = 0;
    s.first = 1;
    s.damp = 0;
    s.prevF = 0.0;
    s.seeded = 0;
    reference_seed(Tp, I, g, I.v);
  }
  I.st[g] = s;
  return a;
}

// End of instance g's round: a failed solve goes to the rescue list (or
// aborts the step when there is none), then the next evaluation point.
// Returns whether the instance is still live.
__device__ __forceinline__ int instance_finish(const DevTopo& Tp, const DevInst& I, const JobParams& P,
                                               int g, int act, int sing, double gmin) {
  if ((act & ACT_SOLVE) && sing) {
    if (I.rescue_list) {
      const int slot = atomicAdd(I.rescue_count, 1);
      RescueItem it;
      it.inst = g;
      it.act = act;
      it.gmin = gmin;
      I.rescue_list[slot] = it;
    } else {
      on_singular(Tp, I, g);
    }
  }
  const InstState st2 = I.st[g];
  set_eval_point(I, P, g, st2);
  return st2.mode != MODE_DONE;
}

// nd_solve spread over a whole CTA: the same packed program in shared memory,
// each phase's items over the CTA's threads, long lists summed by one warp in
// nd_solve's fixed tree, short ones by one thread in order -- so the result
// is nd_solve's, bit for bit.
template <typename T>
__device__ bool nd_solve_cta(T* __restrict__ A, T* __restrict__ y, const int* __restrict__ prog,
                             T gmin, T tiny, T growth_limit) {
  const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bd >> 5;
  const int NL = prog[0], lvt = prog[1], tpb = prog[2], ypb = prog[3], bpb = prog[4];
  bool ok = true;
  T lmax = T(0);
  for (int lv = 0; lv < NL; ++lv) {  // the gmin diagonal, before the elimination
    const int* Lt = prog + lvt + 12 * lv;
    for (int q = tid; q < Lt[1]; q += bd) A[prog[Lt[0] + q]] += gmin;
  }
  __syncthreads();
  for (int lv = 0; lv < NL; ++lv) {
    const int* Lt = prog + lvt + 12 * lv;
    const int po = Lt[0], pc = Lt[1], lo = Lt[2], lc = Lt[3];
    for (int q = tid; q < pc; q += bd) {
      const int d = prog[po + q];
      const T piv = A[d];
      ok = ok && isfinite(piv) && !(fabs(piv) < tiny);
      A[d] = recip(piv);
    }
    __syncthreads();
    for (int e = tid; e < lc; e += bd) {
      const int v = prog[lo + e];
      const int sl = v & 0xFFFF;
      const T l = A[sl] * A[(v >> 16) & 0xFFFF];
      A[sl] = l;
      lmax = fmax(lmax, fabs(l));
    }
    __syncthreads();
    const int to = Lt[4], tsc = Lt[5], tlc = Lt[6];
    for (int t = tid; t < tsc; t += bd) {
      const int h = prog[to + 2 * t], off = tpb + prog[to + 2 * t + 1];
      const int sl = h & 0xFFFF, c = (h >> 16) & 0xFFFF;
      T acc = A[sl];
#pragma unroll 4
      for (int q = 0; q < c; ++q) {
        const int pr = prog[off + q];
        acc -= A[pr & 0xFFFF] * A[(pr >> 16) & 0xFFFF];
      }
      A[sl] = acc;
    }
    const int yo = Lt[7], ysc = Lt[8], ylc = Lt[9];
    for (int r = tid; r < ysc; r += bd) {
      const int h = prog[yo + 2 * r], off = ypb + prog[yo + 2 * r + 1];
      const int row = h & 0xFFFF, c = (h >> 16) & 0xFFFF;
      T acc = y[row];
#pragma unroll 4
      for (int q = 0; q < c; ++q) {
        const int pr = prog[off + q];
        acc -= A[pr & 0xFFFF] * y[(pr >> 16) & 0xFFFF];
      }
      y[row] = acc;
    }
    for (int t = tsc + warp; t < tsc + tlc; t += nw) {
      const int h = prog[to + 2 * t], off = tpb + prog[to + 2 * t + 1];
      const int c = (h >> 16) & 0xFFFF;
      T part = T(0);
      for (int q = lane; q < c; q += 32) {
        const int pr = prog[off + q];
        part += A[pr & 0xFFFF] * A[(pr >> 16) & 0xFFFF];
      }
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) A[h & 0xFFFF] -= part;
    }
    for (int r = ysc + warp; r < ysc + ylc; r += nw) {
      const int h = prog[yo + 2 * r], off = ypb + prog[yo + 2 * r + 1];
      const int c = (h >> 16) & 0xFFFF;
      T part = T(0);
      for (int q = lane; q < c; q += 32) {
        const int pr = prog[off + q];
        part += A[pr & 0xFFFF] * y[(pr >> 16) & 0xFFFF];
      }
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) y[h & 0xFFFF] -= part;
    }
    __syncthreads();
  }
  bool finite = true;
  for (int lv = NL - 1; lv >= 0; --lv) {
    const int* Lt = prog + lvt + 12 * lv;
    const int bo = Lt[10], bc = Lt[11];
    for (int q = tid; q < bc; q += bd) {
      const int a = prog[bo + 2 * q], b = prog[bo + 2 * q + 1];
      const int k = a & 0xFFFF, d = (a >> 16) & 0xFFFF;
      const int c = b & 0xFFFF, off = bpb + ((b >> 16) & 0xFFFF);
      T sv = y[k];
#pragma unroll 4
      for (int j = 0; j < c; ++j) {
        const int pr = prog[off + j];
        sv -= A[pr & 0xFFFF] * y[(pr >> 16) & 0xFFFF];
      }
      sv *= A[d];
      y[k] = sv;
      finite = finite && isfinite(sv);
    }
    __syncthreads();
  }
  return __syncthreads_and(ok && finite && !(lmax > growth_limit)) != 0;
}

// Walks the (item i, listed instance k) pairs e = t, t + step, t + 2 step, ...
// of an m-wide list (i = e / m, k = e % m) with one division per walk rather
// than one per pair; m > 0.
struct PairWalk {
  int i, k, di, dk, m;
  __device__ PairWalk(int t, int step, int m_) : m(m_) {
    i = t / m_;
    k = t - i * m_;
    di = step / m_;
    dk = step - di * m_;
  }
  __device__ void next() {
    k += dk;
    i += di;
    if (k >= m) {
      k -= m;
      ++i;
    }
  }
};

// Control flow + linear solve of a tile of L instances (one CTA): decisions
// from the reductions of k_es, vector updates, the Jacobian tile staged
// into shared memory with cp.async, static-pivot LU with the forward
// substitution fused, x = v + dx, junction limiting, bookkeeping.
template <typename T, bool nd>
__device__ __forceinline__ void lu_round(const DevTopo& Tp, const DevInst& I, const JobParams& P,
                                         int L, int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // level schedule (nd, one warp per instance): A [L][nd_S] ND slots,
  // Y [L][nd_SY], then the packed schedule; else A [nv][L] value slots,
  // Y [n][L] and the packed pivot records
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Y = nd ? A + (size_t)Tp.nd_S * L : A + (size_t)Tp.nv * L;
  int4* rec = (!nd && Tp.lu_rec)
                  ? reinterpret_cast<int4*>(
                        smem_raw + (((size_t)(Tp.nv + Tp.n) * L * sizeof(T) + 15) & ~size_t(15)))
                  : nullptr;
  const int* prog =
      nd ? reinterpret_cast<const int*>(
               smem_raw + (((size_t)(Tp.nd_S + Tp.nd_SY) * L * sizeof(T) + 15) & ~size_t(15)))
         : nullptr;
  if (nd) {  // the packed schedule into shared memory, once per launch
    int4* dst = reinterpret_cast<int4*>(const_cast<int*>(prog));
    const int4* srcp = reinterpret_cast<const int4*>(Tp.nd_prog);
    for (int e = threadIdx.x; e < (Tp.nd_prog_len + 3) / 4; e += blockDim.x) dst[e] = __ldg(&srcp[e]);
  }
  __shared__ int s_live[kMaxLanes], s_act[kMaxLanes], s_sing[kMaxLanes], s_trev[kMaxLanes];
  __shared__ int s_list[kMaxLanes], s_nlist, s_anysolve;
  __shared__ double s_gmin[kMaxLanes], s_hsub[kMaxLanes];

  const int n = Tp.n, nv = Tp.nv;
  const size_t ld = I.ld;
  const int tid = threadIdx.x;
  const int lane = tid % L, row = tid / L, R = blockDim.x / L;
  const int base = blockIdx.x * L;
  const int g = base + lane;
  const int cnt = min(L, I.ni - base);
  if (cnt <= 0) return;

  // 1. decisions (thread per lane, all in warp 0: L <= 32) from the reductions
  //    of k_es; the lanes with an action are listed in order
  int my_live = 0;
  if (tid < 32) {
    int a = 0;
    if (tid < cnt) {
      int trev = 0;
      double gm = 1e-12, hs = P.h;
      a = instance_decide(Tp, I, P, g, my_live, trev, gm, hs);
      s_trev[tid] = trev;  // what this round evaluated
      if (my_live) {
        s_gmin[tid] = gm;
        s_hsub[tid] = hs;
      }
    }
    if (tid < L) {
      s_live[tid] = my_live;
      s_act[tid] = a;
      s_sing[tid] = 0;
    }
    const unsigned acting = __ballot_sync(kFull, a != 0);
    if (a) s_list[__popc(acting & ((1u << tid) - 1u))] = tid;
    const unsigned solving = __ballot_sync(kFull, (a & ACT_SOLVE) != 0);
    if (tid == 0) {
      s_nlist = __popc(acting);
      s_anysolve = solving != 0;
    }
  }
  if (!__syncthreads_or(my_live)) return;
  const int m = s_nlist;  // instances with an action; the vector phases run over
                          // (item, listed instance) pairs spread over the CTA

  // 1b. level schedule: the instances' ND slots start streaming into shared
  //     memory now (asynchronous copies, a warp per slot, a lane per
  //     instance) and land while the vectors are updated
  if (nd) {
    const int lw = tid & 31;
    if (s_anysolve && lw < L) {
      const T* J = reinterpret_cast<const T*>(I.J);
      const int S = Tp.nd_S, nw = blockDim.x >> 5;
      T* dst = A + lw * S;
      const T* srcb = J + base + lw;
      const bool inst = lw < cnt;
#pragma unroll 4
      for (int sl = tid >> 5; sl < Tp.nd_nv; sl += nw) {
        const int src = nd_half(prog, prog[5], sl);
        const bool valid = inst && src != 0xFFFF;
        cp_async_elem<sizeof(T)>(dst + sl, valid ? srcb + (size_t)src * ld : J, valid);
      }
    }
  }

  // 2. vector updates and the right-hand side of the instances that solve
  const int a = s_act[lane];
  const int any_solve = s_anysolve;
  {
    double* __restrict__ X = I.x;
    double* __restrict__ V = I.v;
    double* __restrict__ VT = I.v_tp;
    const double* __restrict__ F = I.F;
#pragma unroll 2
    for (PairWalk w(tid, blockDim.x, m > 0 ? m : 1); m > 0 && w.i < n; w.next()) {
      const int i = w.i, ln = s_list[w.k];
      const int act = s_act[ln];
      const double gmin = s_gmin[ln];
      const size_t o = (size_t)i * ld + base + ln;
      const double fi = F[o];
      double vi;
      if (act & ACT_RESTART) {
        vi = VT[o];
        V[o] = vi;
        X[o] = vi;
      } else if (act & ACT_RESEED) {
        vi = V[o];
        X[o] = vi;
      } else {
        double xi = X[o];
        vi = V[o];
        if (act & ACT_DAMP) {
          xi = vi + 0.5 * (xi - vi);
          X[o] = xi;
        }
        if (act & ACT_ACCEPT) {
          vi = xi;
          V[o] = vi;
        }
        if (act & (ACT_STEP | ACT_TRAN_INIT)) {
          if (P.lte_rel > 0.0 && I.v_tpp)  // the LTE predictor's older point
            I.v_tpp[o] = (act & ACT_TRAN_INIT) ? vi : VT[o];
          VT[o] = vi;
        }
      }
      if (act & ACT_SOLVE)
        Y[nd ? ln * Tp.nd_SY + nd_half(prog, prog[6], i) : i * L + ln] = (T)(-(fi + gmin * vi));
    }
  }
  __syncthreads();

  // 2b. the Jacobian tile of the solving instances into shared memory
  if (any_solve) {
    const T* J = reinterpret_cast<const T*>(I.J);
    const int row_bytes = L * (int)sizeof(T);
    if (nd) {
      // issued in 1b
    } else if (row_bytes % 16 == 0) {
      const int cpr = row_bytes / 16;  // 16-byte chunks per slot row
      const int chunks = nv * cpr;
      for (int c = tid; c < chunks; c += blockDim.x) {
        const int s = c / cpr, part = c - s * cpr;
        cp_async16(reinterpret_cast<char*>(A + (size_t)s * L) + 16 * part,
                   reinterpret_cast<const char*>(J + (size_t)s * ld + base) + 16 * part);
      }
    } else {
      for (int s = row; s < nv; s += R) A[s * L + lane] = J[(size_t)s * ld + g];
    }
    if (rec) stage_pivots(Tp, rec, L);
    cp_async_wait_all();
  }

  // 2c. capacitor history after a completed (sub-)step, waveform samples
  for (PairWalk w(tid, blockDim.x, m > 0 ? m : 1); m > 0 && w.i < Tp.n_cap; w.next()) {
    const int c = w.i, ln = s_list[w.k];
    const int act = s_act[ln];
    if (act & (ACT_TRAN_INIT | ACT_STEP)) {
      const int2 tt = __ldg(&Tp.cap_term[c]);
      const int gl = base + ln;
      const double vc = (tt.x >= 0 ? I.v[tt.x * ld + gl] : 0.0) - (tt.y >= 0 ? I.v[tt.y * ld + gl] : 0.0);
      const size_t ci = (size_t)c * ld + gl;
      if (act & ACT_TRAN_INIT) {
        I.cap_vp[ci] = vc;
        I.cap_ip[ci] = 0.0;
      } else {
        const double C = __ldg(&Tp.cap_c[c]);
        const double h = s_hsub[ln];
        const double ic = P.method == KTRAN_TRAP ? (2.0 * C / h) * (vc - I.cap_vp[ci]) - I.cap_ip[ci]
                                                 : (C / h) * (vc - I.cap_vp[ci]);
        I.cap_vp[ci] = vc;
        I.cap_ip[ci] = ic;
      }
    }
  }
  if ((a & ACT_WAVE) && I.n_wave > 0) {
    const int done_step = I.st[g].step - 1;  // 1-based step just completed
    if (done_step >= 1 && done_step <= I.wave_steps)
      for (int w = row; w < I.n_wave; w += R) {
        const int q = I.wave_pos[w];
        I.wave[((size_t)g * I.wave_steps + (done_step - 1)) * I.n_wave + w] = q >= 0 ? I.v[q * ld + g] : 0.0;
      }
  }
  __syncthreads();

  if (any_solve) {
    if (a & ACT_SOLVE) {
      const T gmin = (T)s_gmin[lane];
      if (!nd)
        for (int i = row; i < n; i += R) A[__ldg(&Tp.lu_hdr[i].w) * L + lane] += gmin;
    }
    if (!nd) __syncthreads();

    // 3. factor + solve: one warp per instance on the level schedule, else
    //    one lane per instance on the pivot program
    const T tiny = sizeof(T) == 8 ? (T)1e-25 : (T)1e-30;
    const T growth = sizeof(T) == 8 ? (T)P.growth64 : (T)fmin(P.growth32, 3.0e38);
    if (nd) {
      const int w = tid >> 5;
      if (w < L && (s_act[w] & ACT_SOLVE)) {
        const bool okw = nd_solve<T>(A + (size_t)w * Tp.nd_S, Y + (size_t)w * Tp.nd_SY, prog,
                                     (T)s_gmin[w], tiny, growth, tid & 31);
        if ((tid & 31) == 0) s_sing[w] = okw ? 0 : 1;
      }
    } else if (tid < L && (s_act[tid] & ACT_SOLVE)) {
      s_sing[tid] = lu_solve<T>(A + tid, Y + tid, L, Tp, rec, tiny, growth) ? 0 : 1;
    }
    __syncthreads();

    // 4. x = v + dx, then junction limiting level by level, over (item,
    //    listed instance) pairs; only instances whose solve succeeded update
    {
      double* __restrict__ X = I.x;
      const double* __restrict__ V = I.v;
#pragma unroll 2
      for (PairWalk w(tid, blockDim.x, m > 0 ? m : 1); m > 0 && w.i < n; w.next()) {
        const int i = w.i, ln = s_list[w.k];
        const int act = s_act[ln];
        if (!(act & ACT_SOLVE) || s_sing[ln]) continue;
        const size_t o = (size_t)i * ld + base + ln;
        double xi = V[o] + (double)Y[nd ? ln * Tp.nd_SY + nd_half(prog, prog[6], i) : i * L + ln];
        if ((act & ACT_LIMIT) && !isfinite(xi)) xi = 0.0;  // SafeUtils::sanitize_vector
        X[o] = xi;
      }
    }
    if (Tp.n_dio > 0) {
      const int lim_lane = tid < L && (s_act[tid] & ACT_SOLVE) && (s_act[tid] & ACT_LIMIT) && !s_sing[tid];
      if (__syncthreads_or(lim_lane)) {
        for (int lvl = 0; lvl < Tp.n_dio_levels; ++lvl) {
          for (PairWalk w(tid, blockDim.x, m); w.i < Tp.n_dio; w.next()) {
            const int d = w.i, ln = s_list[w.k];
            const int act = s_act[ln];
            if ((act & ACT_SOLVE) && (act & ACT_LIMIT) && !s_sing[ln] && __ldg(&Tp.dio_level[d]) == lvl)
              limit_one(Tp, d, I.x, I.v, ld, base + ln);
          }
          __syncthreads();
        }
      }
    }
  }

  // 5. rescue hand-off, next evaluation point, bookkeeping (thread per lane,
  //    all in warp 0)
  if (tid < L) {
    const unsigned mask = L == 32 ? kFull : ((1u << L) - 1u);
    int live = 0, solved = 0, dcev = 0, trev = 0;
    if (tid < cnt && s_live[tid]) {
      const int act = s_act[tid];
      trev = s_trev[tid];
      dcev = !trev;
      solved = (act & ACT_SOLVE) && !s_sing[tid];
      live = instance_finish(Tp, I, P, g, act, s_sing[tid], s_gmin[tid]);
    }
    const int nlive = __popc(__ballot_sync(mask, live));
    const int nsol = __popc(__ballot_sync(mask, solved));
    const int ndc = __popc(__ballot_sync(mask, dcev));
    const int ntr = __popc(__ballot_sync(mask, trev));
    if (tid == 0) {
      if (nlive) atomicAdd(active, nlive);
      if (I.counters) {
        if (ndc) atomicAdd(&I.counters[0], (unsigned long long)ndc);
        if (ntr) atomicAdd(&I.counters[1], (unsigned long long)ntr);
        if (nsol) atomicAdd(&I.counters[2], (unsigned long long)nsol);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kRoundThreads) k_lu(DevTopo Tp, DevInst I, JobParams P, int L,
                                                      int* active) {
  lu_round<T, false>(Tp, I, P, L, active);
}

// The level-scheduled variant: blockDim = 32 L, one warp per instance.
template <typename T>
__global__ void __launch_bounds__(sizeof(T) == 4 ? 1024 : 512)
    k_lu_nd(DevTopo Tp, DevInst I, JobParams P, int L, int* active) {
  lu_round<T, true>(Tp, I, P, L, active);
}

// The level schedule solved by a whole CTA for one instance (the
// block-per-instance schedule): per level the pivots' reciprocals, then the L
// values, then the update targets and right-hand-side rows, each phase spread
// over the CTA's threads; target and row lists longer than Topology::kNdLong
// are summed by one warp with lanes strided and combined in nd_solve's fixed
// tree, and shorter ones by one thread in order, so the results equal
// nd_solve's. Tables are read from global memory. A holds the instance's ND
// slots (shared or global memory), y its right-hand side (ND order) and
// returns the solution. Same failure tests as nd_solve.
template <typename T>
__device__ bool big_solve(T* __restrict__ A, T* __restrict__ y, const DevTopo& Tp, T gmin, T tiny,
                          T growth_limit) {
  const int tid = threadIdx.x, bd = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = bd >> 5;
  bool ok = true, finite = true;
  T lmax = T(0);
  // the gmin diagonal, before the elimination (addDiagonalConditioning)
  for (int q = tid; q < Tp.n; q += bd) A[__ldg(&Tp.nd_diag[q])] += gmin;
  __syncthreads();
  for (int lv = 0; lv < Tp.nd_levels; ++lv) {
    const int p0 = __ldg(&Tp.lv_piv_ptr[lv]), p1 = __ldg(&Tp.lv_piv_ptr[lv + 1]);
    for (int q = p0 + tid; q < p1; q += bd) {
      const int d = __ldg(&Tp.nd_diag[__ldg(&Tp.lv_piv[q])]);
      const T piv = A[d];
      ok = ok && isfinite(piv) && !(fabs(piv) < tiny);
      A[d] = recip(piv);
    }
    __syncthreads();
    const int e0 = __ldg(&Tp.lv_l_ptr[lv]), e1 = __ldg(&Tp.lv_l_ptr[lv + 1]);
    for (int e = e0 + tid; e < e1; e += bd) {
      const int sl = __ldg(&Tp.l_slot[e]);
      const T l = A[sl] * A[__ldg(&Tp.nd_diag[__ldg(&Tp.l_piv[e])])];
      A[sl] = l;
      lmax = fmax(lmax, fabs(l));
    }
    __syncthreads();
    const int t0 = __ldg(&Tp.lv_ts_ptr[lv]), tl = __ldg(&Tp.lv_tl_ptr[lv]), t1 = __ldg(&Tp.lv_ts_ptr[lv + 1]);
    // two targets per thread in flight (no target of a level is read by
    // another of the same level), each summed in its own order
    int t = t0 + tid;
    for (; t + bd < tl; t += 2 * bd) {
      const int sa = __ldg(&Tp.t_slot[t]), sb = __ldg(&Tp.t_slot[t + bd]);
      int qa = __ldg(&Tp.t_off[t]), qb = __ldg(&Tp.t_off[t + bd]);
      const int qa1 = __ldg(&Tp.t_off[t + 1]), qb1 = __ldg(&Tp.t_off[t + bd + 1]);
      T acc_a = A[sa], acc_b = A[sb];
      for (; qa < qa1 && qb < qb1; ++qa, ++qb) {
        const T la = A[__ldg(&Tp.pr_l[qa])], ua = A[__ldg(&Tp.pr_u[qa])];
        const T lb = A[__ldg(&Tp.pr_l[qb])], ub = A[__ldg(&Tp.pr_u[qb])];
        acc_a -= la * ua;
        acc_b -= lb * ub;
      }
      for (; qa < qa1; ++qa) acc_a -= A[__ldg(&Tp.pr_l[qa])] * A[__ldg(&Tp.pr_u[qa])];
      for (; qb < qb1; ++qb) acc_b -= A[__ldg(&Tp.pr_l[qb])] * A[__ldg(&Tp.pr_u[qb])];
      A[sa] = acc_a;
      A[sb] = acc_b;
    }
    if (t < tl) {
      const int sl = __ldg(&Tp.t_slot[t]), q1 = __ldg(&Tp.t_off[t + 1]);
      T acc = A[sl];
      for (int q = __ldg(&Tp.t_off[t]); q < q1; ++q) acc -= A[__ldg(&Tp.pr_l[q])] * A[__ldg(&Tp.pr_u[q])];
      A[sl] = acc;
    }
    const int r0 = __ldg(&Tp.lv_ys_ptr[lv]), rl = __ldg(&Tp.lv_yl_ptr[lv]), r1 = __ldg(&Tp.lv_ys_ptr[lv + 1]);
    for (int r = r0 + tid; r < rl; r += bd) {
      const int row = __ldg(&Tp.y_row[r]), q1 = __ldg(&Tp.y_off[r + 1]);
      T acc = y[row];
      for (int q = __ldg(&Tp.y_off[r]); q < q1; ++q) acc -= A[__ldg(&Tp.yp_l[q])] * y[__ldg(&Tp.yp_k[q])];
      y[row] = acc;
    }
    for (int t = tl + warp; t < t1; t += nw) {  // long target lists: a warp sums
      const int q0 = __ldg(&Tp.t_off[t]), c = __ldg(&Tp.t_off[t + 1]) - q0;
      T part = T(0);
      for (int q = lane; q < c; q += 32) part += A[__ldg(&Tp.pr_l[q0 + q])] * A[__ldg(&Tp.pr_u[q0 + q])];
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) A[__ldg(&Tp.t_slot[t])] -= part;
    }
    for (int r = rl + warp; r < r1; r += nw) {  // long right-hand-side rows
      const int q0 = __ldg(&Tp.y_off[r]), c = __ldg(&Tp.y_off[r + 1]) - q0;
      T part = T(0);
      for (int q = lane; q < c; q += 32) part += A[__ldg(&Tp.yp_l[q0 + q])] * y[__ldg(&Tp.yp_k[q0 + q])];
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) y[__ldg(&Tp.y_row[r])] -= part;
    }
    __syncthreads();
  }
  for (int lv = Tp.nd_levels - 1; lv >= 0; --lv) {
    const int p0 = __ldg(&Tp.lv_piv_ptr[lv]), p1 = __ldg(&Tp.lv_piv_ptr[lv + 1]);
    for (int q = p0 + tid; q < p1; q += bd) {
      const int k = __ldg(&Tp.lv_piv[q]);
      const int b1 = __ldg(&Tp.bs_off[k + 1]);
      T sv = y[k];
      for (int j = __ldg(&Tp.bs_off[k]); j < b1; ++j) sv -= A[__ldg(&Tp.bs_u[j])] * y[__ldg(&Tp.bs_c[j])];
      sv *= A[__ldg(&Tp.nd_diag[k])];
      y[k] = sv;
      finite = finite && isfinite(sv);
    }
    __syncthreads();
  }
  return __syncthreads_and(ok && finite && !(lmax > growth_limit)) != 0;
}

// Control flow + linear solve of one instance per CTA on the level schedule
// (instances whose ND slots do not fit a warp's share of shared memory, and
// the last few live instances of a job): the same round as lu_round with
// every phase spread over the CTA's threads. The ND slots live in dynamic
// shared memory after the right-hand side (gA = false) or in the instance's
// slice of I.lu_ws (gA = true, nd_S elements per instance); with gY the
// right-hand side goes to I.lu_ws as well, for systems whose n values do not
// fit shared memory. With packed,
// the CTA stages the packed program (nd_program) after the slots and solves
// on it (nd_solve_cta) instead of reading the schedule tables from global
// memory. With I.live_in, CTA b takes the b-th listed instance and lists it
// in I.live_out when it stays live.
// What the body of k_lu_big leaves for its caller (shared memory).
struct LuShared {
  int a, live, trev, sing;
  double gmin, hsub;
};

// The body of k_lu_big for instance g, by the whole CTA: the decision, the
// vector updates, the factor/solve and x = v + dx with junction limiting.
// sh receives the action bits, whether the instance was live, whether it
// evaluated a transient point, whether the static pivots failed, and the
// gmin of the solve.
template <typename T, bool gA, bool packed, bool gY = false>
__device__ void lu_big_instance(const DevTopo& Tp, const DevInst& I, const JobParams& P, int g,
                                unsigned char* smem_raw, LuShared& sh) {
  static_assert(!gY || (gA && !packed), "the solve vector goes to global memory only beside global slots");
  int &s_a = sh.a, &s_live = sh.live, &s_trev = sh.trev, &s_sing = sh.sing;
  double &s_gmin = sh.gmin, &s_hsub = sh.hsub;
  const int n = Tp.n, tid = threadIdx.x;
  const size_t ld = I.ld;
  // gY: the solve vector in global memory too, after every instance's slots
  // (I.lu_ws holds ni * (nd_S + nd_SY) elements)
  T* Y = gY ? reinterpret_cast<T*>(I.lu_ws) + (size_t)I.ni * Tp.nd_S + (size_t)g * Tp.nd_SY
            : reinterpret_cast<T*>(smem_raw);
  T* A = gA ? reinterpret_cast<T*>(I.lu_ws) + (size_t)g * Tp.nd_S : Y + Tp.nd_SY;
  const int* prog = nullptr;
  if (packed) {  // after the slots, on a 16-byte boundary
    int* dst = reinterpret_cast<int*>(
        smem_raw + (((size_t)(Tp.nd_SY + Tp.nd_S) * sizeof(T) + 15) & ~size_t(15)));
    const int4* srcp = reinterpret_cast<const int4*>(Tp.nd_prog);
    for (int e = tid; e < (Tp.nd_prog_len + 3) / 4; e += blockDim.x)
      reinterpret_cast<int4*>(dst)[e] = __ldg(&srcp[e]);
    prog = dst;
  }
  if (tid == 0) {
    int live = 0, trev = 0;
    double gm = 1e-12, hs = P.h;
    const int a = g < I.ni ? instance_decide(Tp, I, P, g, live, trev, gm, hs) : 0;
    s_a = a;
    s_live = live;
    s_trev = trev;
    s_gmin = gm;
    s_hsub = hs;
    s_sing = 0;
  }
  __syncthreads();
  if (!s_live) return;
  const int a = s_a;
  const double gmin = s_gmin;

  // the instance's ND slots from its Jacobian value slots
  if (a & ACT_SOLVE) {
    const T* J = reinterpret_cast<const T*>(I.J);
    for (int sl = tid; sl < Tp.nd_nv; sl += blockDim.x) {
      const int src = __ldg(&Tp.nd_src[sl]);
      A[sl] = src >= 0 ? J[(size_t)src * ld + g] : T(0);
    }
  }
  // vector updates and the right-hand side
  {
    double* __restrict__ X = I.x;
    double* __restrict__ V = I.v;
    double* __restrict__ VT = I.v_tp;
    const double* __restrict__ F = I.F;
    for (int i = tid; i < n; i += blockDim.x) {
      const size_t o = (size_t)i * ld + g;
      const double fi = F[o];
      double vi;
      if (a & ACT_RESTART) {
        vi = VT[o];
        V[o] = vi;
        X[o] = vi;
      } else if (a & ACT_RESEED) {
        vi = V[o];
        X[o] = vi;
      } else {
        double xi = X[o];
        vi = V[o];
        if (a & ACT_DAMP) {
          xi = vi + 0.5 * (xi - vi);
          X[o] = xi;
        }
        if (a & ACT_ACCEPT) {
          vi = xi;
          V[o] = vi;
        }
        if (a & (ACT_STEP | ACT_TRAN_INIT)) {
          if (P.lte_rel > 0.0 && I.v_tpp)  // the LTE predictor's older point
            I.v_tpp[o] = (a & ACT_TRAN_INIT) ? vi : VT[o];
          VT[o] = vi;
        }
      }
      if (a & ACT_SOLVE) Y[__ldg(&Tp.nd_pos[i])] = (T)(-(fi + gmin * vi));
    }
  }
  __syncthreads();
  // capacitor history after a completed (sub-)step, waveform samples
  if (a & (ACT_TRAN_INIT | ACT_STEP)) {
    for (int c = tid; c < Tp.n_cap; c += blockDim.x) {
      const int2 tt = __ldg(&Tp.cap_term[c]);
      const double vc = (tt.x >= 0 ? I.v[tt.x * ld + g] : 0.0) - (tt.y >= 0 ? I.v[tt.y * ld + g] : 0.0);
      const size_t ci = (size_t)c * ld + g;
      if (a & ACT_TRAN_INIT) {
        I.cap_vp[ci] = vc;
        I.cap_ip[ci] = 0.0;
      } else {
        const double C = __ldg(&Tp.cap_c[c]);
        const double h = s_hsub;
        const double ic = P.method == KTRAN_TRAP ? (2.0 * C / h) * (vc - I.cap_vp[ci]) - I.cap_ip[ci]
                                                 : (C / h) * (vc - I.cap_vp[ci]);
        I.cap_vp[ci] = vc;
        I.cap_ip[ci] = ic;
      }
    }
  }
  if ((a & ACT_WAVE) && I.n_wave > 0) {
    const int done_step = I.st[g].step - 1;  // 1-based step just completed
    if (done_step >= 1 && done_step <= I.wave_steps)
      for (int w = tid; w < I.n_wave; w += blockDim.x) {
        const int q = I.wave_pos[w];
        I.wave[((size_t)g * I.wave_steps + (done_step - 1)) * I.n_wave + w] = q >= 0 ? I.v[q * ld + g] : 0.0;
      }
  }
  __syncthreads();

  if (a & ACT_SOLVE) {
    const T tiny = sizeof(T) == 8 ? (T)1e-25 : (T)1e-30;
    const T growth = sizeof(T) == 8 ? (T)P.growth64 : (T)fmin(P.growth32, 3.0e38);
    const bool ok = packed ? nd_solve_cta<T>(A, Y, prog, (T)gmin, tiny, growth)
                           : big_solve<T>(A, Y, Tp, (T)gmin, tiny, growth);
    // x = v + dx, then junction limiting level by level
    if (ok) {
      for (int i = tid; i < n; i += blockDim.x) {
        const size_t o = (size_t)i * ld + g;
        double xi = I.v[o] + (double)Y[__ldg(&Tp.nd_pos[i])];
        if ((a & ACT_LIMIT) && !isfinite(xi)) xi = 0.0;  // SafeUtils::sanitize_vector
        I.x[o] = xi;
      }
      if ((a & ACT_LIMIT) && Tp.n_dio > 0) {
        __syncthreads();
        for (int lvl = 0; lvl < Tp.n_dio_levels; ++lvl) {
          for (int d = tid; d < Tp.n_dio; d += blockDim.x)
            if (__ldg(&Tp.dio_level[d]) == lvl) limit_one(Tp, d, I.x, I.v, ld, g);
          __syncthreads();
        }
      }
    }
    if (tid == 0) s_sing = ok ? 0 : 1;
  }
  __syncthreads();
}

template <typename T, bool gA, bool packed, bool gY = false>
__global__ void __launch_bounds__(kBigThreads) k_lu_big(DevTopo Tp, DevInst I, JobParams P, int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ LuShared sh;
  int g = blockIdx.x;
  if (I.live_in) {
    if ((int)blockIdx.x >= *I.live_in_count) return;
    g = I.live_in[blockIdx.x];
  }
  lu_big_instance<T, gA, packed, gY>(Tp, I, P, g, smem_raw, sh);
  if (!sh.live) return;
  // rescue hand-off, next evaluation point, bookkeeping
  if (threadIdx.x == 0) {
    const int a = sh.a, sing = sh.sing;
    if (instance_finish(Tp, I, P, g, a, sing, sh.gmin)) {
      atomicAdd(active, 1);
      if (I.live_out) I.live_out[atomicAdd(I.live_out_count, 1)] = g;
    }
    if (I.counters) {
      atomicAdd(&I.counters[sh.trev ? 1 : 0], 1ull);
      if ((a & ACT_SOLVE) && !sing) atomicAdd(&I.counters[2], 1ull);
    }
  }
}

// The instances not yet done, listed (any order) for the tail rounds.
__global__ void k_live_list(DevInst I, int* list, int* count) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < I.ni && I.st[g].mode != MODE_DONE) list[atomicAdd(count, 1)] = g;
}

// ---------------------------------------------------------------------------
// rescue of the solves whose static pivots failed, one warp per solve:
//   level 1 (mixed precision only; the FP64 path already ran it): the static
//   pivots again, in FP64 on the value slots;
//   level 2: LU with partial pivoting -- the semantics of solveSparse_LU's
//   numeric phase (math/sparse_lu.cpp:216-312) on the permuted system: pivot
//   = largest |a| in the column over the rows not yet pivoted (ties to the
//   lower position), singular below 1e-25, rows with |a| < 1e-30 not
//   eliminated (their entry still enters the forward substitution).
// Level 2 keeps a row in its value slots while every update it receives falls
// on its slots (always so until a row interchange brings another row's
// structure into play); a row that would take fill outside them moves to a
// dense row buffer: a few per warp in shared memory, the rest in the warp's
// global workspace. The arithmetic is that of the dense elimination: each
// entry takes a = fma(-l, u, a) in pivot order, and the only terms left out
// are those with u == 0 (which leave a unchanged); the right-hand side is
// eliminated with its row, in the order of a forward substitution; U is
// written densely and solved in the order of a column-oriented back
// substitution, in blocks of 32 columns.
// ---------------------------------------------------------------------------

// Bytes of the pivot records staged once per rescue CTA (stage_pivots).
__host__ __device__ inline size_t rescue_rec_bytes(int n) {
  return ((size_t)n * (2 * sizeof(int4) + sizeof(int2)) + 15) & ~size_t(15);
}
// Bytes of the slot tables staged once per rescue CTA: row and column
// pointers (n + 1 each), (row, slot) by column and the column of each slot.
__host__ __device__ inline size_t rescue_tab_bytes(int n, int nv) {
  return (sizeof(int) * 2 * ((size_t)n + 1) + sizeof(int2) * (size_t)nv + sizeof(int) * (size_t)nv +
          15) &
         ~size_t(15);
}
// Per-warp shared memory: value slots, right-hand side, K dense row buffers
// and the candidate entries (FP64), then five int arrays of n and the
// candidate rows.
__host__ __device__ inline size_t rescue_warp_bytes(int n, int nv, int K) {
  return (sizeof(double) * ((size_t)nv + n + (size_t)K * n + 32) +
          sizeof(int) * (5 * (size_t)n + 32) + 15) &
         ~size_t(15);
}

struct RescueTab {
  const int2* cent;  // [nv] (row, slot) by column
  const int* cptr;   // [n + 1]
  const int* sptr;   // [n + 1] first slot of each row
  const int* scol;   // [nv] column of each slot (ascending within a row)
};

// Slot of column c in the slot range [s0, s1) of one row, or -1.
__device__ __forceinline__ int find_slot(const int* __restrict__ scol, int s0, int s1, int c) {
  int lo = s0, hi = s1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (scol[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < s1 && scol[lo] == c) ? lo : -1;
}

struct RescueWarp {
  double* vs;   // [nv] value slots (rows kept in their slots)
  double* bp;   // [n] right-hand side by row
  double* fb;   // [K][n] dense row buffers in shared memory
  double* G;    // [n - K][n] dense row buffers in global memory
  double* U;    // [n][n] U by position, row-major (upper part)
  int* pos_of;  // [n] position of each row
  int* row_at;  // [n] row at each position
  int* fat_of;  // [n] row buffer of each row, -1 = in its slots
  int* live;    // rows with a buffer
  int* stk;     // free buffers (shared-memory ones on top)
  int* cr;      // [32] candidate rows of the current column
  double* ca;   // [32] their entries
  int K;
};

__device__ __forceinline__ double* rescue_buf(const RescueWarp& w, int n, int f) {
  return f < w.K ? w.fb + (size_t)f * n : w.G + (size_t)(f - w.K) * n;
}

// One step-i elimination of row r (entry a in column i) by the pivot row:
// prow = its dense buffer, or null when it is in its slots [ps0, ps1); Uc =
// U row i, already written (column-major: Uc[c * n]); top / nlive = buffer
// stack and live list sizes (warp-uniform).
__device__ __forceinline__ void rescue_eliminate(const RescueTab& tb, const RescueWarp& w, int n,
                                                 int i, int r, double a, double piv, double bP,
                                                 const double* prow, int ps0, int ps1,
                                                 const double* Uc, int& top, int& nlive,
                                                 int lane) {
  if (fabs(a) >= 1e-30) {
    const double l = a / piv;
    if (lane == 0) w.bp[r] = fma(-l, bP, w.bp[r]);
    // a non-finite multiplier turns the structural zeros of the dense
    // elimination into NaN too (l * 0): update every column from U row i
    const bool full = !isfinite(l);
    int fr = w.fat_of[r];
    double* fbuf;
    if (fr < 0) {
      const int s0 = tb.sptr[r], s1 = tb.sptr[r + 1];
      if (!prow && !full) {
        // both rows in their slots: in place when the pivot row's nonzero
        // columns past i are all slots of row r
        bool in = true;
        for (int s = ps0 + lane; s < ps1; s += 32) {
          const int c = tb.scol[s];
          if (c > i && w.vs[s] != 0.0 && find_slot(tb.scol, s0, s1, c) < 0) in = false;
        }
        if (__all_sync(kFull, in)) {
          for (int s = ps0 + lane; s < ps1; s += 32) {
            const int c = tb.scol[s];
            const double u = w.vs[s];
            if (c > i && u != 0.0) {
              const int t = find_slot(tb.scol, s0, s1, c);
              w.vs[t] = fma(-l, u, w.vs[t]);
            }
          }
          __syncwarp();
          return;
        }
      }
      // row r moves to a dense row buffer
      fr = w.stk[top - 1];
      fbuf = rescue_buf(w, n, fr);
      __syncwarp();
      if (lane == 0) {
        w.fat_of[r] = fr;
        w.live[nlive] = r;
      }
      --top;
      ++nlive;
      if (prow && !full) {  // (slot value or 0) - l * (pivot row), in one pass
        for (int c = i + 1 + lane; c < n; c += 32) {
          const double u = prow[c];
          fbuf[c] = u != 0.0 ? fma(-l, u, 0.0) : 0.0;
        }
        __syncwarp();
        for (int s = s0 + lane; s < s1; s += 32) {
          const int c = tb.scol[s];
          if (c > i) fbuf[c] = fma(-l, prow[c], w.vs[s]);
        }
        __syncwarp();
        return;
      }
      for (int c = i + 1 + lane; c < n; c += 32) fbuf[c] = 0.0;
      __syncwarp();
      for (int s = s0 + lane; s < s1; s += 32) {
        const int c = tb.scol[s];
        if (c > i) fbuf[c] = w.vs[s];
      }
      __syncwarp();
    } else {
      fbuf = rescue_buf(w, n, fr);
    }
    if (full) {
      for (int c = i + 1 + lane; c < n; c += 32) fbuf[c] = fma(-l, Uc[(size_t)c * n], fbuf[c]);
    } else if (prow) {
      for (int c = i + 1 + lane; c < n; c += 32) {
        const double u = prow[c];
        if (u != 0.0) fbuf[c] = fma(-l, u, fbuf[c]);
      }
    } else {
      for (int s = ps0 + lane; s < ps1; s += 32) {
        const int c = tb.scol[s];
        const double u = w.vs[s];
        if (c > i && u != 0.0) fbuf[c] = fma(-l, u, fbuf[c]);
      }
    }
  } else if (a != 0.0 && lane == 0) {
    w.bp[r] = fma(-a, bP, w.bp[r]);  // not eliminated; still in the forward substitution
  }
  __syncwarp();
}

// Level 2 on the staged system (vs with gmin on the diagonal, bp). Returns
// true with the solution by position in vs, false when singular. U is
// written column-major (U[c * n + r] = u_rc) for a coalesced back
// substitution.
__device__ __forceinline__ bool rescue_pp(const RescueTab& tb, const RescueWarp& w, int n,
                                          int lane) {
  for (int r = lane; r < n; r += 32) {
    w.pos_of[r] = r;
    w.row_at[r] = r;
    w.fat_of[r] = -1;
    w.stk[r] = n - 1 - r;
  }
  int top = n, nlive = 0;  // warp-uniform
  __syncwarp();
  const unsigned below = (1u << lane) - 1u;
  for (int i = 0; i < n; ++i) {
    // 1. candidates: rows at positions >= i with a nonzero entry in column i
    //    (rows in buffers, then rows in slots), listed in cr / ca while they
    //    fit; zeros never win the pivot search unless the column is singular
    int cnt = 0;  // warp-uniform
    for (int q0 = 0; q0 < nlive; q0 += 32) {
      const int qq = q0 + lane;
      int r = -1;
      double a = 0.0;
      if (qq < nlive) {
        r = w.live[qq];
        a = rescue_buf(w, n, w.fat_of[r])[i];
      }
      const bool c = qq < nlive && a != 0.0;
      const unsigned m = __ballot_sync(kFull, c);
      if (c) {
        const int q = cnt + __popc(m & below);
        if (q < 32) {
          w.cr[q] = r;
          w.ca[q] = a;
        }
      }
      cnt += __popc(m);
    }
    const int e0 = tb.cptr[i], e1 = tb.cptr[i + 1];
    for (int b0 = e0; b0 < e1; b0 += 32) {
      const int e = b0 + lane;
      int r = -1;
      double a = 0.0;
      bool c = false;
      if (e < e1) {
        const int2 rs = tb.cent[e];
        r = rs.x;
        if (w.pos_of[r] >= i && w.fat_of[r] < 0) {
          a = w.vs[rs.y];
          c = a != 0.0;
        }
      }
      const unsigned m = __ballot_sync(kFull, c);
      if (c) {
        const int q = cnt + __popc(m & below);
        if (q < 32) {
          w.cr[q] = r;
          w.ca[q] = a;
        }
      }
      cnt += __popc(m);
    }
    __syncwarp();
    // 2. pivot: the largest |a|, ties to the lower position (pos << 16 | row)
    double best = -1.0;
    int bkey = 0x7fffffff;
    if (cnt <= 4) {  // a short list: every lane scans it
      for (int q = 0; q < cnt; ++q) {
        const int r = w.cr[q];
        const double av = fabs(w.ca[q]);
        const int key = w.pos_of[r] << 16 | r;
        if (av > best || (av == best && key < bkey)) {
          best = av;
          bkey = key;
        }
      }
    } else {
      if (cnt <= 32) {
        if (lane < cnt) {
          const int r = w.cr[lane];
          best = fabs(w.ca[lane]);
          bkey = w.pos_of[r] << 16 | r;
        }
      } else {  // more than the list holds: rescan
        for (int q = lane; q < nlive; q += 32) {
          const int r = w.live[q];
          const double av = fabs(rescue_buf(w, n, w.fat_of[r])[i]);
          const int key = w.pos_of[r] << 16 | r;
          if (av > best || (av == best && key < bkey)) {
            best = av;
            bkey = key;
          }
        }
        for (int e = e0 + lane; e < e1; e += 32) {
          const int2 rs = tb.cent[e];
          const int ps = w.pos_of[rs.x];
          if (ps >= i && w.fat_of[rs.x] < 0) {
            const double av = fabs(w.vs[rs.y]);
            const int key = ps << 16 | rs.x;
            if (av > best || (av == best && key < bkey)) {
              best = av;
              bkey = key;
            }
          }
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int ok = __shfl_xor_sync(kFull, bkey, o);
        if (ob > best || (ob == best && ok < bkey)) {
          best = ob;
          bkey = ok;
        }
      }
    }
    if (best < 1e-25) return false;
    const int Pr = bkey & 0xffff, bpos = bkey >> 16;
    const int q = w.row_at[i];
    const int fP = w.fat_of[Pr];
    double* prow = fP >= 0 ? rescue_buf(w, n, fP) : nullptr;
    const int ps0 = tb.sptr[Pr], ps1 = tb.sptr[Pr + 1];
    // the pivot row came from column i's list, so a slot-resident one has that slot
    const double piv = prow ? prow[i] : w.vs[find_slot(tb.scol, ps0, ps1, i)];
    const double bP = w.bp[Pr];
    __syncwarp();
    if (lane == 0) {  // row interchange: positions only
      w.row_at[bpos] = q;
      w.pos_of[q] = bpos;
      w.row_at[i] = Pr;
      w.pos_of[Pr] = i;
    }
    double* Uc = w.U + i;  // U row i: Uc[c * n]

    // 3. the common step of a row interchange chain: the pivot row in a
    //    buffer and one other candidate, in its slots, eliminated with a
    //    finite multiplier -- the candidate takes over the pivot row's
    //    buffer (same values as a fresh buffer)
    bool fast = false;
    int fr = -1, s0 = 0, s1 = 0;
    double fa = 0.0, fl = 0.0;
    if (prow && cnt == 2 && isfinite(bP)) {
      fr = w.cr[0] == Pr ? w.cr[1] : w.cr[0];
      fa = w.cr[0] == Pr ? w.ca[1] : w.ca[0];
      s0 = tb.sptr[fr];
      s1 = tb.sptr[fr + 1];
      if (w.fat_of[fr] < 0 && fabs(fa) >= 1e-30 && s1 - s0 <= 32) {
        fl = fa / piv;
        fast = isfinite(fl);
      }
    }
    if (fast) {
      const double l = fl;
      if (lane == 0) w.bp[fr] = fma(-l, bP, w.bp[fr]);
      int sc = -1;
      double sv = 0.0;
      if (s0 + lane < s1) {
        sc = tb.scol[s0 + lane];
        if (sc > i)
          sv = fma(-l, prow[sc], w.vs[s0 + lane]);
        else
          sc = -1;
      }
      __syncwarp();
      for (int c = i + lane; c < n; c += 32) {
        const double u = prow[c];
        Uc[(size_t)c * n] = u;
        if (c > i) prow[c] = u != 0.0 ? fma(-l, u, 0.0) : 0.0;
      }
      __syncwarp();
      if (sc >= 0) prow[sc] = sv;
      int qi = -1;
      for (int q2 = lane; q2 < nlive; q2 += 32)
        if (w.live[q2] == Pr) qi = q2;
      qi = __reduce_max_sync(kFull, qi);
      if (lane == 0) {
        w.fat_of[fr] = fP;
        w.fat_of[Pr] = -1;
        w.live[qi] = fr;
      }
      __syncwarp();
      continue;
    }

    // 4. general step: U row i, then every other candidate
    if (prow) {
      for (int c = i + lane; c < n; c += 32) Uc[(size_t)c * n] = prow[c];
    } else {
      for (int c = i + lane; c < n; c += 32) Uc[(size_t)c * n] = 0.0;
      __syncwarp();
      for (int s = ps0 + lane; s < ps1; s += 32) {
        const int c = tb.scol[s];
        if (c >= i) Uc[(size_t)c * n] = w.vs[s];
      }
    }
    __syncwarp();
    if (!isfinite(bP)) {
      // the forward substitution's 0 * b of the rows with no entry in
      // column i gives NaN (the others take theirs in the eliminations)
      for (int k = i + 1 + lane; k < n; k += 32) {
        const int r = w.row_at[k];
        double a;
        if (w.fat_of[r] >= 0) {
          a = rescue_buf(w, n, w.fat_of[r])[i];
        } else {
          const int t = find_slot(tb.scol, tb.sptr[r], tb.sptr[r + 1], i);
          a = t >= 0 ? w.vs[t] : 0.0;
        }
        if (a == 0.0) w.bp[r] = fma(-a, bP, w.bp[r]);
      }
      __syncwarp();
    }
    if (cnt <= 32) {
      for (int q2 = 0; q2 < cnt; ++q2) {
        const int r = w.cr[q2];
        if (r != Pr)
          rescue_eliminate(tb, w, n, i, r, w.ca[q2], piv, bP, prow, ps0, ps1, Uc, top, nlive,
                           lane);
      }
    } else {
      // rows in buffers first (the list only grows below), then rows in slots
      for (int q0 = 0; q0 < nlive; q0 += 32) {
        const int qq = q0 + lane;
        int r = -1;
        double a = 0.0;
        if (qq < nlive) {
          r = w.live[qq];
          a = rescue_buf(w, n, w.fat_of[r])[i];
        }
        unsigned m = __ballot_sync(kFull, qq < nlive && r != Pr && a != 0.0);
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          rescue_eliminate(tb, w, n, i, __shfl_sync(kFull, r, src), __shfl_sync(kFull, a, src),
                           piv, bP, prow, ps0, ps1, Uc, top, nlive, lane);
        }
      }
      for (int b0 = e0; b0 < e1; b0 += 32) {
        const int e = b0 + lane;
        int r = -1;
        double a = 0.0;
        bool cand = false;
        if (e < e1) {
          const int2 rs = tb.cent[e];
          r = rs.x;
          if (r != Pr && w.pos_of[r] >= i && w.fat_of[r] < 0) {
            a = w.vs[rs.y];
            cand = a != 0.0;
          }
        }
        unsigned m = __ballot_sync(kFull, cand);
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          rescue_eliminate(tb, w, n, i, __shfl_sync(kFull, r, src), __shfl_sync(kFull, a, src),
                           piv, bP, prow, ps0, ps1, Uc, top, nlive, lane);
        }
      }
    }
    if (fP >= 0) {  // the pivot row's buffer is free again
      int qi = -1;
      for (int q2 = lane; q2 < nlive; q2 += 32)
        if (w.live[q2] == Pr) qi = q2;
      qi = __reduce_max_sync(kFull, qi);
      __syncwarp();
      if (lane == 0) {
        w.live[qi] = w.live[nlive - 1];
        w.stk[top] = fP;
        w.fat_of[Pr] = -1;
      }
      --nlive;
      ++top;
      __syncwarp();
    }
  }

  // back substitution by position, column-oriented in blocks of 32 columns;
  // each lane holds its row's part of the block's triangle in registers
  double* xs = w.vs;
  for (int k = lane; k < n; k += 32) xs[k] = w.bp[w.row_at[k]];
  __syncwarp();
  for (int j1 = n; j1 > 0; j1 -= 32) {
    const int j0 = j1 > 32 ? j1 - 32 : 0;
    const int m = j1 - j0;
    const int k = j0 + lane;
    double u[32];
#pragma unroll
    for (int t = 0; t < 32; ++t)
      u[t] = (t < m && t >= lane) ? w.U[(size_t)(j0 + t) * n + k] : 0.0;
    double acc = k < j1 ? xs[k] : 0.0;
#pragma unroll
    for (int t = 31; t >= 0; --t) {
      if (t < m) {
        if (lane == t) acc = acc / u[t];
        const double xj = __shfl_sync(kFull, acc, t);
        if (lane < t) acc = fma(-u[t], xj, acc);
      }
    }
    if (k < j1) xs[k] = acc;
    __syncwarp();
    // rows above the block: their 32 updates in descending column order
    for (int r0 = 0; r0 < j0; r0 += 32) {
      const int r = r0 + lane;
      if (r < j0) {
        double v[32];
#pragma unroll
        for (int t = 0; t < 32; ++t) v[t] = w.U[(size_t)(j0 + t) * n + r];
        double a2 = xs[r];
#pragma unroll
        for (int t = 31; t >= 0; --t) a2 = fma(-v[t], xs[j0 + t], a2);
        xs[r] = a2;
      }
    }
    __syncwarp();
  }
  return true;
}

// K = dense row buffers per warp in shared memory; blockDim.x / 32 warps per
// CTA, warp w of CTA b owning workspace slot b * warps + w (U and the global
// row buffers, 2 n^2 doubles). Shared memory: pivot records (when the
// static-pivot program has them), slot tables, then the warps' areas.
// Stages the rescue's shared tables (the pivot records when the problem has
// them, the slot tables) at base, by the whole CTA; returns the first byte
// after them. The caller synchronises before using them.
__device__ unsigned char* rescue_setup(const DevTopo& Tp, unsigned char* base, int4*& rec,
                                       RescueTab& tb) {
  const int n = Tp.n, nv = Tp.nv;
  rec = nullptr;
  if (Tp.lu_rec) {
    rec = reinterpret_cast<int4*>(base);
    stage_pivots(Tp, rec, 1);
    base += rescue_rec_bytes(n);
  }
  int2* cent = reinterpret_cast<int2*>(base);
  int* cptr = reinterpret_cast<int*>(cent + nv);
  int* sptr = cptr + n + 1;
  int* scol = sptr + n + 1;
  for (int e = threadIdx.x; e < nv; e += blockDim.x) {
    cent[e] = __ldg(&Tp.csc_ent[e]);
    scol[e] = __ldg(&Tp.slot_rc[e]).y;
  }
  for (int e = threadIdx.x; e <= n; e += blockDim.x) {
    cptr[e] = __ldg(&Tp.csc_ptr[e]);
    sptr[e] = __ldg(&Tp.slot_ptr[e]);
  }
  tb.cent = cent;
  tb.cptr = cptr;
  tb.sptr = sptr;
  tb.scol = scol;
  return base + rescue_tab_bytes(n, nv);
}

// The rescue warp's buffers at base (shared memory, rescue_warp_bytes) and
// workspace slot `slot` of I.rescue_ws.
__device__ RescueWarp rescue_warp(const DevTopo& Tp, const DevInst& I, unsigned char* base, int K,
                                  int slot) {
  const int n = Tp.n, nv = Tp.nv;
  RescueWarp w;
  w.vs = reinterpret_cast<double*>(base);
  w.bp = w.vs + nv;
  w.fb = w.bp + n;
  w.ca = w.fb + (size_t)K * n;
  w.pos_of = reinterpret_cast<int*>(w.ca + 32);
  w.row_at = w.pos_of + n;
  w.fat_of = w.row_at + n;
  w.live = w.fat_of + n;
  w.stk = w.live + n;
  w.cr = w.stk + n;
  w.K = K;
  w.U = I.rescue_ws + (size_t)slot * 2 * n * n;
  w.G = w.U + (size_t)n * n;
  return w;
}

// Rescue of instance g's failed linear solve (action bits act, gmin) by one
// warp: FP64 static pivots first (mixed precision), then the LU with partial
// pivoting. On success x = v + dx (sanitised and junction-limited for DC NR
// iterations) and the instance's rescue count grows; otherwise the
// singular-matrix branch of the control flow runs.
template <typename TJ>
__device__ void rescue_item(const DevTopo& Tp, const DevInst& I, const JobParams& P,
                            const RescueTab& tb, const RescueWarp& w, const int4* rec, int g,
                            int act, double gmin, int lane) {
  const int n = Tp.n, nv = Tp.nv;
  const size_t ld = I.ld;
  const TJ* J = reinterpret_cast<const TJ*>(I.J);
  auto stage = [&]() {
#pragma unroll 4
    for (int s = lane; s < nv; s += 32) w.vs[s] = (double)J[(size_t)s * ld + g];
#pragma unroll 4
    for (int i = lane; i < n; i += 32) {
      const size_t o = (size_t)i * ld + g;
      w.bp[i] = -(I.F[o] + gmin * I.v[o]);
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) w.vs[__ldg(&Tp.lu_hdr[i]).w] += gmin;
    __syncwarp();
  };
  int ok = 0;
  const double* sol = w.bp;
  if (P.precision == KPREC_MIXED) {
    stage();
    if (lane == 0) ok = lu_solve<double>(w.vs, w.bp, 1, Tp, rec, 1e-25, P.growth64) ? 1 : 0;
    ok = __shfl_sync(kFull, ok, 0);
    __syncwarp();
  }
  if (!ok) {
    stage();
    if (rescue_pp(tb, w, n, lane)) {
      ok = 1;
      sol = w.vs;
      if (lane == 0 && I.counters) atomicAdd(&I.counters[4], 1ull);
    }
  }
  if (ok) {
    const bool sanitize = (act & ACT_LIMIT) != 0;
    for (int i = lane; i < n; i += 32) {
      const size_t o = (size_t)i * ld + g;
      double xi = I.v[o] + sol[i];
      if (sanitize && !isfinite(xi)) xi = 0.0;
      I.x[o] = xi;
    }
    __syncwarp();
    if (lane == 0) {
      if (sanitize)
        for (int d = 0; d < Tp.n_dio; ++d) limit_one(Tp, d, I.x, I.v, ld, g);
      I.st[g].rescued += 1;
      if (I.counters) atomicAdd(&I.counters[3], 1ull);
    }
  } else if (lane == 0) {
    on_singular(Tp, I, g);
    set_eval_point(I, P, g, I.st[g]);
  }
  __syncwarp();
}

template <typename TJ>
__global__ void __launch_bounds__(256) k_rescue(DevTopo Tp, DevInst I, JobParams P, int K) {
  extern __shared__ __align__(16) double rs[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
  const int total = *I.rescue_count;
  if ((int)blockIdx.x >= total) return;  // item e runs on CTA e % grid: one solve per SM first
  int4* rec;
  RescueTab tb;
  unsigned char* base = rescue_setup(Tp, reinterpret_cast<unsigned char*>(rs), rec, tb);
  __syncthreads();
  const int slot = blockIdx.x * W + warp;
  if (slot >= I.rescue_slots) return;
  const RescueWarp w = rescue_warp(Tp, I, base + (size_t)warp * rescue_warp_bytes(Tp.n, Tp.nv, K), K, slot);
  for (int e = warp * gridDim.x + blockIdx.x; e < total; e += gridDim.x * W) {
    const RescueItem item = I.rescue_list[e];
    rescue_item<TJ>(Tp, I, P, tb, w, rec, item.inst, item.act, item.gmin, lane);
  }
}

// Threads of the persistent per-instance kernel.
constexpr int kPersistThreads = 512;

// Static shared memory of the persistent kernels' rounds.
struct PersistShared {
  unsigned long long f[kPersistThreads / 32], dv[kPersistThreads / 32];
  int fl[kPersistThreads / 32];
  LuShared lu;
  int rescue;
  int slot;  // rescue workspace slot of this round's rescue
};

// Cycles a CTA waits for a free rescue workspace slot (about 8 s of SM
// clock) before it gives the solve up as singular.
constexpr long long kSlotWaitCycles = 1ll << 34;

// A free slot of the shared rescue workspace (slot_lock[k] == 0 -> 1), tried
// from k = first upward, cyclically; -1 (and *timeouts + 1) when none came free
// within kSlotWaitCycles. Holders release theirs after their rescue, and a
// rescue waits on nothing, so every held slot comes free.
__device__ __forceinline__ int acquire_slot(int* slot_lock, int n_slots, int first, int* timeouts) {
  const long long t0 = clock64();
  for (int k = first % n_slots;; k = k + 1 == n_slots ? 0 : k + 1) {
    if (atomicCAS(&slot_lock[k], 0, 1) == 0) {
      __threadfence();
      return k;
    }
    if (clock64() - t0 > kSlotWaitCycles) {
      if (timeouts) atomicAdd(timeouts, 1);
      return -1;
    }
  }
}

// Every remaining NR round of instance g by the whole CTA: the rounds
// k_es_one + k_lu_big<T, gA, packed> + k_rescue would run one launch each,
// with the same device code, so the results are theirs bit for bit. An
// instance whose static pivots fail is rescued by the CTA's warp 0: in
// workspace slot `slot` when slot_lock is null, else in a slot taken from
// the shared pool slot_lock[0 .. I.rescue_slots) for that rescue (a solve
// that finds no slot within kSlotWaitCycles counts in *slot_timeouts and is
// treated as singular). Stops when the instance is done or after max_rounds
// rounds; then thread 0 adds 1 to *active if the instance is still live and
// raises *rounds_max to the rounds it ran. Dynamic shared memory: the
// largest of the three phases' needs (they run one after another).
template <typename T, bool gA, bool packed>
__device__ void persist_instance(const DevTopo& Tp, const DevInst& I, const JobParams& P, int g,
                                 int slot, int K, int max_rounds, unsigned char* smem_raw,
                                 PersistShared& S, int* active, int* rounds_max,
                                 int* slot_lock = nullptr, int* slot_timeouts = nullptr,
                                 bool slot_values = false) {
  const int tid = threadIdx.x;
  int r = 0;
  bool live = I.ev_heff[g] >= 0.0;
  for (; r < max_rounds && live; ++r) {
    es_one_instance<T, false>(Tp, I, P, g, reinterpret_cast<double*>(smem_raw), S.f, S.dv, S.fl,
                              slot_values);
    __syncthreads();
    lu_big_instance<T, gA, packed>(Tp, I, P, g, smem_raw, S.lu);
    if (!S.lu.live) break;
    const int a = S.lu.a, sing = (a & ACT_SOLVE) ? S.lu.sing : 0;
    if (tid == 0) {
      int rs = -1;
      if (sing && I.rescue_ws != nullptr) {
        if (!slot_lock)
          rs = slot < I.rescue_slots ? slot : -1;
        else if (I.rescue_slots > 0)
          rs = acquire_slot(slot_lock, I.rescue_slots, slot, slot_timeouts);
      }
      S.rescue = rs >= 0;
      S.slot = rs;
      if (S.rescue)
        set_eval_point(I, P, g, I.st[g]);  // as instance_finish does before its hand-off
      else
        instance_finish(Tp, I, P, g, a, sing, S.lu.gmin);
      if (I.counters) {
        atomicAdd(&I.counters[S.lu.trev ? 1 : 0], 1ull);
        if ((a & ACT_SOLVE) && !sing) atomicAdd(&I.counters[2], 1ull);
      }
    }
    __syncthreads();
    if (S.rescue) {
      int4* rec;
      RescueTab tb;
      unsigned char* base = rescue_setup(Tp, smem_raw, rec, tb);
      __syncthreads();
      if (tid < 32) {
        const RescueWarp w = rescue_warp(Tp, I, base, K, S.slot);
        rescue_item<T>(Tp, I, P, tb, w, rec, g, a, S.lu.gmin, tid);
        if (slot_lock) __threadfence();  // the workspace writes before the slot's release
      }
      __syncthreads();
      if (tid == 0 && slot_lock) atomicExch(&slot_lock[S.slot], 0);
    }
    live = I.ev_heff[g] >= 0.0;
    __syncthreads();  // every thread has read the next evaluation point
  }
  if (tid == 0) {
    if (I.st[g].mode != MODE_DONE) atomicAdd(active, 1);
    atomicMax(rounds_max, r);
  }
}

// Byte offsets of one instance's state in shared memory (resident_in),
// each region on a 16-byte boundary; es = the Jacobian value size.
struct ResidentLayout {
  size_t v, x, F, vtp, vtpp, cvp, cip, vsdc, v1, v2, hist, scal, st, J, kp, vth, total;
};
__host__ __device__ inline ResidentLayout resident_layout(const DevTopo& T, size_t es) {
  ResidentLayout L{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o += (bytes + 15) & ~size_t(15);
    return at;
  };
  const size_t n = (size_t)T.n, nc = (size_t)T.n_cap, ns = (size_t)T.n_vs;
  L.v = take(8 * n);
  L.x = take(8 * n);
  L.F = take(8 * n);
  L.vtp = take(8 * n);
  L.vtpp = take(8 * n);
  L.cvp = take(8 * nc);
  L.cip = take(8 * nc);
  L.vsdc = take(8 * ns);
  L.v1 = take(8 * ns);
  L.v2 = take(8 * ns);
  L.hist = take(8 * 2 * KHIST_LEN);
  L.scal = take(8 * 6);  // ev_t, ev_heff, red_f, red_dv, red_flags, ev_lte
  L.st = take(sizeof(InstState));
  L.J = take(es * (size_t)T.nv);
  L.kp = take(4 * (size_t)T.n_mos);
  L.vth = take(4 * (size_t)T.n_mos);
  L.total = o;
  return L;
}

// The state of instance g in shared memory for a persistent CTA: the CTA
// copies the instance's vectors, Jacobian slots, parameters, history and
// state word from the batch's interleaved arrays into `base` (laid out by
// resident_layout), and thread 0 makes R a one-instance view of the copy
// (instance 0, lane stride 1); resident_out writes the mutable part back.
// persist_instance on R runs the arithmetic it would run on the batch's
// arrays, on the same values, so the results are the same bit for bit; only
// the latency of the state changes. Needs a barrier before R is used.
template <typename T>
__device__ void resident_in(const DevTopo& Tp, const DevInst& I, int g, unsigned char* base,
                            DevInst& R) {
  const ResidentLayout L = resident_layout(Tp, sizeof(T));
  const int tid = threadIdx.x, bd = blockDim.x;
  const size_t ld = I.ld;
  double* v = reinterpret_cast<double*>(base + L.v);
  double* x = reinterpret_cast<double*>(base + L.x);
  double* F = reinterpret_cast<double*>(base + L.F);
  double* vtp = reinterpret_cast<double*>(base + L.vtp);
  double* vtpp = reinterpret_cast<double*>(base + L.vtpp);
  double* cvp = reinterpret_cast<double*>(base + L.cvp);
  double* cip = reinterpret_cast<double*>(base + L.cip);
  double* vsdc = reinterpret_cast<double*>(base + L.vsdc);
  double* v1 = reinterpret_cast<double*>(base + L.v1);
  double* v2 = reinterpret_cast<double*>(base + L.v2);
  double* hist = reinterpret_cast<double*>(base + L.hist);
  double* scal = reinterpret_cast<double*>(base + L.scal);
  InstState* st = reinterpret_cast<InstState*>(base + L.st);
  T* Jr = reinterpret_cast<T*>(base + L.J);
  float* kp = reinterpret_cast<float*>(base + L.kp);
  float* vth = reinterpret_cast<float*>(base + L.vth);
  const T* Jg = reinterpret_cast<const T*>(I.J);
  if (tid == 0) {
    R = I;
    R.ni = 1;
    R.ld = 1;
    R.v = v;
    R.x = x;
    R.F = F;
    R.v_tp = vtp;
    R.v_tpp = I.v_tpp ? vtpp : nullptr;
    R.ev_lte = I.ev_lte ? scal + 5 : nullptr;
    R.cap_vp = cvp;
    R.cap_ip = cip;
    R.vs_dc = vsdc;
    R.vs_v1 = v1;
    R.vs_v2 = v2;
    R.hist = hist;
    R.ev_t = scal;
    R.ev_heff = scal + 1;
    R.red_f = reinterpret_cast<unsigned long long*>(scal + 2);
    R.red_dv = reinterpret_cast<unsigned long long*>(scal + 3);
    R.red_flags = reinterpret_cast<int*>(scal + 4);
    R.st = st;
    R.J = Jr;
    R.kp = I.kp ? kp : nullptr;
    R.vth = I.vth ? vth : nullptr;
    R.seed = nullptr;
    R.live_in = nullptr;
    R.live_in_count = nullptr;
    R.live_out = nullptr;
    R.live_out_count = nullptr;
    R.hub_part = nullptr;
    R.hub_cnt = nullptr;
    R.lu_ws = I.lu_ws ? reinterpret_cast<unsigned char*>(I.lu_ws) + (size_t)g * Tp.nd_S * sizeof(T)
                      : nullptr;
    R.wave = I.wave ? I.wave + (size_t)g * I.wave_steps * I.n_wave : nullptr;
    scal[0] = I.ev_t[g];
    scal[1] = I.ev_heff[g];
    reinterpret_cast<unsigned long long*>(scal)[2] = I.red_f[g];
    reinterpret_cast<unsigned long long*>(scal)[3] = I.red_dv[g];
    *reinterpret_cast<int*>(scal + 4) = I.red_flags[g];
    scal[5] = I.ev_lte ? I.ev_lte[g] : -1.0;
    *st = I.st[g];
  }
  for (int i = tid; i < Tp.n; i += bd) {
    const size_t o = (size_t)i * ld + g;
    v[i] = I.v[o];
    x[i] = I.x[o];
    F[i] = I.F[o];
    vtp[i] = I.v_tp[o];
    if (I.v_tpp) vtpp[i] = I.v_tpp[o];
  }
  for (int c = tid; c < Tp.n_cap; c += bd) {
    cvp[c] = I.cap_vp[(size_t)c * ld + g];
    cip[c] = I.cap_ip[(size_t)c * ld + g];
  }
  for (int k = tid; k < Tp.n_vs; k += bd) {
    vsdc[k] = I.vs_dc[(size_t)k * ld + g];
    v1[k] = I.vs_v1[(size_t)k * ld + g];
    v2[k] = I.vs_v2[(size_t)k * ld + g];
  }
  for (int k = tid; k < 2 * KHIST_LEN; k += bd) hist[k] = I.hist[(size_t)k * ld + g];
  for (int k = tid; k < Tp.nv; k += bd) Jr[k] = Jg[(size_t)k * ld + g];
  for (int k = tid; k < Tp.n_mos; k += bd) {
    if (I.kp) kp[k] = I.kp[(size_t)k * ld + g];
    if (I.vth) vth[k] = I.vth[(size_t)k * ld + g];
  }
}

template <typename T>
__device__ void resident_out(const DevTopo& Tp, const DevInst& I, int g, const unsigned char* base) {
  const ResidentLayout L = resident_layout(Tp, sizeof(T));
  const int tid = threadIdx.x, bd = blockDim.x;
  const size_t ld = I.ld;
  const double* v = reinterpret_cast<const double*>(base + L.v);
  const double* x = reinterpret_cast<const double*>(base + L.x);
  const double* F = reinterpret_cast<const double*>(base + L.F);
  const double* vtp = reinterpret_cast<const double*>(base + L.vtp);
  const double* vtpp = reinterpret_cast<const double*>(base + L.vtpp);
  const double* cvp = reinterpret_cast<const double*>(base + L.cvp);
  const double* cip = reinterpret_cast<const double*>(base + L.cip);
  const double* hist = reinterpret_cast<const double*>(base + L.hist);
  const double* scal = reinterpret_cast<const double*>(base + L.scal);
  const InstState* st = reinterpret_cast<const InstState*>(base + L.st);
  const T* Jr = reinterpret_cast<const T*>(base + L.J);
  for (int i = tid; i < Tp.n; i += bd) {
    const size_t o = (size_t)i * ld + g;
    I.v[o] = v[i];
    I.x[o] = x[i];
    I.F[o] = F[i];
    I.v_tp[o] = vtp[i];
    if (I.v_tpp) I.v_tpp[o] = vtpp[i];
  }
  for (int c = tid; c < Tp.n_cap; c += bd) {
    I.cap_vp[(size_t)c * ld + g] = cvp[c];
    I.cap_ip[(size_t)c * ld + g] = cip[c];
  }
  for (int k = tid; k < 2 * KHIST_LEN; k += bd) I.hist[(size_t)k * ld + g] = hist[k];
  T* Jw = reinterpret_cast<T*>(I.J);
  for (int k = tid; k < Tp.nv; k += bd) Jw[(size_t)k * ld + g] = Jr[k];
  if (tid == 0) {
    I.ev_t[g] = scal[0];
    I.ev_heff[g] = scal[1];
    I.red_f[g] = reinterpret_cast<const unsigned long long*>(scal)[2];
    I.red_dv[g] = reinterpret_cast<const unsigned long long*>(scal)[3];
    I.red_flags[g] = *reinterpret_cast<const int*>(scal + 4);
    if (I.ev_lte) I.ev_lte[g] = scal[5];
    I.st[g] = *st;
  }
}

// One instance per CTA, all its remaining rounds in one launch (packed
// program, slots in shared memory; rescue slot blockIdx.x). Instances:
// I.live_in[0 .. *I.live_in_count) when listed, else 0 .. ni - 1.
// With resident_at > 0 the instance's state lives in shared memory from
// that byte offset on (resident_in / resident_out); either way the rounds
// read the instance's buffers through a view R in shared memory. With
// slot_values the evaluation keeps every slot term's value in shared memory
// (es_one_instance).
template <typename T>
__global__ void __launch_bounds__(kPersistThreads) k_persist(DevTopo Tp, DevInst I, JobParams P,
                                                             int max_rounds, int K, int* active,
                                                             int* rounds_max, int resident_at,
                                                             int slot_values) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PersistShared S;
  __shared__ DevInst R;
  int g = blockIdx.x;
  if (I.live_in) {
    if ((int)blockIdx.x >= *I.live_in_count) return;
    g = I.live_in[blockIdx.x];
  }
  if (g >= I.ni) return;
  if (resident_at > 0)
    resident_in<T>(Tp, I, g, smem_raw + resident_at, R);
  else if (threadIdx.x == 0)
    R = I;
  __syncthreads();
  persist_instance<T, false, true>(Tp, R, P, resident_at > 0 ? 0 : g, blockIdx.x, K, max_rounds,
                                   smem_raw, S, active, rounds_max, nullptr, nullptr, slot_values != 0);
  if (resident_at > 0) {
    __syncthreads();
    resident_out<T>(Tp, I, g, smem_raw + resident_at);
  }
}

// Several problems of different sizes in one persistent launch: CTA b runs
// instance b - cta0 of the job whose CTA range holds b (jobs sorted by cta0,
// the first at 0), with that job's factor/solve variant. The job's tables
// are copied into shared memory once; a problem's rescues share its
// workspace slots through the job's slot_lock pool. Dynamic shared memory:
// the largest job's need.
template <typename T>
__global__ void __launch_bounds__(kPersistThreads) k_persist_multi(const PersistJob* __restrict__ jobs,
                                                                   int n_jobs, int max_rounds,
                                                                   int* active, int* rounds_max,
                                                                   int* slot_timeouts) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PersistShared S;
  __shared__ __align__(16) PersistJob J;
  __shared__ DevInst R;
  const int b = blockIdx.x;
  int lo = 0, hi = n_jobs - 1;  // the last job with cta0 <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&jobs[mid].cta0) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  static_assert(sizeof(PersistJob) % 4 == 0, "job copy by words");
  const int* src = reinterpret_cast<const int*>(&jobs[lo]);
  int* dst = reinterpret_cast<int*>(&J);
  for (int e = threadIdx.x; e < (int)(sizeof(PersistJob) / 4); e += blockDim.x) dst[e] = __ldg(&src[e]);
  __syncthreads();
  const int g = b - J.cta0;
  if (g < 0 || g >= J.I.ni) return;
  const int res = J.resident_at;
  if (res > 0)
    resident_in<T>(J.T, J.I, g, smem_raw + res, R);
  else if (threadIdx.x == 0)
    R = J.I;
  __syncthreads();
  const int gl = res > 0 ? 0 : g;
  if (J.variant == 0)
    persist_instance<T, false, true>(J.T, R, J.P, gl, g, J.K, max_rounds, smem_raw, S, active,
                                     rounds_max, J.slot_lock, slot_timeouts, J.slot_values != 0);
  else if (J.variant == 1)
    persist_instance<T, false, false>(J.T, R, J.P, gl, g, J.K, max_rounds, smem_raw, S, active,
                                      rounds_max, J.slot_lock, slot_timeouts, J.slot_values != 0);
  else
    persist_instance<T, true, false>(J.T, R, J.P, gl, g, J.K, max_rounds, smem_raw, S, active,
                                     rounds_max, J.slot_lock, slot_timeouts, J.slot_values != 0);
  if (res > 0) {
    __syncthreads();
    resident_out<T>(J.T, J.I, g, smem_raw + res);
  }
}

// ---------------------------------------------------------------------------
// Small-signal AC: complex static-pivot LU on the packed level program
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_recip(double2 a) {
  const double den = a.x * a.x + a.y * a.y;
  return make_double2(a.x / den, -a.y / den);
}
__device__ __forceinline__ double c_abs(double2 a) { return hypot(a.x, a.y); }

// nd_solve_cta in complex arithmetic: the same packed program (ND slots A,
// right-hand side y in ND positions, gmin on every diagonal first), pivots
// replaced by their reciprocals, multipliers, target updates, forward and back
// substitution level by level. False when a pivot is non-finite or below
// tiny in magnitude, a solution value is non-finite, or a multiplier exceeds
// growth_limit in magnitude.
__device__ bool nd_solve_cta_c(double2* __restrict__ A, double2* __restrict__ y,
                               const int* __restrict__ prog, double gmin, double tiny,
                               double growth_limit) {
  const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bd >> 5;
  const int NL = prog[0], lvt = prog[1], tpb = prog[2], ypb = prog[3], bpb = prog[4];
  bool ok = true;
  double lmax = 0.0;
  for (int lv = 0; lv < NL; ++lv) {
    const int* Lt = prog + lvt + 12 * lv;
    for (int q = tid; q < Lt[1]; q += bd) A[prog[Lt[0] + q]].x += gmin;
  }
  __syncthreads();
  for (int lv = 0; lv < NL; ++lv) {
    const int* Lt = prog + lvt + 12 * lv;
    const int po = Lt[0], pc = Lt[1], lo = Lt[2], lc = Lt[3];
    for (int q = tid; q < pc; q += bd) {
      const int d = prog[po + q];
      const double2 piv = A[d];
      const double m = c_abs(piv);
      ok = ok && isfinite(m) && !(m < tiny);
      A[d] = c_recip(piv);
    }
    __syncthreads();
    for (int e = tid; e < lc; e += bd) {
      const int v = prog[lo + e];
      const int sl = v & 0xFFFF;
      const double2 l = c_mul(A[sl], A[(v >> 16) & 0xFFFF]);
      A[sl] = l;
      lmax = fmax(lmax, c_abs(l));
    }
    __syncthreads();
    const int to = Lt[4], tsc = Lt[5], tlc = Lt[6];
    for (int t = tid; t < tsc; t += bd) {
      const int h = prog[to + 2 * t], off = tpb + prog[to + 2 * t + 1];
      const int sl = h & 0xFFFF, c = (h >> 16) & 0xFFFF;
      double2 acc = A[sl];
      for (int q = 0; q < c; ++q) {
        const int pr = prog[off + q];
        acc = c_sub(acc, c_mul(A[pr & 0xFFFF], A[(pr >> 16) & 0xFFFF]));
      }
      A[sl] = acc;
    }
    const int yo = Lt[7], ysc = Lt[8], ylc = Lt[9];
    for (int r = tid; r < ysc; r += bd) {
      const int h = prog[yo + 2 * r], off = ypb + prog[yo + 2 * r + 1];
      const int row = h & 0xFFFF, c = (h >> 16) & 0xFFFF;
      double2 acc = y[row];
      for (int q = 0; q < c; ++q) {
        const int pr = prog[off + q];
        acc = c_sub(acc, c_mul(A[pr & 0xFFFF], y[(pr >> 16) & 0xFFFF]));
      }
      y[row] = acc;
    }
    for (int t = tsc + warp; t < tsc + tlc; t += nw) {
      const int h = prog[to + 2 * t], off = tpb + prog[to + 2 * t + 1];
      const int c = (h >> 16) & 0xFFFF;
      double2 part = make_double2(0.0, 0.0);
      for (int q = lane; q < c; q += 32) {
        const int pr = prog[off + q];
        part = c_add(part, c_mul(A[pr & 0xFFFF], A[(pr >> 16) & 0xFFFF]));
      }
      for (int o = 16; o > 0; o >>= 1) {
        part.x += __shfl_xor_sync(kFull, part.x, o);
        part.y += __shfl_xor_sync(kFull, part.y, o);
      }
      if (lane == 0) A[h & 0xFFFF] = c_sub(A[h & 0xFFFF], part);
    }
    for (int r = ysc + warp; r < ysc + ylc; r += nw) {
      const int h = prog[yo + 2 * r], off = ypb + prog[yo + 2 * r + 1];
      const int c = (h >> 16) & 0xFFFF;
      double2 part = make_double2(0.0, 0.0);
      for (int q = lane; q < c; q += 32) {
        const int pr = prog[off + q];
        part = c_add(part, c_mul(A[pr & 0xFFFF], y[(pr >> 16) & 0xFFFF]));
      }
      for (int o = 16; o > 0; o >>= 1) {
        part.x += __shfl_xor_sync(kFull, part.x, o);
        part.y += __shfl_xor_sync(kFull, part.y, o);
      }
      if (lane == 0) y[h & 0xFFFF] = c_sub(y[h & 0xFFFF], part);
    }
    __syncthreads();
  }
  bool finite = true;
  for (int lv = NL - 1; lv >= 0; --lv) {
    const int* Lt = prog + lvt + 12 * lv;
    const int bo = Lt[10], bc = Lt[11];
    for (int q = tid; q < bc; q += bd) {
      const int a = prog[bo + 2 * q], b = prog[bo + 2 * q + 1];
      const int k = a & 0xFFFF, d = (a >> 16) & 0xFFFF;
      const int c = b & 0xFFFF, off = bpb + ((b >> 16) & 0xFFFF);
      double2 sv = y[k];
      for (int j = 0; j < c; ++j) {
        const int pr = prog[off + j];
        sv = c_sub(sv, c_mul(A[pr & 0xFFFF], y[(pr >> 16) & 0xFFFF]));
      }
      sv = c_mul(sv, A[d]);
      y[k] = sv;
      finite = finite && isfinite(sv.x) && isfinite(sv.y);
    }
    __syncthreads();
  }
  return __syncthreads_and(ok && finite && !(lmax > growth_limit)) != 0;
}

// One AC point per CTA: blockIdx.x = frequency k, blockIdx.y = instance g.
// Y(j w) from the instance's FP64 Jacobian value slots at its DC point (I.J,
// lane g), plus j w C over each slot's capacitor terms (the transient
// companions' lists), the input node's excitation conductance, and gmin on
// every diagonal inside the solve. Dynamic shared memory: the right-hand side
// [nd_SY] and the ND slots [nd_S] as double2, then (stage_prog) the packed
// program.
__global__ void __launch_bounds__(256) k_ac(DevTopo Tp, DevInst I, AcParams A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int k = blockIdx.x, g = blockIdx.y, tid = threadIdx.x, bd = blockDim.x;
  if (k >= A.n_points || g >= I.ni) return;
  double2* Y = reinterpret_cast<double2*>(smem_raw);
  double2* S = Y + Tp.nd_SY;
  const int* prog = Tp.nd_prog;
  if (A.stage_prog) {
    int* dst = reinterpret_cast<int*>(S + Tp.nd_S);
    const int4* srcp = reinterpret_cast<const int4*>(Tp.nd_prog);
    for (int e = tid; e < (Tp.nd_prog_len + 3) / 4; e += bd) reinterpret_cast<int4*>(dst)[e] = __ldg(&srcp[e]);
    prog = dst;
  }
  const double w = A.omega[k];
  const size_t ld = I.ld;
  const double* J = reinterpret_cast<const double*>(I.J);
  for (int sl = tid; sl < Tp.nd_S; sl += bd) {
    double2 a = make_double2(0.0, 0.0);
    const int src = sl < Tp.nd_nv ? __ldg(&Tp.nd_src[sl]) : -1;
    if (src >= 0) {
      double c = 0.0;
      const int q1 = __ldg(&Tp.jcap_off[src + 1]);
      for (int q = __ldg(&Tp.jcap_off[src]); q < q1; ++q) {
        const int cc = __ldg(&Tp.jcap_code[q]);
        const double C = __ldg(&Tp.cap_c[code_idx(cc)]);
        c = cc < 0 ? c - C : c + C;
      }
      a.x = J[(size_t)src * ld + g] + (src == A.in_slot ? A.g_in : 0.0);
      a.y = w * c;
    }
    S[sl] = a;
  }
  for (int i = tid; i < Tp.nd_SY; i += bd) Y[i] = make_double2(0.0, 0.0);
  __syncthreads();
  if (tid == 0 && A.in_pos >= 0) Y[__ldg(&Tp.nd_pos[A.in_pos])] = make_double2(A.rhs_in, 0.0);
  __syncthreads();
  const bool ok = nd_solve_cta_c(S, Y, prog, A.gmin, A.tiny, A.growth);
  const size_t base = ((size_t)g * A.n_points + k) * (size_t)Tp.n;
  for (int i = tid; i < Tp.n; i += bd) {
    const double2 v = ok ? Y[__ldg(&Tp.nd_pos[i])] : make_double2(0.0, 0.0);
    const size_t o = base + __ldg(&A.perm[i]);
    A.out_re[o] = v.x;
    A.out_im[o] = v.y;
  }
  if (tid == 0) A.status[(size_t)g * A.n_points + k] = ok ? KST_CONVERGED : KST_SINGULAR;
}

// Moves every converged instance into the transient at step 1 (capacitor
// history from the accepted point when init_caps). Thread per instance.
__global__ void k_tran_start(DevTopo T, DevInst I, JobParams P, int init_caps) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= I.ni) return;
  InstState s = I.st[g];
  if (s.status != KST_CONVERGED) return;
  const size_t ld = I.ld;
  for (int i = 0; i < T.n; ++i) {
    const double vi = I.v[i * ld + g];
    I.x[i * ld + g] = vi;
    I.v_tp[i * ld + g] = vi;
    if (init_caps && P.lte_rel > 0.0 && I.v_tpp) I.v_tpp[i * ld + g] = vi;
  }
  if (init_caps) s.hprev = 0.0;  // a fresh transient: no previous sub-step for the LTE test
  if (init_caps)
    for (int c = 0; c < T.n_cap; ++c) {
      const int2 tt = T.cap_term[c];
      I.cap_vp[c * ld + g] = (tt.x >= 0 ? I.v[tt.x * ld + g] : 0.0) - (tt.y >= 0 ? I.v[tt.y * ld + g] : 0.0);
      I.cap_ip[c * ld + g] = 0.0;
    }
  s.mode = MODE_TRAN;
  s.sub = SUB_NR;
  s.step = 1;
  s.first = 1;
  s.it = 0;
  s.depth = 0;
  s.frac = 0;
  s.status = KST_NOCONV;
  I.st[g] = s;
  set_eval_point(I, P, g, s);
  reset_reductions(I, g);
}

// Instance-interleaved permuted voltages -> instance-major node order.
__global__ void k_unpermute(const double* vp, const int* perm, double* out, int ni, int ld, int n) {
  const size_t total = (size_t)n * ld;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int p = (int)(e / ld);
    const int g = (int)(e - (size_t)p * ld);
    if (g < ni) out[(size_t)g * n + perm[p]] = vp[e];
  }
}

// The same for FP32 per-device parameters: [ni][n] in netlist order into
// [n][ld] in SoA order (item p takes netlist item order[p]).
__global__ void k_interleave_f(const float* src, const int* order, float* dst, int ni, int ld, int n) {
  const size_t total = (size_t)n * ld;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int p = (int)(e / ld);
    const int g = (int)(e - (size_t)p * ld);
    dst[e] = g < ni ? src[(size_t)g * n + order[p]] : 0.0f;
  }
}

// Interleaves an instance-major [ni][n] host-order block into [n][ld] permuted.
__global__ void k_interleave(const double* src, const int* perm, double* dst, int ni, int ld, int n) {
  const size_t total = (size_t)n * ld;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int p = (int)(e / ld);
    const int g = (int)(e - (size_t)p * ld);
    dst[e] = g < ni ? src[(size_t)g * n + perm[p]] : 0.0;
  }
}

}  // namespace knr
#endif
