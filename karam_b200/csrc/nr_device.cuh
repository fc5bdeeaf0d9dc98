// nr_device.cuh -- device code of the batched Newton-Raphson inner loop.
//
// One NR "round" = k_eval (device evaluation + stamping at the point x of every
// live instance) followed by an LU round (per-instance control flow, assembly,
// static pivot LU on the filled pattern, triangular solves, junction limiting)
// and, for the rare solves whose static pivots fail, k_rescue (dense partial
// pivoting). The control flow reproduces CircuitSim::solveDC's GMIN / damping /
// pnjlim / convergence logic (solvers/circuitsim_solver.cpp:237-485) and the
// transient NR loop with its attempt loop (circuitsim_solver.cpp:587-660) as a
// per-instance state machine, one decision per round.
//
// This text is compiled twice: by nvcc into the library (with the program
// interpreter InterpFS), and at run time by NVRTC together with a factor-solve
// policy generated for one topology (KARAM_JIT defined), so it includes no
// standard headers.
#ifndef KARAM_NR_DEVICE_CUH
#define KARAM_NR_DEVICE_CUH
#if !defined(__CUDACC_RTC__)
#include "nr_types.h"
#endif

namespace knr {


constexpr int kEvalThreads = 256;
constexpr int kLuThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

enum Act : int {
  ACT_SOLVE = 1,
  ACT_DAMP = 2,
  ACT_ACCEPT = 4,
  ACT_TRAN_INIT = 8,
  ACT_STEP = 16,
  ACT_LIMIT = 32,  // sanitize + pnjlim after the solve (DC NR iterations)
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

__device__ __forceinline__ double source_value(const DevTopo& T, const DevInst& I, int inst,
                                               int s, bool tran, double t) {
  const size_t k = (size_t)inst * T.n_vs + s;
  if (!tran || T.vs_kind[s] != KSRC_PULSE) return I.vs_dc[k];
  return pulse_at(T.vs_pulse + 7 * s, I.vs_v1[k], I.vs_v2[k], t);
}

// seedInitialGuess (circuitsim_solver.cpp:32-116) in the permuted space;
// single thread.
__device__ void reference_seed(const DevTopo& T, const DevInst& I, int inst, double* v) {
  for (int i = 0; i < T.n; ++i) v[i] = 0.0;
  double vsup = 5.0;
  for (int s = 0; s < T.n_vs; ++s) {
    const double val = I.vs_dc[(size_t)inst * T.n_vs + s];
    const int p = T.seed_vs[s];
    if (p >= 0) v[p] = val;
    if (val > vsup) vsup = val;
  }
  for (int d = 0; d < T.n_seed_anode; ++d) {
    const int p = T.seed_anode[d];
    if (p >= 0) v[p] = fmax(v[p], 0.6);
  }
  for (int s = 0; s < T.n_is; ++s) {
    const int p = T.is_term[s].x;
    if (p >= 0 && v[p] == 0.0) v[p] = vsup * 0.5;
  }
}

// ---------------------------------------------------------------------------
// init: seed, state
// ---------------------------------------------------------------------------
#if !defined(KARAM_JIT)
__global__ void k_init(DevTopo T, DevInst I, JobParams P) {
  const int inst = blockIdx.x;
  if (inst >= I.ni) return;
  double* v = I.v + (size_t)inst * T.n;
  double* x = I.x + (size_t)inst * T.n;
  const bool seeded = P.seeded && I.seed != nullptr;
  if (seeded) {
    for (int i = threadIdx.x; i < T.n; i += blockDim.x) v[i] = I.seed[(size_t)inst * T.n + i];
  } else if (threadIdx.x == 0) {
    reference_seed(T, I, inst, v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) x[i] = v[i];
  if (threadIdx.x == 0) {
    if (I.counters) atomicAdd(&I.counters[0], 1ull);
    InstState s = {};
    s.mode = MODE_DC;
    s.sub = SUB_NR;
    s.g = seeded ? P.gmin_steps - 1 : 0;
    s.first = 1;
    s.status = KST_NOCONV;
    s.seeded = seeded ? 1 : 0;
    s.prevF = 0.0;
    s.prev_dv = -1.0;
    I.st[inst] = s;
  }
}
#endif  // !KARAM_JIT

// ---------------------------------------------------------------------------
// evaluation + stamping
// ---------------------------------------------------------------------------
constexpr int kMaxEvalInst = 8;

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

#if !defined(KARAM_JIT)
// One CTA evaluates up to NE instances: every gather-table load (device
// terminals, stamp codes) is made once and applied to all of them, so the
// index latency is amortised and the per-instance accumulations run side by
// side. Shared memory per instance: x (n), MOSFET gm/gds/ids, diode g/i.
// Summation order per Jacobian entry is the stamp order (bit-exact FP64).
template <typename TJ>
__global__ void __launch_bounds__(kEvalThreads) k_eval(DevTopo T, DevInst I, JobParams P, int NE) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && I.rescue_count) *I.rescue_count = 0;
  extern __shared__ double sm[];
  __shared__ int s_inst[kMaxEvalInst], s_tran[kMaxEvalInst];
  __shared__ double s_t[kMaxEvalInst], s_heff[kMaxEvalInst];
  __shared__ double red[kEvalThreads / 32][kMaxEvalInst];
  __shared__ int s_cnt;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int cnt = 0;
    const int units = 1 << P.max_halvings;
    for (int k = 0; k < NE; ++k) {
      const int inst = blockIdx.x * NE + k;
      if (inst >= I.ni) break;
      const InstState st = I.st[inst];
      if (st.mode == MODE_DONE) continue;
      const bool tran = st.mode == MODE_TRAN;
      // transient sub-step: size h / 2^depth ending at
      // ((step - 1) * units + frac + size) * h / units
      const int size = units >> st.depth;
      const double hsub = P.h * size / units;
      s_inst[cnt] = inst;
      s_tran[cnt] = tran;
      s_t[cnt] = tran ? P.t0 + (double)((st.step - 1) * units + st.frac + size) * (P.h / units) : 0.0;
      s_heff[cnt] = P.method == KTRAN_TRAP ? hsub : 2.0 * hsub;
      cnt++;
    }
    s_cnt = cnt;
  }
  __syncthreads();
  const int ne = s_cnt;
  if (ne == 0) return;
  const int n = T.n, nm = T.n_mos, nd = T.n_dio;
  const int per = n + 3 * nm + 2 * nd;
  auto xs = [&](int k) { return sm + (size_t)k * per; };
  for (int e = tid; e < ne * n; e += blockDim.x) {
    const int k = e / n, i = e - k * n;
    xs(k)[i] = I.x[(size_t)s_inst[k] * n + i];
  }
  __syncthreads();

  for (int m = tid; m < nm; m += blockDim.x) {
    const int4 tm = T.mos_term[m];
    const double2 geo = T.mos_geo[m];
    const double2 card = T.mos_card[m];
    const double sign = T.mos_pmos[m] ? -1.0 : 1.0;
#pragma unroll
    for (int k = 0; k < kMaxEvalInst; ++k) {
      if (k >= ne) break;
      const double* x = xs(k);
      const size_t pi = (size_t)s_inst[k] * nm + m;
      const double kpm = I.kp ? (double)I.kp[pi] : card.x;
      const double vthm = I.vth ? (double)I.vth[pi] : card.y;
      double ids, gm, gds;
      mosfet_eval(tm.x >= 0 ? x[tm.x] : 0.0, tm.y >= 0 ? x[tm.y] : 0.0, tm.z >= 0 ? x[tm.z] : 0.0,
                  sign, kpm, vthm, geo.x, geo.y, ids, gm, gds);
      double* dv = xs(k) + n;
      dv[m] = gm;
      dv[nm + m] = gds;
      dv[2 * nm + m] = ids;
    }
  }
  for (int d = tid; d < nd; d += blockDim.x) {
    const int2 tt = T.dio_term[d];
    const double4 par = T.dio_par[d];
#pragma unroll
    for (int k = 0; k < kMaxEvalInst; ++k) {
      if (k >= ne) break;
      const double* x = xs(k);
      double id, gd;
      diode_eval((tt.x >= 0 ? x[tt.x] : 0.0) - (tt.y >= 0 ? x[tt.y] : 0.0), par, id, gd);
      double* dv = xs(k) + n + 3 * nm;
      dv[d] = gd;
      dv[nd + d] = id;
    }
  }
  __syncthreads();

  // Jacobian at x: linear part + gathered device terms, in stamp order.
  for (int f = tid; f < T.nf; f += blockDim.x) {
    double acc[kMaxEvalInst];
    const double base = T.jlin_dc[f];
#pragma unroll
    for (int k = 0; k < kMaxEvalInst; ++k) acc[k] = base;
    for (int q = T.jcap_off[f]; q < T.jcap_off[f + 1]; ++q) {
      const int c = T.jcap_code[q];
      const double cc = 2.0 * T.cap_c[code_idx(c)];
#pragma unroll
      for (int k = 0; k < kMaxEvalInst; ++k) {
        if (k >= ne || !s_tran[k]) continue;
        const double g = cc / s_heff[k];
        acc[k] = c < 0 ? acc[k] - g : acc[k] + g;
      }
    }
    for (int q = T.jt_off[f]; q < T.jt_off[f + 1]; ++q) {
      const int c = T.jt_code[q];
      const int idx = code_idx(c), kind = code_kind(c);
      const int off = kind == 0 ? n + nm + idx : (kind == 1 ? n + idx : n + 3 * nm + idx);
#pragma unroll
      for (int k = 0; k < kMaxEvalInst; ++k) {
        if (k >= ne) break;
        const double val = xs(k)[off];
        acc[k] = c < 0 ? acc[k] - val : acc[k] + val;
      }
    }
#pragma unroll
    for (int k = 0; k < kMaxEvalInst; ++k) {
      if (k >= ne) break;
      reinterpret_cast<TJ*>(I.J)[(size_t)s_inst[k] * T.nf + f] = (TJ)acc[k];
    }
  }

  // KCL residual at x: currents leaving every node (no gmin).
  double lmax[kMaxEvalInst];
  bool bad = false;
#pragma unroll
  for (int k = 0; k < kMaxEvalInst; ++k) lmax[k] = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    double acc[kMaxEvalInst];
#pragma unroll
    for (int k = 0; k < kMaxEvalInst; ++k) acc[k] = 0.0;
    for (int q = T.ft_off[i]; q < T.ft_off[i + 1]; ++q) {
      const int c = T.ft_code[q];
      const int idx = code_idx(c), kind = code_kind(c);
      int2 tt = make_int2(-1, -1);
      double g = 0.0;
      if (kind == 0) {
        tt = T.res_term[idx];
        g = T.res_g[idx];
      } else if (kind == 1) {
        tt = T.vs_term[idx];
      } else if (kind == 3) {
        tt = T.cap_term[idx];
        g = 2.0 * T.cap_c[idx];
      }
#pragma unroll
      for (int k = 0; k < kMaxEvalInst; ++k) {
        if (k >= ne) break;
        const double* x = xs(k);
        const double va = tt.x >= 0 ? x[tt.x] : 0.0, vb = tt.y >= 0 ? x[tt.y] : 0.0;
        double cur = 0.0;
        switch (kind) {
          case 0:  // resistor
            cur = g * (va - vb);
            break;
          case 1:  // Norton voltage source, G = 1e3 S
            cur = 1.0e3 * ((va - vb) - source_value(T, I, s_inst[k], idx, s_tran[k], s_t[k]));
            break;
          case 2:
            cur = T.is_amp[idx];
            break;
          case 3:  // capacitor companion
            if (s_tran[k]) {
              const size_t ci = (size_t)s_inst[k] * T.n_cap + idx;
              cur = (g / s_heff[k]) * ((va - vb) - I.cap_vp[ci]);
              if (P.method == KTRAN_TRAP) cur -= I.cap_ip[ci];
            }
            break;
          case 4:
            cur = x[n + 3 * nm + nd + idx];
            break;
          default:
            cur = x[n + 2 * nm + idx];
            break;
        }
        acc[k] = c < 0 ? acc[k] - cur : acc[k] + cur;
      }
    }
#pragma unroll
    for (int k = 0; k < kMaxEvalInst; ++k) {
      if (k >= ne) break;
      I.F[(size_t)s_inst[k] * n + i] = acc[k];
      if (!isfinite(acc[k])) bad = true;
      lmax[k] = fmax(lmax[k], fabs(acc[k]));
    }
  }
  bad = __any_sync(kFull, bad);
#pragma unroll
  for (int k = 0; k < kMaxEvalInst; ++k) {
    double m = lmax[k];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(kFull, m, o));
    if ((tid & 31) == 0) red[tid >> 5][k] = bad ? __longlong_as_double(0x7ff0000000000000LL) : m;
  }
  __syncthreads();
  if (tid < ne) {
    double m = 0.0;
    bool nf = false;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      if (isinf(red[w][tid])) nf = true;
      m = fmax(m, red[w][tid]);
    }
    I.Fmax[s_inst[tid]] = nf ? __longlong_as_double(0x7ff8000000000000LL) : m;
  }
}
#endif  // !KARAM_JIT

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

__device__ int start_polish(InstState& s, double& gmin_out) {
  s.sub = SUB_POLISH;
  s.pol_cnt = 0;
  s.prev_dv = -1.0;
  gmin_out = 1e-12;
  return ACT_SOLVE;
}

// One decision of the NR control flow for the trial point x whose KCL
// residual is F (vconv / pok / dv compare x against the accepted point v).
__device__ int decide(InstState& s, double F, bool vconv, bool pok, double dv,
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
      return ACT_ACCEPT | step_done(s, P, hsub);
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
  if (pok || dv == 0.0 || stalled || s.pol_cnt >= P.polish_max)
    return ACT_ACCEPT | step_done(s, P, hsub);
  s.prev_dv = dv;
  gmin_out = 1e-12;
  return ACT_ACCEPT | ACT_SOLVE;
}

// applyPnJunctionLimits (circuitsim_solver.cpp:118-169) for diode d on x
// against v. The temperature-scaled Vt and vcrit (pnjlim's compute_vcrit,
// physics/device_physics.h:175-179) are per-diode constants the host computes
// with the reference's expressions once per topology.
__device__ __forceinline__ void limit_one(const DevTopo& T, int d, double* x, const double* v) {
  const int2 tt = T.dio_term[d];
  const int p = tt.x, q = tt.y;
  if (p < 0 && q < 0) return;
  const double2 lim = T.dio_lim[d];
  const double vt = lim.x, vcrit = lim.y;
  const double vjo = (p >= 0 ? v[p] : 0.0) - (q >= 0 ? v[q] : 0.0);
  const double vjn = (p >= 0 ? x[p] : 0.0) - (q >= 0 ? x[q] : 0.0);
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
      x[p] -= corr * 0.5;
      x[q] += corr * 0.5;
    } else if (p >= 0) {
      x[p] -= corr;
    } else {
      x[q] += corr;
    }
  }
}

// The reference limits diodes one after another; diodes of one level share
// no node with each other, and every earlier diode sharing a node has a lower
// level, so level-by-level parallel limiting gives the sequential result.
__device__ void limit_junctions_warp(const DevTopo& T, double* x, const double* v, int lane) {
  for (int lvl = 0; lvl < T.n_dio_levels; ++lvl) {
    for (int d = lane; d < T.n_dio; d += 32)
      if (T.dio_level[d] == lvl) limit_one(T, d, x, v);
    __syncwarp();
  }
}

__device__ void limit_junctions(const DevTopo& T, double* x, const double* v) {
  for (int d = 0; d < T.n_dio; ++d) limit_one(T, d, x, v);
}

// Static-pivot LU + forward/back substitution, one instance per thread, on
// the numerically non-zero part of the filled pattern. A: the instance's value
// row (gmin already on the diagonal); y: right-hand side in, solution out.
// Pivot k of the program lists Lrow/Lpos (rows i > k with A[i][k] != 0 and
// their positions), Ucol/Upos (columns j > k of row k) and the update targets
// A[i][j] for every (i, j) pair. Returns false when the static pivots are
// unusable: a tiny or non-finite pivot, a multiplier above growth_limit (the
// elimination order amplifies rounding, e.g. a supply hub eliminated after a
// chain of high-gain stages), or a non-finite solution; such solves are redone
// with partial pivoting. InterpFS reads the program from memory; a policy
// generated per topology replaces it with straight-line code.
struct InterpFS {
  template <typename T>
  __device__ static bool run(T* __restrict__ A, T* __restrict__ y, const DevTopo& Tp, T tiny,
                             T growth_limit) {
    const int4* __restrict__ hdr = Tp.lu_hdr;
    const int* __restrict__ data = Tp.lu_data;
    const int n = Tp.n;
    bool ok = true;
    T lmax = T(0);
    for (int k = 0; k < n; ++k) {
      const int4 h = __ldg(hdr + k);
      const int nl = h.y, nu = h.z;
      const int* lp = data + h.x + nl;
      const int* up = lp + nl + nu;
      const int* tp = up + nu;
      const T piv = A[h.w];
      ok = ok && isfinite(piv) && !(fabs(piv) < tiny);
      const T r = T(1) / piv;
      A[h.w] = r;
      for (int a = 0; a < nl; ++a) {
        const int la = __ldg(lp + a);
        const T l = A[la] * r;
        lmax = fmax(lmax, fabs(l));
        A[la] = l;
        const int* trow = tp + a * nu;
        for (int b2 = 0; b2 < nu; ++b2) A[__ldg(trow + b2)] -= l * A[__ldg(up + b2)];
      }
    }
    for (int k = 0; k < n; ++k) {
      const int4 h = __ldg(hdr + k);
      const int nl = h.y;
      const int* lr = data + h.x;
      const int* lp = lr + nl;
      const T yk = y[k];
      for (int a = 0; a < nl; ++a) y[__ldg(lr + a)] -= A[__ldg(lp + a)] * yk;
    }
    bool finite = true;
    for (int k = n - 1; k >= 0; --k) {
      const int4 h = __ldg(hdr + k);
      const int nl = h.y, nu = h.z;
      const int* uc = data + h.x + 2 * nl;
      const int* up = uc + nu;
      T s = y[k];
      for (int b2 = 0; b2 < nu; ++b2) s -= A[__ldg(up + b2)] * y[__ldg(uc + b2)];
      y[k] = s * A[h.w];
      finite = finite && isfinite(y[k]);
    }
    return ok && finite && !(lmax > growth_limit);
  }
};

// What the control flow does when a linear solve of a DC NR iteration fails
// for good (the reference's singular-matrix branch, circuitsim_solver.cpp:358-366):
// a seeded start falls back to the reference seed, anything else stops.
__device__ void on_singular(const DevTopo& Tp, const DevInst& I, int inst) {
  InstState s = I.st[inst];
  if (s.mode == MODE_DC && s.sub == SUB_NR) s.iters += 2 * (s.it + 1);
  if (s.mode == MODE_DC && s.sub == SUB_NR && s.seeded) {
    double* v = I.v + (size_t)inst * Tp.n;
    double* x = I.x + (size_t)inst * Tp.n;
    reference_seed(Tp, I, inst, v);
    for (int i = 0; i < Tp.n; ++i) x[i] = v[i];
    s.g = 0;
    s.it = 0;
    s.first = 1;
    s.damp = 0;
    s.prevF = 0.0;
    s.seeded = 0;
  } else {
    s.status = KST_SINGULAR;
    s.mode = MODE_DONE;
  }
  I.st[inst] = s;
}

// One round of the control flow + linear solve for NI instances (one CTA).
template <typename T, typename FS>
__device__ __forceinline__ void lu_round(const DevTopo& Tp, const DevInst& I, const JobParams& P,
                                         int NI, int S, int Sv, int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* vals = reinterpret_cast<T*>(smem_raw);
  T* vec = vals + (size_t)NI * S;
  __shared__ int act[32];
  __shared__ int vconv_s[32], pok_s[32], sing_s[32], solve_list[32];
  __shared__ double dv_s[32], gmin_s[32], hsub_s[32];
  __shared__ int n_solve;

  const int n = Tp.n, nf = Tp.nf;
  const int base = blockIdx.x * NI;
  const int cnt = min(NI, I.ni - base);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (cnt <= 0) return;

  // 1. compare the trial point x with the accepted point v (warp per instance)
  for (int k = warp; k < cnt; k += nw) {
    const int inst = base + k;
    bool vc = true, pk = true;
    double dvm = 0.0;
    if (I.st[inst].mode != MODE_DONE) {
      const double* x = I.x + (size_t)inst * n;
      const double* v = I.v + (size_t)inst * n;
      for (int i = lane; i < n; i += 32) {
        const double xi = x[i], vi = v[i];
        const double d = fabs(xi - vi), m = fmax(fabs(xi), fabs(vi));
        if (d > P.reltol * m + P.vntol) vc = false;
        if (d > P.polish_rel * m + P.polish_abs) pk = false;
        dvm = fmax(dvm, d);
      }
      vc = __all_sync(kFull, vc);
      pk = __all_sync(kFull, pk);
      for (int o = 16; o > 0; o >>= 1) dvm = fmax(dvm, __shfl_xor_sync(kFull, dvm, o));
    }
    if (lane == 0) {
      vconv_s[k] = vc;
      pok_s[k] = pk;
      dv_s[k] = dvm;
    }
  }
  __syncthreads();

  // 2. decisions (thread per instance)
  if (tid < 32) {
    int a = 0;
    if (tid < cnt) {
      const int inst = base + tid;
      InstState s = I.st[inst];
      double gm = 1e-12, hs = P.h;
      a = decide(s, I.Fmax[inst], vconv_s[tid], pok_s[tid], dv_s[tid], P, gm, hs);
      hsub_s[tid] = hs;
      if (a & ACT_RESEED) {
        s.g = 0;
        s.it = 0;
        s.first = 1;
        s.damp = 0;
        s.prevF = 0.0;
        s.seeded = 0;
      }
      gmin_s[tid] = gm;
      I.st[inst] = s;
    }
    act[tid] = a;
    sing_s[tid] = 0;
    const unsigned m = __ballot_sync(kFull, a & ACT_SOLVE);
    if (a & ACT_SOLVE) solve_list[__popc(m & ((1u << tid) - 1u))] = tid;
    if (tid == 0) n_solve = __popc(m);
  }
  __syncthreads();

  // 3. vector updates (warp per instance)
  for (int k = warp; k < cnt; k += nw) {
    const int a = act[k];
    if (!(a & (ACT_DAMP | ACT_ACCEPT | ACT_TRAN_INIT | ACT_STEP | ACT_RESEED | ACT_RESTART)))
      continue;
    const int inst = base + k;
    double* x = I.x + (size_t)inst * n;
    double* v = I.v + (size_t)inst * n;
    if (a & ACT_RESEED) {
      if (lane == 0) reference_seed(Tp, I, inst, v);
      __syncwarp();
      for (int i = lane; i < n; i += 32) x[i] = v[i];
      continue;
    }
    if (a & ACT_RESTART) {
      const double* vtp = I.v_tp + (size_t)inst * n;
      for (int i = lane; i < n; i += 32) {
        v[i] = vtp[i];
        x[i] = vtp[i];
      }
      continue;
    }
    if (a & ACT_DAMP)
      for (int i = lane; i < n; i += 32) x[i] = v[i] + 0.5 * (x[i] - v[i]);
    if (a & ACT_ACCEPT)
      for (int i = lane; i < n; i += 32) v[i] = x[i];
    __syncwarp();
    if (a & (ACT_STEP | ACT_TRAN_INIT)) {
      double* vtp = I.v_tp + (size_t)inst * n;
      for (int i = lane; i < n; i += 32) vtp[i] = v[i];
    }
    if ((a & ACT_WAVE) && I.n_wave > 0) {
      const int done_step = I.st[inst].step - 1;  // 1-based step just completed
      if (done_step >= 1 && done_step <= I.wave_steps)
        for (int w = lane; w < I.n_wave; w += 32) {
          const int q = I.wave_pos[w];
          I.wave[((size_t)inst * I.wave_steps + (done_step - 1)) * I.n_wave + w] = q >= 0 ? v[q] : 0.0;
        }
    }
    if (a & (ACT_TRAN_INIT | ACT_STEP)) {
      for (int c = lane; c < Tp.n_cap; c += 32) {
        const int2 tt = Tp.cap_term[c];
        const double vc = (tt.x >= 0 ? v[tt.x] : 0.0) - (tt.y >= 0 ? v[tt.y] : 0.0);
        const size_t ci = (size_t)inst * Tp.n_cap + c;
        if (a & ACT_TRAN_INIT) {
          I.cap_vp[ci] = vc;
          I.cap_ip[ci] = 0.0;
        } else {
          const double C = Tp.cap_c[c];
          const double h = hsub_s[k];
          const double ic = P.method == KTRAN_TRAP
                                ? (2.0 * C / h) * (vc - I.cap_vp[ci]) - I.cap_ip[ci]
                                : (C / h) * (vc - I.cap_vp[ci]);
          I.cap_vp[ci] = vc;
          I.cap_ip[ci] = ic;
        }
      }
    }
  }
  __syncthreads();

  // 4. assembly of the instances that solve this round
  const int ns = n_solve;
  if (ns > 0) {
    const T* Jall = reinterpret_cast<const T*>(I.J);
    for (int e = tid; e < ns * nf; e += blockDim.x) {
      const int j = e / nf, f = e - j * nf;
      const int k = solve_list[j];
      vals[(size_t)k * S + f] = Jall[(size_t)(base + k) * nf + f];
    }
    for (int e = tid; e < ns * n; e += blockDim.x) {
      const int j = e / n, i = e - j * n;
      const int k = solve_list[j];
      const size_t o = (size_t)(base + k) * n + i;
      vec[(size_t)k * Sv + i] = (T)(-(I.F[o] + gmin_s[k] * I.v[o]));
    }
    __syncthreads();
    for (int e = tid; e < ns * n; e += blockDim.x) {
      const int j = e / n, i = e - j * n;
      const int k = solve_list[j];
      vals[(size_t)k * S + __ldg(&Tp.lu_hdr[i].w)] += (T)gmin_s[k];
    }
    __syncthreads();

    // 5. factor + solve: one instance per lane of warp 0
    if (warp == 0 && lane < cnt && (act[lane] & ACT_SOLVE)) {
      const T tiny = sizeof(T) == 8 ? (T)1e-25 : (T)1e-30;
      const T growth = sizeof(T) == 8 ? (T)1e10 : (T)1e4;
      const bool ok = FS::template run<T>(vals + (size_t)lane * S, vec + (size_t)lane * Sv, Tp,
                                          tiny, growth);
      sing_s[lane] = ok ? 0 : 1;
    }
    __syncthreads();

    // 6. x = v + dx
    for (int k = warp; k < cnt; k += nw) {
      const int a = act[k];
      if (!(a & ACT_SOLVE) || sing_s[k]) continue;
      const int inst = base + k;
      double* x = I.x + (size_t)inst * n;
      const double* v = I.v + (size_t)inst * n;
      const T* dx = vec + (size_t)k * Sv;
      const bool sanitize = (a & ACT_LIMIT) != 0;
      for (int i = lane; i < n; i += 32) {
        double xi = v[i] + (double)dx[i];
        if (sanitize && !isfinite(xi)) xi = 0.0;  // SafeUtils::sanitize_vector
        x[i] = xi;
      }
      __syncwarp();
      if (sanitize && Tp.n_dio > 0) limit_junctions_warp(Tp, x, v, lane);
    }
    __syncthreads();
  }

  // 7. singular pivots, junction limiting, bookkeeping (thread per instance)
  if (tid < 32) {
    int live = 0;
    if (tid < cnt) {
      const int inst = base + tid;
      const int a = act[tid];
      if ((a & ACT_SOLVE) && sing_s[tid]) {
        // static pivots unusable: hand the solve to the partial-pivoting rescue
        if (I.rescue_list) {
          const int slot = atomicAdd(I.rescue_count, 1);
          RescueItem it;
          it.inst = inst;
          it.act = a;
          it.gmin = gmin_s[tid];
          I.rescue_list[slot] = it;
        } else {
          on_singular(Tp, I, inst);
        }
      }
      const int md = I.st[inst].mode;
      live = (md != MODE_DONE) ? (md == MODE_TRAN ? 2 : 1) : 0;
    }
    const unsigned m = __ballot_sync(kFull, live != 0);
    const unsigned mt = __ballot_sync(kFull, live == 2);
    const unsigned ms = __ballot_sync(kFull, tid < cnt && (act[tid] & ACT_SOLVE) && !sing_s[tid]);
    if (tid == 0) {
      if (m) atomicAdd(active, __popc(m));
      if (I.counters) {
        // instances alive now are evaluated by the next round
        if (m & ~mt) atomicAdd(&I.counters[0], (unsigned long long)__popc(m & ~mt));
        if (mt) atomicAdd(&I.counters[1], (unsigned long long)__popc(mt));
        if (ms) atomicAdd(&I.counters[2], (unsigned long long)__popc(ms));
      }
    }
  }
}

// Dense FP64 LU with partial pivoting for the flagged instances: the
// semantics of solveSparse_LU's numeric phase (math/sparse_lu.cpp:216-312) on
// the permuted system: pivot = largest |a| in the column (ties to the lower
// row), singular below 1e-25, rows with |a| < 1e-30 skipped. One CTA per
// solve, matrix in a global workspace slot, right-hand side in shared memory.
#if !defined(KARAM_JIT)
template <typename TJ>
__global__ void __launch_bounds__(256) k_rescue(DevTopo Tp, DevInst I, JobParams P) {
  extern __shared__ double rs[];
  const int n = Tp.n, nf = Tp.nf;
  double* b = rs;                                  // n
  double* lval = b + n;                            // n
  int* rows = reinterpret_cast<int*>(lval + n);    // n
  __shared__ double red_v[8];
  __shared__ int red_r[8];
  __shared__ int s_piv, s_cnt, s_sing;
  __shared__ double s_aii;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int total = *I.rescue_count;
  double* A = I.rescue_ws + (size_t)blockIdx.x * n * n;
  for (int e = blockIdx.x; e < total; e += gridDim.x) {
    const RescueItem item = I.rescue_list[e];
    const int inst = item.inst;
    const double gmin = item.gmin;
    const TJ* J = reinterpret_cast<const TJ*>(I.J) + (size_t)inst * nf;
    for (size_t q = tid; q < (size_t)n * n; q += blockDim.x) A[q] = 0.0;
    __syncthreads();
    for (int f = tid; f < nf; f += blockDim.x)
      A[(size_t)Tp.f_row[f] * n + Tp.f_colp[f]] = (double)J[f];
    for (int i = tid; i < n; i += blockDim.x) {
      const size_t o = (size_t)inst * n + i;
      b[i] = -(I.F[o] + gmin * I.v[o]);
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) A[(size_t)i * n + i] += gmin;
    if (tid == 0) s_sing = 0;
    __syncthreads();

    for (int i = 0; i < n; ++i) {
      // pivot search + rows to eliminate
      if (tid == 0) s_cnt = 0;
      __syncthreads();
      double best = -1.0;
      int brow = n;
      for (int r = i + tid; r < n; r += blockDim.x) {
        const double a = fabs(A[(size_t)r * n + i]);
        if (a > best || (a == best && r < brow)) {
          best = a;
          brow = r;
        }
        if (r > i && a >= 1e-30) rows[atomicAdd(&s_cnt, 1)] = r;
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int orow = __shfl_xor_sync(kFull, brow, o);
        if (ob > best || (ob == best && orow < brow)) {
          best = ob;
          brow = orow;
        }
      }
      if (lane == 0) {
        red_v[warp] = best;
        red_r[warp] = brow;
      }
      __syncthreads();
      if (tid == 0) {
        double bv = red_v[0];
        int br = red_r[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
          if (red_v[w] > bv || (red_v[w] == bv && red_r[w] < br)) {
            bv = red_v[w];
            br = red_r[w];
          }
        if (bv < 1e-25) s_sing = 1;
        s_piv = br;
        s_aii = fabs(A[(size_t)i * n + i]);
      }
      __syncthreads();
      if (s_sing) break;
      const int p = s_piv;
      if (p != i) {
        for (int c = tid; c < n; c += blockDim.x) {
          const double t = A[(size_t)i * n + c];
          A[(size_t)i * n + c] = A[(size_t)p * n + c];
          A[(size_t)p * n + c] = t;
        }
        if (tid == 0) {
          const double t = b[i];
          b[i] = b[p];
          b[p] = t;
          // row p now holds the old row i: it stays in the list only if its
          // entry in column i is not negligible
          if (!(s_aii >= 1e-30))
            for (int q = 0; q < s_cnt; ++q)
              if (rows[q] == p) {
                rows[q] = rows[s_cnt - 1];
                s_cnt--;
                break;
              }
        }
      }
      __syncthreads();
      const int m = s_cnt;
      const double piv = A[(size_t)i * n + i];
      for (int q = tid; q < m; q += blockDim.x) {
        const int r = rows[q];
        const double l = A[(size_t)r * n + i] / piv;
        A[(size_t)r * n + i] = l;
        lval[q] = l;
      }
      __syncthreads();
      const int w = n - i - 1;
      for (int e2 = tid; e2 < m * w; e2 += blockDim.x) {
        const int q = e2 / w, c = i + 1 + (e2 - q * w);
        A[(size_t)rows[q] * n + c] -= lval[q] * A[(size_t)i * n + c];
      }
      __syncthreads();
    }
    if (!s_sing) {
      for (int j = 0; j < n; ++j) {  // forward substitution, unit lower
        const double bj = b[j];
        for (int r = j + 1 + tid; r < n; r += blockDim.x) b[r] -= A[(size_t)r * n + j] * bj;
        __syncthreads();
      }
      for (int j = n - 1; j >= 0; --j) {  // back substitution
        if (tid == 0) b[j] /= A[(size_t)j * n + j];
        __syncthreads();
        const double xj = b[j];
        for (int r = tid; r < j; r += blockDim.x) b[r] -= A[(size_t)r * n + j] * xj;
        __syncthreads();
      }
      double* x = I.x + (size_t)inst * n;
      const double* v = I.v + (size_t)inst * n;
      const bool sanitize = (item.act & ACT_LIMIT) != 0;
      for (int i = tid; i < n; i += blockDim.x) {
        double xi = v[i] + b[i];
        if (sanitize && !isfinite(xi)) xi = 0.0;
        x[i] = xi;
      }
      __syncthreads();
      if (tid == 0) {
        if (sanitize && Tp.n_dio > 0) limit_junctions(Tp, x, v);
        I.st[inst].rescued += 1;
        if (I.counters) atomicAdd(&I.counters[3], 1ull);
      }
    } else if (tid == 0) {
      on_singular(Tp, I, inst);
    }
    __syncthreads();
  }
}
#endif  // !KARAM_JIT

#if !defined(KARAM_JIT)
__global__ void k_tran_start(DevTopo T, DevInst I, int init_caps) {
  const int inst = blockIdx.x;
  if (inst >= I.ni) return;
  InstState s = I.st[inst];
  if (s.status != KST_CONVERGED) return;
  __syncthreads();
  const double* v = I.v + (size_t)inst * T.n;
  double* x = I.x + (size_t)inst * T.n;
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) x[i] = v[i];
  if (init_caps)
    for (int c = threadIdx.x; c < T.n_cap; c += blockDim.x) {
      const int2 tt = T.cap_term[c];
      const size_t ci = (size_t)inst * T.n_cap + c;
      I.cap_vp[ci] = (tt.x >= 0 ? v[tt.x] : 0.0) - (tt.y >= 0 ? v[tt.y] : 0.0);
      I.cap_ip[ci] = 0.0;
    }
  double* vtp = I.v_tp + (size_t)inst * T.n;
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) vtp[i] = v[i];
  if (threadIdx.x == 0) {
    if (I.counters) atomicAdd(&I.counters[1], 1ull);
    s.mode = MODE_TRAN;
    s.sub = SUB_NR;
    s.step = 1;
    s.first = 1;
    s.it = 0;
    s.depth = 0;
    s.frac = 0;
    s.status = KST_NOCONV;
    I.st[inst] = s;
  }
}
#endif  // !KARAM_JIT

#if !defined(KARAM_JIT)
__global__ void k_unpermute(const double* vp, const int* perm, double* out, int ni, int n) {
  const size_t total = (size_t)ni * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t inst = e / n;
    const int p = (int)(e - inst * n);
    out[inst * n + perm[p]] = vp[e];
  }
}
#endif  // !KARAM_JIT


}  // namespace knr
#endif
