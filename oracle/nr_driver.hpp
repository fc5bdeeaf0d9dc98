// nr_driver.hpp -- the oracle's Newton-Raphson driver (TEST INFRASTRUCTURE ONLY).
//
// One composition, two backends: ref_harness.cpp plugs in the reference's own
// tensorisation, stamping, CSR assembly and LU; port.cpp plugs in this
// project's restatement of the same functions. The driver itself restates
// CircuitSim::solveDC (solvers/circuitsim_solver.cpp:176-485) and the NR loop
// of CircuitSim::stepTransient (circuitsim_solver.cpp:600-635) with these
// documented deviations:
//   * KCL residual. calculatePhysicalResiduals (physics/circuitsim.h:1250-1671)
//     sums device currents per node but hardcodes MOSFET KP/VTO/LAMBDA by
//     model-name substring, so it disagrees with the stamps whenever model
//     cards are used and the reference never converges. The oracle keeps its
//     structure (a KCL sum of device currents, no gmin) with the currents of
//     the SoA kernels at the tensorised parameters, so it is exactly J(v) v -
//     rhs(v) of the same stamps in real arithmetic, without the cancellation of
//     forming J v and rhs separately (1e3 S source rows).
//   * Transient. The reference re-tensorises every step (which zeroes the SoA
//     capacitor history), has no PULSE in the SoA path and picks dt adaptively.
//     The oracle runs fixed steps with the companions of
//     math/integration_method.h:47-115, PULSE of physics/circuitsim.h:2155-2170
//     and the history update of circuitsim_solver.cpp:669-699, starting from the
//     DC solution (v_prev = DC capacitor voltage, i_prev = 0).
//   * Polishing (optional, opts.polish_max > 0): after the reference criterion
//     holds, Newton steps continue at the final gmin until every update is
//     below polish_rel*|v| + polish_abs or the update stops shrinking, so two
//     correct solvers meet at the same FP64 fixed point.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace oracle {

// pnjlim and compute_vcrit: physics/device_physics.h:132-179 (SPICE3f5 form).
inline double pnjlim(double vnew, double vold, double vt, double vcrit) {
  double vlim = vnew;
  if (vold > 30.0 * vt && vnew > 30.0 * vt) return vnew;
  if (vold < -5.0 * vt && vnew < -5.0 * vt) return vnew;
  if (vnew > vcrit && std::fabs(vnew - vold) > 2.0 * vt) {
    if (vold > 0.0) {
      double arg = 1.0 + (vnew - vold) / vt;
      if (arg > 0.0)
        vlim = vold + vt * std::log(arg);
      else
        vlim = vcrit;
    } else {
      vlim = vt * std::log(vnew / vt);
    }
  } else if (vnew < -5.0 * vt) {
    vlim = std::max(vnew, vold - 5.0 * vt);
  }
  return vlim;
}
inline double compute_vcrit(double vt, double is) {
  return vt * std::log(vt / (std::sqrt(2.0) * is));
}

// PULSE waveform, physics/circuitsim.h:2155-2170.
inline double pulse_value(const double* p, double time) {
  const double v1 = p[0], v2 = p[1], td = p[2], tr = p[3], tf = p[4], pw = p[5], per = p[6];
  double t = time - td;
  if (!(t > 0)) return v1;
  double period = per > 0 ? per : 1e99;
  t = std::fmod(t, period);
  if (t < tr) return v1 + (v2 - v1) * (t / tr);
  if (t < tr + pw) return v2;
  if (t < tr + pw + tf) return v2 + (v1 - v2) * ((t - tr - pw) / tf);
  return v1;
}

// Per-instance source values: DC value and (for PULSE) the scaled pulse
// levels, per the karam_instances contract in include/karam.h.
struct SourceSet {
  std::vector<int> pos, neg, kind;
  std::vector<double> dc;
  std::vector<double> pulse;  // [n][7]
  double value_at(int i, double t, bool transient) const {
    if (!transient || kind[i] != KARAM_SRC_PULSE) return dc[i];
    return pulse_value(&pulse[7 * i], t);
  }
};

inline void make_sources(const karam_netlist* nl, const karam_instances* inst, int idx,
                         SourceSet& s) {
  int n = nl->n_vsrc;
  s.pos.assign(nl->vs_pos, nl->vs_pos + n);
  s.neg.assign(nl->vs_neg, nl->vs_neg + n);
  s.kind.assign(n, KARAM_SRC_DC);
  s.dc.assign(nl->vs_dc, nl->vs_dc + n);
  s.pulse.assign(7 * n, 0.0);
  for (int i = 0; i < n; ++i) {
    if (nl->vs_kind) s.kind[i] = nl->vs_kind[i];
    if (s.kind[i] == KARAM_SRC_PULSE && nl->vs_pulse)
      for (int k = 0; k < 7; ++k) s.pulse[7 * i + k] = nl->vs_pulse[7 * i + k];
    if (inst && inst->vs_dc) {
      double nv = inst->vs_dc[(size_t)idx * n + i];
      if (s.kind[i] == KARAM_SRC_PULSE && nl->vs_dc[i] != 0.0) {
        double sc = nv / nl->vs_dc[i];
        s.pulse[7 * i + 0] *= sc;
        s.pulse[7 * i + 1] *= sc;
      }
      s.dc[i] = nv;
    }
  }
}

struct Csr {
  int n = 0;
  std::vector<int> row_ptr, col, diag;
};

// Sparse matrix-vector residual: F = J v - rhs, max |F_i| (same row-major
// accumulation as matrixMultiplication in math/linalg.h).
inline double residual_max(const Csr& p, const std::vector<double>& vals,
                           const std::vector<double>& v, const std::vector<double>& rhs,
                           bool* nonfinite) {
  double m = 0.0;
  for (int i = 0; i < p.n; ++i) {
    double s = 0.0;
    for (int k = p.row_ptr[i]; k < p.row_ptr[i + 1]; ++k) s += vals[k] * v[p.col[k]];
    double f = s - rhs[i];
    if (!std::isfinite(f)) *nonfinite = true;
    m = std::max(m, std::fabs(f));
  }
  return m;
}

// checkConvergence, physics/circuitsim.h:1218-1241.
inline bool check_convergence(const oracle_opts& o, const std::vector<double>& vn,
                              const std::vector<double>& vo, double kcl, double kcl_tol) {
  if (kcl < o.kcl_shortcut) return true;
  for (size_t i = 0; i < vn.size(); ++i) {
    double diff = std::fabs(vn[i] - vo[i]);
    double lim = o.reltol * std::max(std::fabs(vn[i]), std::fabs(vo[i])) + o.vntol;
    if (diff > lim) return false;
  }
  return !(kcl > kcl_tol);
}

// Polishing test on one update: every node inside polish_rel*|v|+polish_abs.
inline bool polish_done(const oracle_opts& o, const std::vector<double>& vn,
                        const std::vector<double>& vo, double* dvmax) {
  bool ok = true;
  double m = 0.0;
  for (size_t i = 0; i < vn.size(); ++i) {
    double d = std::fabs(vn[i] - vo[i]);
    m = std::max(m, d);
    if (d > o.polish_rel * std::max(std::fabs(vn[i]), std::fabs(vo[i])) + o.polish_abs) ok = false;
  }
  *dvmax = m;
  return ok;
}

// Backend interface (both implementations provide it):
//   int n; Csr pat; SourceSet src;
//   std::vector<int> dio_a, dio_c; std::vector<double> dio_is, dio_vt;   (SoA order)
//   std::vector<int> cap_n1, cap_n2; std::vector<double> cap_c;          (SoA order)
//   std::vector<int> seed_dio_anode;                                     (netlist order)
//   std::vector<int> isrc_pos; double temp_k;
//   void stamp(const std::vector<double>& v, double h, int method,
//              const std::vector<double>& cvp, const std::vector<double>& cip,
//              double t, std::vector<double>& vals, std::vector<double>& rhs);
//   void kcl(v, h, method, cvp, cip, t, F): node currents at the point of the
//              last stamp() call (device kernel outputs of that call);
//   bool solve(const std::vector<double>& vals_gmin, const std::vector<double>& rhs,
//              std::vector<double>& x, int solver);
template <class B>
struct Driver {
  B& b;
  oracle_opts o;
  std::vector<double> vals, rhs, tmp_vals, tmp_rhs, cvp, cip;

  Driver(B& be, const oracle_opts& oo) : b(be), o(oo) {}

  // DC convergence history (ConvergenceStep records, circuitsim_solver.cpp:
  // 408-425): residual and max |v_new - v_old| of every DC NR iteration, and
  // the stagnation / divergence flags of :427-443.
  std::vector<double> h_res, h_dv;
  bool h_stag = false, h_div = false, h_sing = false;

  void record(int it, double prev_kcl, double kcl, const std::vector<double>& x,
              const std::vector<double>& v) {
    double md = 0.0;
    for (int i = 0; i < b.n; ++i) md = std::max(md, std::fabs(x[i] - v[i]));
    h_res.push_back(kcl);
    h_dv.push_back(md);
    if (it > 0 && std::fabs(prev_kcl - kcl) < 1e-15 && kcl > o.kcl_tol) h_stag = true;
    const size_t z = h_res.size();
    if (z >= 3 && h_res[z - 1] > h_res[z - 2] && h_res[z - 2] > h_res[z - 3]) h_div = true;
  }

  // ConvergenceEngine::classifyFailure (solvers/convergence_engine.h:26-87),
  // numbered as ConvergenceFailureType (infrastructure/simtrace.h:39-47).
  int classify() const {
    if (h_sing) return 1;
    const size_t z = h_res.size();
    if (z == 0) return 0;
    for (double d : h_dv)
      if (d > 100.0) return 6;
    if (z >= 5) {
      bool up = true;
      for (size_t i = z - 4; i < z; ++i)
        if (h_res[i] <= h_res[i - 1]) up = false;
      if (up) return 2;
    }
    if (z >= 4) {
      int ch = 0;
      for (size_t i = 2; i < z; ++i) {
        const double pd = h_res[i - 1] - h_res[i - 2], cd = h_res[i] - h_res[i - 1];
        if ((pd > 0 && cd < 0) || (pd < 0 && cd > 0)) ch++;
      }
      if ((double)ch / (double)(z - 2) > 0.6) return 3;
    }
    if (z >= 10) {
      const double a = h_res[z - 10], c = h_res.back();
      if (a > 0.0 && c > 0.5 * a) return 4;
    }
    return 0;
  }

  void add_gmin(std::vector<double>& v, double gmin) {
    for (int i = 0; i < b.n; ++i) v[b.pat.diag[i]] += gmin;
  }

  std::vector<double> fvec;

  // KCL residual at x (DC: h = 0): currents leaving every node through the
  // devices, evaluated by the backend from the device-kernel outputs at x.
  double kcl_at(const std::vector<double>& x, double h, int method, double t, bool* nf) {
    b.stamp(x, h, method, cvp, cip, t, tmp_vals, tmp_rhs);
    b.kcl(x, h, method, cvp, cip, t, fvec);
    double m = 0.0;
    for (double f : fvec) {
      if (!std::isfinite(f)) *nf = true;
      m = std::max(m, std::fabs(f));
    }
    return m;
  }

  // seedInitialGuess, circuitsim_solver.cpp:32-116 (no BJTs on this path).
  void seed(std::vector<double>& v) {
    const size_t N = v.size();
    for (size_t i = 0; i < b.src.pos.size(); ++i) {
      int idx = b.src.pos[i] - 1;
      if (idx >= 0 && (size_t)idx < N) v[idx] = b.src.dc[i];
    }
    for (int a : b.seed_dio_anode) {
      int idx = a - 1;
      if (idx >= 0 && (size_t)idx < N) v[idx] = std::max(v[idx], 0.6);
    }
    double vsup = 5.0;
    for (double d : b.src.dc) vsup = std::max(vsup, d);
    for (int p : b.isrc_pos) {
      int idx = p - 1;
      if (idx < 0 || (size_t)idx >= N) continue;
      if (v[idx] == 0.0) v[idx] = vsup * 0.5;
    }
  }

  // applyPnJunctionLimits, circuitsim_solver.cpp:118-169 (diodes).
  void limit(std::vector<double>& vn, const std::vector<double>& vo) {
    const double ts = b.temp_k / 300.15;
    const int N = (int)vn.size();
    for (size_t i = 0; i < b.dio_a.size(); ++i) {
      double vt = b.dio_vt[i], is = b.dio_is[i];
      vt *= ts;
      is *= std::pow(ts, 3.0) * std::exp(1.11 / (vt / ts) - 1.11 / vt);
      int p = b.dio_a[i] - 1, q = b.dio_c[i] - 1;
      if (p < 0 && q < 0) continue;
      if (p >= N || q >= N) continue;
      double vcrit = compute_vcrit(vt, is);
      double vjo = (p >= 0 ? vo[p] : 0.0) - (q >= 0 ? vo[q] : 0.0);
      double vjn = (p >= 0 ? vn[p] : 0.0) - (q >= 0 ? vn[q] : 0.0);
      double vl = pnjlim(vjn, vjo, vt, vcrit);
      double corr = vjn - vl;
      if (std::fabs(corr) > 1e-12) {
        if (p >= 0 && q >= 0) {
          vn[p] -= corr * 0.5;
          vn[q] += corr * 0.5;
        } else if (p >= 0) {
          vn[p] -= corr;
        } else if (q >= 0) {
          vn[q] += corr;
        }
      }
    }
  }

  // One Newton solve at v with gmin; false when the LU reports singular.
  bool newton_point(const std::vector<double>& v, double gmin, double h, int method,
                    double t, std::vector<double>& x) {
    b.stamp(v, h, method, cvp, cip, t, vals, rhs);
    add_gmin(vals, gmin);
    return b.solve(vals, rhs, x, o.linear_solver);
  }

  // GMIN-stepping NR (circuitsim_solver.cpp:237-485). g_first > 0 starts at a
  // later GMIN step (seeded start). Returns converged; updates v and stats.
  bool gmin_loop(std::vector<double>& v, int g_first, int iter_cap, oracle_stats* st) {
    const int G = o.gmin_steps;
    double final_kcl = 0.0;
    bool converged = false;
    std::vector<double> x(b.n);
    for (int g = g_first; g < G; ++g) {
      double gmin = std::pow(10.0, -(3.0 + g * 0.5));
      if (gmin < 1e-12) gmin = 1e-12;
      st->gmin_step = g;
      bool gconv = false;
      int it = 0;
      int cap = iter_cap > 0 ? iter_cap : o.max_nr_iter;
      for (; it < cap; ++it) {
        if (!newton_point(v, gmin, 0.0, 0, 0.0, x)) {
          final_kcl = 1e9;
          st->singular = 1;
          h_sing = true;
          st->iterations += it + 1;
          break;
        }
        for (double& e : x)
          if (!std::isfinite(e)) e = 0.0;  // SafeUtils::sanitize_vector
        limit(x, v);
        bool nf = false;
        double kcl = kcl_at(x, 0.0, 0, 0.0, &nf);
        if (it > 0 && kcl >= final_kcl) {
          for (int i = 0; i < b.n; ++i) x[i] = v[i] + 0.5 * (x[i] - v[i]);
          kcl = kcl_at(x, 0.0, 0, 0.0, &nf);
          st->damped++;
          if (kcl >= final_kcl) {
            for (int i = 0; i < b.n; ++i) x[i] = v[i] + 0.5 * (x[i] - v[i]);
            kcl = kcl_at(x, 0.0, 0, 0.0, &nf);
            st->damped++;
          }
        }
        record(it, final_kcl, kcl, x, v);
        final_kcl = kcl;
        double tol = (g == G - 1) ? o.kcl_tol : 1.0;
        if (check_convergence(o, x, v, kcl, tol)) {
          v = x;
          gconv = true;
          st->iterations += it + 1;
          break;
        }
        v = x;
      }
      if (!gconv) st->iterations += it + 1;
      if (g == G - 1 && gconv) {
        converged = true;
        break;
      }
      if (!gconv) {
        if (final_kcl < 1.0) continue;
        break;
      }
    }
    st->residual = final_kcl;
    return converged;
  }

  // Polishing Newton steps at the final gmin (DC: h = 0; transient: companions).
  // Each step is the reference's linear solve applied to the residual
  // (dx = J^-1 (rhs - J v), v += dx), i.e. iterative refinement of the
  // reference solution, so the fixed point is set by the FP64 residual rather
  // than by the rounding of a solve for v itself.
  bool refine_step(const std::vector<double>& v, double h, int method, double t,
                   std::vector<double>& x) {
    b.stamp(v, h, method, cvp, cip, t, vals, rhs);
    b.kcl(v, h, method, cvp, cip, t, fvec);
    add_gmin(vals, 1e-12);
    std::vector<double> r(b.n);
    for (int i = 0; i < b.n; ++i) r[i] = -(fvec[i] + 1e-12 * v[i]);
    std::vector<double> dx;
    if (!b.solve(vals, r, dx, o.linear_solver)) return false;
    x.resize(b.n);
    for (int i = 0; i < b.n; ++i) x[i] = v[i] + dx[i];
    return true;
  }

  void polish(std::vector<double>& v, double h, int method, double t, oracle_stats* st) {
    if (o.polish_max <= 0) return;
    std::vector<double> x(b.n);
    double prev = -1.0;
    for (int p = 0; p < o.polish_max; ++p) {
      if (!refine_step(v, h, method, t, x)) break;
      double dv = 0.0;
      bool ok = polish_done(o, x, v, &dv);
      v = x;
      st->polish_iters++;
      if (ok || dv == 0.0 || (prev >= 0.0 && dv > 0.5 * prev)) break;
      prev = dv;
    }
  }

  void final_residual(const std::vector<double>& v, double h, int method, double t,
                      oracle_stats* st) {
    bool nf = false;
    st->residual = kcl_at(v, h, method, t, &nf);
  }

  int solve_dc(const double* v0, std::vector<double>& v, oracle_stats* st) {
    std::memset(st, 0, sizeof(*st));
    h_res.clear();
    h_dv.clear();
    h_stag = h_div = h_sing = false;
    v.assign(b.n, 0.0);
    bool conv = false;
    if (o.seeded && v0) {
      v.assign(v0, v0 + b.n);
      oracle_stats s2{};
      conv = gmin_loop(v, o.gmin_steps - 1, o.seed_max_iter, &s2);
      st->iterations += s2.iterations;
      st->damped += s2.damped;
      if (conv) {
        st->seeded_ok = 1;
        st->gmin_step = s2.gmin_step;
      } else {
        v.assign(b.n, 0.0);
      }
    }
    if (!conv) {
      seed(v);
      oracle_stats s3{};
      conv = gmin_loop(v, 0, 0, &s3);
      st->iterations += s3.iterations;
      st->damped += s3.damped;
      st->gmin_step = s3.gmin_step;
      st->singular = s3.singular;
    }
    st->converged = conv ? 1 : 0;
    if (conv) polish(v, 0.0, 0, 0.0, st);
    final_residual(v, 0.0, 0, 0.0, st);
    st->failure_type = classify();
    st->stagnation = h_stag ? 1 : 0;
    st->divergence = h_div ? 1 : 0;
    st->history_len = (int32_t)h_res.size();
    return 0;
  }

  // NR of one transient (sub-)step from guess at time t with step h.
  // Returns the number of iterations used; conv tells whether it converged.
  int tran_nr(std::vector<double>& guess, double h, int method, double t, bool* conv,
              oracle_stats* st) {
    std::vector<double> x(b.n);
    *conv = false;
    int it = 0;
    for (; it < o.max_nr_iter; ++it) {
      if (!newton_point(guess, 1e-12, h, method, t, x)) {
        st->singular = 1;
        return it + 1;
      }
      bool nf = false;
      double kcl = kcl_at(x, h, method, t, &nf);
      if (check_convergence(o, x, guess, kcl, o.kcl_tol)) {
        guess = x;
        *conv = true;
        return it + 1;
      }
      guess = x;
    }
    return it + 1;
  }

  // Fixed-step transient (see header comment). A step whose NR does not
  // converge within max_nr_iter is retried from the last accepted time point
  // with half the step, as the attempt loop of CircuitSim::stepTransient does
  // (circuitsim_solver.cpp:587-660, MAX_ATTEMPTS = 4, i.e. three halvings;
  // o.max_halvings sets the count); the halved sub-steps then complete the
  // step, so results stay on the output grid.
  int transient(const std::vector<double>& v_start, double dt, int n_steps, int method,
                const int32_t* wave_nodes, int n_wave, double* wave_out,
                std::vector<double>& v, oracle_stats* st) {
    std::memset(st, 0, sizeof(*st));
    v = v_start;
    const size_t nc = b.cap_c.size();
    cvp.assign(nc, 0.0);
    cip.assign(nc, 0.0);
    auto vnode = [&](const std::vector<double>& vv, int node) {
      return node > 0 ? vv[node - 1] : 0.0;
    };
    for (size_t i = 0; i < nc; ++i) cvp[i] = vnode(v, b.cap_n1[i]) - vnode(v, b.cap_n2[i]);
    std::vector<double> guess, v_prev = v;  // v_prev: the accepted point before v
    double h_prev = 0.0;                     // size of the last accepted sub-step
    st->converged = 1;
    const int H = o.max_halvings, units = 1 << H;
    const double unit = dt / units;
    for (int s = 1; s <= n_steps && st->converged; ++s) {
      int depth = 0, frac = 0;
      while (frac < units) {
        const int size = units >> depth;
        const double h = dt * size / units;
        const double t = (double)((s - 1) * units + frac + size) * unit;
        guess = v;
        bool conv = false;
        int its = tran_nr(guess, h, method, t, &conv, st);
        st->iterations += its;
        st->max_step_iters = std::max(st->max_step_iters, its);
        if (!conv) {
          if (st->singular || depth == H) {
            st->converged = 0;
            v = guess;
            break;
          }
          depth++;
          st->halvings++;
          continue;
        }
        polish(guess, h, method, t, st);
        // LTE step control (the product's documented rule, karam_solver_opts
        // lte_reltol): the accepted point against the linear extrapolation
        // from the two previous accepted points; a failing sub-step is redone
        // with half the step while halvings remain
        if (o.lte_rel > 0.0 && h_prev > 0.0 && depth < H) {
          const double r = h / h_prev;
          bool ok = true;
          for (int i = 0; i < b.n && ok; ++i) {
            const double p = v[i] + r * (v[i] - v_prev[i]);
            if (std::fabs(guess[i] - p) > o.lte_rel * std::fmax(std::fabs(guess[i]), std::fabs(v[i])) + o.lte_abs)
              ok = false;
          }
          if (!ok) {
            depth++;
            st->halvings++;
            st->lte_rejects++;
            continue;
          }
        }
        // capacitor history, circuitsim_solver.cpp:669-699
        for (size_t i = 0; i < nc; ++i) {
          double vc = vnode(guess, b.cap_n1[i]) - vnode(guess, b.cap_n2[i]);
          double C = b.cap_c[i];
          double ic = (method == KARAM_TRAN_TRAP) ? (2.0 * C / h) * (vc - cvp[i]) - cip[i]
                                                  : (C / h) * (vc - cvp[i]);
          cvp[i] = vc;
          cip[i] = ic;
        }
        v_prev = v;
        v = guess;
        h_prev = h;
        frac += size;
      }
      if (st->converged && wave_out && n_wave > 0)
        for (int k = 0; k < n_wave; ++k)
          wave_out[(size_t)(s - 1) * n_wave + k] = vnode(v, wave_nodes[k]);
    }
    st->residual = 0.0;
    return 0;
  }
};

// ---------------------------------------------------------------------------
// Small-signal AC (ACSolver::solveAC_Sparse, solvers/ac_solver.h:711-773)
// ---------------------------------------------------------------------------

// Log-spaced sweep frequencies, solveAC_Sparse's formula (ac_solver.h:724-729).
inline std::vector<double> ac_frequencies(double f_start, double f_stop, int n_points) {
  std::vector<double> f(n_points > 0 ? n_points : 0);
  const double lo = std::log10(std::max(f_start, 1e-3));
  const double hi = std::log10(std::max(f_stop, f_start + 1.0));
  for (int i = 0; i < n_points; ++i)
    f[i] = std::pow(10.0, lo + (hi - lo) * i / std::max(n_points - 1, 1));
  return f;
}

// Position of (r, c) in the pattern's row r, or -1.
inline int csr_at(const Csr& p, int r, int c) {
  for (int q = p.row_ptr[r]; q < p.row_ptr[r + 1]; ++q)
    if (p.col[q] == c) return q;
  return -1;
}

// Y(jw) on the stamp pattern p at one frequency w: the real part is the NR
// Jacobian at the DC point (jac, without gmin) plus 1e-12 on every diagonal
// (the conditioning of ac_solver.h:701-702) plus the excitation's 1e6 at the
// input node's diagonal (ac_solver.h:751-763); the imaginary part is w C from
// each capacitor's four stamps (ac_solver.h:658-660). rhs_re: 1e6 * amplitude
// at the input node. Nodes are 1-based, 0 = ground.
inline void ac_matrix(const Csr& p, const std::vector<double>& jac, const std::vector<int>& cap_n1,
                      const std::vector<int>& cap_n2, const std::vector<double>& cap_c, double w,
                      int input_node, double amplitude, std::vector<double>& re,
                      std::vector<double>& im, std::vector<double>& rhs_re) {
  const int n = p.n;
  re = jac;
  im.assign(jac.size(), 0.0);
  rhs_re.assign(n, 0.0);
  auto add_im = [&](int a, int b, double y) {
    if (a <= 0 || b <= 0) return;
    const int q = csr_at(p, a - 1, b - 1);
    if (q >= 0) im[q] += y;
  };
  for (size_t k = 0; k < cap_c.size(); ++k) {
    const double y = w * cap_c[k];
    const int a = cap_n1[k], b = cap_n2[k];
    add_im(a, a, y);
    add_im(a, b, -y);
    add_im(b, a, -y);
    add_im(b, b, y);
  }
  for (int i = 0; i < n; ++i) re[p.diag[i]] += 1e-12;
  if (input_node > 0 && input_node <= n) {
    const double g_large = 1e6;
    re[p.diag[input_node - 1]] += g_large;
    rhs_re[input_node - 1] += g_large * amplitude;
  }
}

}  // namespace oracle
