// port.cpp -- CPU restatement of the reference's NR inner loop
// (TEST INFRASTRUCTURE ONLY; built by oracle/Makefile into oracle/_build/).
//
// Plain C++ written for this project. Each function names the reference
// file:line whose behaviour it restates; floating-point operations keep the
// reference's evaluation order so that results agree bit for bit with the
// library built from the reference sources (ref_harness.cpp), which the tests
// check. The NR driver is shared with that library (nr_driver.hpp).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "nr_driver.hpp"

namespace {

// ---------------------------------------------------------------------------
// SoA tensors (tensors/physics_tensors.h:24-419) -- only the fields used here.
// ---------------------------------------------------------------------------
struct Mos {
  int d, g, s, b;
  double W, L, Kp, Vth, lam;
  bool pmos;
};
struct Dio {
  int a, c;
  double Is, N, Vt;
};
struct Two {
  int n1, n2;
  double val;
};

struct Soa {
  std::vector<Mos> mos;
  std::vector<Dio> dio;
  std::vector<Two> res, cap, isrc;
  std::vector<int> vs_pos, vs_neg;
  std::vector<int> mos_order, dio_order;  // soa index -> netlist index
};

// tensorizeNetlist (tensors/physics_tensors.cpp:305-493): devices are
// collected into per-model-name buckets (std::map, so ascending name order)
// and flushed bucket by bucket; linear elements keep netlist order. MOSFET
// KP/VTO/LAMBDA come from the model card with the defaults of :424-441;
// diode Vt is scaled by T/300.15 (:419).
Soa tensorize(const karam_netlist* nl) {
  Soa s;
  auto mname = [&](int m) { return std::string(nl->model_name[m]); };
  std::map<std::string, std::vector<int>> mb, db;
  for (int i = 0; i < nl->n_mos; ++i) mb[mname(nl->m_model[i])].push_back(i);
  for (int i = 0; i < nl->n_dio; ++i) {
    int m = nl->d_model ? nl->d_model[i] : -1;
    db[m >= 0 ? mname(m) : std::string("diode_generic")].push_back(i);
  }
  const double tscale = nl->temp_k / 300.15;
  for (auto& kv : db)
    for (int i : kv.second) {
      s.dio.push_back({nl->d_anode[i], nl->d_cathode[i], nl->d_is[i], nl->d_n[i],
                       nl->d_vt[i] * tscale});
      s.dio_order.push_back(i);
    }
  for (auto& kv : mb)
    for (int i : kv.second) {
      int m = nl->m_model[i];
      bool pmos = nl->model_type[m] == KARAM_MODEL_PMOS;
      auto card = [&](const double* arr, double dflt) {
        return (arr && !std::isnan(arr[m])) ? arr[m] : dflt;
      };
      double kp = card(nl->model_kp, pmos ? 100e-6 : 200e-6);
      double vth = card(nl->model_vto, pmos ? -0.7 : 0.7);
      double lam = card(nl->model_lambda, 0.02);
      s.mos.push_back({nl->m_d[i], nl->m_g[i], nl->m_s[i], nl->m_b[i], nl->m_w[i], nl->m_l[i], kp,
                       vth, lam, pmos});
      s.mos_order.push_back(i);
    }
  for (int i = 0; i < nl->n_res; ++i) s.res.push_back({nl->r_n1[i], nl->r_n2[i], nl->r_ohm[i]});
  for (int i = 0; i < nl->n_cap; ++i) s.cap.push_back({nl->c_n1[i], nl->c_n2[i], nl->c_farad[i]});
  for (int i = 0; i < nl->n_isrc; ++i) s.isrc.push_back({nl->is_pos[i], nl->is_neg[i], nl->is_amp[i]});
  for (int i = 0; i < nl->n_vsrc; ++i) {
    s.vs_pos.push_back(nl->vs_pos[i]);
    s.vs_neg.push_back(nl->vs_neg[i]);
  }
  return s;
}

// ---------------------------------------------------------------------------
// Triplet stamping (physics/circuitsim.h:2413-2666) + gmin diagonal (:2857)
// ---------------------------------------------------------------------------
struct Stamp {
  std::vector<int> r, c;
  std::vector<double> v;
  std::vector<double> rhs;
  void add(int row, int col, double val) {
    r.push_back(row);
    c.push_back(col);
    v.push_back(val);
  }
  void clear(int n) {
    r.clear();
    c.clear();
    v.clear();
    rhs.assign(n, 0.0);
  }
};

// Two-terminal conductance: 4 triplets if both ends are nodes, else 1.
inline void stamp_g(Stamp& st, int n1, int n2, double g) {
  if (n1 != 0 && n2 != 0) {
    st.add(n1 - 1, n1 - 1, g);
    st.add(n2 - 1, n2 - 1, g);
    st.add(n1 - 1, n2 - 1, -g);
    st.add(n2 - 1, n1 - 1, -g);
  } else if (n1 != 0) {
    st.add(n1 - 1, n1 - 1, g);
  } else if (n2 != 0) {
    st.add(n2 - 1, n2 - 1, g);
  }
}

struct Eval {
  // per-device state written by the kernels (physics_tensors.cpp:19-104)
  std::vector<double> vgs, vds, ids, gm, gds;
  std::vector<double> vd, id, gd;
};

// batchDiodePhysics_generic, tensors/physics_tensors.cpp:19-51
void diode_physics(const std::vector<Dio>& dio, const std::vector<double>& v, Eval& e) {
  const int nv = (int)v.size();
  e.vd.resize(dio.size());
  e.id.resize(dio.size());
  e.gd.resize(dio.size());
  for (size_t i = 0; i < dio.size(); ++i) {
    int a = dio[i].a, c = dio[i].c;
    double va = (a > 0 && a <= nv) ? v[a - 1] : 0.0;
    double vc = (c > 0 && c <= nv) ? v[c - 1] : 0.0;
    e.vd[i] = va - vc;
    double nvt = dio[i].N * dio[i].Vt;
    double vcrit = 30.0 * nvt;
    double arg = e.vd[i] / nvt;
    double ex = std::exp(std::min(arg, 30.0));
    double ibase = dio[i].Is * (ex - 1.0);
    double gbase = (dio[i].Is / nvt) * ex;
    double delta = std::max(0.0, e.vd[i] - vcrit);
    e.id[i] = ibase + delta * gbase;
    e.gd[i] = std::max(1e-12, gbase);
  }
}

// batchMosfetPhysics_generic, tensors/physics_tensors.cpp:53-104
void mosfet_physics(const std::vector<Mos>& mos, const std::vector<double>& v, Eval& e) {
  const int nv = (int)v.size();
  size_t m = mos.size();
  e.vgs.resize(m);
  e.vds.resize(m);
  e.ids.resize(m);
  e.gm.resize(m);
  e.gds.resize(m);
  for (size_t i = 0; i < m; ++i) {
    const Mos& q = mos[i];
    double vd = (q.d > 0 && q.d <= nv) ? v[q.d - 1] : 0.0;
    double vg = (q.g > 0 && q.g <= nv) ? v[q.g - 1] : 0.0;
    double vs = (q.s > 0 && q.s <= nv) ? v[q.s - 1] : 0.0;
    double sign = q.pmos ? -1.0 : 1.0;
    e.vgs[i] = vg - vs;
    e.vds[i] = vd - vs;
    double lvgs = sign * e.vgs[i];
    double lvds = sign * e.vds[i];
    double lvth = sign * q.Vth;
    double K = 0.5 * q.Kp * (q.W / q.L);
    double vov = lvgs - lvth;
    if (vov <= 0.0) {
      e.ids[i] = 0.0;
      e.gm[i] = 0.0;
      e.gds[i] = 1e-12;
    } else if (lvds < vov) {
      e.ids[i] = sign * K * (2.0 * vov * lvds - lvds * lvds);
      e.gm[i] = 2.0 * K * lvds;
      e.gds[i] = 2.0 * K * (vov - lvds);
    } else {
      e.ids[i] = sign * K * vov * vov * (1.0 + q.lam * lvds);
      e.gm[i] = 2.0 * K * vov * (1.0 + q.lam * lvds);
      e.gds[i] = K * vov * vov * q.lam;
    }
    if (e.gds[i] < 1e-12) e.gds[i] = 1e-12;
  }
}

// stampSoABlock, physics/circuitsim.h:2413-2666 (no BJTs, no inductors, no
// registry models). h_eff > 0 stamps the trapezoidal capacitor companion with
// history g*v_prev + i_prev (:2480-2505).
void stamp_soa(const Soa& s, const std::vector<double>& vdc, const std::vector<double>& v,
               double h_eff, const std::vector<double>& cvp, const std::vector<double>& cip,
               Stamp& st, Eval& e) {
  for (const Two& r : s.res) stamp_g(st, r.n1, r.n2, 1.0 / r.val);
  for (size_t i = 0; i < s.vs_pos.size(); ++i) {
    int p = s.vs_pos[i], q = s.vs_neg[i];
    const double gint = 1.0e3;
    double ieq = vdc[i] * gint;
    stamp_g(st, p, q, gint);
    if (p != 0) st.rhs[p - 1] += ieq;
    if (q != 0) st.rhs[q - 1] -= ieq;
  }
  for (const Two& cs : s.isrc) {
    if (cs.n1 != 0) st.rhs[cs.n1 - 1] -= cs.val;
    if (cs.n2 != 0) st.rhs[cs.n2 - 1] += cs.val;
  }
  if (!s.cap.empty() && h_eff > 0.0) {
    for (size_t i = 0; i < s.cap.size(); ++i) {
      const Two& c = s.cap[i];
      double geq = (2.0 * c.val) / h_eff;
      double ihist = geq * cvp[i] + cip[i];
      stamp_g(st, c.n1, c.n2, geq);
      if (c.n1 != 0) st.rhs[c.n1 - 1] += ihist;
      if (c.n2 != 0) st.rhs[c.n2 - 1] -= ihist;
    }
  }
  diode_physics(s.dio, v, e);
  mosfet_physics(s.mos, v, e);
  for (size_t i = 0; i < s.dio.size(); ++i) {
    int a = s.dio[i].a, c = s.dio[i].c;
    double g = e.gd[i];
    double ieq = e.id[i] - g * e.vd[i];
    stamp_g(st, a, c, g);
    if (a != 0) st.rhs[a - 1] -= ieq;
    if (c != 0) st.rhs[c - 1] += ieq;
  }
  for (size_t i = 0; i < s.mos.size(); ++i) {
    const Mos& q = s.mos[i];
    int d = q.d, g = q.g, so = q.s, b = q.b;
    double gm = e.gm[i], gmb = 0.0, gds = e.gds[i];
    double vbs = (b != 0) ? (v[b - 1] - (so != 0 ? v[so - 1] : 0.0)) : 0.0;
    double ieq = e.ids[i] - (gm * e.vgs[i] + gmb * vbs + gds * e.vds[i]);
    stamp_g(st, d, so, gds);
    if (d != 0) {
      if (g != 0) st.add(d - 1, g - 1, gm);
      if (so != 0) st.add(d - 1, so - 1, -gm);
    }
    if (so != 0) {
      if (g != 0) st.add(so - 1, g - 1, -gm);
      st.add(so - 1, so - 1, gm);
    }
    if (d != 0) {
      if (b != 0) st.add(d - 1, b - 1, gmb);
      if (so != 0) st.add(d - 1, so - 1, -gmb);
    }
    if (so != 0) {
      if (b != 0) st.add(so - 1, b - 1, -gmb);
      st.add(so - 1, so - 1, gmb);
    }
    if (d != 0) st.rhs[d - 1] -= ieq;
    if (so != 0) st.rhs[so - 1] += ieq;
  }
}

// ---------------------------------------------------------------------------
// CSR pattern and assembly (math/linalg.h:82-107, 281-465)
// ---------------------------------------------------------------------------
struct Pattern {
  int n = 0;
  std::vector<int> row_ptr, col;
  std::unordered_map<int64_t, int> pos;
  int index_of(int r, int c) const {
    auto it = pos.find((int64_t(r) << 32) | int64_t(unsigned(c)));
    return it == pos.end() ? -1 : it->second;
  }
};

// createCsr's sort + dedup reduced to the pattern: rows ascending, columns
// ascending within a row, duplicates merged.
Pattern build_pattern(int n, const Stamp& st) {
  std::vector<std::pair<int, int>> rc;
  rc.reserve(st.r.size());
  for (size_t k = 0; k < st.r.size(); ++k)
    if (st.r[k] < n && st.c[k] < n) rc.emplace_back(st.r[k], st.c[k]);
  std::sort(rc.begin(), rc.end());
  rc.erase(std::unique(rc.begin(), rc.end()), rc.end());
  Pattern p;
  p.n = n;
  p.row_ptr.assign(n + 1, 0);
  for (auto& e : rc) p.row_ptr[e.first + 1]++;
  for (int i = 0; i < n; ++i) p.row_ptr[i + 1] += p.row_ptr[i];
  p.col.resize(rc.size());
  for (size_t k = 0; k < rc.size(); ++k) {
    p.col[k] = rc[k].second;
    p.pos[(int64_t(rc[k].first) << 32) | int64_t(unsigned(rc[k].second))] = (int)k;
  }
  return p;
}

// assembleFast: values summed in triplet insertion order.
void assemble(const Pattern& p, const Stamp& st, std::vector<double>& vals) {
  vals.assign(p.col.size(), 0.0);
  for (size_t k = 0; k < st.r.size(); ++k) {
    int idx = p.index_of(st.r[k], st.c[k]);
    if (idx >= 0) vals[idx] += st.v[k];
  }
}

// ---------------------------------------------------------------------------
// Dense partial-pivot LU, solveLU_Pivoted (math/linalg.h:742-854), and the
// same elimination on a permuted system (solveSparse_LU, sparse_lu.cpp:134-330,
// which adds the |a| < 1e-30 row skip).
// ---------------------------------------------------------------------------
bool dense_lu_solve(std::vector<double>& A, std::vector<double>& b, int n, bool skip_tiny,
                    std::vector<double>& x) {
  for (int i = 0; i < n; ++i) {
    double maxv = 0.0;
    int maxr = i;
    for (int k = i; k < n; ++k) {
      double val = std::fabs(A[(size_t)k * n + i]);
      if (val > maxv) {
        maxv = val;
        maxr = k;
      } else if (val == maxv && k < maxr) {
        maxr = k;
      }
    }
    if (maxv < 1e-25) return false;
    if (maxr != i) {
      for (int k = 0; k < n; ++k) std::swap(A[(size_t)i * n + k], A[(size_t)maxr * n + k]);
      std::swap(b[i], b[maxr]);
    }
    for (int j = i + 1; j < n; ++j) {
      if (skip_tiny && std::fabs(A[(size_t)j * n + i]) < 1e-30) continue;
      A[(size_t)j * n + i] /= A[(size_t)i * n + i];
      double l = A[(size_t)j * n + i];
      for (int k = i + 1; k < n; ++k) A[(size_t)j * n + k] -= l * A[(size_t)i * n + k];
    }
  }
  std::vector<double> y(n, 0.0);
  for (int i = 0; i < n; ++i) {
    y[i] = b[i];
    for (int j = 0; j < i; ++j) y[i] -= A[(size_t)i * n + j] * y[j];
  }
  x.assign(n, 0.0);
  for (int i = n - 1; i >= 0; --i) {
    x[i] = y[i];
    for (int j = i + 1; j < n; ++j) x[i] -= A[(size_t)i * n + j] * x[j];
    x[i] /= A[(size_t)i * n + i];
  }
  return true;
}

// ---------------------------------------------------------------------------
// FactorGraph::fromTensorizedBlock (infrastructure/factor_graph.cpp:9-162) and
// the Min-Fill loop of TreewidthAnalyzer::analyze (treewidth_analyzer.cpp:14-141)
// ---------------------------------------------------------------------------
struct MinFill {
  std::vector<uint32_t> ordering;
  int treewidth = 0;
};

MinFill min_fill(const Soa& s, int n) {
  std::vector<std::vector<uint32_t>> factors;
  std::set<uint32_t> volt;
  auto f2 = [&](std::initializer_list<int> nodes, bool branch, uint32_t& bid) {
    std::vector<uint32_t> f;
    for (int x : nodes)
      if (x > 0) {
        f.push_back((uint32_t)x);
        volt.insert((uint32_t)x);
      }
    if (branch) f.push_back(bid++);
    factors.push_back(f);
  };
  uint32_t bid = (uint32_t)n;  // branch ids start at numCircuitNodes
  uint32_t nbranch = 0;
  for (const Dio& d : s.dio) f2({d.a, d.c}, false, bid);
  for (const Mos& m : s.mos) f2({m.d, m.g, m.s, m.b}, false, bid);
  for (const Two& r : s.res) f2({r.n1, r.n2}, false, bid);
  for (const Two& c : s.cap) f2({c.n1, c.n2}, false, bid);
  for (size_t i = 0; i < s.vs_pos.size(); ++i) {
    f2({s.vs_pos[i], s.vs_neg[i]}, true, bid);
    nbranch++;
  }
  for (const Two& c : s.isrc) f2({c.n1, c.n2}, false, bid);

  std::vector<uint32_t> vars(volt.begin(), volt.end());
  for (uint32_t k = 0; k < nbranch; ++k) vars.push_back((uint32_t)n + k);

  std::map<uint32_t, std::set<uint32_t>> adj;
  for (uint32_t v : vars) adj[v];
  for (auto& f : factors)
    for (size_t i = 0; i < f.size(); ++i)
      for (size_t j = i + 1; j < f.size(); ++j)
        if (f[i] != f[j]) {
          adj[f[i]].insert(f[j]);
          adj[f[j]].insert(f[i]);
        }

  MinFill out;
  std::vector<uint32_t> remaining = vars;
  std::sort(remaining.begin(), remaining.end());
  uint32_t maxclique = 0;
  const size_t N = vars.size();
  for (size_t step = 0; step < N; ++step) {
    uint32_t best = remaining[0];
    uint32_t bestfill = UINT32_MAX;
    for (uint32_t v : remaining) {
      const std::set<uint32_t>& nb = adj[v];
      std::vector<uint32_t> nv(nb.begin(), nb.end());
      uint32_t fill = 0;
      for (size_t i = 0; i < nv.size(); ++i)
        for (size_t j = i + 1; j < nv.size(); ++j)
          if (!adj[nv[i]].count(nv[j])) ++fill;
      if (fill < bestfill || (fill == bestfill && v < best)) {
        bestfill = fill;
        best = v;
      }
    }
    out.ordering.push_back(best);
    std::vector<uint32_t> nv(adj[best].begin(), adj[best].end());
    maxclique = std::max<uint32_t>(maxclique, (uint32_t)nv.size() + 1);
    for (size_t i = 0; i < nv.size(); ++i)
      for (size_t j = i + 1; j < nv.size(); ++j) {
        adj[nv[i]].insert(nv[j]);
        adj[nv[j]].insert(nv[i]);
      }
    for (uint32_t u : nv) adj[u].erase(best);
    adj.erase(best);
    remaining.erase(std::find(remaining.begin(), remaining.end(), best));
  }
  out.treewidth = maxclique > 0 ? (int)maxclique - 1 : 0;
  return out;
}

// Translation of the raw ordering to a 0-based permutation of the n unknowns:
// ids in 1..n kept, repeats dropped, minus one; unknowns no device touches
// (absent from the factor graph) go last in id order.
std::vector<uint32_t> translate(const std::vector<uint32_t>& raw, int n) {
  std::vector<uint32_t> perm;
  std::vector<char> seen(n + 1, 0);
  for (uint32_t id : raw)
    if (id >= 1 && id <= (uint32_t)n && !seen[id]) {
      seen[id] = 1;
      perm.push_back(id - 1);
    }
  for (int i = 1; i <= n; ++i)
    if (!seen[i]) perm.push_back(i - 1);
  return perm;
}

// symbolicFactorize, math/sparse_lu.cpp:14-128
struct Symbolic {
  std::vector<int> perm, iperm, row_ptr, col;
  int fill = 0;
};

Symbolic symbolic(const Pattern& p, const std::vector<uint32_t>& ord) {
  const int n = p.n;
  Symbolic s;
  s.perm.resize(n);
  s.iperm.resize(n);
  for (int i = 0; i < n; ++i) {
    s.perm[i] = (int)ord[i];
    s.iperm[ord[i]] = i;
  }
  std::vector<std::set<int>> adj(n);
  for (int r = 0; r < n; ++r)
    for (int k = p.row_ptr[r]; k < p.row_ptr[r + 1]; ++k) {
      int c = p.col[k];
      if (c != r) {
        adj[r].insert(c);
        adj[c].insert(r);
      }
    }
  std::vector<std::set<int>> rows(n);
  for (int i = 0; i < n; ++i) rows[i].insert(i);
  for (int step = 0; step < n; ++step) {
    int v = (int)ord[step];
    std::vector<int> nb(adj[v].begin(), adj[v].end());
    for (int u : nb) {
      int pc = s.iperm[u];
      rows[step].insert(pc);
      rows[pc].insert(step);
    }
    for (size_t i = 0; i < nb.size(); ++i)
      for (size_t j = i + 1; j < nb.size(); ++j)
        if (!adj[nb[i]].count(nb[j])) {
          adj[nb[i]].insert(nb[j]);
          adj[nb[j]].insert(nb[i]);
          ++s.fill;
        }
    for (int u : nb) adj[u].erase(v);
    adj[v].clear();
  }
  s.row_ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    s.row_ptr[i] = (int)s.col.size();
    for (int c : rows[i]) s.col.push_back(c);
  }
  s.row_ptr[n] = (int)s.col.size();
  return s;
}

// ---------------------------------------------------------------------------
// Backend for the shared driver
// ---------------------------------------------------------------------------
struct PortBackend {
  int n = 0;
  oracle::Csr pat;
  oracle::SourceSet src;
  std::vector<int> dio_a, dio_c;
  std::vector<double> dio_is, dio_vt;
  std::vector<int> cap_n1, cap_n2;
  std::vector<double> cap_c;
  std::vector<int> seed_dio_anode, isrc_pos;
  double temp_k = 300.15;

  Soa soa;
  Pattern cp;
  Stamp st;
  Eval ev;
  Symbolic sym;
  bool have_sym = false;

  Pattern pattern_for(bool transient) {
    std::vector<double> v(n, 0.0), z(soa.cap.size(), 0.0), vdc(soa.vs_pos.size(), 0.0);
    Stamp s2;
    s2.clear(n);
    Eval e2;
    stamp_soa(soa, vdc, v, transient ? 1.0 : 0.0, z, z, s2, e2);
    for (int i = 0; i < n; ++i) s2.add(i, i, 1e-12);
    return build_pattern(n, s2);
  }

  void build(const karam_netlist* nl) {
    soa = tensorize(nl);
    temp_k = nl->temp_k;
    int nmax = nl->n_nodes;
    auto touch = [&](int x) { nmax = std::max(nmax, x); };
    for (const Mos& m : soa.mos) { touch(m.d); touch(m.g); touch(m.s); touch(m.b); }
    for (const Dio& d : soa.dio) { touch(d.a); touch(d.c); }
    for (const Two& r : soa.res) { touch(r.n1); touch(r.n2); }
    for (const Two& c : soa.cap) { touch(c.n1); touch(c.n2); }
    for (const Two& c : soa.isrc) { touch(c.n1); touch(c.n2); }
    for (size_t i = 0; i < soa.vs_pos.size(); ++i) { touch(soa.vs_pos[i]); touch(soa.vs_neg[i]); }
    n = nmax;
    for (const Dio& d : soa.dio) {
      dio_a.push_back(d.a);
      dio_c.push_back(d.c);
      dio_is.push_back(d.Is);
      dio_vt.push_back(d.Vt);
    }
    for (const Two& c : soa.cap) {
      cap_n1.push_back(c.n1);
      cap_n2.push_back(c.n2);
      cap_c.push_back(c.val);
    }
    for (int i = 0; i < nl->n_dio; ++i) seed_dio_anode.push_back(nl->d_anode[i]);
    for (int i = 0; i < nl->n_isrc; ++i) isrc_pos.push_back(nl->is_pos[i]);
    cp = pattern_for(true);
    pat.n = n;
    pat.row_ptr = cp.row_ptr;
    pat.col = cp.col;
    pat.diag.assign(n, -1);
    for (int i = 0; i < n; ++i) pat.diag[i] = cp.index_of(i, i);
  }

  void set_instance(const karam_netlist* nl, const karam_instances* inst, int idx) {
    oracle::make_sources(nl, inst, idx, src);
    if (!inst) return;
    for (size_t j = 0; j < soa.mos.size(); ++j) {
      size_t k = (size_t)idx * nl->n_mos + soa.mos_order[j];
      if (inst->mos_kp) soa.mos[j].Kp = (double)inst->mos_kp[k];
      if (inst->mos_vto) soa.mos[j].Vth = (double)inst->mos_vto[k];
    }
  }

  void stamp(const std::vector<double>& v, double h, int method, const std::vector<double>& cvp,
             const std::vector<double>& cip, double t, std::vector<double>& vals,
             std::vector<double>& rhs) {
    bool tran = h > 0.0;
    std::vector<double> vdc(src.dc.size());
    for (size_t i = 0; i < vdc.size(); ++i) vdc[i] = src.value_at((int)i, t, tran);
    double h_eff = 0.0;
    std::vector<double> ip;
    if (tran) {
      // backward Euler (C/h, (C/h) v_prev) == trapezoidal stamp at 2h, i_prev 0
      h_eff = method == KARAM_TRAN_TRAP ? h : 2.0 * h;
      ip = method == KARAM_TRAN_TRAP ? cip : std::vector<double>(cip.size(), 0.0);
    }
    st.clear(n);
    stamp_soa(soa, vdc, v, h_eff, cvp, ip, st, ev);
    assemble(cp, st, vals);
    rhs = st.rhs;
  }

  // Currents leaving every node at v (the stamp() just run at v left the
  // device-kernel outputs in ev): R (v1 - v2)/R, Norton sources
  // 1e3 ((v+ - v-) - V), current sources, capacitor companions, diodes, MOSFETs.
  void kcl(const std::vector<double>& v, double h, int method, const std::vector<double>& cvp,
           const std::vector<double>& cip, double t, std::vector<double>& F) {
    F.assign(n, 0.0);
    auto vn = [&](int node) { return node > 0 ? v[node - 1] : 0.0; };
    auto add = [&](int node, double cur) {
      if (node > 0) F[node - 1] += cur;
    };
    const bool tran = h > 0.0;
    for (const Two& r : soa.res) {
      double i = (vn(r.n1) - vn(r.n2)) / r.val;
      add(r.n1, i);
      add(r.n2, -i);
    }
    for (size_t k = 0; k < soa.vs_pos.size(); ++k) {
      double i = 1.0e3 * ((vn(soa.vs_pos[k]) - vn(soa.vs_neg[k])) - src.value_at((int)k, t, tran));
      add(soa.vs_pos[k], i);
      add(soa.vs_neg[k], -i);
    }
    for (const Two& c : soa.isrc) {
      add(c.n1, c.val);
      add(c.n2, -c.val);
    }
    if (tran) {
      const double heff = method == KARAM_TRAN_TRAP ? h : 2.0 * h;
      for (size_t k = 0; k < soa.cap.size(); ++k) {
        const Two& c = soa.cap[k];
        double g = (2.0 * c.val) / heff;
        double i = g * ((vn(c.n1) - vn(c.n2)) - cvp[k]);
        if (method == KARAM_TRAN_TRAP) i -= cip[k];
        add(c.n1, i);
        add(c.n2, -i);
      }
    }
    for (size_t k = 0; k < soa.dio.size(); ++k) {
      add(soa.dio[k].a, ev.id[k]);
      add(soa.dio[k].c, -ev.id[k]);
    }
    for (size_t k = 0; k < soa.mos.size(); ++k) {
      add(soa.mos[k].d, ev.ids[k]);
      add(soa.mos[k].s, -ev.ids[k]);
    }
  }

  void ensure_symbolic() {
    if (have_sym) return;
    MinFill mf = min_fill(soa, n);
    sym = symbolic(cp, translate(mf.ordering, n));
    have_sym = true;
  }

  bool solve(const std::vector<double>& vals, const std::vector<double>& rhs,
             std::vector<double>& x, int solver) {
    std::vector<double> A((size_t)n * n, 0.0);
    if (solver == ORACLE_LS_SPARSE) {
      ensure_symbolic();
      for (int r = 0; r < n; ++r)
        for (int k = pat.row_ptr[r]; k < pat.row_ptr[r + 1]; ++k)
          A[(size_t)sym.iperm[r] * n + sym.iperm[pat.col[k]]] = vals[k];
      std::vector<double> b(n), xp;
      for (int i = 0; i < n; ++i) b[i] = rhs[sym.perm[i]];
      if (!dense_lu_solve(A, b, n, true, xp)) return false;
      x.assign(n, 0.0);
      for (int i = 0; i < n; ++i) x[sym.perm[i]] = xp[i];
      return true;
    }
    for (int r = 0; r < n; ++r)
      for (int k = pat.row_ptr[r]; k < pat.row_ptr[r + 1]; ++k) A[(size_t)r * n + pat.col[k]] = vals[k];
    std::vector<double> b = rhs;
    return dense_lu_solve(A, b, n, false, x);
  }
};

struct Session {
  PortBackend b;
  Session(const karam_netlist* nl, const karam_instances* inst, int idx) {
    b.build(nl);
    b.set_instance(nl, inst, idx);
  }
};

template <class F>
int guarded(F f) {
  try {
    return f();
  } catch (const std::exception& e) {
    fprintf(stderr, "oracle(port): %s\n", e.what());
    return -1;
  }
}

// solveComplexLU_Sparse (math/linalg.h:993-1078) restated: the CSR values
// into a dense row-major matrix, LU with partial pivoting on the complex
// magnitude (hypot; on equal magnitudes the earlier row), rows swapped with
// the right-hand side, multipliers by complex division over |d|^2, forward
// substitution with the unit lower factor, back substitution. Returns false
// when a pivot's magnitude is below 1e-25 (rank deficient).
bool complex_lu_solve(const oracle::Csr& p, const std::vector<double>& vre,
                      const std::vector<double>& vim, const std::vector<double>& rre,
                      const std::vector<double>& rim, std::vector<double>& xre,
                      std::vector<double>& xim) {
  const int n = p.n;
  xre.assign(n, 0.0);
  xim.assign(n, 0.0);
  if (n == 0) return true;
  std::vector<double> Are((size_t)n * n, 0.0), Aim((size_t)n * n, 0.0);
  for (int r = 0; r < n; ++r)
    for (int q = p.row_ptr[r]; q < p.row_ptr[r + 1]; ++q) {
      Are[(size_t)r * n + p.col[q]] = vre[q];
      Aim[(size_t)r * n + p.col[q]] = vim[q];
    }
  std::vector<double> bre(rre), bim(rim);
  for (int i = 0; i < n; ++i) {
    double best = 0.0;
    int row = i;
    for (int k = i; k < n; ++k) {
      const double mag = std::hypot(Are[(size_t)k * n + i], Aim[(size_t)k * n + i]);
      if (mag > best) {
        best = mag;
        row = k;
      } else if (mag == best && k < row) {
        row = k;
      }
    }
    if (best < 1e-25) return false;
    if (row != i) {
      for (int k = 0; k < n; ++k) {
        std::swap(Are[(size_t)i * n + k], Are[(size_t)row * n + k]);
        std::swap(Aim[(size_t)i * n + k], Aim[(size_t)row * n + k]);
      }
      std::swap(bre[i], bre[row]);
      std::swap(bim[i], bim[row]);
    }
    const double dre = Are[(size_t)i * n + i], dim = Aim[(size_t)i * n + i];
    const double den = dre * dre + dim * dim;
    for (int j = i + 1; j < n; ++j) {
      const double ar = Are[(size_t)j * n + i], ai = Aim[(size_t)j * n + i];
      const double fre = (ar * dre + ai * dim) / den;
      const double fim = (ai * dre - ar * dim) / den;
      Are[(size_t)j * n + i] = fre;
      Aim[(size_t)j * n + i] = fim;
      for (int k = i + 1; k < n; ++k) {
        Are[(size_t)j * n + k] -= fre * Are[(size_t)i * n + k] - fim * Aim[(size_t)i * n + k];
        Aim[(size_t)j * n + k] -= fre * Aim[(size_t)i * n + k] + fim * Are[(size_t)i * n + k];
      }
    }
  }
  std::vector<double> yre(n), yim(n);
  for (int i = 0; i < n; ++i) {
    yre[i] = bre[i];
    yim[i] = bim[i];
    for (int j = 0; j < i; ++j) {
      yre[i] -= Are[(size_t)i * n + j] * yre[j] - Aim[(size_t)i * n + j] * yim[j];
      yim[i] -= Are[(size_t)i * n + j] * yim[j] + Aim[(size_t)i * n + j] * yre[j];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double sre = yre[i], sim = yim[i];
    for (int j = i + 1; j < n; ++j) {
      sre -= Are[(size_t)i * n + j] * xre[j] - Aim[(size_t)i * n + j] * xim[j];
      sim -= Are[(size_t)i * n + j] * xim[j] + Aim[(size_t)i * n + j] * xre[j];
    }
    const double dre = Are[(size_t)i * n + i], dim = Aim[(size_t)i * n + i];
    const double den = dre * dre + dim * dim;
    xre[i] = (sre * dre + sim * dim) / den;
    xim[i] = (sim * dre - sre * dim) / den;
  }
  return true;
}

}  // namespace

extern "C" {

void oracle_default_opts(oracle_opts* o) {
  o->max_nr_iter = 50;
  o->gmin_steps = 19;
  o->reltol = 1e-3;
  o->vntol = 1e-6;
  o->kcl_shortcut = 1e-9;
  o->kcl_tol = 1e-12;
  o->polish_max = 0;
  o->polish_rel = 0.0;
  o->polish_abs = 0.0;
  o->linear_solver = ORACLE_LS_DENSE;
  o->seeded = 0;
  o->seed_max_iter = 10;
  o->max_halvings = 3;
  o->lte_rel = 0.0;
  o->lte_abs = 0.0;
}

int oracle_tensorize(const karam_netlist* nl, int32_t* mos_order, int32_t* dio_order) {
  return guarded([&] {
    Soa s = tensorize(nl);
    std::copy(s.mos_order.begin(), s.mos_order.end(), mos_order);
    std::copy(s.dio_order.begin(), s.dio_order.end(), dio_order);
    return 0;
  });
}

int oracle_pattern(const karam_netlist* nl, int32_t transient, int32_t* row_ptr, int32_t* col,
                   int32_t cap) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    Pattern p = s.b.pattern_for(transient != 0);
    if (row_ptr) std::copy(p.row_ptr.begin(), p.row_ptr.end(), row_ptr);
    if (col && (int)p.col.size() <= cap) std::copy(p.col.begin(), p.col.end(), col);
    return (int)p.col.size();
  });
}

int oracle_stamp_map(const karam_netlist* nl, int32_t* slot_csr, int32_t cap) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    auto& b = s.b;
    std::vector<double> v(b.n, 0.0), z(b.cap_c.size(), 0.0), vdc(b.soa.vs_pos.size(), 0.0);
    Stamp st;
    st.clear(b.n);
    Eval e;
    stamp_soa(b.soa, vdc, v, 1.0, z, z, st, e);
    for (int i = 0; i < b.n; ++i) st.add(i, i, 1e-12);
    int nt = (int)st.r.size();
    if (slot_csr && nt <= cap)
      for (int k = 0; k < nt; ++k) slot_csr[k] = b.cp.index_of(st.r[k], st.c[k]);
    return nt;
  });
}

int oracle_stamp(const karam_netlist* nl, const karam_instances* inst, int32_t idx,
                 const double* v, double h, int32_t method, const double* cap_vprev,
                 const double* cap_iprev, double t, double* vals, double* rhs) {
  return guarded([&] {
    Session s(nl, inst, idx);
    auto& b = s.b;
    std::vector<double> vv(v, v + b.n), cvp(b.cap_c.size(), 0.0), cip(b.cap_c.size(), 0.0);
    if (cap_vprev) cvp.assign(cap_vprev, cap_vprev + b.cap_c.size());
    if (cap_iprev) cip.assign(cap_iprev, cap_iprev + b.cap_c.size());
    std::vector<double> vl, r;
    b.stamp(vv, h, method, cvp, cip, t, vl, r);
    std::copy(vl.begin(), vl.end(), vals);
    std::copy(r.begin(), r.end(), rhs);
    return 0;
  });
}

int oracle_stamp_abs(const karam_netlist* nl, const karam_instances* inst, int32_t idx,
                     const double* v, double h, int32_t method, const double* cap_vprev,
                     const double* cap_iprev, double t, double* abs_vals, int32_t* n_terms) {
  return guarded([&] {
    Session s(nl, inst, idx);
    auto& b = s.b;
    std::vector<double> vv(v, v + b.n), cvp(b.cap_c.size(), 0.0), cip(b.cap_c.size(), 0.0);
    if (cap_vprev) cvp.assign(cap_vprev, cap_vprev + b.cap_c.size());
    if (cap_iprev) cip.assign(cap_iprev, cap_iprev + b.cap_c.size());
    std::vector<double> vl, r;
    b.stamp(vv, h, method, cvp, cip, t, vl, r);
    std::fill(abs_vals, abs_vals + vl.size(), 0.0);
    std::fill(n_terms, n_terms + vl.size(), 0);
    for (size_t k = 0; k < b.st.r.size(); ++k) {
      const int at = b.cp.index_of(b.st.r[k], b.st.c[k]);
      if (at < 0) continue;
      abs_vals[at] += std::fabs(b.st.v[k]);
      n_terms[at] += 1;
    }
    return 0;
  });
}

int oracle_ordering(const karam_netlist* nl, uint32_t* raw, int32_t* raw_len, int32_t* perm) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    MinFill mf = min_fill(s.b.soa, s.b.n);
    if (raw) std::copy(mf.ordering.begin(), mf.ordering.end(), raw);
    if (raw_len) *raw_len = (int32_t)mf.ordering.size();
    std::vector<uint32_t> p = translate(mf.ordering, s.b.n);
    if (perm) std::copy(p.begin(), p.end(), perm);
    return mf.treewidth;
  });
}

int oracle_symbolic(const karam_netlist* nl, int32_t* perm, int32_t* iperm, int32_t* f_row_ptr,
                    int32_t* f_col, int32_t* fill_in, int32_t cap) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    s.b.ensure_symbolic();
    const Symbolic& sy = s.b.sym;
    if (perm) std::copy(sy.perm.begin(), sy.perm.end(), perm);
    if (iperm) std::copy(sy.iperm.begin(), sy.iperm.end(), iperm);
    if (f_row_ptr) std::copy(sy.row_ptr.begin(), sy.row_ptr.end(), f_row_ptr);
    if (f_col && (int)sy.col.size() <= cap) std::copy(sy.col.begin(), sy.col.end(), f_col);
    if (fill_in) *fill_in = sy.fill;
    return (int)sy.col.size();
  });
}

int oracle_linsolve(const karam_netlist* nl, const double* vals, double gmin, const double* rhs,
                    int32_t solver, double* x) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    auto& b = s.b;
    std::vector<double> vl(vals, vals + b.pat.col.size()), r(rhs, rhs + b.n), xx;
    for (int i = 0; i < b.n; ++i) vl[b.pat.diag[i]] += gmin;
    if (!b.solve(vl, r, xx, solver)) return 1;
    std::copy(xx.begin(), xx.end(), x);
    return 0;
  });
}

int oracle_solve_dc(const karam_netlist* nl, const karam_instances* inst, int32_t idx,
                    const oracle_opts* opts, const double* v0, double* v_out, oracle_stats* st) {
  return guarded([&] {
    Session s(nl, inst, idx);
    oracle::Driver<PortBackend> d(s.b, *opts);
    std::vector<double> v;
    d.solve_dc(v0, v, st);
    std::copy(v.begin(), v.end(), v_out);
    return 0;
  });
}

int oracle_transient(const karam_netlist* nl, const karam_instances* inst, int32_t idx,
                     const oracle_opts* opts, const double* v_start, double dt, int32_t n_steps,
                     int32_t method, const int32_t* wave_nodes, int32_t n_wave, double* wave_out,
                     double* v_out, oracle_stats* st) {
  return guarded([&] {
    Session s(nl, inst, idx);
    oracle::Driver<PortBackend> d(s.b, *opts);
    std::vector<double> vs(v_start, v_start + s.b.n), v;
    d.transient(vs, dt, n_steps, method, wave_nodes, n_wave, wave_out, v, st);
    std::copy(v.begin(), v.end(), v_out);
    return 0;
  });
}

int oracle_run_batch(const karam_netlist* nl, const karam_instances* inst, int32_t i0, int32_t i1,
                     const oracle_opts* opts, double dt, int32_t n_steps, int32_t method,
                     int32_t n_threads, double* v_out, oracle_stats* st) {
  return guarded([&] {
    int count = i1 - i0;
    if (count <= 0) return 0;
    int nt = std::max(1, std::min<int>(n_threads, count));
    int n = 0;
    {
      Session probe(nl, nullptr, 0);
      n = probe.b.n;
    }
    std::vector<std::thread> pool;
    for (int w = 0; w < nt; ++w) {
      pool.emplace_back([&, w] {
        for (int i = i0 + w; i < i1; i += nt) {
          Session s(nl, inst, i);
          oracle::Driver<PortBackend> d(s.b, *opts);
          std::vector<double> v, v2;
          oracle_stats s1{}, s2{};
          d.solve_dc(nullptr, v, &s1);
          if (n_steps > 0 && s1.converged) {
            d.transient(v, dt, n_steps, method, nullptr, 0, nullptr, v2, &s2);
            v = v2;
            s1.iterations += s2.iterations;
            s1.polish_iters += s2.polish_iters;
            s1.converged = s2.converged;
            s1.max_step_iters = s2.max_step_iters;
          }
          std::copy(v.begin(), v.end(), v_out + (size_t)(i - i0) * n);
          st[i - i0] = s1;
        }
      });
    }
    for (auto& th : pool) th.join();
    return 0;
  });
}

int oracle_ac(const karam_netlist* nl, const karam_instances* inst, int32_t idx, const double* v_dc,
              double f_start, double f_stop, int32_t n_points, int32_t input_node, double amplitude,
              int32_t rule, double* out_re, double* out_im) {
  return guarded([&] {
    if (rule != 1) throw std::runtime_error("the port restates the Jacobian rule (1) only");
    Session s(nl, inst, idx);
    auto& b = s.b;
    std::vector<double> v(v_dc, v_dc + b.n), z(b.cap_c.size(), 0.0), jac, rhs;
    b.stamp(v, 0.0, KARAM_TRAN_BE, z, z, 0.0, jac, rhs);
    const std::vector<double> f = oracle::ac_frequencies(f_start, f_stop, n_points);
    int singular = 0;
    std::vector<double> re, im, rre, rim(b.n, 0.0), xre, xim;
    for (int k = 0; k < n_points; ++k) {
      oracle::ac_matrix(b.pat, jac, b.cap_n1, b.cap_n2, b.cap_c, 2.0 * M_PI * f[k], input_node,
                        amplitude, re, im, rre);
      if (!complex_lu_solve(b.pat, re, im, rre, rim, xre, xim)) {
        ++singular;
        std::fill(xre.begin(), xre.end(), 0.0);
        std::fill(xim.begin(), xim.end(), 0.0);
      }
      std::copy(xre.begin(), xre.end(), out_re + (size_t)k * b.n);
      std::copy(xim.begin(), xim.end(), out_im + (size_t)k * b.n);
    }
    return singular;
  });
}

}  // extern "C"
