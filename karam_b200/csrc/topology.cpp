// topology.cpp -- host symbolic layer (see topology.hpp).
#include "topology.hpp"

#include <algorithm>
#include <functional>
#include <iterator>
#include <cmath>
#include <cstdlib>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>

namespace karam {
namespace {

// Largest problem (unknowns, or Min-Fill vertices) whose host analysis keeps
// its structures as bit rows; larger ones use sorted vectors, ordered sets and
// hash sets. Both give identical tables. KARAM_BITROW_MAX, read once, moves
// the switch so that tests can run the large-problem code on small cases.
int bitrow_max() {
  static const int v = [] {
    const char* e = std::getenv("KARAM_BITROW_MAX");
    return e && *e ? std::atoi(e) : 16384;
  }();
  return v;
}

void require(bool ok, const std::string& msg) {
  if (!ok) throw std::runtime_error(msg);
}

inline int64_t key(int r, int c) { return (int64_t(r) << 32) | int64_t(uint32_t(c)); }

// Two-terminal conductance stamp: 4 triplets, or 1 when a terminal is ground
// (the pattern of every linear and diode stamp in stampSoABlock).
void stamp_g(std::vector<Triplet>& t, int n1, int n2, int kind, int idx) {
  if (n1 != 0 && n2 != 0) {
    t.push_back({n1 - 1, n1 - 1, -1, kind, idx, false});
    t.push_back({n2 - 1, n2 - 1, -1, kind, idx, false});
    t.push_back({n1 - 1, n2 - 1, -1, kind, idx, true});
    t.push_back({n2 - 1, n1 - 1, -1, kind, idx, true});
  } else if (n1 != 0) {
    t.push_back({n1 - 1, n1 - 1, -1, kind, idx, false});
  } else if (n2 != 0) {
    t.push_back({n2 - 1, n2 - 1, -1, kind, idx, false});
  }
}

void tensorize(const karam_netlist* nl, Topology& T) {
  require(nl != nullptr, "netlist is NULL");
  require(nl->n_nodes >= 0, "n_nodes must not be negative");
  require(nl->n_models >= 0 && nl->n_mos >= 0 && nl->n_dio >= 0 && nl->n_res >= 0 &&
              nl->n_cap >= 0 && nl->n_vsrc >= 0 && nl->n_isrc >= 0,
          "negative device count");
  int nmax = nl->n_nodes;
  auto node = [&](int x, const char* what) {
    require(x >= 0, std::string("negative node id in ") + what);
    nmax = std::max(nmax, x);
    return x;
  };
  auto model_name = [&](int m) {
    require(m >= 0 && m < nl->n_models && nl->model_name && nl->model_name[m],
            "model index out of range");
    return std::string(nl->model_name[m]);
  };
  T.temp_k = nl->temp_k > 0 ? nl->temp_k : 300.15;
  const double tscale = T.temp_k / 300.15;

  // Devices regrouped per model name, std::map order (physics_tensors.cpp:481-490).
  std::map<std::string, std::vector<int>> mb, db;
  for (int i = 0; i < nl->n_mos; ++i) {
    int m = nl->m_model ? nl->m_model[i] : -1;
    std::string nm = model_name(m);
    int ty = nl->model_type[m];
    require(ty == KARAM_MODEL_NMOS || ty == KARAM_MODEL_PMOS, "MOSFET model is not NMOS/PMOS");
    mb[nm].push_back(i);
  }
  for (int i = 0; i < nl->n_dio; ++i) {
    int m = nl->d_model ? nl->d_model[i] : -1;
    db[m >= 0 ? model_name(m) : std::string("diode_generic")].push_back(i);
  }
  for (auto& kv : db)
    for (int i : kv.second) {
      require(nl->d_is[i] > 0 && nl->d_n[i] > 0 && nl->d_vt[i] > 0, "diode Is/N/Vt must be > 0");
      T.dio.push_back({node(nl->d_anode[i], "diode"), node(nl->d_cathode[i], "diode"), nl->d_is[i],
                       nl->d_n[i], nl->d_vt[i] * tscale});
      T.dio_order.push_back(i);
    }
  for (auto& kv : mb)
    for (int i : kv.second) {
      int m = nl->m_model[i];
      bool pmos = nl->model_type[m] == KARAM_MODEL_PMOS;
      auto card = [&](const double* a, double dflt) {
        return (a && !std::isnan(a[m])) ? a[m] : dflt;
      };
      require(nl->m_w[i] > 0 && nl->m_l[i] > 0, "MOSFET W and L must be > 0");
      Topology::Mos q;
      q.d = node(nl->m_d[i], "mosfet");
      q.g = node(nl->m_g[i], "mosfet");
      q.s = node(nl->m_s[i], "mosfet");
      q.b = node(nl->m_b[i], "mosfet");
      q.w = nl->m_w[i];
      q.l = nl->m_l[i];
      q.wl = q.w / q.l;
      q.kp_card = card(nl->model_kp, pmos ? 100e-6 : 200e-6);
      q.vto_card = card(nl->model_vto, pmos ? -0.7 : 0.7);
      q.lam = card(nl->model_lambda, 0.02);
      q.pmos = pmos;
      T.mos.push_back(q);
      T.mos_order.push_back(i);
    }
  for (int i = 0; i < nl->n_res; ++i) {
    require(nl->r_ohm[i] > 0 && std::isfinite(nl->r_ohm[i]), "resistance must be finite and > 0");
    T.res.push_back({node(nl->r_n1[i], "resistor"), node(nl->r_n2[i], "resistor"), nl->r_ohm[i]});
  }
  for (int i = 0; i < nl->n_cap; ++i) {
    require(nl->c_farad[i] >= 0 && std::isfinite(nl->c_farad[i]), "capacitance must be >= 0");
    T.cap.push_back({node(nl->c_n1[i], "capacitor"), node(nl->c_n2[i], "capacitor"), nl->c_farad[i]});
  }
  for (int i = 0; i < nl->n_isrc; ++i)
    T.isrc.push_back({node(nl->is_pos[i], "isource"), node(nl->is_neg[i], "isource"), nl->is_amp[i]});
  for (int i = 0; i < nl->n_vsrc; ++i) {
    Topology::Vs v{};
    v.pos = node(nl->vs_pos[i], "vsource");
    v.neg = node(nl->vs_neg[i], "vsource");
    v.kind = nl->vs_kind ? nl->vs_kind[i] : KARAM_SRC_DC;
    require(v.kind == KARAM_SRC_DC || v.kind == KARAM_SRC_PULSE, "unknown source kind");
    v.dc = nl->vs_dc[i];
    if (v.kind == KARAM_SRC_PULSE) {
      require(nl->vs_pulse != nullptr, "PULSE source without parameters");
      for (int k = 0; k < 7; ++k) v.pulse[k] = nl->vs_pulse[7 * i + k];
    }
    T.vs.push_back(v);
  }
  for (int i = 0; i < nl->n_dio; ++i) T.seed_anodes.push_back(nl->d_anode[i]);
  T.n = nmax;
  require(T.n >= 1, "netlist has no unknowns");
}

// Stamp slots in stampSoABlock order (transient pattern: capacitor companions
// included) followed by the gmin diagonal of addDiagonalConditioning.
void stamps(Topology& T) {
  auto& t = T.trip;
  for (size_t i = 0; i < T.res.size(); ++i) stamp_g(t, T.res[i].n1, T.res[i].n2, SS_RES, (int)i);
  for (size_t i = 0; i < T.vs.size(); ++i) stamp_g(t, T.vs[i].pos, T.vs[i].neg, SS_VS, (int)i);
  for (size_t i = 0; i < T.cap.size(); ++i) stamp_g(t, T.cap[i].n1, T.cap[i].n2, SS_CAP, (int)i);
  for (size_t i = 0; i < T.dio.size(); ++i) stamp_g(t, T.dio[i].a, T.dio[i].c, SS_DIO, (int)i);
  for (size_t i = 0; i < T.mos.size(); ++i) {
    const auto& q = T.mos[i];
    int d = q.d, g = q.g, s = q.s, b = q.b, k = (int)i;
    stamp_g(t, d, s, SS_MOS_GDS, k);
    if (d != 0) {
      if (g != 0) t.push_back({d - 1, g - 1, -1, SS_MOS_GM, k, false});
      if (s != 0) t.push_back({d - 1, s - 1, -1, SS_MOS_GM, k, true});
    }
    if (s != 0) {
      if (g != 0) t.push_back({s - 1, g - 1, -1, SS_MOS_GM, k, true});
      t.push_back({s - 1, s - 1, -1, SS_MOS_GM, k, false});
    }
    if (d != 0) {
      if (b != 0) t.push_back({d - 1, b - 1, -1, SS_MOS_GMB, k, false});
      if (s != 0) t.push_back({d - 1, s - 1, -1, SS_MOS_GMB, k, true});
    }
    if (s != 0) {
      if (b != 0) t.push_back({s - 1, b - 1, -1, SS_MOS_GMB, k, true});
      t.push_back({s - 1, s - 1, -1, SS_MOS_GMB, k, false});
    }
  }
  for (int i = 0; i < T.n; ++i) t.push_back({i, i, -1, SS_GMIN, i, false});

  // CSR pattern: sorted (row, col), duplicates merged (createCsr, linalg.h:281-411).
  std::vector<int64_t> keys;
  keys.reserve(t.size());
  for (auto& x : t) keys.push_back(key(x.row, x.col));
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  T.row_ptr.assign(T.n + 1, 0);
  T.col.resize(keys.size());
  std::unordered_map<int64_t, int> pos;
  pos.reserve(keys.size() * 2);
  for (size_t k = 0; k < keys.size(); ++k) {
    int r = int(keys[k] >> 32);
    T.row_ptr[r + 1]++;
    T.col[k] = int(uint32_t(keys[k]));
    pos[keys[k]] = (int)k;
  }
  for (int i = 0; i < T.n; ++i) T.row_ptr[i + 1] += T.row_ptr[i];
  T.slot_csr.resize(t.size());
  for (size_t k = 0; k < t.size(); ++k) T.slot_csr[k] = pos[key(t[k].row, t[k].col)];
}

// Factor graph of FactorGraph::fromTensorizedBlock: one factor per device over
// its non-ground terminals; voltage sources add a branch-current variable whose
// id starts at the node count (so the first one shares its id with node n).
void ordering(Topology& T) {
  std::vector<std::vector<uint32_t>> factors;
  std::set<uint32_t> volt;
  uint32_t bid = (uint32_t)T.n, nbranch = 0;
  auto add = [&](std::initializer_list<int> nodes, bool branch) {
    std::vector<uint32_t> f;
    for (int x : nodes)
      if (x > 0) {
        f.push_back((uint32_t)x);
        volt.insert((uint32_t)x);
      }
    if (branch) {
      f.push_back(bid++);
      ++nbranch;
    }
    factors.push_back(std::move(f));
  };
  for (auto& d : T.dio) add({d.a, d.c}, false);
  for (auto& m : T.mos) add({m.d, m.g, m.s, m.b}, false);
  for (auto& r : T.res) add({r.n1, r.n2}, false);
  for (auto& c : T.cap) add({c.n1, c.n2}, false);
  for (auto& v : T.vs) add({v.pos, v.neg}, true);
  for (auto& c : T.isrc) add({c.n1, c.n2}, false);
  std::vector<uint32_t> vars(volt.begin(), volt.end());
  for (uint32_t k = 0; k < nbranch; ++k) vars.push_back((uint32_t)T.n + k);
  MinFillResult mf = min_fill(factors, vars);
  T.raw_order = mf.ordering;
  T.treewidth = mf.treewidth;
  // Translation to a 0-based permutation of the unknowns: ids 1..n kept in
  // order of first appearance, branch ids and repeats dropped; unknowns no
  // device touches go last.
  std::vector<char> seen(T.n + 1, 0);
  T.perm.clear();
  for (uint32_t id : mf.ordering)
    if (id >= 1 && id <= (uint32_t)T.n && !seen[id]) {
      seen[id] = 1;
      T.perm.push_back((int)id - 1);
    }
  for (int i = 1; i <= T.n; ++i)
    if (!seen[i]) T.perm.push_back(i - 1);
  T.iperm.assign(T.n, 0);
  for (int i = 0; i < T.n; ++i) T.iperm[T.perm[i]] = i;
}

// symbolicFactorize (math/sparse_lu.cpp:14-128): eliminate in permuted order
// on the undirected CSR graph; row k of U (and column k of L) holds the
// permuted indices of the neighbours of the k-th eliminated unknown.
void symbolic(Topology& T, std::vector<std::vector<int>>& urow) {
  const int n = T.n;
  std::vector<std::unordered_set<int>> adj(n);
  for (int r = 0; r < n; ++r)
    for (int k = T.row_ptr[r]; k < T.row_ptr[r + 1]; ++k) {
      int c = T.col[k];
      if (c != r) {
        adj[r].insert(c);
        adj[c].insert(r);
      }
    }
  urow.assign(n, {});
  int fill = 0;
  std::vector<int> nb;
  for (int step = 0; step < n; ++step) {
    int v = T.perm[step];
    nb.assign(adj[v].begin(), adj[v].end());
    std::sort(nb.begin(), nb.end());
    auto& ur = urow[step];
    for (int u : nb) ur.push_back(T.iperm[u]);
    std::sort(ur.begin(), ur.end());
    for (size_t i = 0; i < nb.size(); ++i)
      for (size_t j = i + 1; j < nb.size(); ++j)
        if (adj[nb[i]].insert(nb[j]).second) {
          adj[nb[j]].insert(nb[i]);
          ++fill;
        }
    for (int u : nb) adj[u].erase(v);
    adj[v].clear();
  }
  T.fill_in = fill;
  // filled CSR (symmetric structure): row i = {k < i : i in urow[k]} + {i} + urow[i]
  std::vector<std::vector<int>> lcols(n);
  for (int k = 0; k < n; ++k)
    for (int j : urow[k]) lcols[j].push_back(k);
  T.f_row_ptr.assign(n + 1, 0);
  T.f_col.clear();
  T.f_diag.assign(n, -1);
  for (int i = 0; i < n; ++i) {
    T.f_row_ptr[i] = (int)T.f_col.size();
    for (int k : lcols[i]) T.f_col.push_back(k);  // ascending by construction
    T.f_diag[i] = (int)T.f_col.size();
    T.f_col.push_back(i);
    for (int j : urow[i]) T.f_col.push_back(j);
  }
  T.f_row_ptr[n] = (int)T.f_col.size();
}

void device_tables(Topology& T, const std::vector<std::vector<int>>& urow) {
  const int n = T.n, nf = T.nnz_filled();
  // position of (pr, pc) in the filled CSR: each row's columns ascend
  auto fp = [&](int pr, int pc) {
    const int* row = T.f_col.data() + T.f_row_ptr[pr];
    const int* end = T.f_col.data() + T.f_row_ptr[pr + 1];
    const int* it = std::lower_bound(row, end, pc);
    require(it != end && *it == pc, "filled pattern misses a position");
    return (int)(it - T.f_col.data());
  };
  for (auto& x : T.trip) x.f = fp(T.iperm[x.row], T.iperm[x.col]);

  auto flatten = [](const std::vector<std::vector<int>>& v, std::vector<int>& off,
                    std::vector<int>& code) {
    off.assign(v.size() + 1, 0);
    code.clear();
    for (size_t i = 0; i < v.size(); ++i) {
      off[i] = (int)code.size();
      code.insert(code.end(), v[i].begin(), v[i].end());
    }
    off[v.size()] = (int)code.size();
  };
  // KCL gather tables per permuted node: currents leaving the node.
  std::vector<std::vector<int>> ft(n);
  auto two = [&](int n1, int n2, int kind, int idx) {
    if (n1 > 0) ft[T.iperm[n1 - 1]].push_back(term(kind, idx, false));
    if (n2 > 0) ft[T.iperm[n2 - 1]].push_back(term(kind, idx, true));
  };
  for (size_t i = 0; i < T.res.size(); ++i) two(T.res[i].n1, T.res[i].n2, FK_RES, (int)i);
  for (size_t i = 0; i < T.vs.size(); ++i) two(T.vs[i].pos, T.vs[i].neg, FK_VS, (int)i);
  for (size_t i = 0; i < T.isrc.size(); ++i) two(T.isrc[i].n1, T.isrc[i].n2, FK_IS, (int)i);
  for (size_t i = 0; i < T.cap.size(); ++i) two(T.cap[i].n1, T.cap[i].n2, FK_CAP, (int)i);
  for (size_t i = 0; i < T.dio.size(); ++i) two(T.dio[i].a, T.dio[i].c, FK_DIO, (int)i);
  for (size_t i = 0; i < T.mos.size(); ++i) two(T.mos[i].d, T.mos[i].s, FK_MOS, (int)i);
  flatten(ft, T.ft_off, T.ft_code);

  // LU program on the numerically non-zero part of the filled pattern. The
  // filled pattern of symbolicFactorize is symmetric, but the MNA stamps are
  // not (a MOSFET stamps its drain/source rows, never its gate row), so many
  // positions of it hold zeros that stay zero through the elimination. The
  // program keeps the reference's ordering and pattern and skips those: it
  // eliminates on the unsymmetric structure of the stamps (gmb stamps, always
  // zero in the level-1 kernel, excluded), which is a subset of the filled
  // pattern, so results equal the full static elimination's.
  // Structure as bit rows and columns up to 16384 unknowns, else sorted
  // vectors (row -> cols, col -> rows, permuted); L and U of a pivot come out
  // ascending either way.
  const bool nzbits = n <= bitrow_max();
  const size_t W = ((size_t)n + 63) / 64;
  std::vector<uint64_t> nzrb(nzbits ? W * (size_t)n : 0), nzcb(nzbits ? W * (size_t)n : 0);
  std::vector<std::vector<int>> nzr(nzbits ? 0 : n), nzc(nzbits ? 0 : n);
  auto add_nz = [&](int r, int c) {
    if (nzbits) {
      nzrb[(size_t)r * W + (c >> 6)] |= 1ull << (c & 63);
      nzcb[(size_t)c * W + (r >> 6)] |= 1ull << (r & 63);
      return;
    }
    auto& row = nzr[r];
    auto it = std::lower_bound(row.begin(), row.end(), c);
    if (it != row.end() && *it == c) return;
    row.insert(it, c);
    auto& col = nzc[c];
    col.insert(std::lower_bound(col.begin(), col.end(), r), r);
  };
  for (auto& x : T.trip)
    if (x.kind != SS_MOS_GMB) add_nz(T.iperm[x.row], T.iperm[x.col]);
  T.lu_hdr.assign(4 * (size_t)n, 0);
  T.lu_data.clear();
  T.lu_ops = 0;
  T.max_d = 0;
  std::vector<int> L, U, merged;
  for (int k = 0; k < n; ++k) {
    L.clear();
    U.clear();
    if (nzbits) {
      auto above = [&](const std::vector<uint64_t>& B, std::vector<int>& out) {
        const uint64_t* row = &B[(size_t)k * W];
        const size_t q0 = (size_t)(k + 1) >> 6;
        for (size_t q = q0; q < W; ++q) {
          uint64_t c = row[q];
          if (q == q0) c &= ~0ull << ((k + 1) & 63);
          for (; c; c &= c - 1) out.push_back((int)(q * 64 + (size_t)__builtin_ctzll(c)));
        }
      };
      above(nzcb, L);
      above(nzrb, U);
    } else {
      for (int i : nzc[k])
        if (i > k) L.push_back(i);
      for (int j : nzr[k])
        if (j > k) U.push_back(j);
    }
    if (nzbits) {
      for (int i : L)
        for (int j : U) add_nz(i, j);
    } else {  // L and U ascend: one sorted union per row and per column
      for (int i : L) {
        merged.clear();
        std::set_union(nzr[i].begin(), nzr[i].end(), U.begin(), U.end(), std::back_inserter(merged));
        nzr[i].swap(merged);
      }
      for (int j : U) {
        merged.clear();
        std::set_union(nzc[j].begin(), nzc[j].end(), L.begin(), L.end(), std::back_inserter(merged));
        nzc[j].swap(merged);
      }
    }
    const int nl = (int)L.size(), nu = (int)U.size();
    T.max_d = std::max({T.max_d, nl, nu});
    T.lu_hdr[4 * k + 0] = (int)T.lu_data.size();
    T.lu_hdr[4 * k + 1] = nl;
    T.lu_hdr[4 * k + 2] = nu;
    T.lu_hdr[4 * k + 3] = T.f_diag[k];
    for (int i : L) T.lu_data.push_back(i);
    for (int i : L) T.lu_data.push_back(fp(i, k));
    for (int j : U) T.lu_data.push_back(j);
    for (int j : U) T.lu_data.push_back(fp(k, j));
    // positions of (i, j), j in U, by one walk along row i's filled columns
    // (U ascends and lies in them)
    const int* fcol = T.f_col.data();
    for (int i : L) {
      const int* end = fcol + T.f_row_ptr[i + 1];
      const int* it = nu ? std::lower_bound(fcol + T.f_row_ptr[i], end, U.front()) : end;
      for (int j : U) {
        while (it != end && *it < j) ++it;
        require(it != end && *it == j, "filled pattern misses a position");
        T.lu_data.push_back((int)(it - fcol));
      }
    }
    T.lu_ops += nl + nl * nu;
  }

  // Value slots: the filled positions the static-pivot elimination can make
  // non-zero (every position the program reads or writes), numbered
  // row-major. The device stores and factors only these.
  T.f_slot.assign(nf, -1);
  for (int k = 0; k < n; ++k) {
    const int off = T.lu_hdr[4 * k], nl = T.lu_hdr[4 * k + 1], nu = T.lu_hdr[4 * k + 2];
    T.f_slot[T.lu_hdr[4 * k + 3]] = 0;
    for (int q = off + nl; q < off + 2 * nl; ++q) T.f_slot[T.lu_data[q]] = 0;
    for (int q = off + 2 * nl + nu; q < off + 2 * nl + 2 * nu + nl * nu; ++q) T.f_slot[T.lu_data[q]] = 0;
  }
  T.nv = 0;
  T.slot_row.clear();
  T.slot_col.clear();
  for (int i = 0; i < n; ++i)
    for (int f = T.f_row_ptr[i]; f < T.f_row_ptr[i + 1]; ++f)
      if (T.f_slot[f] >= 0) {
        T.f_slot[f] = T.nv++;
        T.slot_row.push_back(i);
        T.slot_col.push_back(T.f_col[f]);
      }
  for (int k = 0; k < n; ++k) {
    const int off = T.lu_hdr[4 * k], nl = T.lu_hdr[4 * k + 1], nu = T.lu_hdr[4 * k + 2];
    T.lu_hdr[4 * k + 3] = T.f_slot[T.lu_hdr[4 * k + 3]];
    for (int q = off + nl; q < off + 2 * nl; ++q) T.lu_data[q] = T.f_slot[T.lu_data[q]];
    for (int q = off + 2 * nl + nu; q < off + 2 * nl + 2 * nu + nl * nu; ++q)
      T.lu_data[q] = T.f_slot[T.lu_data[q]];
  }

  // Jacobian gather tables per value slot, summation order = triplet order.
  std::vector<std::vector<int>> jt(T.nv), jc(T.nv);
  T.jlin_dc.assign(T.nv, 0.0);
  for (auto& x : T.trip) {
    if (x.kind == SS_MOS_GMB || x.kind == SS_GMIN) continue;  // gmb is always 0; gmin is added per solve
    const int sl = T.f_slot[x.f];
    require(sl >= 0, "a stamped position is outside the LU structure");
    switch (x.kind) {
      case SS_RES: {
        double g = 1.0 / T.res[x.idx].val;
        T.jlin_dc[sl] += x.neg ? -g : g;
        break;
      }
      case SS_VS:
        T.jlin_dc[sl] += x.neg ? -1.0e3 : 1.0e3;
        break;
      case SS_CAP:
        jc[sl].push_back(term(0, x.idx, x.neg));
        break;
      case SS_DIO:
        jt[sl].push_back(term(JK_DIO_G, x.idx, x.neg));
        break;
      case SS_MOS_GDS:
        jt[sl].push_back(term(JK_MOS_GDS, x.idx, x.neg));
        break;
      case SS_MOS_GM:
        jt[sl].push_back(term(JK_MOS_GM, x.idx, x.neg));
        break;
      default:
        break;
    }
  }
  flatten(jt, T.jt_off, T.jt_code);
  flatten(jc, T.jcap_off, T.jcap_code);

  // Pivot records for programs whose pivots all have nL <= 1 and nU <= 2
  // (chain-like circuits), 8 ints per pivot:
  //   meta = nL | nU << 4 | chain << 8 | back-forwarding << 9
  //   then diagonal slot, Lslot0, Lrow0, Uslot0, Uslot1, T00, T01
  // and 2 ints per pivot for the back substitution: Ucol0, Ucol1 (lu_rec2).
  // "chain" marks a pivot whose L value and second target are the previous
  // pivot's targets and whose L row's right-hand side the previous pivot wrote
  // (so the device keeps them in registers), with no other read touching what
  // the previous pivot wrote (so its loads may be issued early).
  // Back-forwarding bit b: Ucol b is the unknown the previous back-substitution
  // step solved.
  T.lu_small = T.n < (1 << 24) && T.nv < (1 << 24);
  for (int k = 0; k < n && T.lu_small; ++k)
    if (T.lu_hdr[4 * k + 1] > 1 || T.lu_hdr[4 * k + 2] > 2) T.lu_small = false;
  T.lu_rec.clear();
  T.lu_rec2.clear();
  if (T.lu_small) {
    T.lu_rec.assign(8 * (size_t)n, 0);
    T.lu_rec2.assign(2 * (size_t)n, 0);
    struct Piv { int d, nl, nu, lr, ls, us[2], uc[2], t[2]; };
    std::vector<Piv> pv(n);
    for (int k = 0; k < n; ++k) {
      const int off = T.lu_hdr[4 * k], nl = T.lu_hdr[4 * k + 1], nu = T.lu_hdr[4 * k + 2];
      const int* d = &T.lu_data[off];
      Piv& q = pv[k];
      q = Piv{};
      q.d = T.lu_hdr[4 * k + 3];
      q.nl = nl;
      q.nu = nu;
      if (nl > 0) {
        q.lr = d[0];
        q.ls = d[1];
      }
      for (int b = 0; b < nu; ++b) {
        q.uc[b] = d[2 * nl + b];
        q.us[b] = d[2 * nl + nu + b];
        if (nl > 0) q.t[b] = d[2 * nl + 2 * nu + b];
      }
    }
    for (int k = 0; k < n; ++k) {
      const Piv& q = pv[k];
      bool chain = false;
      if (k > 0 && q.nl == 1 && q.nu == 2) {
        const Piv& p = pv[k - 1];
        auto written = [&](int slot) {
          if (slot == p.d) return true;
          if (p.nl > 0 && slot == p.ls) return true;
          for (int b = 0; b < p.nu && p.nl > 0; ++b)
            if (slot == p.t[b]) return true;
          return false;
        };
        chain = p.nl == 1 && p.nu == 2 && q.ls == p.t[0] && q.t[1] == p.t[1] && q.lr == p.lr &&
                !written(q.d) && !written(q.us[0]) && !written(q.us[1]) && !written(q.t[0]) &&
                k != p.lr;
      }
      unsigned fb = 0;
      if (k + 1 < n) {
        if (q.nu > 0 && q.uc[0] == k + 1) fb |= 1u;
        if (q.nu > 1 && q.uc[1] == k + 1) fb |= 2u;
      }
      int* w = &T.lu_rec[8 * (size_t)k];
      w[0] = (int)((unsigned)q.nl | (unsigned)q.nu << 4 | (chain ? 1u : 0u) << 8 | fb << 9);
      w[1] = q.d;
      w[2] = q.ls;
      w[3] = q.lr;
      w[4] = q.us[0];
      w[5] = q.us[1];
      w[6] = q.t[0];
      w[7] = q.t[1];
      T.lu_rec2[2 * (size_t)k] = q.uc[0];
      T.lu_rec2[2 * (size_t)k + 1] = q.uc[1];
    }
  }

  // Junction limiting constants (applyPnJunctionLimits, circuitsim_solver.cpp:118-169):
  // the reference recomputes them on every call with these expressions.
  const double ts = T.temp_k / 300.15;
  std::vector<int> last(n + 1, -1);
  T.dio_lim.clear();
  T.dio_level.clear();
  T.n_dio_levels = 0;
  for (const auto& d : T.dio) {
    double vt = d.vt * ts;
    double is = d.is * std::pow(ts, 3.0) * std::exp(1.11 / (vt / ts) - 1.11 / vt);
    T.dio_lim.push_back(vt);
    T.dio_lim.push_back(vt * std::log(vt / (std::sqrt(2.0) * is)));
    int lvl = 0;
    if (d.a > 0) lvl = std::max(lvl, last[d.a] + 1);
    if (d.c > 0) lvl = std::max(lvl, last[d.c] + 1);
    if (d.a > 0) last[d.a] = lvl;
    if (d.c > 0) last[d.c] = lvl;
    T.dio_level.push_back(lvl);
    T.n_dio_levels = std::max(T.n_dio_levels, lvl + 1);
  }

  auto pn = [&](int node) { return node > 0 ? T.iperm[node - 1] : -1; };
  for (auto& m : T.mos) {
    T.mos_term.push_back(pn(m.d));
    T.mos_term.push_back(pn(m.g));
    T.mos_term.push_back(pn(m.s));
    T.mos_term.push_back(pn(m.b));
  }
  for (auto& d : T.dio) {
    T.dio_term.push_back(pn(d.a));
    T.dio_term.push_back(pn(d.c));
  }
  for (auto& r : T.res) { T.res_term.push_back(pn(r.n1)); T.res_term.push_back(pn(r.n2)); }
  for (auto& c : T.cap) { T.cap_term.push_back(pn(c.n1)); T.cap_term.push_back(pn(c.n2)); }
  for (auto& v : T.vs) { T.vs_term.push_back(pn(v.pos)); T.vs_term.push_back(pn(v.neg)); }
  for (auto& c : T.isrc) { T.is_term.push_back(pn(c.n1)); T.is_term.push_back(pn(c.n2)); }
}

// Level schedule of the factor/solve kernel's LU (Topology::nd_*): the
// static-pivot elimination of the Min-Fill system in a nested-dissection
// order, so that pivots with no dependency between them run side by side.
//  - Order: vertices of degree > 32 (supply hubs) last; the rest by recursive
//    bisection with the middle BFS level from a pseudo-peripheral vertex as
//    separator, separators after both halves (deterministic: ties to the
//    smallest index).
//  - Structure: the stamped positions and the diagonal, eliminated
//    unsymmetrically (pivot k fills (i, j) for i in L_k, j in U_k).
//  - Levels: pivot m depends on k when k's elimination writes row or column
//    m (m in L_k or U_k); level(m) = 1 + the largest level it depends on.
//    Within a level no pivot reads what another writes; two pivots updating
//    the same target are summed in one list, in pivot order.
void nd_schedule(Topology& T) {
  const int n = T.n;
  T.nd_levels = 0;
  // past ~7e4 unknowns the host build takes minutes and one CTA per instance
  // is the wrong shape for the factorization
  if (n < 2 || n > 70000) return;
  auto key = [](int r, int c) { return (int64_t(r) << 32) | int64_t(unsigned(c)); };
  // stamped positions (Min-Fill permuted space)
  std::vector<std::pair<int, int>> pos;
  for (const auto& x : T.trip) {
    const int sl = T.f_slot[x.f];
    if (sl >= 0) pos.emplace_back(T.slot_row[sl], T.slot_col[sl]);
  }
  for (int i = 0; i < n; ++i) pos.emplace_back(i, i);
  std::vector<std::vector<int>> adj(n);
  for (auto& q : pos)
    if (q.first != q.second) {
      adj[q.first].push_back(q.second);
      adj[q.second].push_back(q.first);
    }
  for (auto& a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  std::vector<char> hub(n, 0);
  for (int i = 0; i < n; ++i) hub[i] = adj[i].size() > 32;
  std::vector<int> order;
  order.reserve(n);
  std::vector<int> mark(n, -1), lev(n, -1);
  int stamp = 0;
  // recursive nested dissection on the vertex set `nodes` (sorted)
  std::function<void(std::vector<int>&)> nd = [&](std::vector<int>& nodes) {
    if (nodes.size() <= 2) {
      order.insert(order.end(), nodes.begin(), nodes.end());
      return;
    }
    const int in_set = stamp++;
    for (int v : nodes) mark[v] = in_set;
    // components, each from its smallest vertex
    std::vector<std::vector<int>> comps;
    const int seen = stamp++;
    for (int s0 : nodes) {
      if (mark[s0] != in_set) continue;
      std::vector<int> comp{s0};
      mark[s0] = seen;
      for (size_t h = 0; h < comp.size(); ++h)
        for (int w : adj[comp[h]])
          if (mark[w] == in_set) {
            mark[w] = seen;
            comp.push_back(w);
          }
      std::sort(comp.begin(), comp.end());
      comps.push_back(std::move(comp));
    }
    if (comps.size() > 1) {
      for (auto& c : comps) nd(c);
      return;
    }
    std::vector<int>& comp = comps[0];
    const int cur = stamp++;
    for (int v : comp) mark[v] = cur;
    auto bfs = [&](int src, std::vector<int>& seq) {
      seq.clear();
      seq.push_back(src);
      const int vis = stamp++;
      lev[src] = 0;
      std::vector<int> visited{src};
      mark[src] = vis;
      for (size_t h = 0; h < seq.size(); ++h)
        for (int w : adj[seq[h]])
          if (mark[w] == cur) {
            mark[w] = vis;
            lev[w] = lev[seq[h]] + 1;
            seq.push_back(w);
          }
      for (int v : seq) mark[v] = cur;  // back into the component
    };
    std::vector<int> seq;
    bfs(comp[0], seq);
    int far = seq[0];
    for (int v : seq)
      if (lev[v] > lev[far] || (lev[v] == lev[far] && v < far)) far = v;
    bfs(far, seq);
    int L = 0;
    for (int v : seq) L = std::max(L, lev[v]);
    if (L < 2) {
      order.insert(order.end(), comp.begin(), comp.end());
      return;
    }
    const int mid = L / 2;
    std::vector<int> a, b, sep;
    for (int v : comp) (lev[v] < mid ? a : (lev[v] > mid ? b : sep)).push_back(v);
    nd(a);
    nd(b);
    order.insert(order.end(), sep.begin(), sep.end());
  };
  std::vector<int> rest;
  for (int i = 0; i < n; ++i)
    if (!hub[i]) rest.push_back(i);
  // hubs leave the graph the dissection sees
  for (int i = 0; i < n; ++i)
    if (hub[i]) mark[i] = -2;
  {
    std::vector<std::vector<int>> adj2(n);
    for (int i = 0; i < n; ++i)
      if (!hub[i])
        for (int w : adj[i])
          if (!hub[w]) adj2[i].push_back(w);
    adj.swap(adj2);
  }
  nd(rest);
  for (int i = 0; i < n; ++i)
    if (hub[i]) order.push_back(i);
  if ((int)order.size() != n) return;
  T.nd_perm = order;
  T.nd_pos.assign(n, 0);
  for (int p = 0; p < n; ++p) T.nd_pos[order[p]] = p;

  // unsymmetric symbolic elimination in ND order (rows and columns as bit
  // rows up to 16384 unknowns, else sorted vectors; the same structure either
  // way), then each row's columns in ascending order
  std::vector<std::vector<int>> Lk(n), Uk(n), Rrow(n);
  if (n <= bitrow_max()) {
    const size_t W = ((size_t)n + 63) / 64;
    std::vector<uint64_t> Rb(W * (size_t)n, 0), Cb(W * (size_t)n, 0);
    auto set_bit = [&](std::vector<uint64_t>& B, int a, int b) { B[(size_t)a * W + (b >> 6)] |= 1ull << (b & 63); };
    for (auto& q : pos) {
      const int r = T.nd_pos[q.first], c = T.nd_pos[q.second];
      set_bit(Rb, r, c);
      set_bit(Cb, c, r);
    }
    auto above = [&](const std::vector<uint64_t>& B, int k, std::vector<int>& out) {
      const uint64_t* row = &B[(size_t)k * W];
      for (size_t q = (size_t)(k + 1) >> 6; q < W; ++q) {
        uint64_t c = row[q];
        if (q == ((size_t)(k + 1) >> 6)) c &= ~0ull << ((k + 1) & 63);
        while (c) {
          out.push_back((int)(q * 64 + (size_t)__builtin_ctzll(c)));
          c &= c - 1;
        }
      }
    };
    std::vector<uint64_t> ub(W);
    for (int k = 0; k < n; ++k) {
      above(Cb, k, Lk[k]);
      above(Rb, k, Uk[k]);
      if (Uk[k].empty()) continue;
      std::fill(ub.begin(), ub.end(), 0ull);
      for (int j : Uk[k]) ub[j >> 6] |= 1ull << (j & 63);
      const size_t q0 = (size_t)Uk[k].front() >> 6, q1 = (size_t)Uk[k].back() >> 6;
      for (int i : Lk[k]) {
        uint64_t* ri = &Rb[(size_t)i * W];
        for (size_t q = q0; q <= q1; ++q) {
          uint64_t fresh = ub[q] & ~ri[q];
          ri[q] |= ub[q];
          while (fresh) {
            const int j = (int)(q * 64 + (size_t)__builtin_ctzll(fresh));
            set_bit(Cb, j, i);
            fresh &= fresh - 1;
          }
        }
      }
    }
    for (int r = 0; r < n; ++r) {  // every column of the row, ascending
      const uint64_t* row = &Rb[(size_t)r * W];
      for (size_t q = 0; q < W; ++q)
        for (uint64_t c = row[q]; c; c &= c - 1) Rrow[r].push_back((int)(q * 64 + (size_t)__builtin_ctzll(c)));
    }
  } else {  // sorted vectors; pivot k's fill is one sorted union per row and per column
    std::vector<std::vector<int>> R(n), Cc(n);
    for (auto& q : pos) {
      const int r = T.nd_pos[q.first], c = T.nd_pos[q.second];
      R[r].push_back(c);
      Cc[c].push_back(r);
    }
    for (auto* v : {&R, &Cc})
      for (auto& x : *v) {
        std::sort(x.begin(), x.end());
        x.erase(std::unique(x.begin(), x.end()), x.end());
      }
    std::vector<int> merged;
    for (int k = 0; k < n; ++k) {
      Lk[k].assign(std::upper_bound(Cc[k].begin(), Cc[k].end(), k), Cc[k].end());
      Uk[k].assign(std::upper_bound(R[k].begin(), R[k].end(), k), R[k].end());
      for (int i : Lk[k]) {
        merged.clear();
        std::set_union(R[i].begin(), R[i].end(), Uk[k].begin(), Uk[k].end(), std::back_inserter(merged));
        R[i].swap(merged);
      }
      for (int j : Uk[k]) {
        merged.clear();
        std::set_union(Cc[j].begin(), Cc[j].end(), Lk[k].begin(), Lk[k].end(), std::back_inserter(merged));
        Cc[j].swap(merged);
      }
    }
    for (int r = 0; r < n; ++r) Rrow[r].swap(R[r]);
  }
  // ND slots, row-major: slot (r, c) = first slot of row r + rank of c among
  // the row's ascending columns
  std::vector<int> row_first(n + 1, 0);
  for (int r = 0; r < n; ++r) row_first[r + 1] = row_first[r] + (int)Rrow[r].size();
  T.nd_nv = row_first[n];
  T.nd_src.clear();
  std::unordered_map<int64_t, int> mf;
  for (int sl = 0; sl < T.nv; ++sl) mf[key(T.slot_row[sl], T.slot_col[sl])] = sl;
  for (int r = 0; r < n; ++r)
    for (int c : Rrow[r]) {
      auto f = mf.find(key(order[r], order[c]));
      T.nd_src.push_back(f == mf.end() ? -1 : f->second);
    }
  auto S = [&](int r, int c) {
    const auto& row = Rrow[r];
    const auto it = std::lower_bound(row.begin(), row.end(), c);
    if (it == row.end() || *it != c) throw std::logic_error("level schedule: position outside the structure");
    return row_first[r] + (int)(it - row.begin());
  };
  T.nd_diag.assign(n, 0);
  for (int k = 0; k < n; ++k) T.nd_diag[k] = S(k, k);
  // levels
  std::vector<int> level(n, 0);
  for (int k = 0; k < n; ++k) {
    for (int m : Lk[k]) level[m] = std::max(level[m], level[k] + 1);
    for (int m : Uk[k]) level[m] = std::max(level[m], level[k] + 1);
  }
  const int NL = 1 + *std::max_element(level.begin(), level.end());
  std::vector<std::vector<int>> piv(NL);
  for (int k = 0; k < n; ++k) piv[level[k]].push_back(k);
  for (auto* v : {&T.lv_piv, &T.lv_piv_ptr, &T.lv_l_ptr, &T.l_slot, &T.l_piv, &T.lv_ts_ptr,
                  &T.lv_tl_ptr, &T.t_slot, &T.t_off, &T.pr_l, &T.pr_u, &T.lv_ys_ptr, &T.lv_yl_ptr,
                  &T.y_row, &T.y_off, &T.yp_l, &T.yp_k, &T.bs_off, &T.bs_u, &T.bs_c})
    v->clear();
  T.t_off.push_back(0);
  T.y_off.push_back(0);
  for (int lv = 0; lv < NL; ++lv) {
    T.lv_piv_ptr.push_back((int)T.lv_piv.size());
    T.lv_l_ptr.push_back((int)T.l_slot.size());
    // update pairs by target slot and right-hand-side pairs by row, each in
    // pivot order within its target (a stable sort of the emission order)
    struct Rec {
      int key, a, b;
    };
    std::vector<Rec> tc, yc;
    for (int k : piv[lv]) {
      T.lv_piv.push_back(k);
      for (int i : Lk[k]) {
        const int sik = S(i, k);
        T.l_slot.push_back(sik);
        T.l_piv.push_back(k);
        yc.push_back({i, sik, k});
        if (Uk[k].empty()) continue;
        // row i holds every column of U_k (fill): walk both ascending lists
        const auto& row = Rrow[i];
        size_t p = (size_t)(std::lower_bound(row.begin(), row.end(), Uk[k].front()) - row.begin());
        for (int j : Uk[k]) {
          while (p < row.size() && row[p] < j) ++p;
          if (p == row.size() || row[p] != j) throw std::logic_error("level schedule: fill outside the structure");
          tc.push_back({row_first[i] + (int)p, sik, S(k, j)});
        }
      }
    }
    auto by_key = [](const Rec& x, const Rec& y) { return x.key < y.key; };
    std::stable_sort(tc.begin(), tc.end(), by_key);
    std::stable_sort(yc.begin(), yc.end(), by_key);
    // groups of equal keys in key order: short lists, then long ones
    auto emit = [&](const std::vector<Rec>& recs, std::vector<int>& keys, std::vector<int>& off,
                    std::vector<int>& pa, std::vector<int>& pb, std::vector<int>& short_ptr,
                    std::vector<int>& long_ptr) {
      for (int pass = 0; pass < 2; ++pass) {
        (pass ? long_ptr : short_ptr).push_back((int)keys.size());
        for (size_t g0 = 0; g0 < recs.size();) {
          size_t g1 = g0;
          while (g1 < recs.size() && recs[g1].key == recs[g0].key) ++g1;
          if (((int)(g1 - g0) > Topology::kNdLong) == (pass == 1)) {
            keys.push_back(recs[g0].key);
            for (size_t q = g0; q < g1; ++q) {
              pa.push_back(recs[q].a);
              pb.push_back(recs[q].b);
            }
            off.push_back((int)pa.size());
          }
          g0 = g1;
        }
      }
    };
    emit(tc, T.t_slot, T.t_off, T.pr_l, T.pr_u, T.lv_ts_ptr, T.lv_tl_ptr);
    emit(yc, T.y_row, T.y_off, T.yp_l, T.yp_k, T.lv_ys_ptr, T.lv_yl_ptr);
  }
  T.lv_piv_ptr.push_back((int)T.lv_piv.size());
  T.lv_l_ptr.push_back((int)T.l_slot.size());
  T.lv_ts_ptr.push_back((int)T.t_slot.size());
  T.lv_tl_ptr.push_back((int)T.t_slot.size());
  T.lv_ys_ptr.push_back((int)T.y_row.size());
  T.lv_yl_ptr.push_back((int)T.y_row.size());
  T.bs_off.push_back(0);
  for (int k = 0; k < n; ++k) {
    for (int j : Uk[k]) {
      T.bs_u.push_back(S(k, j));
      T.bs_c.push_back(j);
    }
    T.bs_off.push_back((int)T.bs_u.size());
  }
  T.nd_levels = NL;
}

// The level schedule packed into one int array that a CTA stages into shared
// memory (lo | hi << 16, 16-bit fields):
//   [0] levels, [1] section offset of the level table, [2] of the target
//   pairs, [3] of the right-hand-side pairs, [4] of the back-substitution
//   pairs, [5] of nd_src (two per int, 0xFFFF = none), [6] of nd_pos (two per
//   int), [7] total ints;
//   level table, 12 ints per level: offsets and counts of its pivots (diag
//   slots), L entries (slot | diag << 16), short targets and long targets
//   (int2: slot | count << 16, first pair), short and long right-hand-side
//   rows (int2: row | count << 16, first pair), back-substitution pivots
//   (int2: pivot | diag << 16, count | first pair << 16);
//   pairs: target (l slot | u slot << 16), right-hand side (l slot | pivot <<
//   16), back substitution (u slot | column << 16).
void nd_program(Topology& T) {
  T.nd_prog.clear();
  if (T.nd_levels == 0) return;
  const int NL = T.nd_levels;
  if (T.nd_nv >= 0xFFFF || T.n >= 0xFFFF || (int)T.pr_l.size() >= 0xFFFF ||
      (int)T.yp_l.size() >= 0xFFFF || (int)T.bs_u.size() >= 0xFFFF)
    return;
  auto pk = [](int lo, int hi) { return (int)((unsigned)lo | ((unsigned)hi << 16)); };
  std::vector<int> body, tp, yp, bp;
  std::vector<int> lvt(12 * (size_t)NL);
  for (int lv = 0; lv < NL; ++lv) {
    int* L = &lvt[12 * (size_t)lv];
    L[0] = (int)body.size();
    for (int q = T.lv_piv_ptr[lv]; q < T.lv_piv_ptr[lv + 1]; ++q) body.push_back(T.nd_diag[T.lv_piv[q]]);
    L[1] = (int)body.size() - L[0];
    L[2] = (int)body.size();
    for (int e = T.lv_l_ptr[lv]; e < T.lv_l_ptr[lv + 1]; ++e)
      body.push_back(pk(T.l_slot[e], T.nd_diag[T.l_piv[e]]));
    L[3] = (int)body.size() - L[2];
    auto items = [&](int a, int b, const std::vector<int>& key, const std::vector<int>& off,
                     const std::vector<int>& pl, const std::vector<int>& ph, std::vector<int>& pairs,
                     int* o, int* c) {
      *o = (int)body.size();
      for (int t = a; t < b; ++t) {
        body.push_back(pk(key[t], off[t + 1] - off[t]));
        body.push_back((int)pairs.size());
        for (int q = off[t]; q < off[t + 1]; ++q) pairs.push_back(pk(pl[q], ph[q]));
      }
      *c = b - a;
    };
    items(T.lv_ts_ptr[lv], T.lv_tl_ptr[lv], T.t_slot, T.t_off, T.pr_l, T.pr_u, tp, &L[4], &L[5]);
    int tl_off;
    items(T.lv_tl_ptr[lv], T.lv_ts_ptr[lv + 1], T.t_slot, T.t_off, T.pr_l, T.pr_u, tp, &tl_off, &L[6]);
    items(T.lv_ys_ptr[lv], T.lv_yl_ptr[lv], T.y_row, T.y_off, T.yp_l, T.yp_k, yp, &L[7], &L[8]);
    int yl_off;
    items(T.lv_yl_ptr[lv], T.lv_ys_ptr[lv + 1], T.y_row, T.y_off, T.yp_l, T.yp_k, yp, &yl_off, &L[9]);
    L[10] = (int)body.size();
    for (int q = T.lv_piv_ptr[lv]; q < T.lv_piv_ptr[lv + 1]; ++q) {
      const int k = T.lv_piv[q];
      body.push_back(pk(k, T.nd_diag[k]));
      body.push_back(pk(T.bs_off[k + 1] - T.bs_off[k], (int)bp.size()));
      for (int b = T.bs_off[k]; b < T.bs_off[k + 1]; ++b) bp.push_back(pk(T.bs_u[b], T.bs_c[b]));
    }
    L[11] = T.lv_piv_ptr[lv + 1] - T.lv_piv_ptr[lv];
  }
  if (tp.size() >= 0xFFFF || yp.size() >= 0xFFFF || bp.size() >= 0xFFFF) return;
  std::vector<int> src((T.nd_nv + 1) / 2), ps((T.n + 1) / 2);
  for (int i = 0; i < T.nd_nv; ++i) {
    const unsigned v = T.nd_src[i] < 0 ? 0xFFFFu : (unsigned)T.nd_src[i];
    src[i / 2] = (int)((unsigned)src[i / 2] | (v << (16 * (i & 1))));
  }
  for (int i = 0; i < T.n; ++i)
    ps[i / 2] = (int)((unsigned)ps[i / 2] | ((unsigned)T.nd_pos[i] << (16 * (i & 1))));
  std::vector<int>& P = T.nd_prog;
  P.assign(8, 0);
  P[0] = NL;
  P[1] = (int)P.size();
  P.insert(P.end(), lvt.begin(), lvt.end());
  const int body_at = (int)P.size();
  P.insert(P.end(), body.begin(), body.end());
  // level-table offsets are absolute in the program
  for (int lv = 0; lv < NL; ++lv)
    for (int f : {0, 2, 4, 7, 10}) P[P[1] + 12 * lv + f] += body_at;
  P[2] = (int)P.size();
  P.insert(P.end(), tp.begin(), tp.end());
  P[3] = (int)P.size();
  P.insert(P.end(), yp.begin(), yp.end());
  P[4] = (int)P.size();
  P.insert(P.end(), bp.begin(), bp.end());
  P[5] = (int)P.size();
  P.insert(P.end(), src.begin(), src.end());
  P[6] = (int)P.size();
  P.insert(P.end(), ps.begin(), ps.end());
  P[7] = (int)P.size();
}

}  // namespace

// Min-Fill on sparse adjacency. Adjacency is a sorted vector per vertex and
// membership tests go through stamp arrays, so memory and time follow the
// graph's size, not n^2. Fill counts are updated from the elimination's new
// edges instead of being recounted. With u eliminated, K = N(u), and for a
// neighbour w: A = N(w) \ {u}, C = the vertices of K that become new
// neighbours of w (w's new edges), E_A = the new edges with both ends in A,
//   fill'(w) = fill(w) - |A \ K| - E_A + sum over c in C of |(A \ K) \ N(c)|
// (the pairs (u, y) leave, new edges inside A stop being missing, and each new
// neighbour c is missing exactly the old neighbours outside K it is not
// adjacent to). Every vertex outside K and u loses one missing pair per new
// edge with both ends among its neighbours. Integer counts, so the order is
// the recount's, ties included.
static MinFillResult min_fill_sparse(const std::vector<std::vector<uint32_t>>& factors,
                                     const std::unordered_map<uint32_t, int>& dense,
                                     const std::vector<uint32_t>& ids, std::vector<int> extra,
                                     size_t n_listed) {
  const int nv = (int)ids.size();
  std::vector<std::vector<int>> adj(nv);
  for (const auto& f : factors)
    for (size_t i = 0; i < f.size(); ++i)
      for (size_t j = i + 1; j < f.size(); ++j)
        if (f[i] != f[j]) {
          const int a = dense.at(f[i]), b = dense.at(f[j]);
          adj[a].push_back(b);
          adj[b].push_back(a);
        }
  for (auto& r : adj) {
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
  }
  // stamp arrays: mark[x] == g tags x in the current set
  std::vector<uint32_t> in_k(nv, 0), mark(nv, 0);
  uint32_t gk = 0, gm = 0;
  std::vector<uint32_t> fill(nv, 0);
  for (int u = 0; u < nv; ++u) {
    ++gm;
    for (int x : adj[u]) mark[x] = gm;
    uint64_t inside = 0;
    for (int x : adj[u])
      for (int y : adj[x]) inside += mark[y] == gm;
    const uint64_t k = adj[u].size();
    fill[u] = (uint32_t)((k * (k - 1) - inside) / 2);
  }
  std::set<std::pair<uint32_t, uint32_t>> pq;  // (fill, id)
  for (int u = 0; u < nv; ++u) pq.insert({fill[u], ids[u]});
  std::vector<char> alive(nv, 1);
  std::vector<int> ghosts(nv, 0);
  MinFillResult out;
  out.ordering.reserve(n_listed);
  uint32_t maxclique = 0;
  std::vector<int> nb, touched, merged;
  std::vector<std::vector<int>> partners;  // per position in nb: new neighbours, ascending
  std::vector<uint32_t> dec(nv, 0);
  std::vector<uint32_t> newfill;
  while (!pq.empty()) {
    auto top = *pq.begin();
    pq.erase(pq.begin());
    const int u = dense.at(top.second);
    out.ordering.push_back(top.second);
    if (!alive[u]) {  // repeated listing: isolated by now
      maxclique = std::max<uint32_t>(maxclique, 1);
      if (--ghosts[u] > 0) pq.insert({0u, ids[u]});
      continue;
    }
    nb = adj[u];
    const int k = (int)nb.size();
    maxclique = std::max<uint32_t>(maxclique, (uint32_t)k + 1);
    ++gk;
    in_k[u] = gk;
    for (int w : nb) in_k[w] = gk;
    // new edges: for each a in K, the members of K \ {a} it is not adjacent to
    if ((int)partners.size() < k) partners.resize(k);
    for (int i = 0; i < k; ++i) {
      const int a = nb[i];
      auto& pa = partners[i];
      pa.clear();
      const auto& ra = adj[a];
      size_t p = 0;
      for (int j = 0; j < k; ++j) {
        const int b = nb[j];
        if (b == a) continue;
        while (p < ra.size() && ra[p] < b) ++p;
        if (p == ra.size() || ra[p] != b) pa.push_back(b);
      }
    }
    // vertices outside K and u adjacent to both ends of a new edge
    touched.clear();
    for (int i = 0; i < k; ++i) {
      const int a = nb[i];
      for (int b : partners[i]) {
        if (b < a) continue;
        const auto& ra = adj[a];
        const auto& rb = adj[b];
        size_t p = 0, q = 0;
        while (p < ra.size() && q < rb.size()) {
          if (ra[p] < rb[q]) {
            ++p;
          } else if (rb[q] < ra[p]) {
            ++q;
          } else {
            const int w = ra[p];
            if (in_k[w] != gk && dec[w]++ == 0) touched.push_back(w);
            ++p;
            ++q;
          }
        }
      }
    }
    // neighbours of u: the update rule above, on the old adjacency
    newfill.assign(k, 0);
    for (int i = 0; i < k; ++i) {
      const int w = nb[i];
      ++gm;
      int64_t out_k = 0;  // |A \ K|
      for (int x : adj[w]) {
        mark[x] = gm;
        out_k += in_k[x] != gk;
      }
      int64_t e_a = 0;
      for (int j = 0; j < k; ++j) {
        const int a = nb[j];
        if (a == w || mark[a] != gm) continue;
        for (int b : partners[j])
          if (b > a && b != w && mark[b] == gm) ++e_a;
      }
      int64_t cross = 0;
      for (int c : partners[i]) {
        int64_t seen = 0;
        for (int x : adj[c]) seen += mark[x] == gm && in_k[x] != gk;
        cross += out_k - seen;
      }
      newfill[i] = (uint32_t)((int64_t)fill[w] - out_k - e_a + cross);
    }
    // new adjacency: N(a) \ {u} merged with a's new neighbours
    for (int i = 0; i < k; ++i) {
      const int a = nb[i];
      const auto& ra = adj[a];
      const auto& pa = partners[i];
      merged.clear();
      merged.reserve(ra.size() + pa.size());
      size_t p = 0, q = 0;
      while (p < ra.size() || q < pa.size()) {
        if (q == pa.size() || (p < ra.size() && ra[p] < pa[q])) {
          if (ra[p] != u) merged.push_back(ra[p]);
          ++p;
        } else {
          merged.push_back(pa[q++]);
        }
      }
      adj[a].swap(merged);
    }
    adj[u].clear();
    adj[u].shrink_to_fit();
    alive[u] = 0;
    for (int w : touched) {
      pq.erase({fill[w], ids[w]});
      fill[w] -= dec[w];
      dec[w] = 0;
      pq.insert({fill[w], ids[w]});
    }
    for (int i = 0; i < k; ++i) {
      const int w = nb[i];
      pq.erase({fill[w], ids[w]});
      fill[w] = newfill[i];
      pq.insert({fill[w], ids[w]});
    }
    if (extra[u] > 0) {
      ghosts[u] = extra[u];
      pq.insert({0u, ids[u]});
      extra[u] = 0;
    }
  }
  out.treewidth = maxclique > 0 ? (int)maxclique - 1 : 0;
  return out;
}

// Min-Fill elimination with the reference's choice rule: at every step the
// vertex with the fewest missing neighbour pairs, ties to the smallest id
// (treewidth_analyzer.cpp:72-102). Instead of rescanning every vertex, fill
// counts live in an ordered set keyed (fill, id) and only vertices whose
// neighbourhood changed are updated (min_fill_sparse above). A variable id
// listed twice (the reference's branch id that equals the node count) is
// eliminated twice, the second time as an isolated vertex, which is what the
// reference's map-keyed adjacency does.
MinFillResult min_fill(const std::vector<std::vector<uint32_t>>& factors,
                       const std::vector<uint32_t>& variables) {
  std::unordered_map<uint32_t, int> dense;
  std::vector<uint32_t> ids;
  std::vector<int> extra;  // repeated listings per dense vertex
  for (uint32_t id : variables) {
    auto it = dense.find(id);
    if (it == dense.end()) {
      dense[id] = (int)ids.size();
      ids.push_back(id);
      extra.push_back(0);
    } else {
      extra[it->second]++;
    }
  }
  return min_fill_sparse(factors, dense, ids, std::move(extra), variables.size());
}

namespace {

// KCL term records (terminals + coefficient per term of ft_code).
void node_term_records(Topology& T) {
  T.ft_a.clear();
  T.ft_b.clear();
  T.ft_coef.clear();
  for (int c : T.ft_code) {
    const int kind = (c >> 24) & 0x7f, idx = c & 0xffffff;
    int a = -1, b = -1;
    double coef = 0.0;
    switch (kind) {
      case FK_RES:
        a = T.res_term[2 * idx];
        b = T.res_term[2 * idx + 1];
        coef = 1.0 / T.res[idx].val;
        break;
      case FK_VS:
        a = T.vs_term[2 * idx];
        b = T.vs_term[2 * idx + 1];
        break;
      case FK_IS:
        coef = T.isrc[idx].val;
        break;
      case FK_CAP:
        a = T.cap_term[2 * idx];
        b = T.cap_term[2 * idx + 1];
        coef = 2.0 * T.cap[idx].val;
        break;
      default:
        break;
    }
    T.ft_a.push_back(a);
    T.ft_b.push_back(b);
    T.ft_coef.push_back(coef);
  }
}

// Shared-memory layout of a block's device values: 96 doubles per device, 32
// lanes each of {gm or diode g, gds or diode i, MOSFET ids}. A slot term is
// stored as its sign bit | the offset of its value for lane 0; a node
// device term keeps its code and carries that offset in its fourth field.
int es_slot_term(int code, int local_dev) {
  const int kind = (code >> 24) & 0x7f;  // JK_MOS_GDS, JK_MOS_GM, JK_DIO_G
  return (code & int32_t(0x80000000u)) | (local_dev * 96 + (kind == JK_MOS_GDS ? 32 : 0));
}
int es_node_term_offset(int code, int local_dev) {
  const int kind = (code >> 24) & 0x7f;  // FK_DIO: diode current, FK_MOS: ids
  return local_dev * 96 + (kind == FK_DIO ? 32 : 64);
}

// Packs the stamp items into evaluation + stamping blocks. Items go in row
// order (the slots of a row, then its node), so a block covers a stretch of
// the ordering and the devices it needs are mostly its own; a device shared
// by two blocks is evaluated by both.
void es_blocks(Topology& T) {
  const int n = T.n, nv = T.nv, nm = (int)T.mos.size();
  T.es_block.clear();
  T.es_item.clear();
  T.es_dev.clear();
  T.es_jt.clear();
  T.es_ft.clear();
  T.es_fc.clear();
  T.es_hub.clear();
  T.es_hubc.clear();
  T.n_hub_groups = 0;
  T.n_hub_rows = 0;
  T.es_max_dev = kEsMaxDev;
  // device of a slot term / node term (-1: none)
  auto slot_dev = [&](int c) {
    const int kind = (c >> 24) & 0x7f, idx = c & 0xffffff;
    return kind == JK_DIO_G ? nm + idx : idx;
  };
  auto node_dev = [&](int c) {
    const int kind = (c >> 24) & 0x7f, idx = c & 0xffffff;
    if (kind == FK_DIO) return nm + idx;
    if (kind == FK_MOS) return idx;
    return -1;
  };
  auto item_devs = [&](int it, std::vector<int>& out) {
    out.clear();
    if (it < nv) {
      for (int q = T.jt_off[it]; q < T.jt_off[it + 1]; ++q) out.push_back(slot_dev(T.jt_code[q]));
    } else {
      const int i = it - nv;
      for (int q = T.ft_off[i]; q < T.ft_off[i + 1]; ++q) {
        const int d = node_dev(T.ft_code[q]);
        if (d >= 0) out.push_back(d);
      }
    }
  };
  // Item order: row by row (the slots of a row, then its node), the rows in
  // Cuthill-McKee order of the graph in which two rows are adjacent when a
  // device stamps into both. Consecutive rows then share most of their
  // devices, so few devices are evaluated by more than one block. Hub rows
  // (nodes with more devices than a block holds) stay out of the graph; their
  // slots follow the row of their column, whose devices they need, and the
  // hub nodes (and the slots in hub columns) come last.
  std::vector<int> order;
  {
    std::vector<int> dv;
    std::vector<int> row_first(n + 1, nv);
    for (int s = nv - 1; s >= 0; --s) row_first[T.slot_row[s]] = s;
    for (int r = n - 1; r >= 0; --r) row_first[r] = std::min(row_first[r], row_first[r + 1]);
    std::vector<std::vector<int>> dev_rows;
    std::vector<char> hub_row(n, 0);
    for (int r = 0; r < n; ++r) {
      item_devs(nv + r, dv);
      std::sort(dv.begin(), dv.end());
      dv.erase(std::unique(dv.begin(), dv.end()), dv.end());
      if ((int)dv.size() > kEsMaxDev) {
        hub_row[r] = 1;
        continue;
      }
      for (int d : dv) {
        if (d >= (int)dev_rows.size()) dev_rows.resize(d + 1);
        dev_rows[d].push_back(r);
      }
    }
    std::vector<std::vector<int>> adj(n);
    for (const auto& rows : dev_rows)
      for (int a : rows)
        for (int b : rows)
          if (a != b) adj[a].push_back(b);
    for (auto& a : adj) {
      std::sort(a.begin(), a.end());
      a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    auto degree_less = [&](int a, int b) {
      return adj[a].size() != adj[b].size() ? adj[a].size() < adj[b].size() : a < b;
    };
    std::vector<int> level(n, -1);
    auto bfs = [&](int root, std::vector<int>& out) {  // Cuthill-McKee from root
      out.clear();
      out.push_back(root);
      level[root] = 0;
      for (size_t h = 0; h < out.size(); ++h) {
        std::vector<int> nb;
        for (int b : adj[out[h]])
          if (level[b] < 0) nb.push_back(b);
        std::sort(nb.begin(), nb.end(), degree_less);
        for (int b : nb) {
          level[b] = level[out[h]] + 1;
          out.push_back(b);
        }
      }
    };
    std::vector<int> rows, comp;
    std::vector<char> done(n, 0);
    for (int r = 0; r < n; ++r) done[r] = hub_row[r];
    // each component starts at its lowest-degree row (ties to the smallest
    // index): the first row not yet done in one sorted list
    std::vector<int> by_degree;
    for (int r = 0; r < n; ++r)
      if (!done[r]) by_degree.push_back(r);
    std::sort(by_degree.begin(), by_degree.end(), degree_less);
    size_t next_root = 0;
    while (true) {
      while (next_root < by_degree.size() && done[by_degree[next_root]]) ++next_root;
      if (next_root == by_degree.size()) break;
      const int root = by_degree[next_root];
      // pseudo-peripheral start: the last row of a BFS from the
      // lowest-degree row of the component
      bfs(root, comp);
      const int far = comp.back();
      for (int r : comp) level[r] = -1;
      bfs(far, comp);
      for (int r : comp) {
        done[r] = 1;
        rows.push_back(r);
      }
    }
    std::vector<std::vector<int>> hub_slots_of_col(n);
    for (int s = 0; s < nv; ++s)
      if (hub_row[T.slot_row[s]] && !hub_row[T.slot_col[s]]) hub_slots_of_col[T.slot_col[s]].push_back(s);
    for (int r : rows) {
      for (int s = row_first[r]; s < nv && T.slot_row[s] == r; ++s) order.push_back(s);
      order.push_back(nv + r);
      for (int s : hub_slots_of_col[r]) order.push_back(s);
    }
    for (int r = 0; r < n; ++r)
      if (hub_row[r]) {
        for (int s = row_first[r]; s < nv && T.slot_row[s] == r; ++s)
          if (hub_row[T.slot_col[s]]) order.push_back(s);
        order.push_back(nv + r);
      }
  }
  std::vector<int> cur_items, cur_devs, devs;
  std::unordered_map<int, int> local;
  std::vector<int> hubs;  // items with more devices than one block holds
  auto emit = [&](const std::vector<int>& items, const std::vector<int>& dlist, bool) {
    if (items.empty()) return;
    std::unordered_map<int, int> lid;
    for (size_t k = 0; k < dlist.size(); ++k) lid[dlist[k]] = (int)k;
    T.es_block.push_back((int)T.es_item.size() / 4);
    T.es_block.push_back((int)items.size());
    T.es_block.push_back((int)T.es_dev.size());
    T.es_block.push_back((int)dlist.size());
    for (int k = 0; k < 4; ++k) T.es_hubc.push_back(0);
    T.es_dev.insert(T.es_dev.end(), dlist.begin(), dlist.end());
    for (int it : items) {
      T.es_item.push_back(it);
      if (it < nv) {
        T.es_item.push_back((int)T.es_jt.size());
        T.es_item.push_back(T.jt_off[it + 1] - T.jt_off[it]);
        T.es_item.push_back(0);
        for (int q = T.jt_off[it]; q < T.jt_off[it + 1]; ++q) {
          const int c = T.jt_code[q];
          T.es_jt.push_back(es_slot_term(c, lid.at(slot_dev(c))));
        }
      } else {
        const int i = it - nv;
        T.es_item.push_back((int)T.es_ft.size() / 4);
        T.es_item.push_back(T.ft_off[i + 1] - T.ft_off[i]);
        T.es_item.push_back(0);
        for (int q = T.ft_off[i]; q < T.ft_off[i + 1]; ++q) {
          const int c = T.ft_code[q];
          const int d = node_dev(c);
          T.es_ft.push_back(d >= 0 ? ((c & int32_t(0xFF000000u)) | lid.at(d)) : c);
          T.es_ft.push_back(T.ft_a[q]);
          T.es_ft.push_back(T.ft_b[q]);
          T.es_ft.push_back(d >= 0 ? es_node_term_offset(c, lid.at(d)) : 0);
          T.es_fc.push_back(T.ft_coef[q]);
        }
      }
    }
  };
  for (int it : order) {
    item_devs(it, devs);
    std::vector<int> fresh;
    for (int d : devs)
      if (!local.count(d) && std::find(fresh.begin(), fresh.end(), d) == fresh.end()) fresh.push_back(d);
    std::vector<int> own;  // the item's own distinct devices, in term order
    for (int d : devs)
      if (std::find(own.begin(), own.end(), d) == own.end()) own.push_back(d);
    if ((int)own.size() > kEsMaxDev) {
      hubs.push_back(it);  // emitted after the normal blocks, grouped
      continue;
    }
    if ((int)(cur_devs.size() + fresh.size()) > kEsMaxDev || (int)cur_items.size() >= kEsMaxItems) {
      emit(cur_items, cur_devs, false);
      cur_items.clear();
      cur_devs.clear();
      local.clear();
      fresh = own;
    }
    for (int d : fresh) {
      local[d] = (int)cur_devs.size();
      cur_devs.push_back(d);
    }
    cur_items.push_back(it);
  }
  emit(cur_items, cur_devs, false);
  const size_t normal_blocks = T.es_block.size();

  // Hub items (the supply node and its diagonal slot): groups of up to
  // kEsMaxHubs share the union of their devices, split into chunks of
  // kEsMaxDev with one block per chunk. Each chunk block sums the group's
  // terms of its chunk into partial rows; the last block of the group to
  // finish (per tile of 32 instances) adds the partials in chunk order. The
  // union is in first-occurrence order; a group is kept only if every item's
  // device indices never decrease along its terms (so the terms of one chunk
  // are contiguous and es_hub can bound them), otherwise each hub forms a
  // group of its own over its term occurrences.
  auto terms_of = [&](int it, std::vector<int>& out) {  // device per term, -1 = linear
    out.clear();
    if (it < nv) {
      for (int q = T.jt_off[it]; q < T.jt_off[it + 1]; ++q) out.push_back(slot_dev(T.jt_code[q]));
    } else {
      const int i = it - nv;
      for (int q = T.ft_off[i]; q < T.ft_off[i + 1]; ++q) out.push_back(node_dev(T.ft_code[q]));
    }
  };
  auto emit_group = [&](const std::vector<int>& items, const std::vector<int>& dlist,
                        const std::vector<std::vector<int>>& lidx) {
    const int nch = ((int)dlist.size() + kEsMaxDev - 1) / kEsMaxDev;
    for (int c = 0; c < nch; ++c) {
      T.es_block.push_back((int)T.es_item.size() / 4);
      T.es_block.push_back(-(int)items.size());
      T.es_block.push_back((int)T.es_dev.size() + c * kEsMaxDev);
      T.es_block.push_back(std::min(kEsMaxDev, (int)dlist.size() - c * kEsMaxDev));
      T.es_hubc.push_back(c);
      T.es_hubc.push_back(nch);
      T.es_hubc.push_back(T.n_hub_groups);
      T.es_hubc.push_back(T.n_hub_rows);
    }
    ++T.n_hub_groups;
    T.n_hub_rows += (int)items.size() * nch;
    T.es_dev.insert(T.es_dev.end(), dlist.begin(), dlist.end());
    for (size_t m = 0; m < items.size(); ++m) {
      const int it = items[m];
      T.es_item.push_back(it);
      const std::vector<int>& li = lidx[m];
      // term index where each device chunk starts (linear terms go with the
      // chunk of the device term before them), and the end
      const int hb = (int)T.es_hub.size();
      {
        int c = 0;
        T.es_hub.push_back(0);
        for (int t = 0; t < (int)li.size(); ++t)
          while (li[t] >= 0 && li[t] / kEsMaxDev > c) {
            T.es_hub.push_back(t);
            ++c;
          }
        while (c < nch) {
          T.es_hub.push_back((int)li.size());
          ++c;
        }
      }
      if (it < nv) {
        T.es_item.push_back((int)T.es_jt.size());
        T.es_item.push_back(T.jt_off[it + 1] - T.jt_off[it]);
        T.es_item.push_back(hb);
        for (int q = T.jt_off[it], t = 0; q < T.jt_off[it + 1]; ++q, ++t)
          T.es_jt.push_back(es_slot_term(T.jt_code[q], li[t] % kEsMaxDev));  // chunk-local
      } else {
        const int i = it - nv;
        T.es_item.push_back((int)T.es_ft.size() / 4);
        T.es_item.push_back(T.ft_off[i + 1] - T.ft_off[i]);
        T.es_item.push_back(hb);
        for (int q = T.ft_off[i], t = 0; q < T.ft_off[i + 1]; ++q, ++t) {
          const int c = T.ft_code[q];
          T.es_ft.push_back(li[t] >= 0 ? ((c & int32_t(0xFF000000u)) | li[t]) : c);
          T.es_ft.push_back(T.ft_a[q]);
          T.es_ft.push_back(T.ft_b[q]);
          T.es_ft.push_back(li[t] >= 0 ? es_node_term_offset(c, li[t] % kEsMaxDev) : 0);
          T.es_fc.push_back(T.ft_coef[q]);
        }
      }
    }
  };
  std::vector<int> tdev;
  for (size_t h0 = 0; h0 < hubs.size(); h0 += kEsMaxHubs) {
    std::vector<int> items(hubs.begin() + h0, hubs.begin() + std::min(hubs.size(), h0 + kEsMaxHubs));
    std::vector<int> dlist;
    std::unordered_map<int, int> uid;
    std::vector<std::vector<int>> lidx(items.size());
    bool monotone = true;
    for (size_t m = 0; m < items.size(); ++m) {
      terms_of(items[m], tdev);
      int last_chunk = 0;
      for (int d : tdev) {
        if (d < 0) {
          lidx[m].push_back(-1);
          continue;
        }
        auto f = uid.find(d);
        int id;
        if (f == uid.end()) {
          id = (int)dlist.size();
          uid[d] = id;
          dlist.push_back(d);
        } else {
          id = f->second;
        }
        lidx[m].push_back(id);
        if (id / kEsMaxDev < last_chunk) monotone = false;
        last_chunk = std::max(last_chunk, id / kEsMaxDev);
      }
    }
    if (monotone) {
      emit_group(items, dlist, lidx);
      continue;
    }
    for (int it : items) {  // each hub over its own term occurrences
      terms_of(it, tdev);
      std::vector<int> occ;
      std::vector<std::vector<int>> li(1);
      for (int d : tdev) {
        li[0].push_back(d >= 0 ? (int)occ.size() : -1);
        if (d >= 0) occ.push_back(d);
      }
      emit_group({it}, occ, li);
    }
  }
  // hub blocks run longest: put them first so the grid starts them first
  std::rotate(T.es_block.begin(), T.es_block.begin() + normal_blocks, T.es_block.end());
  std::rotate(T.es_hubc.begin(), T.es_hubc.begin() + normal_blocks, T.es_hubc.end());
}

}  // namespace

Topology build_topology(const karam_netlist* nl) {
  Topology T;
  tensorize(nl, T);
  stamps(T);
  ordering(T);
  std::vector<std::vector<int>> urow;
  symbolic(T, urow);
  device_tables(T, urow);
  node_term_records(T);
  es_blocks(T);
  nd_schedule(T);
  nd_program(T);
  return T;
}

}  // namespace karam
