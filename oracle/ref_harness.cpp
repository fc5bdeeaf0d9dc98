// ref_harness.cpp -- oracle backend built on the reference's own sources
// (TEST INFRASTRUCTURE ONLY; built by oracle/Makefile into oracle/_ref/).
//
// Every numeric step here is a call into the reference: TensorNetlist adders
// (netlist/circuit.h:1139-1216), tensorizeNetlist (tensors/physics_tensors.cpp:305),
// the generic device kernels via KernelDispatcher, CircuitSim::stampSoABlock
// (physics/circuitsim.h:2413-2751), MatrixConstructor::buildPattern/assembleFast
// (math/linalg.h:421-465), solveLU_Pivoted (math/linalg.h:742), symbolicFactorize
// and solveSparse_LU (math/sparse_lu.cpp), FactorGraph::fromTensorizedBlock and
// TreewidthAnalyzer::analyze. Only the NR driver composition (nr_driver.hpp)
// and the instance-parameter injection are this project's.
//
// CircuitSim keeps its matrix builder and RHS private; this test-only unit
// opens them with a preprocessor switch so the stamps can be read back.
#define private public
#include "acutesim_engine/physics/circuitsim.h"
#undef private
#include "acutesim_engine/infrastructure/factor_graph.h"
#include "acutesim_engine/infrastructure/treewidth_analyzer.h"
#include "acutesim_engine/math/sparse_lu.h"
#include "acutesim_engine/math/portable_rng.h"
#include "acutesim_engine/solvers/ac_solver.h"

#include <algorithm>
#include <cmath>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "nr_driver.hpp"

namespace {

std::string model_name(const karam_netlist* nl, int m) {
  return std::string(nl->model_name[m]);
}

// Netlist-order -> SoA-order maps. tensorizeNetlist buckets devices in a
// std::map keyed by model name (physics_tensors.cpp:481-490), so the SoA order
// is a stable sort of the netlist order by model name; checked against the
// tensorised terminals below.
std::vector<int> bucket_order(int n, const std::vector<std::string>& names) {
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return names[a] < names[b]; });
  return ord;
}

struct RefBackend {
  int n = 0;
  oracle::Csr pat;
  oracle::SourceSet src;
  std::vector<int> dio_a, dio_c;
  std::vector<double> dio_is, dio_vt;
  std::vector<int> cap_n1, cap_n2;
  std::vector<double> cap_c;
  std::vector<int> seed_dio_anode, isrc_pos;
  double temp_k = 300.15;

  TensorNetlist net;
  TensorizedBlock soa;
  std::unique_ptr<CircuitSim> sim;
  CachedCsrPattern cpat;
  std::vector<int> mos_order, dio_order;

  void build(const karam_netlist* nl) {
    net.environment.ambient_temp_K = nl->temp_k;
    temp_k = nl->temp_k;
    for (int m = 0; m < nl->n_models; ++m) {
      ModelCard c;
      c.name = model_name(nl, m);
      int ty = nl->model_type[m];
      c.type = ty == KARAM_MODEL_PMOS ? "PMOS" : (ty == KARAM_MODEL_NMOS ? "NMOS" : "D");
      if (nl->model_kp && !std::isnan(nl->model_kp[m])) c.params["KP"] = nl->model_kp[m];
      if (nl->model_vto && !std::isnan(nl->model_vto[m])) c.params["VTO"] = nl->model_vto[m];
      if (nl->model_lambda && !std::isnan(nl->model_lambda[m]))
        c.params["LAMBDA"] = nl->model_lambda[m];
      net.addModelCard(c);
    }
    for (int i = 0; i < nl->n_vsrc; ++i) {
      bool pulse = nl->vs_kind && nl->vs_kind[i] == KARAM_SRC_PULSE;
      net.addVoltageSource(nl->vs_pos[i], nl->vs_neg[i], nl->vs_dc[i], pulse ? "PULSE" : "");
      if (pulse) {
        auto& vs = net.globalBlock.voltageSources.back();
        const double* p = nl->vs_pulse + 7 * i;
        vs.pulse_v1 = p[0]; vs.pulse_v2 = p[1]; vs.pulse_td = p[2]; vs.pulse_tr = p[3];
        vs.pulse_tf = p[4]; vs.pulse_pw = p[5]; vs.pulse_per = p[6];
      }
    }
    for (int i = 0; i < nl->n_isrc; ++i)
      net.addCurrentSource(nl->is_pos[i], nl->is_neg[i], nl->is_amp[i]);
    for (int i = 0; i < nl->n_res; ++i) net.addResistor(nl->r_n1[i], nl->r_n2[i], nl->r_ohm[i]);
    for (int i = 0; i < nl->n_cap; ++i)
      net.addCapacitor(nl->c_n1[i], nl->c_n2[i], nl->c_farad[i]);
    std::vector<std::string> dnames(nl->n_dio), mnames(nl->n_mos);
    for (int i = 0; i < nl->n_dio; ++i) {
      net.globalBlock.addDiode("D" + std::to_string(i + 1), nl->d_anode[i], nl->d_cathode[i],
                               nl->d_is[i], nl->d_n[i], nl->d_vt[i]);
      int mi = nl->d_model ? nl->d_model[i] : -1;
      dnames[i] = mi >= 0 ? model_name(nl, mi) : std::string("diode_generic");
      net.globalBlock.diodes.back().modelName = dnames[i];
      net.numGlobalNodes = std::max({net.numGlobalNodes, nl->d_anode[i], nl->d_cathode[i]});
    }
    for (int i = 0; i < nl->n_mos; ++i) {
      mnames[i] = model_name(nl, nl->m_model[i]);
      net.addMosfet("M" + std::to_string(i + 1), nl->m_d[i], nl->m_g[i], nl->m_s[i], nl->m_b[i],
                    mnames[i], nl->m_w[i], nl->m_l[i]);
    }
    net.numGlobalNodes = std::max(net.numGlobalNodes, nl->n_nodes);
    n = net.numGlobalNodes;

    soa = tensorizeNetlist(net);
    mos_order = bucket_order(nl->n_mos, mnames);
    dio_order = bucket_order(nl->n_dio, dnames);
    for (size_t j = 0; j < soa.mosfets.size(); ++j) {
      int k = mos_order[j];
      if (soa.mosfets.drains[j] != nl->m_d[k] || soa.mosfets.gates[j] != nl->m_g[k] ||
          soa.mosfets.sources[j] != nl->m_s[k] || soa.mosfets.bodies[j] != nl->m_b[k])
        throw std::runtime_error("MOSFET SoA order mismatch");
    }
    for (size_t j = 0; j < soa.diodes.size(); ++j) {
      int k = dio_order[j];
      if (soa.diodes.node_a[j] != nl->d_anode[k] || soa.diodes.node_c[j] != nl->d_cathode[k])
        throw std::runtime_error("diode SoA order mismatch");
    }

    // devices the driver needs (SoA order for pnjlim and history)
    dio_a.assign(soa.diodes.node_a.begin(), soa.diodes.node_a.end());
    dio_c.assign(soa.diodes.node_c.begin(), soa.diodes.node_c.end());
    dio_is.assign(soa.diodes.Is.begin(), soa.diodes.Is.end());
    dio_vt.assign(soa.diodes.Vt.begin(), soa.diodes.Vt.end());
    cap_n1.assign(soa.capacitors.plates1.begin(), soa.capacitors.plates1.end());
    cap_n2.assign(soa.capacitors.plates2.begin(), soa.capacitors.plates2.end());
    cap_c.assign(soa.capacitors.C.begin(), soa.capacitors.C.end());
    for (const auto& d : net.globalBlock.diodes) seed_dio_anode.push_back(d.anode);
    for (const auto& c : net.globalBlock.currentSources) isrc_pos.push_back(c.nodePositive);

    sim = std::make_unique<CircuitSim>();
    sim->execMode = CircuitSim::ExecutionMode::TENSOR_SOA_SCALAR;
    build_pattern(true);
  }

  // Pattern from one full stamping pass plus gmin (the reference builds it
  // after addDiagonalConditioning, circuitsim_solver.cpp:256-264).
  CachedCsrPattern pattern_for(bool transient) {
    std::vector<double> v(n, 0.0);
    auto& mb = sim->matrixBuilder;
    mb.clear();
    mb.setDimensions(n, n);
    sim->rhsVector.assign(n, 0.0);
    for (size_t i = 0; i < soa.capacitors.size(); ++i) {
      soa.capacitors.v_prev[i] = 0.0;
      soa.capacitors.i_prev[i] = 0.0;
    }
    sim->stampSoABlock(soa, v, transient ? 1.0 : 0.0);
    sim->addDiagonalConditioning(n, 1e-12);
    return mb.buildPattern();
  }

  void build_pattern(bool transient) {
    cpat = pattern_for(transient);
    pat.n = n;
    pat.row_ptr = cpat.row_pointer;
    pat.col = cpat.col_indices;
    pat.diag.assign(n, -1);
    for (int i = 0; i < n; ++i)
      for (int k = pat.row_ptr[i]; k < pat.row_ptr[i + 1]; ++k)
        if (pat.col[k] == i) pat.diag[i] = k;
  }

  void set_instance(const karam_netlist* nl, const karam_instances* inst, int idx) {
    oracle::make_sources(nl, inst, idx, src);
    if (inst) {
      for (size_t j = 0; j < soa.mosfets.size(); ++j) {
        size_t k = (size_t)idx * nl->n_mos + mos_order[j];
        if (inst->mos_kp) soa.mosfets.Kp[j] = (double)inst->mos_kp[k];
        if (inst->mos_vto) soa.mosfets.Vth[j] = (double)inst->mos_vto[k];
      }
    }
    for (size_t i = 0; i < soa.voltageSources.size(); ++i) soa.voltageSources.voltages[i] = src.dc[i];
  }

  void stamp(const std::vector<double>& v, double h, int method, const std::vector<double>& cvp,
             const std::vector<double>& cip, double t, std::vector<double>& vals,
             std::vector<double>& rhs) {
    bool tran = h > 0.0;
    for (size_t i = 0; i < soa.voltageSources.size(); ++i)
      soa.voltageSources.voltages[i] = src.value_at((int)i, t, tran);
    double h_eff = 0.0;
    if (tran) {
      // stampSoABlock always stamps the trapezoidal companion 2C/h with
      // history g*v_prev + i_prev (physics/circuitsim.h:2480-2505). Backward
      // Euler (C/h, (C/h) v_prev) is the same stamp at 2h with i_prev = 0.
      h_eff = method == KARAM_TRAN_TRAP ? h : 2.0 * h;
      for (size_t i = 0; i < soa.capacitors.size(); ++i) {
        soa.capacitors.v_prev[i] = cvp[i];
        soa.capacitors.i_prev[i] = method == KARAM_TRAN_TRAP ? cip[i] : 0.0;
      }
    }
    auto& mb = sim->matrixBuilder;
    mb.clear();
    mb.setDimensions(n, n);
    sim->rhsVector.assign(n, 0.0);
    sim->stampSoABlock(soa, v, h_eff);
    Csr_matrix m = mb.assembleFast(cpat);
    vals = m.values;
    rhs = sim->rhsVector;
  }

  // Currents leaving every node at v, with the device currents the
  // reference kernels left in the SoA tensors during the last stamp() at v.
  void kcl(const std::vector<double>& v, double h, int method, const std::vector<double>& cvp,
           const std::vector<double>& cip, double t, std::vector<double>& F) {
    F.assign(n, 0.0);
    auto vn = [&](int node) { return node > 0 ? v[node - 1] : 0.0; };
    auto add = [&](int node, double cur) {
      if (node > 0) F[node - 1] += cur;
    };
    const bool tran = h > 0.0;
    const auto& R = soa.resistors;
    for (size_t k = 0; k < R.size(); ++k) {
      double i = (vn(R.nodes1[k]) - vn(R.nodes2[k])) / R.R[k];
      add(R.nodes1[k], i);
      add(R.nodes2[k], -i);
    }
    const auto& V = soa.voltageSources;
    for (size_t k = 0; k < V.size(); ++k) {
      double i = 1.0e3 * ((vn(V.nodesPos[k]) - vn(V.nodesNeg[k])) - src.value_at((int)k, t, tran));
      add(V.nodesPos[k], i);
      add(V.nodesNeg[k], -i);
    }
    const auto& I = soa.currentSources;
    for (size_t k = 0; k < I.size(); ++k) {
      add(I.nodesPos[k], I.currents[k]);
      add(I.nodesNeg[k], -I.currents[k]);
    }
    if (tran) {
      const double heff = method == KARAM_TRAN_TRAP ? h : 2.0 * h;
      const auto& Cp = soa.capacitors;
      for (size_t k = 0; k < Cp.size(); ++k) {
        double g = (2.0 * Cp.C[k]) / heff;
        double i = g * ((vn(Cp.plates1[k]) - vn(Cp.plates2[k])) - cvp[k]);
        if (method == KARAM_TRAN_TRAP) i -= cip[k];
        add(Cp.plates1[k], i);
        add(Cp.plates2[k], -i);
      }
    }
    const auto& D = soa.diodes;
    for (size_t k = 0; k < D.size(); ++k) {
      add(D.node_a[k], D.i_d[k]);
      add(D.node_c[k], -D.i_d[k]);
    }
    const auto& M = soa.mosfets;
    for (size_t k = 0; k < M.size(); ++k) {
      add(M.drains[k], M.ids[k]);
      add(M.sources[k], -M.ids[k]);
    }
  }

  Csr_matrix as_csr(const std::vector<double>& vals) const {
    Csr_matrix m;
    m.rows = n;
    m.cols = n;
    m.nnz = (int)vals.size();
    m.row_pointer = pat.row_ptr;
    m.col_indices = pat.col;
    m.values = vals;
    return m;
  }

  std::unique_ptr<SymbolicFactorization> sym;

  std::vector<uint32_t> translated_ordering(std::vector<uint32_t>* raw_out, int* tw) {
    FactorGraph fg = FactorGraph::fromTensorizedBlock(soa, (uint32_t)n);
    TreewidthAnalysis ta = TreewidthAnalyzer::analyze(fg);
    if (raw_out) *raw_out = ta.eliminationOrdering;
    if (tw) *tw = (int)ta.estimatedTreewidth;
    // The raw ordering mixes 1-based node ids with branch ids that start at
    // n (colliding with node n, factor_graph.cpp:23,127-138); symbolicFactorize
    // wants a 0-based permutation of size n. Keep ids 1..n, first occurrence
    // wins, subtract one.
    std::vector<uint32_t> perm;
    std::vector<char> seen(n + 1, 0);
    for (uint32_t id : ta.eliminationOrdering) {
      if (id >= 1 && id <= (uint32_t)n && !seen[id]) {
        seen[id] = 1;
        perm.push_back(id - 1);
      }
    }
    for (int i = 1; i <= n; ++i)
      if (!seen[i]) perm.push_back(i - 1);  // isolated unknowns last
    return perm;
  }

  bool solve(const std::vector<double>& vals, const std::vector<double>& rhs,
             std::vector<double>& x, int solver) {
    Csr_matrix m = as_csr(vals);
    SolverResult r;
    if (solver == ORACLE_LS_SPARSE) {
      if (!sym) sym = std::make_unique<SymbolicFactorization>(
                    symbolicFactorize(cpat, translated_ordering(nullptr, nullptr)));
      r = solveSparse_LU(m, rhs, *sym);
    } else {
      r = solveLU_Pivoted(m, rhs);
    }
    if (!r.converged) return false;
    x = r.solution;
    return true;
  }
};

struct Session {
  RefBackend b;
  Session(const karam_netlist* nl, const karam_instances* inst, int idx) {
    b.build(nl);
    b.set_instance(nl, inst, idx);
  }
};

template <class F>
int guarded(F f) {
  // The reference reports clamps and singular pivots on std::cerr; formatting
  // those messages inside this library crashed the host process, so its
  // diagnostics are silenced here (the results are returned, not printed).
  static const bool quiet = [] {
    std::cerr.setstate(std::ios::badbit);
    return true;
  }();
  (void)quiet;
  try {
    return f();
  } catch (const std::exception& e) {
    fprintf(stderr, "oracle(ref): %s\n", e.what());
    return -1;
  }
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
    Session s(nl, nullptr, 0);
    for (size_t i = 0; i < s.b.mos_order.size(); ++i) mos_order[i] = s.b.mos_order[i];
    for (size_t i = 0; i < s.b.dio_order.size(); ++i) dio_order[i] = s.b.dio_order[i];
    return 0;
  });
}

int oracle_pattern(const karam_netlist* nl, int32_t transient, int32_t* row_ptr, int32_t* col,
                   int32_t cap) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    CachedCsrPattern p = s.b.pattern_for(transient != 0);
    if (row_ptr) std::copy(p.row_pointer.begin(), p.row_pointer.end(), row_ptr);
    if (col && p.nnz <= cap) std::copy(p.col_indices.begin(), p.col_indices.end(), col);
    return p.nnz;
  });
}

int oracle_stamp_map(const karam_netlist* nl, int32_t* slot_csr, int32_t cap) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    auto& b = s.b;
    std::vector<double> v(b.n, 0.0);
    auto& mb = b.sim->matrixBuilder;
    mb.clear();
    mb.setDimensions(b.n, b.n);
    b.sim->rhsVector.assign(b.n, 0.0);
    b.sim->stampSoABlock(b.soa, v, 1.0);
    b.sim->addDiagonalConditioning(b.n, 1e-12);
    const auto& rows = mb.thread_rows[0];
    const auto& cols = mb.thread_cols[0];
    int nt = (int)rows.size();
    if (slot_csr && nt <= cap)
      for (int k = 0; k < nt; ++k) slot_csr[k] = b.cpat.indexOf(rows[k], cols[k]);
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

int oracle_ordering(const karam_netlist* nl, uint32_t* raw, int32_t* raw_len, int32_t* perm) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    std::vector<uint32_t> r;
    int tw = 0;
    std::vector<uint32_t> p = s.b.translated_ordering(&r, &tw);
    if (raw) std::copy(r.begin(), r.end(), raw);
    if (raw_len) *raw_len = (int32_t)r.size();
    if (perm) std::copy(p.begin(), p.end(), perm);
    return tw;
  });
}

int oracle_symbolic(const karam_netlist* nl, int32_t* perm, int32_t* iperm, int32_t* f_row_ptr,
                    int32_t* f_col, int32_t* fill_in, int32_t cap) {
  return guarded([&] {
    Session s(nl, nullptr, 0);
    SymbolicFactorization sf = symbolicFactorize(s.b.cpat, s.b.translated_ordering(nullptr, nullptr));
    if (perm) std::copy(sf.perm.begin(), sf.perm.end(), perm);
    if (iperm) std::copy(sf.iperm.begin(), sf.iperm.end(), iperm);
    if (f_row_ptr)
      std::copy(sf.filledPattern.row_pointer.begin(), sf.filledPattern.row_pointer.end(), f_row_ptr);
    if (f_col && sf.filledPattern.nnz <= cap)
      std::copy(sf.filledPattern.col_indices.begin(), sf.filledPattern.col_indices.end(), f_col);
    if (fill_in) *fill_in = sf.estimatedFillIn;
    return sf.filledPattern.nnz;
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
    oracle::Driver<RefBackend> d(s.b, *opts);
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
    oracle::Driver<RefBackend> d(s.b, *opts);
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
    std::vector<std::thread> pool;
    std::vector<int> rc(nt, 0);
    int n = 0;
    {
      Session probe(nl, nullptr, 0);
      n = probe.b.n;
    }
    for (int w = 0; w < nt; ++w) {
      pool.emplace_back([&, w] {
        for (int i = i0 + w; i < i1; i += nt) {
          Session s(nl, inst, i);
          oracle::Driver<RefBackend> d(s.b, *opts);
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

// Draws of the reference's seeded normal sampler (math/portable_rng.h:15-95):
// PortableRNG(seed) feeding PortableNormalDist(mean, sd), `count` calls in a row.
// Used to pin the Monte-Carlo parameter sampler of the test circuits.
int oracle_ref_normals(uint64_t seed, double mean, double sd, int32_t count, double* out) {
  acutesim::math::PortableRNG rng(seed);
  acutesim::math::PortableNormalDist dist(mean, sd);
  for (int32_t i = 0; i < count; ++i) out[i] = dist(rng);
  return 0;
}

int oracle_ac(const karam_netlist* nl, const karam_instances* inst, int32_t idx, const double* v_dc,
              double f_start, double f_stop, int32_t n_points, int32_t input_node, double amplitude,
              int32_t rule, double* out_re, double* out_im) {
  return guarded([&] {
    Session s(nl, inst, idx);
    auto& b = s.b;
    const int n = b.n;
    std::vector<double> v(v_dc, v_dc + n);
    int singular = 0;
    if (rule == 0) {  // the reference's sweep as it stands
      ACSolver::ACResult r =
          ACSolver::solveAC_Sparse(b.net, v, f_start, f_stop, n_points, input_node, amplitude);
      for (int k = 0; k < n_points; ++k)
        for (int i = 0; i < n; ++i) {
          out_re[(size_t)k * n + i] = r.nodeVoltages[k][i].real();
          out_im[(size_t)k * n + i] = r.nodeVoltages[k][i].imag();
        }
      return 0;
    }
    // the NR Jacobian of the reference's stamps at the DC point, solved by
    // the reference's complex LU
    std::vector<double> z(b.cap_c.size(), 0.0), jac, rhs;
    b.stamp(v, 0.0, KARAM_TRAN_BE, z, z, 0.0, jac, rhs);
    const std::vector<double> f = oracle::ac_frequencies(f_start, f_stop, n_points);
    std::vector<double> re, im, rre, rim(n, 0.0);
    for (int k = 0; k < n_points; ++k) {
      oracle::ac_matrix(b.pat, jac, b.cap_n1, b.cap_n2, b.cap_c, 2.0 * M_PI * f[k], input_node,
                        amplitude, re, im, rre);
      ComplexCsr Y;
      Y.rows = Y.cols = n;
      Y.nnz = (int)b.pat.col.size();
      Y.row_pointer = b.pat.row_ptr;
      Y.col_indices = b.pat.col;
      Y.values_real = re;
      Y.values_imag = im;
      ComplexSolverResult sol = solveComplexLU_Sparse(Y, rre, rim);
      if (sol.rankDeficient && !sol.converged) ++singular;
      std::copy(sol.solution_real.begin(), sol.solution_real.end(), out_re + (size_t)k * n);
      std::copy(sol.solution_imag.begin(), sol.solution_imag.end(), out_im + (size_t)k * n);
    }
    return singular;
  });
}

}  // extern "C"
