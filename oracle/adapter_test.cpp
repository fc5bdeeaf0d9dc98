// adapter_test.cpp -- C entry points that drive the reference-side adapter
// (karam_b200/adapter/karam_adapter.cpp) from a test (TEST INFRASTRUCTURE
// ONLY; built by oracle/Makefile, target adapter, into oracle/_ref/).
//
// A karam_netlist from the tests' builders becomes a reference TensorNetlist
// through the reference's own adders (netlist/circuit.h:1139-1216); the
// adapter then flattens it back and solves through libkaram_b200.so, either
// directly (KaramSolver::solveDC, CircuitSim::solveDC's replacement) or
// through the reference's AnalysisRegistry with the handlers it registers.
#include <algorithm>
#include <cstring>
#include <string>

#include "acutesim_engine/physics/circuitsim.h"
#include "acutesim_engine/solvers/analysis_registry.h"
#include "karam_adapter.hpp"

namespace {

TensorNetlist to_tensor_netlist(const karam_netlist* nl) {
  TensorNetlist net;
  net.environment.ambient_temp_K = nl->temp_k;
  for (int m = 0; m < nl->n_models; ++m) {
    ModelCard c;
    c.name = nl->model_name[m];
    const int ty = nl->model_type[m];
    c.type = ty == KARAM_MODEL_PMOS ? "PMOS" : (ty == KARAM_MODEL_NMOS ? "NMOS" : "D");
    if (nl->model_kp && !std::isnan(nl->model_kp[m])) c.params["KP"] = nl->model_kp[m];
    if (nl->model_vto && !std::isnan(nl->model_vto[m])) c.params["VTO"] = nl->model_vto[m];
    if (nl->model_lambda && !std::isnan(nl->model_lambda[m])) c.params["LAMBDA"] = nl->model_lambda[m];
    net.addModelCard(c);
  }
  for (int i = 0; i < nl->n_vsrc; ++i) {
    const bool pulse = nl->vs_kind && nl->vs_kind[i] == KARAM_SRC_PULSE;
    net.addVoltageSource(nl->vs_pos[i], nl->vs_neg[i], nl->vs_dc[i], pulse ? "PULSE" : "");
    if (pulse) {
      auto& vs = net.globalBlock.voltageSources.back();
      const double* p = nl->vs_pulse + 7 * i;
      vs.pulse_v1 = p[0]; vs.pulse_v2 = p[1]; vs.pulse_td = p[2]; vs.pulse_tr = p[3];
      vs.pulse_tf = p[4]; vs.pulse_pw = p[5]; vs.pulse_per = p[6];
    }
  }
  for (int i = 0; i < nl->n_isrc; ++i) net.addCurrentSource(nl->is_pos[i], nl->is_neg[i], nl->is_amp[i]);
  for (int i = 0; i < nl->n_res; ++i) net.addResistor(nl->r_n1[i], nl->r_n2[i], nl->r_ohm[i]);
  for (int i = 0; i < nl->n_cap; ++i) net.addCapacitor(nl->c_n1[i], nl->c_n2[i], nl->c_farad[i]);
  for (int i = 0; i < nl->n_dio; ++i) {
    net.globalBlock.addDiode("D" + std::to_string(i + 1), nl->d_anode[i], nl->d_cathode[i], nl->d_is[i],
                             nl->d_n[i], nl->d_vt[i]);
    const int mi = nl->d_model ? nl->d_model[i] : -1;
    net.globalBlock.diodes.back().modelName = mi >= 0 ? std::string(nl->model_name[mi]) : "diode_generic";
    net.numGlobalNodes = std::max({net.numGlobalNodes, nl->d_anode[i], nl->d_cathode[i]});
  }
  for (int i = 0; i < nl->n_mos; ++i)
    net.addMosfet("M" + std::to_string(i + 1), nl->m_d[i], nl->m_g[i], nl->m_s[i], nl->m_b[i],
                  nl->model_name[nl->m_model[i]], nl->m_w[i], nl->m_l[i]);
  net.numGlobalNodes = std::max(net.numGlobalNodes, nl->n_nodes);
  return net;
}

}  // namespace

extern "C" {

// DC operating point of nl through the adapter: via_registry = 0 calls
// KaramSolver::solveDC, 1 dispatches AnalysisTypeDTO::DC through the
// reference's AnalysisRegistry. v_out[0 .. n) receives the node voltages of
// nodes 1..n; returns 0 or -1 (message in err, 256 bytes).
int adapter_test_dc(const karam_netlist* nl, int32_t via_registry, double* v_out, int32_t* n_out,
                    int32_t* iterations, int32_t* converged, char* err) {
  try {
    TensorNetlist net = to_tensor_netlist(nl);
    std::vector<double> v;
    if (via_registry) {
      acutesim::orchestration::SimulationRequestDTO req;
      req.analysis = acutesim::orchestration::AnalysisTypeDTO::DC;
      CircuitSim sim;
      const auto r = acutesim::compute::AnalysisRegistry::instance().dispatch(req.analysis, req, net, sim);
      if (r.waveformPoints.empty()) throw std::runtime_error("no result: " + r.errorDetail);
      v = r.waveformPoints[0].nodeVoltages;
      *iterations = r.iterations;
      *converged = r.converged ? 1 : 0;
    } else {
      const SolverStep s = karam_adapter::thread_solver().solveDC(net);
      v = s.nodeVoltages;
      *iterations = s.stats.iterations;
      *converged = s.stats.converged ? 1 : 0;
    }
    *n_out = (int32_t)v.size() - 1;
    for (size_t i = 1; i < v.size(); ++i) v_out[i - 1] = v[i];
    return 0;
  } catch (const std::exception& e) {
    std::strncpy(err, e.what(), 255);
    err[255] = 0;
    return -1;
  }
}

// Whether the reference's registry now serves DC, TRANSIENT and MONTE_CARLO.
int adapter_test_registered(void) {
  auto& reg = acutesim::compute::AnalysisRegistry::instance();
  using acutesim::orchestration::AnalysisTypeDTO;
  return reg.supports(AnalysisTypeDTO::DC) && reg.supports(AnalysisTypeDTO::TRANSIENT) &&
         reg.supports(AnalysisTypeDTO::MONTE_CARLO);
}

// BE transient of nl through the registry's TRANSIENT handler: `steps` steps
// of dt after the DC point; wave_out[k][i] = node i + 1 after step k + 1.
int adapter_test_tran(const karam_netlist* nl, double dt, int32_t steps, double* wave_out,
                      int32_t* converged, char* err) {
  try {
    TensorNetlist net = to_tensor_netlist(nl);
    acutesim::orchestration::SimulationRequestDTO req;
    req.analysis = acutesim::orchestration::AnalysisTypeDTO::TRANSIENT;
    req.transient.stepSizeS = dt;
    req.transient.stopTimeS = dt * steps;
    CircuitSim sim;
    const auto r = acutesim::compute::AnalysisRegistry::instance().dispatch(req.analysis, req, net, sim);
    *converged = r.converged ? 1 : 0;
    if ((int)r.waveformPoints.size() != steps + 1) throw std::runtime_error("waveform length: " + r.errorDetail);
    const int n = (int)r.waveformPoints[0].nodeVoltages.size() - 1;
    for (int k = 0; k < steps; ++k)
      for (int i = 0; i < n; ++i) wave_out[(size_t)k * n + i] = r.waveformPoints[k + 1].nodeVoltages[i + 1];
    return 0;
  } catch (const std::exception& e) {
    std::strncpy(err, e.what(), 255);
    err[255] = 0;
    return -1;
  }
}

}  // extern "C"
