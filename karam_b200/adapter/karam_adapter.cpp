// karam_adapter.cpp -- reference-side binding of the B200 NR inner loop (see
// karam_adapter.hpp): TensorNetlist -> karam_netlist, SolverStep results and
// the AnalysisRegistry handlers for DC / TRANSIENT / MONTE_CARLO.
#include "karam_adapter.hpp"

#include <cmath>
#include <limits>
#include <map>
#include <stdexcept>

#include "acutesim_engine/math/portable_rng.h"
#include "acutesim_engine/physics/circuitsim.h"
#include "acutesim_engine/solvers/analysis_registry.h"

namespace karam_adapter {

namespace {
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();
double card_param(const ModelCard& c, const char* key) {
  auto it = c.params.find(key);
  return it == c.params.end() ? kNaN : it->second;
}
}  // namespace

FlatNetlist::FlatNetlist(const TensorNetlist& net) {
  const TensorBlock& b = net.globalBlock;
  // model cards in the netlist's (name-ordered) map, then the device model
  // names that have no card: tensorizeNetlist buckets devices by model name
  // (tensors/physics_tensors.cpp:481-490), so every name must exist
  std::map<std::string, int> idx;
  auto add_model = [&](const std::string& name, int type, double kp, double vto, double lam) {
    idx[name] = (int)names_.size();
    names_.push_back(name);
    mt_.push_back(type);
    kp_.push_back(kp);
    vto_.push_back(vto);
    lam_.push_back(lam);
  };
  for (const auto& kv : net.modelCards) {
    const ModelCard& c = kv.second;
    const int type = c.type == "PMOS" ? KARAM_MODEL_PMOS : c.type == "NMOS" ? KARAM_MODEL_NMOS : KARAM_MODEL_DIODE;
    add_model(kv.first, type, card_param(c, "KP"), card_param(c, "VTO"), card_param(c, "LAMBDA"));
  }
  for (const Mosfet& m : b.mosfets)
    if (!idx.count(m.modelName)) add_model(m.modelName, KARAM_MODEL_NMOS, kNaN, kNaN, kNaN);  // no card: NMOS defaults
  for (const Diode& d : b.diodes)
    if (!idx.count(d.modelName)) add_model(d.modelName, KARAM_MODEL_DIODE, kNaN, kNaN, kNaN);

  for (const VoltageSource& v : b.voltageSources) {
    vp_.push_back(v.nodePositive);
    vn_.push_back(v.nodeNegative);
    vdc_.push_back(v.voltage_V);
    const bool pulse = v.type == "PULSE";
    vk_.push_back(pulse ? KARAM_SRC_PULSE : KARAM_SRC_DC);
    for (double p : {v.pulse_v1, v.pulse_v2, v.pulse_td, v.pulse_tr, v.pulse_tf, v.pulse_pw, v.pulse_per})
      vpulse_.push_back(pulse ? p : 0.0);
  }
  for (const CurrentSource& i : b.currentSources) {
    ip_.push_back(i.nodePositive);
    in_.push_back(i.nodeNegative);
    iamp_.push_back(i.current_A);
  }
  for (const Resistor& r : b.resistors) {
    r1_.push_back(r.nodeTerminal1);
    r2_.push_back(r.nodeTerminal2);
    r_.push_back(r.resistance_ohms);
  }
  for (const Capacitor& c : b.capacitors) {
    c1_.push_back(c.nodePlate1);
    c2_.push_back(c.nodePlate2);
    c_.push_back(c.capacitance_farads);
  }
  for (const Diode& d : b.diodes) {
    da_.push_back(d.anode);
    dc_.push_back(d.cathode);
    dis_.push_back(d.saturationCurrent_I_S_A);
    dn_.push_back(d.emissionCoefficient_N);
    dvt_.push_back(d.thermalVoltage_V_T_V);
    dm_.push_back(d.modelName == "diode_generic" ? -1 : idx.at(d.modelName));
  }
  for (const Mosfet& m : b.mosfets) {
    md_.push_back(m.drain);
    mg_.push_back(m.gate);
    ms_.push_back(m.source);
    mb_.push_back(m.body);
    mw_.push_back(m.w);
    ml_.push_back(m.l);
    mm_.push_back(idx.at(m.modelName));
  }
  for (const std::string& s : names_) cnames_.push_back(s.c_str());

  nl_.n_nodes = net.numGlobalNodes;
  nl_.temp_k = net.environment.ambient_temp_K;
  nl_.n_vsrc = (int32_t)vdc_.size();
  nl_.vs_pos = vp_.data();
  nl_.vs_neg = vn_.data();
  nl_.vs_dc = vdc_.data();
  nl_.vs_kind = vk_.data();
  nl_.vs_pulse = vpulse_.data();
  nl_.n_isrc = (int32_t)iamp_.size();
  nl_.is_pos = ip_.data();
  nl_.is_neg = in_.data();
  nl_.is_amp = iamp_.data();
  nl_.n_res = (int32_t)r_.size();
  nl_.r_n1 = r1_.data();
  nl_.r_n2 = r2_.data();
  nl_.r_ohm = r_.data();
  nl_.n_cap = (int32_t)c_.size();
  nl_.c_n1 = c1_.data();
  nl_.c_n2 = c2_.data();
  nl_.c_farad = c_.data();
  nl_.n_dio = (int32_t)dis_.size();
  nl_.d_anode = da_.data();
  nl_.d_cathode = dc_.data();
  nl_.d_is = dis_.data();
  nl_.d_n = dn_.data();
  nl_.d_vt = dvt_.data();
  nl_.d_model = dm_.data();
  nl_.n_mos = (int32_t)mw_.size();
  nl_.m_d = md_.data();
  nl_.m_g = mg_.data();
  nl_.m_s = ms_.data();
  nl_.m_b = mb_.data();
  nl_.m_w = mw_.data();
  nl_.m_l = ml_.data();
  nl_.m_model = mm_.data();
  nl_.n_models = (int32_t)names_.size();
  nl_.model_name = cnames_.data();
  nl_.model_type = mt_.data();
  nl_.model_kp = kp_.data();
  nl_.model_vto = vto_.data();
  nl_.model_lambda = lam_.data();
}

KaramSolver::KaramSolver(int device) {
  if (karam_ctx_create(device, &ctx_) != KARAM_OK)
    throw std::runtime_error(std::string("karam_ctx_create: ") + karam_last_error(nullptr));
}

KaramSolver::~KaramSolver() {
  karam_problem_destroy(prob_);
  karam_ctx_destroy(ctx_);
}

// The problem of this netlist's content with room for `instances`: reused
// while the netlist's fingerprint (karam_netlist_hash: structure and values,
// the role of TensorBlock::topologyHash at circuitsim_solver.cpp:262-268) and
// the batch fit; the library's own symbolic cache makes a rebuild cheap.
karam_problem* KaramSolver::problem(const TensorNetlist& net, int instances) {
  FlatNetlist flat(net);
  uint64_t h = 0;
  karam_netlist_hash(&flat.get(), &h);
  if (prob_ && h == hash_ && instances <= cap_) return prob_;
  karam_problem_destroy(prob_);
  prob_ = nullptr;
  if (karam_problem_create(ctx_, &flat.get(), instances, &prob_) != KARAM_OK) {
    err_ = karam_last_error(ctx_);
    prob_ = nullptr;
    return nullptr;
  }
  karam_problem_info info{};
  karam_problem_info_get(prob_, &info);
  hash_ = h;
  cap_ = instances;
  n_ = info.n;
  return prob_;
}

// SolverStep of one instance (circuitsim_solver.cpp:529-554): voltages with
// ground at index 0, iterations, residual, convergence, failure diagnostics.
SolverStep KaramSolver::step_of(const karam_instance_stats& st, const double* v, int n, int rc,
                                double t) {
  SolverStep step;
  step.time = t;
  step.nodeVoltages.assign(n + 1, 0.0);
  for (int i = 0; i < n; ++i) step.nodeVoltages[i + 1] = v[i];
  SolverStats& s = step.stats;
  s.converged = rc == KARAM_OK && st.status == KARAM_ST_CONVERGED;
  s.iterations = st.iterations;
  s.residual = st.residual;
  s.method = "Newton-Raphson";
  s.gminSteppingUsed = st.gmin_step > 0;
  s.failureType = static_cast<ConvergenceFailureType>(st.failure_type);
  s.stagnationDetected = st.stagnation != 0;
  s.divergenceDetected = st.divergence != 0;
  s.rankDeficient = st.status == KARAM_ST_SINGULAR;
  if (!s.converged) {
    s.error_detail = rc != KARAM_OK ? std::string(karam_last_error(ctx_))
                     : st.status == KARAM_ST_SINGULAR ? "singular matrix"
                     : st.status == KARAM_ST_NAN      ? "non-finite residual"
                     : st.status == KARAM_ST_TIMEOUT  ? "round budget exhausted"
                                                      : "NR did not converge";
  }
  return step;
}

SolverStep KaramSolver::solveDC(const TensorNetlist& net, const karam_solver_opts* opts) {
  karam_problem* p = problem(net, 1);
  if (!p) {
    SolverStep step;
    step.stats.error_detail = err_;
    return step;
  }
  karam_set_instances(p, nullptr);  // the netlist's own values
  karam_solver_opts o;
  if (opts)
    o = *opts;
  else
    karam_default_opts(&o);
  std::vector<double> v(n_);
  karam_instance_stats st{};
  const int rc = karam_solve_dc(p, &o, nullptr, v.data(), &st);
  return step_of(st, v.data(), n_, rc, 0.0);
}

SolverStep KaramSolver::stepTransient(const TensorNetlist& net, double dt, int method,
                                      const karam_solver_opts* opts) {
  karam_problem* p = problem(net, 1);
  if (!p) {
    SolverStep step;
    step.stats.error_detail = err_;
    return step;
  }
  karam_solver_opts o;
  if (opts)
    o = *opts;
  else
    karam_default_opts(&o);
  std::vector<double> v(n_);
  karam_instance_stats st{};
  const int rc = karam_step_transient(p, &o, dt, 1, method, nullptr, 0, nullptr, v.data(), &st);
  return step_of(st, v.data(), n_, rc, 0.0);
}

std::vector<SolverStep> KaramSolver::runMonteCarlo(const TensorNetlist& net,
                                                   const karam_instances& inst, double dt,
                                                   int n_steps, const karam_solver_opts* opts) {
  std::vector<SolverStep> out;
  karam_problem* p = problem(net, inst.n_instances);
  if (!p) return out;
  karam_solver_opts o;
  if (opts)
    o = *opts;
  else
    karam_default_opts(&o);
  std::vector<double> v((size_t)inst.n_instances * n_);
  std::vector<karam_instance_stats> st(inst.n_instances);
  const int rc = karam_run_mc(p, &inst, &o, dt, n_steps, KARAM_TRAN_BE, v.data(), st.data());
  for (int i = 0; i < inst.n_instances; ++i)
    out.push_back(step_of(st[i], v.data() + (size_t)i * n_, n_, rc, dt * n_steps));
  return out;
}

KaramSolver& thread_solver() {
  thread_local std::unique_ptr<KaramSolver> s;
  if (!s) s = std::make_unique<KaramSolver>(0);
  return *s;
}

}  // namespace karam_adapter

// ---------------------------------------------------------------------------
// AnalysisRegistry handlers (solvers/analysis_registry.h:25-63)
// ---------------------------------------------------------------------------
namespace {

using acutesim::orchestration::SimulationRequestDTO;
using acutesim::orchestration::SimulationResponseDTO;
using acutesim::orchestration::WaveformPointDTO;

void fill(SimulationResponseDTO& r, const SolverStep& s, const char* kind) {
  r.success = s.stats.converged;
  r.converged = s.stats.converged;
  r.iterations = s.stats.iterations;
  r.residual = s.stats.residual;
  r.errorDetail = s.stats.error_detail;
  r.analysisType = kind;
  r.solverProvenance = "karam_b200 (B200 NR inner loop): " + s.stats.provenance();
  WaveformPointDTO w;
  w.timeS = s.time;
  w.nodeVoltages = s.nodeVoltages;
  r.waveformPoints.push_back(std::move(w));
}

// DC operating point.
SimulationResponseDTO karamDcHandler(const SimulationRequestDTO&, const TensorNetlist& net, CircuitSim&) {
  SimulationResponseDTO r;
  fill(r, karam_adapter::thread_solver().solveDC(net), "DC");
  return r;
}

// DC, then fixed backward-Euler steps of transient.stepSizeS up to
// transient.stopTimeS; one waveform point per step.
SimulationResponseDTO karamTranHandler(const SimulationRequestDTO& req, const TensorNetlist& net,
                                       CircuitSim&) {
  SimulationResponseDTO r;
  karam_adapter::KaramSolver& S = karam_adapter::thread_solver();
  SolverStep dc = S.solveDC(net);
  fill(r, dc, "TRANSIENT");
  const double h = req.transient.stepSizeS;
  if (!dc.stats.converged || !(h > 0)) return r;
  const int steps = (int)std::llround(req.transient.stopTimeS / h);
  for (int k = 1; k <= steps; ++k) {
    SolverStep s = S.stepTransient(net, h);
    s.time = k * h;
    WaveformPointDTO w;
    w.timeS = s.time;
    w.nodeVoltages = s.nodeVoltages;
    r.waveformPoints.push_back(std::move(w));
    r.iterations += s.stats.iterations;
    r.residual = s.stats.residual;
    if (!s.stats.converged) {
      r.success = r.converged = false;
      r.errorDetail = s.stats.error_detail;
      break;
    }
  }
  return r;
}

// Monte Carlo: parameters["mc_runs"] instances of Gaussian KP (5 %) / VTO
// (30 mV) variation per MOSFET from the reference's PortableRNG seeded
// req.mcSeed + run, the DC point of each in one batch; one waveform point
// (t = 0) per run.
SimulationResponseDTO karamMcHandler(const SimulationRequestDTO& req, const TensorNetlist& net,
                                     CircuitSim&) {
  SimulationResponseDTO r;
  karam_adapter::FlatNetlist flat(net);
  const karam_netlist& nl = flat.get();
  auto it = req.parameters.find("mc_runs");
  const int runs = it == req.parameters.end() ? 1 : std::max(1, (int)it->second);
  std::vector<float> kp((size_t)runs * nl.n_mos), vto((size_t)runs * nl.n_mos);
  for (int i = 0; i < runs; ++i) {
    acutesim::math::PortableRNG rng(req.mcSeed + (uint64_t)i);
    acutesim::math::PortableNormalDist nd(0.0, 1.0);
    for (int m = 0; m < nl.n_mos; ++m) {
      const int c = nl.m_model[m];
      const double zv = nd(rng), zk = nd(rng);
      vto[(size_t)i * nl.n_mos + m] = (float)(nl.model_vto[c] + 0.03 * zv);
      kp[(size_t)i * nl.n_mos + m] = (float)(nl.model_kp[c] * (1.0 + 0.05 * zk));
    }
  }
  karam_instances inst{};
  inst.n_instances = runs;
  inst.mos_kp = kp.data();
  inst.mos_vto = vto.data();
  std::vector<SolverStep> steps = karam_adapter::thread_solver().runMonteCarlo(net, inst, 0.0, 0);
  r.success = r.converged = !steps.empty();
  r.analysisType = "MONTE_CARLO";
  for (const SolverStep& s : steps) {
    r.converged = r.converged && s.stats.converged;
    r.iterations += s.stats.iterations;
    WaveformPointDTO w;
    w.nodeVoltages = s.nodeVoltages;
    r.waveformPoints.push_back(std::move(w));
  }
  r.success = r.converged;
  return r;
}

using acutesim::compute::RegisterAnalysis;
using acutesim::orchestration::AnalysisTypeDTO;
RegisterAnalysis<AnalysisTypeDTO::DC, &karamDcHandler> s_karam_dc;
RegisterAnalysis<AnalysisTypeDTO::TRANSIENT, &karamTranHandler> s_karam_tran;
RegisterAnalysis<AnalysisTypeDTO::MONTE_CARLO, &karamMcHandler> s_karam_mc;

}  // namespace
