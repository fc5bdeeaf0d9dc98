// karam_adapter.hpp -- the reference-side binding of the B200 NR inner loop.
//
// This is the translation unit a maintainer of the reference engine adds to
// route its DC, transient and Monte-Carlo analyses through libkaram_b200.so:
// it flattens a TensorNetlist (netlist/circuit.h:1056-1216) into the C ABI's
// karam_netlist, keeps one karam_problem per topology, returns SolverStep /
// SolverStats (infrastructure/simtrace.h:76-136) filled the way
// CircuitSim::solveDC fills them (solvers/circuitsim_solver.cpp:529-554), and
// registers DC / TRANSIENT / MONTE_CARLO handlers with the reference's
// AnalysisRegistry (solvers/analysis_registry.h:25-63), which ships handlers
// for TF / PZ / FOURIER only (solvers/register_analyses.cpp:132-138). It is
// compiled against the reference's headers (oracle/Makefile, target adapter).
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "acutesim_engine/infrastructure/simtrace.h"
#include "acutesim_engine/netlist/circuit.h"
#include "karam.h"

namespace karam_adapter {

// The C ABI's view of a TensorNetlist's global block; the arrays live as
// long as the object.
class FlatNetlist {
 public:
  explicit FlatNetlist(const TensorNetlist& net);
  const karam_netlist& get() const { return nl_; }
  // model card index of each MOSFET, in netlist order
  const std::vector<int32_t>& mos_models() const { return mm_; }

 private:
  std::vector<int32_t> vp_, vn_, vk_, ip_, in_, r1_, r2_, c1_, c2_, da_, dc_, dm_, md_, mg_, ms_, mb_, mm_, mt_;
  std::vector<double> vdc_, vpulse_, iamp_, r_, c_, dis_, dn_, dvt_, mw_, ml_, kp_, vto_, lam_;
  std::vector<std::string> names_;
  std::vector<const char*> cnames_;
  karam_netlist nl_{};
};

// One GPU context and the problem of the last topology it solved.
class KaramSolver {
 public:
  explicit KaramSolver(int device = 0);
  ~KaramSolver();
  KaramSolver(const KaramSolver&) = delete;
  KaramSolver& operator=(const KaramSolver&) = delete;

  // CircuitSim::solveDC (physics/circuitsim.h:1110): plain FP64 NR (or the
  // precision of opts) on the netlist's own values. nodeVoltages[0] is ground.
  SolverStep solveDC(const TensorNetlist& net, const karam_solver_opts* opts = nullptr);
  // CircuitSim::stepTransient (physics/circuitsim.h:1111): one step of dt
  // from the last accepted point (the DC point after solveDC).
  SolverStep stepTransient(const TensorNetlist& net, double dt, int method = KARAM_TRAN_BE,
                           const karam_solver_opts* opts = nullptr);
  // A Monte-Carlo batch (SessionImpl::runMonteCarlo's role, engine_impl.cpp:259-281):
  // DC then n_steps transient steps of every instance; one SolverStep each.
  std::vector<SolverStep> runMonteCarlo(const TensorNetlist& net, const karam_instances& inst,
                                        double dt, int n_steps, const karam_solver_opts* opts = nullptr);
  const std::string& lastError() const { return err_; }

 private:
  karam_problem* problem(const TensorNetlist& net, int instances);
  SolverStep step_of(const karam_instance_stats& st, const double* v, int n, int rc, double t);
  karam_ctx* ctx_ = nullptr;
  karam_problem* prob_ = nullptr;
  uint64_t hash_ = 0;
  int cap_ = 0, n_ = 0;
  std::string err_;
};

// The thread's solver (created on first use, device 0), as the registry
// handlers use it.
KaramSolver& thread_solver();

}  // namespace karam_adapter
