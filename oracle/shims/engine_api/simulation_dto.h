// Build shim: the DTOs of engine_api/simulation_dto.h, which the reference
// includes (solvers/analysis_registry.h:17, engine_impl.cpp:25) but does not
// ship. Only the fields the reference's own code reads and writes are here
// (engine_impl.cpp:41-61,121-320; solvers/register_analyses.cpp:33-53), so its
// analysis registry and the adapter compile against it. TEST / INTEGRATION
// INFRASTRUCTURE ONLY.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace acutesim {
namespace orchestration {

enum class AnalysisTypeDTO { DC, AC, TRANSIENT, MONTE_CARLO, TF, TRANSFER_FUNCTION, POLE_ZERO, FOURIER };
enum class PrecisionMode { Native_F64, Emulated_F64, Mixed };

struct SourceDTO {
  std::string payload;  // netlist text
  std::string format;   // "spice", ...
};

struct TransientDTO {
  double stopTimeS = 0.0;
  double stepSizeS = 0.0;
};

struct CornerDTO {
  std::string processCorner = "TT";
  double temperature = 27.0;
  double supplyVoltage = 1.8;
};

struct SimulationRequestDTO {
  SourceDTO source;
  AnalysisTypeDTO analysis = AnalysisTypeDTO::DC;
  TransientDTO transient;
  CornerDTO corner;
  std::map<std::string, double> parameters;
  uint64_t topologyHash = 0;
  uint64_t mcSeed = 0;
};

struct WaveformPointDTO {
  double timeS = 0.0;
  std::vector<double> nodeVoltages;
};

struct SimulationResponseDTO {
  std::string jobId;
  bool converged = false;
  bool success = false;
  int iterations = 0;
  double residual = 0.0;
  std::string errorDetail;
  std::vector<WaveformPointDTO> waveformPoints;
  std::string solverProvenance;
  PrecisionMode precisionMode = PrecisionMode::Native_F64;
  double solveTimeMs = 0.0;
  std::string analysisType;
  uint64_t topologyHash = 0;
};

struct MonteCarloConfigDTO {
  int numRuns = 0;
  uint64_t seed = 0;
};

}  // namespace orchestration
}  // namespace acutesim
