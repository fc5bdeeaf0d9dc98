// jit.cpp -- the LU round compiled at run time for one topology.
//
// The LU program of a topology (fixed pattern, fixed ordering, fixed static
// pivots) is turned into straight-line CUDA: every value position is an
// immediate offset into the instance's shared-memory row, so the compiler
// schedules the whole elimination with no index loads on the critical path.
// The text is compiled by NVRTC for sm_100a together with nr_device.cuh (the
// same control flow the static kernels use) and loaded with the CUDA runtime's
// library API. NVRTC is opened with dlopen; without it the static interpreter
// kernel runs instead.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "device.hpp"
#include "topology.hpp"

namespace karam {
namespace {

#include "jit_sources.inc"  // kNrTypesSource, kNrDeviceSource (generated by build.py)

// Generated code above this many LU operations compiles too slowly to pay off.
constexpr int kMaxJitOps = 120000;

struct Nvrtc {
  void* h = nullptr;
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
  decltype(&nvrtcGetErrorString) err = nullptr;
  bool ok() const { return h && create && compile && log_size && log && cubin_size && cubin && destroy; }
};

Nvrtc& nvrtc() {
  static Nvrtc n = [] {
    Nvrtc r;
    const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
    for (const char* nm : names) {
      r.h = dlopen(nm, RTLD_NOW | RTLD_LOCAL);
      if (r.h) break;
    }
    if (!r.h) return r;
    r.create = (decltype(r.create))dlsym(r.h, "nvrtcCreateProgram");
    r.compile = (decltype(r.compile))dlsym(r.h, "nvrtcCompileProgram");
    r.log_size = (decltype(r.log_size))dlsym(r.h, "nvrtcGetProgramLogSize");
    r.log = (decltype(r.log))dlsym(r.h, "nvrtcGetProgramLog");
    r.cubin_size = (decltype(r.cubin_size))dlsym(r.h, "nvrtcGetCUBINSize");
    r.cubin = (decltype(r.cubin))dlsym(r.h, "nvrtcGetCUBIN");
    r.destroy = (decltype(r.destroy))dlsym(r.h, "nvrtcDestroyProgram");
    r.err = (decltype(r.err))dlsym(r.h, "nvrtcGetErrorString");
    return r;
  }();
  return n;
}

// Straight-line restatement of InterpFS::run for this topology's program.
std::string generate_factor_solve(const Topology& T) {
  std::ostringstream o;
  const int n = T.n;
  o << "struct GenFS {\n  template <typename T>\n"
       "  __device__ static bool run(T* __restrict__ A, T* __restrict__ y, const DevTopo& Tp,\n"
       "                             T tiny, T growth_limit) {\n"
       "    bool ok = true;\n    T lmax = T(0);\n    T r, l, s;\n";
  for (int k = 0; k < n; ++k) {
    const int off = T.lu_hdr[4 * k], nl = T.lu_hdr[4 * k + 1], nu = T.lu_hdr[4 * k + 2],
              dp = T.lu_hdr[4 * k + 3];
    const int* lp = &T.lu_data[off + nl];
    const int* up = lp + nl + nu;
    const int* tp = up + nu;
    o << "    r = A[" << dp << "]; ok = ok && isfinite(r) && !(fabs(r) < tiny); r = T(1) / r; A["
      << dp << "] = r;\n";
    for (int a = 0; a < nl; ++a) {
      o << "    l = A[" << lp[a] << "] * r; lmax = fmax(lmax, fabs(l)); A[" << lp[a] << "] = l;";
      for (int b = 0; b < nu; ++b) o << " A[" << tp[a * nu + b] << "] -= l * A[" << up[b] << "];";
      o << "\n";
    }
  }
  for (int k = 0; k < n; ++k) {
    const int off = T.lu_hdr[4 * k], nl = T.lu_hdr[4 * k + 1];
    if (nl == 0) continue;
    const int* lr = &T.lu_data[off];
    const int* lp = lr + nl;
    o << "    s = y[" << k << "];";
    for (int a = 0; a < nl; ++a) o << " y[" << lr[a] << "] -= A[" << lp[a] << "] * s;";
    o << "\n";
  }
  for (int k = n - 1; k >= 0; --k) {
    const int off = T.lu_hdr[4 * k], nl = T.lu_hdr[4 * k + 1], nu = T.lu_hdr[4 * k + 2],
              dp = T.lu_hdr[4 * k + 3];
    const int* uc = &T.lu_data[off + 2 * nl];
    const int* up = uc + nu;
    o << "    s = y[" << k << "];";
    for (int b = 0; b < nu; ++b) o << " s -= A[" << up[b] << "] * y[" << uc[b] << "];";
    o << " y[" << k << "] = s * A[" << dp << "];\n";
  }
  o << "    bool fin = true;\n    for (int i = 0; i < " << n
    << "; ++i) fin = fin && isfinite(y[i]);\n"
       "    return ok && fin && !(lmax > growth_limit);\n  }\n};\n";
  o << "extern \"C\" __global__ void __launch_bounds__(256) karam_lu_jit_f32(DevTopo Tp, DevInst I,\n"
       "    JobParams P, int NI, int S, int Sv, int* active) {\n"
       "  knr::lu_round<float, GenFS>(Tp, I, P, NI, S, Sv, active);\n}\n";
  o << "extern \"C\" __global__ void __launch_bounds__(256) karam_lu_jit_f64(DevTopo Tp, DevInst I,\n"
       "    JobParams P, int NI, int S, int Sv, int* active) {\n"
       "  knr::lu_round<double, GenFS>(Tp, I, P, NI, S, Sv, active);\n}\n";
  return o.str();
}

}  // namespace

void jit_build(const Topology& T, JitLu& J) {
  J = JitLu{};
  // Opt-in: NVRTC spends seconds on the straight-line code of a few hundred
  // pivots, more than a short job gains back.
  const char* env = getenv("KARAM_JIT");
  if (!env || std::strcmp(env, "1") != 0) {
    J.status = "interpreter (run-time compiled LU not requested; KARAM_JIT=1 enables it)";
    return;
  }
  if (T.lu_ops > kMaxJitOps) {
    J.status = "LU program too large for straight-line code";
    return;
  }
  Nvrtc& N = nvrtc();
  if (!N.ok()) {
    J.status = "NVRTC not available";
    return;
  }
  auto t0 = std::chrono::steady_clock::now();
  std::string src = std::string(kNrTypesSource) + "\n" + kNrDeviceSource + "\n" +
                    "using namespace knr;\n" + generate_factor_solve(T);
  nvrtcProgram prog = nullptr;
  if (N.create(&prog, src.c_str(), "karam_lu_jit.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
    J.status = "nvrtcCreateProgram failed";
    return;
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-DKARAM_JIT", "-lineinfo"};
  nvrtcResult rc = N.compile(prog, 4, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t ls = 0;
    N.log_size(prog, &ls);
    std::string log(ls, '\0');
    if (ls) N.log(prog, &log[0]);
    J.status = "NVRTC compile failed: " + log.substr(0, 2000);
    N.destroy(&prog);
    return;
  }
  size_t cs = 0;
  N.cubin_size(prog, &cs);
  std::vector<char> cubin(cs);
  N.cubin(prog, cubin.data());
  N.destroy(&prog);
  cudaLibrary_t lib = nullptr;
  cudaError_t e = cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
  if (e != cudaSuccess) {
    J.status = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return;
  }
  cudaKernel_t k32 = nullptr, k64 = nullptr;
  if (cudaLibraryGetKernel(&k32, lib, "karam_lu_jit_f32") != cudaSuccess ||
      cudaLibraryGetKernel(&k64, lib, "karam_lu_jit_f64") != cudaSuccess) {
    J.status = "kernel lookup failed";
    cudaGetLastError();
    cudaLibraryUnload(lib);
    return;
  }
  J.library = lib;
  J.kernel_f32 = (void*)k32;
  J.kernel_f64 = (void*)k64;
  J.ok = true;
  J.status = "ready";
  J.compile_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void jit_release(JitLu& J) {
  if (J.library) cudaLibraryUnload((cudaLibrary_t)J.library);
  J = JitLu{};
}

void configure_jit(const JitLu& J, const LuLaunch& L) {
  if (!J.ok) return;
  cudaFuncSetAttribute((const void*)J.kernel_f32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)L.smem);
  cudaFuncSetAttribute((const void*)J.kernel_f64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)L.smem);
}

void launch_lu_jit(const JitLu& J, const DevTopo& T, const DevInst& I, const JobParams& P,
                   const LuLaunch& L, int prec, int* active, cudaStream_t s) {
  DevTopo t = T;
  DevInst in = I;
  JobParams p = P;
  int ni = L.ni_per_cta, S = L.S, Sv = L.Sv;
  void* args[] = {&t, &in, &p, &ni, &S, &Sv, &active};
  const void* k = prec == KPREC_MIXED ? J.kernel_f32 : J.kernel_f64;
  cudaLaunchKernel(k, dim3(L.grid), dim3(256), args, L.smem, s);
}

}  // namespace karam
