// device.hpp -- host-side declarations of the kernel launchers. The data
// layout the kernels share with the host is in nr_types.h.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <string>

#include "nr_types.h"

namespace karam {

struct Topology;

// Launch geometry of the LU round: NI instances per CTA, one lane each.
struct LuLaunch {
  int ni_per_cta;  // instances per CTA
  int S;           // odd stride of the value rows
  int Sv;          // odd stride of the vector rows
  size_t smem;     // dynamic shared memory bytes
  int grid;
};

void launch_init(const DevTopo& T, const DevInst& I, const JobParams& P, cudaStream_t s);
// Moves every converged instance into the transient at step 1 (capacitor
// history from the accepted point when init_caps).
void launch_tran_start(const DevTopo& T, const DevInst& I, int init_caps, cudaStream_t s);
void launch_eval(const DevTopo& T, const DevInst& I, const JobParams& P, int prec,
                 cudaStream_t s);
void launch_lu(const DevTopo& T, const DevInst& I, const JobParams& P, const LuLaunch& L,
               int prec, int* active, cudaStream_t s);
size_t eval_smem_bytes(const DevTopo& T);
// Sets the dynamic shared-memory limits of the kernels (call outside stream capture).
void configure_kernels(const DevTopo& T, const LuLaunch& L);
LuLaunch plan_lu(const DevTopo& T, int ni, int prec, int max_smem, int num_sms);
void unpermute(const double* v_perm, const int* perm, double* out, int ni, int n, cudaStream_t s);
// Dense FP64 partial-pivoting solves for the instances the LU kernel flagged.
void launch_rescue(const DevTopo& T, const DevInst& I, const JobParams& P, int prec, int grid,
                   cudaStream_t s);
size_t rescue_smem_bytes(const DevTopo& T);

// ---- LU round compiled at run time for one topology (jit.cpp) --------------
// Straight-line factor + solve code generated from the topology's LU program,
// compiled with NVRTC for sm_100a together with nr_device.cuh and loaded as a
// CUDA library. The interpreter is used when NVRTC is unavailable.
struct JitLu {
  bool ok = false;
  std::string status;          // "ready", or why the interpreter is used
  void* kernel_f32 = nullptr;  // cudaKernel_t
  void* kernel_f64 = nullptr;
  void* library = nullptr;     // cudaLibrary_t
  double compile_ms = 0.0;
};
void jit_build(const Topology& T, JitLu& out);
void jit_release(JitLu& j);
void launch_lu_jit(const JitLu& J, const DevTopo& T, const DevInst& I, const JobParams& P,
                   const LuLaunch& L, int prec, int* active, cudaStream_t s);
void configure_jit(const JitLu& J, const LuLaunch& L);

}  // namespace karam
