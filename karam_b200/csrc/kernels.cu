// kernels.cu -- statically compiled sm_100a kernels and their launchers. The
// device code lives in nr_device.cuh; the LU round here uses the program
// interpreter (the run-time compiled module replaces it per topology).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/karam.h"
#include "device.hpp"
#include "nr_device.cuh"

namespace karam {

using namespace knr;

template <typename T>
__global__ void __launch_bounds__(kLuThreads) k_lu_static(DevTopo Tp, DevInst I, JobParams P,
                                                            int NI, int S, int Sv, int* active) {
  lu_round<T, InterpFS>(Tp, I, P, NI, S, Sv, active);
}


// Shared memory of one instance in the evaluation kernel (x, MOSFET gm/gds/ids,
// diode g/i), and the number of instances one CTA evaluates together.
size_t eval_smem_bytes(const DevTopo& T) {
  return sizeof(double) * ((size_t)T.n + 3 * (size_t)T.n_mos + 2 * (size_t)T.n_dio);
}

int eval_instances_per_cta(const DevTopo& T) {
  const size_t per = eval_smem_bytes(T);
  int ne = (int)((96 * 1024) / (per > 0 ? per : 1));
  return std::max(1, std::min(ne, kMaxEvalInst));
}

void launch_init(const DevTopo& T, const DevInst& I, const JobParams& P, cudaStream_t s) {
  k_init<<<I.ni, 128, 0, s>>>(T, I, P);
}

void launch_tran_start(const DevTopo& T, const DevInst& I, int init_caps, cudaStream_t s) {
  k_tran_start<<<I.ni, 128, 0, s>>>(T, I, init_caps);
}

void configure_kernels(const DevTopo& T, const LuLaunch& L) {
  const int sm = (int)(eval_smem_bytes(T) * eval_instances_per_cta(T));
  cudaFuncSetAttribute(k_eval<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_eval<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_lu_static<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem);
  cudaFuncSetAttribute(k_lu_static<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem);
  const int rsm = (int)rescue_smem_bytes(T);
  cudaFuncSetAttribute(k_rescue<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
  cudaFuncSetAttribute(k_rescue<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, rsm);
}

void launch_eval(const DevTopo& T, const DevInst& I, const JobParams& P, int prec,
                 cudaStream_t s) {
  const int ne = eval_instances_per_cta(T);
  const size_t sm = eval_smem_bytes(T) * ne;
  const int grid = (I.ni + ne - 1) / ne;
  if (prec == KARAM_PREC_MIXED)
    k_eval<float><<<grid, kEvalThreads, sm, s>>>(T, I, P, ne);
  else
    k_eval<double><<<grid, kEvalThreads, sm, s>>>(T, I, P, ne);
}

LuLaunch plan_lu(const DevTopo& T, int ni, int prec, int max_smem, int num_sms) {
  LuLaunch L{};
  const size_t es = prec == KARAM_PREC_MIXED ? sizeof(float) : sizeof(double);
  L.S = T.nf | 1;
  L.Sv = T.n | 1;
  const size_t per = es * ((size_t)L.S + (size_t)L.Sv);
  const size_t reserve = 2048;  // static shared memory of k_lu
  int max_ni = (int)std::min<size_t>(32, (max_smem > (int)reserve ? (max_smem - reserve) : 0) / per);
  if (max_ni < 1) {
    L.ni_per_cta = 0;
    return L;
  }
  int want = (ni + num_sms - 1) / num_sms;
  if (want < 1) want = 1;
  L.ni_per_cta = std::min(max_ni, want);
  L.grid = (ni + L.ni_per_cta - 1) / L.ni_per_cta;
  L.smem = per * L.ni_per_cta;
  return L;
}

void launch_lu(const DevTopo& T, const DevInst& I, const JobParams& P, const LuLaunch& L, int prec,
               int* active, cudaStream_t s) {
  if (prec == KARAM_PREC_MIXED)
    k_lu_static<float><<<L.grid, kLuThreads, L.smem, s>>>(T, I, P, L.ni_per_cta, L.S, L.Sv, active);
  else
    k_lu_static<double><<<L.grid, kLuThreads, L.smem, s>>>(T, I, P, L.ni_per_cta, L.S, L.Sv, active);
}

size_t rescue_smem_bytes(const DevTopo& T) { return (size_t)T.n * (2 * sizeof(double) + sizeof(int)); }

void launch_rescue(const DevTopo& T, const DevInst& I, const JobParams& P, int prec, int grid,
                   cudaStream_t s) {
  const size_t sm = rescue_smem_bytes(T);
  if (prec == KARAM_PREC_MIXED)
    k_rescue<float><<<grid, 256, sm, s>>>(T, I, P);
  else
    k_rescue<double><<<grid, 256, sm, s>>>(T, I, P);
}

void unpermute(const double* v_perm, const int* perm, double* out, int ni, int n, cudaStream_t s) {
  const size_t total = (size_t)ni * n;
  int blocks = (int)std::min<size_t>((total + 255) / 256, 4096);
  if (blocks < 1) blocks = 1;
  k_unpermute<<<blocks, 256, 0, s>>>(v_perm, perm, out, ni, n);
}

}  // namespace karam
