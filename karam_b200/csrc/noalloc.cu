// noalloc.cu -- evaluation + stamping into caller buffers without any device
// allocation (karam_eval_stamp_noalloc).
//
// Some callers cannot call cudaMalloc at the moment they need a Jacobian: code
// whose device memory is owned by its own pool allocator and must not be
// bypassed, or latency-critical loops where cudaMalloc / cudaFree would
// synchronise the device. For them the per-call scratch of the evaluation +
// stamping kernel (interleaved voltages, Jacobian value slots, residual,
// evaluation points, reductions, CSR map) lives in one fixed device array,
// kScratchBytes large, which every GPU that loads this library holds until the
// process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/karam.h"
#include "device.hpp"
#include "noalloc.hpp"

namespace karam {

namespace {

// The shared scratch array. Host code must not pass `g_scratch` itself to a
// kernel: on the host the name stands for a host-side placeholder, not for the
// device address; the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Lanes of the batch start at a DC point; lanes past it never evaluate; the
// reductions start neutral, the hub chunk counters at 0.
__global__ void k_noalloc_init(DevInst I, int hub_cnt_len) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < hub_cnt_len) I.hub_cnt[g] = 0;
  if (g >= I.ld) return;
  I.ev_t[g] = 0.0;
  I.ev_heff[g] = g < I.ni ? 0.0 : -1.0;
  I.red_f[g] = 0ull;
  I.red_dv[g] = 0ull;
  I.red_flags[g] = 3;
}

// Value slots -> CSR order (0 where the CSR position is structurally zero for
// the static-pivot LU), permuted residual -> node order.
template <typename TJ>
__global__ void k_noalloc_out(const TJ* J, const double* F, const int* csr_slot, const int* perm,
                              int ni, int ld, int nnz, int n, double* jac, double* f) {
  const size_t tj = (size_t)ni * nnz, tf = (size_t)ni * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tj + tf;
       e += (size_t)gridDim.x * blockDim.x) {
    if (e < tj) {
      const int i = (int)(e / nnz), j = (int)(e - (size_t)i * nnz);
      const int s = csr_slot[j];
      jac[e] = s >= 0 ? (double)J[(size_t)s * ld + i] : 0.0;
    } else {
      const size_t q = e - tj;
      const int i = (int)(q / n), k = (int)(q - (size_t)i * n);
      f[(size_t)i * n + perm[k]] = F[(size_t)k * ld + i];
    }
  }
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

// Looked up on every call rather than cached: the lookup allocates nothing
// and costs little, and an address kept from an earlier context would be
// stale after a device reset in the same process.
void* noalloc_scratch(const char** err) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return nullptr;
  }
  return p;
}

size_t noalloc_bytes(int n, int nv, int nnz, int ld, int hub_rows, int hub_groups) {
  const size_t L = (size_t)ld;
  return up256(8 * (size_t)n * L) * 2 + up256(8 * (size_t)nv * L) + up256(8 * L) * 4 +
         up256(4 * L) + up256(4 * (size_t)nnz) + up256(8 * (size_t)hub_rows * L) +
         up256(4 * (size_t)hub_groups * (L / 32));
}

cudaError_t noalloc_eval_stamp(void* scratch, const DevTopo& T, DevInst I, int prec,
                               const double* d_v, const int* perm, const int* h_csr_slot, int nnz,
                               double* d_jac, double* d_f, cudaStream_t s) {
  unsigned char* p = static_cast<unsigned char*>(scratch);
  const size_t L = (size_t)I.ld;
  auto take = [&](size_t bytes) {
    unsigned char* q = p;
    p += up256(bytes);
    return q;
  };
  double* x = reinterpret_cast<double*>(take(8 * (size_t)T.n * L));
  double* F = reinterpret_cast<double*>(take(8 * (size_t)T.n * L));
  void* J = take(8 * (size_t)T.nv * L);
  double* ev_t = reinterpret_cast<double*>(take(8 * L));
  double* ev_h = reinterpret_cast<double*>(take(8 * L));
  auto* rf = reinterpret_cast<unsigned long long*>(take(8 * L));
  auto* rd = reinterpret_cast<unsigned long long*>(take(8 * L));
  int* rfl = reinterpret_cast<int*>(take(4 * L));
  int* csr = reinterpret_cast<int*>(take(4 * (size_t)nnz));
  double* hub_part = reinterpret_cast<double*>(take(8 * (size_t)T.n_hub_rows * L));
  const int hub_cnt_len = T.n_hub_groups * (int)(L / 32);
  int* hub_cnt = reinterpret_cast<int*>(take(4 * (size_t)hub_cnt_len));
  // every instance evaluates a DC point; v is only read for the convergence
  // measures the stamping kernel folds, which this call does not report
  I.x = x;
  I.v = x;
  I.F = F;
  I.J = J;
  I.ev_t = ev_t;
  I.ev_heff = ev_h;
  I.red_f = rf;
  I.red_dv = rd;
  I.red_flags = rfl;
  I.seed = nullptr;
  I.counters = nullptr;
  I.wave = nullptr;
  I.rescue_count = nullptr;
  I.hub_part = hub_part;
  I.hub_cnt = hub_cnt;
  cudaError_t e = cudaMemcpyAsync(csr, h_csr_slot, sizeof(int) * (size_t)nnz,
                                  cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  interleave(d_v, perm, x, I.ni, I.ld, T.n, s);
  k_noalloc_init<<<(std::max(I.ld, hub_cnt_len) + 255) / 256, 256, 0, s>>>(I, hub_cnt_len);
  JobParams P{};
  P.precision = prec;
  P.reltol = 1e-3;
  P.vntol = 1e-6;
  launch_eval_stamp(T, I, P, RoundLaunch{}, prec, s);
  const size_t total = (size_t)I.ni * ((size_t)nnz + T.n);
  const int grid = (int)std::min<size_t>((total + 255) / 256, 4096);
  if (prec == KARAM_PREC_MIXED)
    k_noalloc_out<float><<<grid, 256, 0, s>>>(static_cast<const float*>(J), F, csr, perm, I.ni,
                                               I.ld, nnz, T.n, d_jac, d_f);
  else
    k_noalloc_out<double><<<grid, 256, 0, s>>>(static_cast<const double*>(J), F, csr, perm,
                                                I.ni, I.ld, nnz, T.n, d_jac, d_f);
  return cudaGetLastError();
}

}  // namespace karam
