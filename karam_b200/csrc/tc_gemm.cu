// tc_gemm.cu -- BF16 x BF16 -> FP32 GEMM on the tcgen05 tensor cores.
//
// One CTA of 128 threads computes a 128 x 128 tile of C = A B^T (both
// operands K-major). The K loop runs in blocks of 64 through a ring of
// kStages shared-memory stages:
//   * thread 0 (the producer) loads each block of A and B with one 2-D TMA
//     copy each (cp.async.bulk.tensor, 128-byte swizzle: the K-major SW128
//     canonical layout the tensor cores read), completing on the stage's
//     "full" mbarrier;
//   * thread 32 (the MMA issuer) waits for a full stage and issues four
//     tcgen05.mma (M 128, N 128, K 16) into a 128-column FP32 accumulator in
//     tensor memory, then tcgen05.commit frees the stage through its "empty"
//     mbarrier; after the last block a final commit signals "done";
//   * all four warps then read their 32 accumulator lanes (rows) back with
//     tcgen05.ld and write C.
// Every mbarrier wait is bounded (about a second of SM clock); a wait that
// gives up sets *err, and the kernel still waits (bounded) for the work it
// has issued before it frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "tc_gemm.hpp"

namespace karam {

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 64, kStages = 4;
constexpr int kTmemCols = 128;  // FP32 accumulator: one column per N
constexpr uint32_t kStageBytes = (uint32_t)(kBM + kBN) * kBK * sizeof(__nv_bfloat16);
// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits
// 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 =
// 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);
constexpr long long kWaitCycles = 1ll << 31;

struct __align__(1024) TcSmem {
  __nv_bfloat16 a[kStages][kBM * kBK];  // 16 KiB per stage, 1024-byte aligned (swizzle atoms)
  __nv_bfloat16 b[kStages][kBN * kBK];
  unsigned long long full[kStages], empty[kStages], done;
  uint32_t tmem;
};

__device__ __forceinline__ uint32_t sm_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void bar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the completion of the barrier's phase with this parity; false
// when about a second of SM clock passed first.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!bar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
// 2-D TMA load of a box at (x = inner coordinate, y) into shared memory.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle:
// start address >> 4 (bits 0-13), leading byte offset 1 (unused for this
// layout, bits 16-29), stride byte offset 1024 >> 4 between 8-row groups
// (bits 32-45), version 1 (bits 46-47), layout SWIZZLE_128B = 2 (bits 61-63).
__device__ __forceinline__ uint64_t kmajor_sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
// Arrives once on the barrier when every tcgen05 operation this thread issued
// before it has completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 32 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__global__ void __launch_bounds__(128) k_gemm_tc(const __grid_constant__ CUtensorMap ta,
                                                 const __grid_constant__ CUtensorMap tb, int M,
                                                 int N, int K, float* __restrict__ C, int ldc,
                                                 int acc, int* err, TcEpilogue ep) {
  extern __shared__ unsigned char tc_raw[];
  const uint32_t pad = (1024u - (sm_addr(tc_raw) & 1023u)) & 1023u;
  TcSmem* S = reinterpret_cast<TcSmem*>(tc_raw + pad);
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int nk = (K + kBK - 1) / kBK;
  if (tid == 0) {
    for (int st = 0; st < kStages; ++st) {
      bar_init(sm_addr(&S->full[st]), 1);
      bar_init(sm_addr(&S->empty[st]), 1);
    }
    bar_init(sm_addr(&S->done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  if (warp == 0) {  // the accumulator's tensor-memory columns (the whole warp)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm_addr(&S->tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S->tmem;

  if (warp == 0) {
    if (lane == 0) {  // producer: TMA copies of A and B, one K block per stage
      for (int kb = 0; kb < nk; ++kb) {
        const int st = kb % kStages, use = kb / kStages;
        if (use > 0 && !bar_wait(sm_addr(&S->empty[st]), (use - 1) & 1)) {
          s_fail = 1;
          break;
        }
        const uint32_t full = sm_addr(&S->full[st]);
        bar_expect_tx(full, kStageBytes);
        tma_load_2d(sm_addr(S->a[st]), &ta, kb * kBK, m0, full);
        tma_load_2d(sm_addr(S->b[st]), &tb, kb * kBK, n0, full);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      for (int kb = 0; kb < nk; ++kb) {
        const int st = kb % kStages, use = kb / kStages;
        if (!bar_wait(sm_addr(&S->full[st]), use & 1)) {
          s_fail = 1;
          break;
        }
        tc_fence_after();
        const uint32_t a0 = sm_addr(S->a[st]), b0 = sm_addr(S->b[st]);
#pragma unroll
        for (int kk = 0; kk < kBK / 16; ++kk)  // K 16 per MMA: 32 bytes along the swizzled rows
          umma_bf16(tmem, kmajor_sw128_desc(a0 + 32 * kk), kmajor_sw128_desc(b0 + 32 * kk), kIdesc,
                    (kb | kk) != 0);
        umma_commit(sm_addr(&S->empty[st]));  // the stage is free once these MMAs have read it
      }
      umma_commit(sm_addr(&S->done));  // every MMA issued above has completed
    }
    __syncwarp();
  }
  __syncthreads();  // the roles have issued their work (s_fail is final)

  // epilogue: warp w holds accumulator lanes (tile rows) 32 w .. 32 w + 31
  const bool done = bar_wait(sm_addr(&S->done), 0);
  tc_fence_after();
  if (done && !s_fail) {
    const int row = m0 + warp * 32 + lane;
    const bool vec = (ldc & 3) == 0;
    for (int c0 = 0; c0 < kBN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row >= M) continue;
      const int nv = N - (n0 + c0);
      if (nv <= 0) continue;
      if (ep.bias)
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += j < nv ? __ldg(&ep.bias[n0 + c0 + j]) : 0.0f;
      if (ep.out_bf16) {
        __nv_bfloat16* orow = ep.out_bf16 + (size_t)row * ep.ld_out + n0 + c0;
        if (nv >= 32) {  // 16-byte stores: ld_out and the column offset are multiples of 8
#pragma unroll
          for (int j = 0; j < 32; j += 8) {
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16_rn(ep.gelu ? seeder_gelu(v[j + q]) : v[j + q]);
            *reinterpret_cast<uint4*>(orow + j) = *reinterpret_cast<const uint4*>(h);
          }
        } else {
          for (int j = 0; j < nv; ++j) orow[j] = __float2bfloat16_rn(ep.gelu ? seeder_gelu(v[j]) : v[j]);
        }
      }
      if (!C) continue;
      float* crow = C + (size_t)row * ldc + n0 + c0;
      if (vec && nv >= 32) {
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          float4 o = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
          if (acc) {
            const float4 c = *reinterpret_cast<const float4*>(crow + j);
            o.x += c.x;
            o.y += c.y;
            o.z += c.z;
            o.w += c.w;
          }
          *reinterpret_cast<float4*>(crow + j) = o;
        }
      } else {
        for (int j = 0; j < 32 && j < nv; ++j) crow[j] = acc ? crow[j] + v[j] : v[j];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  if (tid == 0 && (!done || s_fail) && err) atomicExch(err, 1);
}

// dst[r][c] = src[r][c] or src[c][r] as BF16 through a 32 x 32 tile (both
// sides coalesced).
__global__ void k_to_bf16(const float* __restrict__ src, int ld_src, int trans, int rows, int cols,
                          __nv_bfloat16* __restrict__ dst, int ld_dst) {
  __shared__ float t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 256 threads: 32 x 8
  for (int i = ty; i < 32; i += 8) {
    float v = 0.0f;
    if (trans) {  // src[c][r]: read along r
      const int c = c0 + i, r = r0 + tx;
      if (c < cols && r < rows) v = src[(size_t)c * ld_src + r];
      t[tx][i] = v;
    } else {
      const int r = r0 + i, c = c0 + tx;
      if (r < rows && c < cols) v = src[(size_t)r * ld_src + c];
      t[i][tx] = v;
    }
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + tx;
    if (r < rows && c < cols) dst[(size_t)r * ld_dst + c] = __float2bfloat16_rn(t[i][tx]);
  }
}


}  // namespace

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of a K-major BF16 operand with `rows` rows of K values (row
// stride ld elements): boxes of 64 K values x 128 rows, 128-byte swizzle,
// zeros outside the matrix.
bool kmajor_map(CUtensorMap* map, const __nv_bfloat16* base, int rows, int K, int ld) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(__nv_bfloat16)};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBM};
  const cuuint32_t es[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides,
             box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

cudaError_t tc_gemm_bf16(int M, int N, int K, const __nv_bfloat16* A, int lda,
                         const __nv_bfloat16* B, int ldb, float* C, int ldc, int acc, int* err,
                         cudaStream_t s, const TcEpilogue* ep) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  const TcEpilogue e = ep ? *ep : TcEpilogue{};
  if (e.out_bf16 && ((e.ld_out & 7) || (reinterpret_cast<uintptr_t>(e.out_bf16) & 15)))
    return cudaErrorInvalidValue;  // the epilogue's 16-byte stores
  if (!C && !e.out_bf16) return cudaErrorInvalidValue;
  if (K <= 0) {  // an empty sum
    if (acc || e.bias || e.out_bf16) return cudaErrorInvalidValue;
    return cudaMemset2DAsync(C, (size_t)ldc * sizeof(float), 0, (size_t)N * sizeof(float), M, s);
  }
  if ((lda & 7) || (ldb & 7) || (reinterpret_cast<uintptr_t>(A) & 15) ||
      (reinterpret_cast<uintptr_t>(B) & 15))
    return cudaErrorInvalidValue;  // TMA: 16-byte aligned bases and row strides
  CUtensorMap ta, tb;
  if (!kmajor_map(&ta, A, M, K, lda) || !kmajor_map(&tb, B, N, K, ldb)) return cudaErrorInvalidValue;
  const int smem = (int)sizeof(TcSmem) + 1024;
  static std::once_flag attr;
  cudaError_t ea = cudaSuccess;
  std::call_once(attr, [&] {
    ea = cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  });
  if (ea != cudaSuccess) return ea;
  const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  k_gemm_tc<<<grid, 128, smem, s>>>(ta, tb, M, N, K, C, ldc, acc, err, e);
  return cudaGetLastError();
}

void to_bf16(const float* src, int ld_src, int trans, int rows, int cols, __nv_bfloat16* dst,
             int ld_dst, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  const dim3 grid((cols + 31) / 32, (rows + 31) / 32);
  k_to_bf16<<<grid, 256, 0, s>>>(src, ld_src, trans, rows, cols, dst, ld_dst);
}


}  // namespace karam
