// tc_gemm.hpp -- BF16 GEMM on the 5th-generation tensor cores (tcgen05) with
// TMA operand staging, for the learned seeder's layers (tc_gemm.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace karam {

// C[M][N] = A[M][K] * B[N][K]^T (acc = 0) or C += that (acc = 1), FP32 result
// and accumulation. A and B are BF16 and K-major (row r holds its K values
// contiguously) with row strides lda / ldb elements, multiples of 8, and
// 16-byte aligned bases; C is FP32 row-major with row stride ldc. Rows and K
// beyond the matrices read as zeros. *err (device, may be null) is set to 1
// when a bounded wait of the kernel gave up; the result is then not valid.
// Optional epilogue of tc_gemm_bf16, applied to each result z (FP32): z +=
// bias[col] (bias may be null), then, with out_bf16, out_bf16[row][col] (row
// stride ld_out elements, a multiple of 8) = BF16 of gelu(z) (gelu = 1) or
// z: the next layer's K-major operand. C may then be null (no FP32 result).
struct TcEpilogue {
  const float* bias = nullptr;
  int gelu = 0;
  __nv_bfloat16* out_bf16 = nullptr;
  int ld_out = 0;
};

cudaError_t tc_gemm_bf16(int M, int N, int K, const __nv_bfloat16* A, int lda,
                         const __nv_bfloat16* B, int ldb, float* C, int ldc, int acc, int* err,
                         cudaStream_t s, const TcEpilogue* ep = nullptr);

#ifdef __CUDACC__
// GELU of the seeder network, 0.5 z (1 + erf(z / sqrt 2)), shared by the
// training kernels and the GEMM epilogue so both compute the same values.
__device__ __forceinline__ float seeder_gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678f)); }
#endif

// dst[r][c] (BF16, row stride ld_dst) = src[r][c] (trans = 0, row stride
// ld_src) or src[c][r] (trans = 1) for r < rows, c < cols: the K-major
// operands of tc_gemm_bf16 from FP32 matrices in either orientation.
void to_bf16(const float* src, int ld_src, int trans, int rows, int cols, __nv_bfloat16* dst,
             int ld_dst, cudaStream_t s);

}  // namespace karam
