// noalloc.hpp -- evaluation + stamping without device allocation (noalloc.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "nr_types.h"

namespace karam {

// Size of the library's fixed device scratch array (per GPU, held until exit).
constexpr size_t kScratchBytes = size_t(16) << 20;

// Device address of the scratch array on the current device, looked up with
// cudaGetSymbolAddress on every call; returns null and sets *err when that
// fails.
void* noalloc_scratch(const char** err);

// Scratch bytes one call needs for a topology of n unknowns, nv value slots,
// nnz CSR entries, hub_rows hub chunk partial rows and hub_groups hub groups,
// at lane stride ld.
size_t noalloc_bytes(int n, int nv, int nnz, int ld, int hub_rows, int hub_groups);

// Evaluation + stamping of I's instances at d_v ([ni][n], node order, device)
// into d_jac ([ni][nnz], CSR order) and d_f ([ni][n], node order), every
// intermediate in `scratch`. Enqueued on s; the caller synchronises.
cudaError_t noalloc_eval_stamp(void* scratch, const DevTopo& T, DevInst I, int prec,
                               const double* d_v, const int* perm, const int* h_csr_slot, int nnz,
                               double* d_jac, double* d_f, cudaStream_t s);

}  // namespace karam
