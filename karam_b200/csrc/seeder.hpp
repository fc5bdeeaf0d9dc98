// seeder.hpp -- the learned NR seeder: a multilayer perceptron that maps an
// instance's sampled device parameters and source values to an initial guess
// of its node voltages (the role of solvers/neural_seeder.h in the reference,
// whose learned model is future work there). Weights are used in BF16 by the
// tensor-core GEMMs with FP32 accumulation; master weights, Adam moments and
// activations are FP32. Everything lives on one device and runs on the
// caller's stream.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "nr_types.h"

namespace karam {

struct Mlp;

// hidden: hidden layers of `width` units (GELU); one linear output layer.
// Throws std::runtime_error on bad sizes or CUDA errors.
Mlp* mlp_create(int n_in, int n_out, int width, int hidden, uint64_t seed, cudaStream_t s);
void mlp_destroy(Mlp* m);
int mlp_n_in(const Mlp* m);
int mlp_n_out(const Mlp* m);
int mlp_samples(const Mlp* m);

// Appends n training samples (raw features X[n][n_in], raw targets
// Y[n][n_out], FP32, device memory, row-major) to the training set.
void mlp_add_samples(Mlp* m, const float* dX, const float* dY, int n, cudaStream_t s);

// Adam on the mean squared error of the normalised targets. The feature and
// target normalisations (per-column mean and standard deviation) are taken
// from the training set at the first call. Returns the mean loss of the last
// epoch (normalised units).
float mlp_train(Mlp* m, int epochs, int batch, float lr, uint64_t shuffle_seed, cudaStream_t s);

// Raw outputs for n rows of raw features (device memory). `out` is written
// as out[i * out_ld + r] for output i of row r when out_ld > 0 (column
// layout, e.g. instance-interleaved seeds), else row-major out[r][n_out].
void mlp_predict(Mlp* m, const float* dX, int n, double* out, int out_ld, cudaStream_t s);

// One GEMM of the engine, exposed for tests: C[M][N] = op(A) op(B) with
// op(A)[m][k] = transA ? A[k * lda + m] : A[m * lda + k] (B likewise),
// operands rounded to BF16, FP32 accumulation. accumulate: C += instead of =.
void mlp_gemm(int M, int N, int K, const float* A, int lda, int transA, const float* B, int ldb,
              int transB, float* C, int ldc, int accumulate, cudaStream_t s);

// Features (VTO per MOSFET, KP per MOSFET, DC value per source) of instances
// idx[0..rows) (or 0..rows) into X[rows][2 n_mos + n_vs], and their node
// voltages (permuted order) into Y[rows][n] when Y is not null.
void seeder_features(const DevTopo& T, const DevInst& I, const int* idx, int rows, float* X,
                     float* Y, cudaStream_t s);

}  // namespace karam
