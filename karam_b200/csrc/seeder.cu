// seeder.cu -- training and inference kernels of the learned NR seeder (see
// seeder.hpp). The GEMMs run on the tcgen05 tensor cores (tc_gemm.cu) with
// BF16 operands staged by TMA and FP32 accumulation in tensor memory; each
// operand is first converted to a K-major BF16 copy, transposed where the
// product needs it. The network is small (config 2: 1026 -> 512 -> 512 ->
// 512 -> 322, 1.2 M weights), so a batch of 4096 instances costs a few GFLOP.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "nr_types.h"
#include "seeder.hpp"
#include "tc_gemm.hpp"

namespace karam {

namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

__device__ __forceinline__ float gelu(float z) { return seeder_gelu(z); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678f)) + z * 0.39894228f * expf(-0.5f * z * z);
}

// Z += b (kept for the backward pass); H = gelu(Z) unless H is null.
__global__ void k_bias_act(float* Z, const float* b, float* H, int rows, int cols) {
  const size_t n = (size_t)rows * cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const float z = Z[e] + b[e % cols];
    Z[e] = z;
    if (H) H[e] = gelu(z);
  }
}

__global__ void k_gelu_bwd(float* dH, const float* Z, int rows, int cols) {
  const size_t n = (size_t)rows * cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x)
    dH[e] *= gelu_d(Z[e]);
}

// dY = 2 (Y - T) / (rows cols); loss += mean squared error.
__global__ void k_mse(const float* Y, const float* T, float* dY, int rows, int cols, float* loss) {
  const size_t n = (size_t)rows * cols;
  const float s = 1.0f / (float)n;
  float part = 0.0f;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const float d = Y[e] - T[e];
    dY[e] = 2.0f * s * d;
    part += d * d * s;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

__global__ void k_colsum(const float* G, int rows, int cols, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += G[(size_t)r * cols + c];
  out[c] = s;
}

// Adam update of n parameters for one training step: the step's bias
// corrections c1, c2 come from the epoch's table c12[2 q], c12[2 q + 1], q =
// ctr[0] the step within the epoch (so a captured step replays unchanged).
__global__ void k_adam_step(float* w, const float* g, float* m, float* v, int n, float lr,
                            const float* c12, const int* ctr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int q = *ctr;
  const float c1 = c12[2 * q], c2 = c12[2 * q + 1];
  const float gi = g[i];
  const float mi = 0.9f * m[i] + 0.1f * gi;
  const float vi = 0.999f * v[i] + 0.001f * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

// The step within the epoch advances (the last kernel of a captured step).
__global__ void k_step_advance(int* ctr) {
  if (blockIdx.x == 0 && threadIdx.x == 0) ctr[0] += 1;
}

// k_norm_rows over the batch of step ctr[0]: rows idx[ctr[0] * B + r].
__global__ void k_norm_rows_step(const float* src, const int* idx, const int* ctr, int B, int cols,
                                 const float* mean, const float* istd, float* out) {
  const int* bi = idx + (size_t)(*ctr) * B;
  const size_t n = (size_t)B * cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / cols), j = (int)(e - (size_t)r * cols);
    out[e] = (src[(size_t)bi[r] * cols + j] - mean[j]) * istd[j];
  }
}

// out[r][j] = (src[row(r)][j] - mean[j]) * istd[j], row(r) = idx ? idx[r] : r.
__global__ void k_norm_rows(const float* src, const int* idx, int rows, int cols,
                            const float* mean, const float* istd, float* out) {
  const size_t n = (size_t)rows * cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / cols), j = (int)(e - (size_t)r * cols);
    const int sr = idx ? idx[r] : r;
    out[e] = (src[(size_t)sr * cols + j] - mean[j]) * istd[j];
  }
}

// k_norm_rows into a K-major BF16 operand [rows][ld] (the first layer's A):
// the same FP32 arithmetic, rounded to BF16 as the GEMM's operand copy would.
__global__ void k_norm_rows_bf16(const float* src, int rows, int cols, const float* mean,
                                 const float* istd, __nv_bfloat16* out, int ld) {
  const size_t n = (size_t)rows * cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / cols), j = (int)(e - (size_t)r * cols);
    out[(size_t)r * ld + j] = __float2bfloat16_rn((src[(size_t)r * cols + j] - mean[j]) * istd[j]);
  }
}

// Column mean and 1 / standard deviation (0 for a constant column).
__global__ void k_col_stats(const float* X, int rows, int cols, float* mean, float* istd,
                            float* sd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double s = 0.0;
  for (int r = 0; r < rows; ++r) s += X[(size_t)r * cols + c];
  const double mu = s / rows;
  double q = 0.0;
  for (int r = 0; r < rows; ++r) {
    const double d = X[(size_t)r * cols + c] - mu;
    q += d * d;
  }
  const double sdv = sqrt(q / rows);
  mean[c] = (float)mu;
  istd[c] = sdv > 0.0 ? (float)(1.0 / sdv) : 0.0f;
  if (sd) sd[c] = (float)sdv;
}

__global__ void k_denorm(const float* Y, int rows, int cols, const float* mean, const float* sd,
                         double* out, int out_ld) {
  const size_t n = (size_t)rows * cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / cols), i = (int)(e - (size_t)r * cols);
    const double v = (double)Y[e] * sd[i] + mean[i];
    if (out_ld > 0)
      out[(size_t)i * out_ld + r] = v;
    else
      out[e] = v;
  }
}

// Uniform(-a, a) from a counter hash (splitmix64), deterministic per seed.
__global__ void k_init_uniform(float* w, int n, float a, unsigned long long seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const float u = (float)((z >> 40) * (1.0 / 16777216.0));  // [0, 1)
  w[i] = (2.0f * u - 1.0f) * a;
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 4096); }

struct Buf {
  float* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    n = count;
    if (count) ck(cudaMalloc(&p, count * sizeof(float)), "seeder alloc");
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

struct BBuf {  // device BF16 array
  __nv_bfloat16* p = nullptr;
  size_t n = 0;
  void need(size_t count) {
    if (count <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = count;
    ck(cudaMalloc(&p, count * sizeof(__nv_bfloat16)), "seeder alloc");
  }
  BBuf() = default;
  BBuf(const BBuf&) = delete;
  BBuf& operator=(const BBuf&) = delete;
  BBuf(BBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  ~BBuf() {
    if (p) cudaFree(p);
  }
};

inline int pad8(int k) { return (k + 7) & ~7; }

// BF16 copies of a GEMM's operands and its kernel's error flag.
struct GemmWs {
  __nv_bfloat16* a = nullptr;
  __nv_bfloat16* b = nullptr;
  size_t na = 0, nb = 0;
  int* err = nullptr;
  void need(size_t ea, size_t eb) {
    if (ea > na) {
      if (a) cudaFree(a);
      a = nullptr;
      ck(cudaMalloc(&a, ea * sizeof(__nv_bfloat16)), "seeder gemm workspace");
      na = ea;
    }
    if (eb > nb) {
      if (b) cudaFree(b);
      b = nullptr;
      ck(cudaMalloc(&b, eb * sizeof(__nv_bfloat16)), "seeder gemm workspace");
      nb = eb;
    }
    if (!err) {
      ck(cudaMalloc(&err, sizeof(int)), "seeder gemm flag");
      ck(cudaMemset(err, 0, sizeof(int)), "seeder gemm flag");
    }
  }
  int* err_flag() {
    if (!err) {
      ck(cudaMalloc(&err, sizeof(int)), "seeder gemm flag");
      ck(cudaMemset(err, 0, sizeof(int)), "seeder gemm flag");
    }
    return err;
  }
  ~GemmWs() {
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    if (err) cudaFree(err);
  }
};

}  // namespace

struct Mlp {
  std::vector<int> dims;  // n_in, width x hidden, n_out
  int L = 0;              // weight layers
  std::vector<Buf> W, b, gW, gb, mW, vW, mb, vb;
  Buf Xs, Ys;  // training samples (raw)
  int ns = 0;
  Buf fmean, fistd, tmean, tistd, tsd;
  bool normed = false;
  int bcap = 0;
  std::vector<Buf> act, pre;  // act[0..L-1] inputs of each layer, pre[1..L] pre-activations
  Buf g1, g2, tgt, loss;
  int* idx = nullptr;
  int idx_cap = 0;
  long step = 0;
  GemmWs ws;
  // inference: K-major BF16 weights ([N][pad8(K)] per layer, converted again
  // when training has changed them) and BF16 activations ([rows][pad8(K)])
  std::vector<BBuf> wbf, abf;
  long wbf_step = -1;
  // training: the step counter of a captured step and the epoch's Adam
  // bias-correction table
  Buf c12;
  int* ctr = nullptr;
  ~Mlp() {
    if (ctr) cudaFree(ctr);
    if (idx) cudaFree(idx);
  }
};

namespace {

void ensure_batch(Mlp* m, int B) {
  if (B <= m->bcap) return;
  int maxd = *std::max_element(m->dims.begin(), m->dims.end());
  m->act.resize(m->L);
  m->pre.resize(m->L + 1);
  for (int l = 0; l < m->L; ++l) m->act[l].alloc((size_t)B * m->dims[l]);
  for (int l = 1; l <= m->L; ++l) m->pre[l].alloc((size_t)B * m->dims[l]);
  m->g1.alloc((size_t)B * maxd);
  m->g2.alloc((size_t)B * maxd);
  m->tgt.alloc((size_t)B * m->dims[m->L]);
  m->bcap = B;
}

// C[M][N] (+)= op(A)[M][K] op(B)[K][N] for FP32 matrices: both operands
// become K-major BF16 copies (A as [M][K], B as [N][K]; rows padded to a
// multiple of 8 values for the TMA strides), then the tcgen05 GEMM.
void gemm(int M, int N, int K, const float* A, int lda, int tA, const float* B, int ldb, int tB,
          float* C, int ldc, int acc, GemmWs& ws, cudaStream_t s) {
  if (M <= 0 || N <= 0) return;
  const int kp = (K + 7) & ~7;
  ws.need((size_t)M * kp, (size_t)N * kp);
  to_bf16(A, lda, tA, M, K, ws.a, kp, s);       // A[m][k] = op(A)
  to_bf16(B, ldb, tB ? 0 : 1, N, K, ws.b, kp, s);  // B[n][k] = op(B)[k][n]
  ck(tc_gemm_bf16(M, N, K, ws.a, kp, ws.b, kp, C, ldc, acc, ws.err, s), "tcgen05 gemm launch");
}

// Synchronises s and reports a GEMM whose bounded waits gave up.
void check_gemm(GemmWs& ws, cudaStream_t s) {
  if (!ws.err) return;
  int e = 0;
  ck(cudaMemcpyAsync(&e, ws.err, sizeof(int), cudaMemcpyDeviceToHost, s), "gemm flag");
  ck(cudaStreamSynchronize(s), "gemm sync");
  if (e) {
    cudaMemsetAsync(ws.err, 0, sizeof(int), s);
    throw std::runtime_error("seeder GEMM: a bounded wait of the tensor-core kernel gave up");
  }
}

// Forward pass of B rows whose normalised inputs are in act[0]; the output
// (normalised units) is left in pre[L].
void forward(Mlp* m, int B, cudaStream_t s) {
  for (int l = 1; l <= m->L; ++l) {
    const int K = m->dims[l - 1], N = m->dims[l];
    gemm(B, N, K, m->act[l - 1].p, K, 0, m->W[l - 1].p, N, 0, m->pre[l].p, N, 0, m->ws, s);
    const size_t e = (size_t)B * N;
    k_bias_act<<<grid_for(e), 256, 0, s>>>(m->pre[l].p, m->b[l - 1].p,
                                           l < m->L ? m->act[l].p : nullptr, B, N);
  }
}

}  // namespace

Mlp* mlp_create(int n_in, int n_out, int width, int hidden, uint64_t seed, cudaStream_t s) {
  if (n_in < 1 || n_out < 1 || width < 1 || hidden < 0 || hidden > 16)
    throw std::runtime_error("seeder: bad network sizes");
  Mlp* m = new Mlp;
  try {
    m->dims.push_back(n_in);
    for (int h = 0; h < hidden; ++h) m->dims.push_back(width);
    m->dims.push_back(n_out);
    m->L = (int)m->dims.size() - 1;
    for (auto* v : {&m->W, &m->b, &m->gW, &m->gb, &m->mW, &m->vW, &m->mb, &m->vb}) v->resize(m->L);
    for (int l = 0; l < m->L; ++l) {
      const size_t nw = (size_t)m->dims[l] * m->dims[l + 1], nb = m->dims[l + 1];
      m->W[l].alloc(nw);
      m->gW[l].alloc(nw);
      m->mW[l].alloc(nw);
      m->vW[l].alloc(nw);
      m->b[l].alloc(nb);
      m->gb[l].alloc(nb);
      m->mb[l].alloc(nb);
      m->vb[l].alloc(nb);
      // uniform with variance 1 / fan_in (GELU layers) and zero biases
      const float a = std::sqrt(3.0f / (float)m->dims[l]);
      k_init_uniform<<<(int)((nw + 255) / 256), 256, 0, s>>>(m->W[l].p, (int)nw, a,
                                                              seed + 7919ull * (l + 1));
      ck(cudaMemsetAsync(m->b[l].p, 0, nb * sizeof(float), s), "seeder init");
      for (Buf* z : {&m->mW[l], &m->vW[l]}) ck(cudaMemsetAsync(z->p, 0, nw * sizeof(float), s), "seeder init");
      for (Buf* z : {&m->mb[l], &m->vb[l]}) ck(cudaMemsetAsync(z->p, 0, nb * sizeof(float), s), "seeder init");
    }
    m->fmean.alloc(n_in);
    m->fistd.alloc(n_in);
    m->tmean.alloc(n_out);
    m->tistd.alloc(n_out);
    m->tsd.alloc(n_out);
    m->loss.alloc(1);
    ck(cudaGetLastError(), "seeder init launch");
  } catch (...) {
    delete m;
    throw;
  }
  return m;
}

void mlp_destroy(Mlp* m) { delete m; }
int mlp_n_in(const Mlp* m) { return m->dims.front(); }
int mlp_n_out(const Mlp* m) { return m->dims.back(); }
int mlp_samples(const Mlp* m) { return m->ns; }

void mlp_add_samples(Mlp* m, const float* dX, const float* dY, int n, cudaStream_t s) {
  if (n <= 0) return;
  const int ni = m->dims.front(), no = m->dims.back();
  const size_t need = (size_t)(m->ns + n);
  if (need > m->Xs.n / std::max(1, ni)) {
    size_t cap = std::max<size_t>(need, 2 * (size_t)m->ns);
    Buf X2, Y2;
    X2.alloc(cap * ni);
    Y2.alloc(cap * no);
    if (m->ns) {
      ck(cudaMemcpyAsync(X2.p, m->Xs.p, (size_t)m->ns * ni * sizeof(float), cudaMemcpyDeviceToDevice, s), "seeder copy");
      ck(cudaMemcpyAsync(Y2.p, m->Ys.p, (size_t)m->ns * no * sizeof(float), cudaMemcpyDeviceToDevice, s), "seeder copy");
    }
    ck(cudaStreamSynchronize(s), "seeder sync");
    std::swap(m->Xs.p, X2.p);
    std::swap(m->Xs.n, X2.n);
    std::swap(m->Ys.p, Y2.p);
    std::swap(m->Ys.n, Y2.n);
  }
  ck(cudaMemcpyAsync(m->Xs.p + (size_t)m->ns * ni, dX, (size_t)n * ni * sizeof(float),
                     cudaMemcpyDeviceToDevice, s), "seeder copy");
  ck(cudaMemcpyAsync(m->Ys.p + (size_t)m->ns * no, dY, (size_t)n * no * sizeof(float),
                     cudaMemcpyDeviceToDevice, s), "seeder copy");
  m->ns += n;
}

float mlp_train(Mlp* m, int epochs, int batch, float lr, uint64_t shuffle_seed, cudaStream_t s) {
  if (m->ns < 1) throw std::runtime_error("seeder: no training samples");
  if (epochs < 1 || batch < 1 || !(lr > 0.0f)) throw std::runtime_error("seeder: bad training options");
  const int ni = m->dims.front(), no = m->dims.back();
  if (!m->normed) {
    k_col_stats<<<(ni + 127) / 128, 128, 0, s>>>(m->Xs.p, m->ns, ni, m->fmean.p, m->fistd.p, nullptr);
    k_col_stats<<<(no + 127) / 128, 128, 0, s>>>(m->Ys.p, m->ns, no, m->tmean.p, m->tistd.p, m->tsd.p);
    m->normed = true;
  }
  const int B = std::min(batch, m->ns);
  const int nb = m->ns / B;
  ensure_batch(m, B);
  if (m->idx_cap < m->ns) {
    if (m->idx) cudaFree(m->idx);
    m->idx = nullptr;
    ck(cudaMalloc(&m->idx, (size_t)m->ns * sizeof(int)), "seeder alloc");
    m->idx_cap = m->ns;
  }
  if (!m->ctr) {
    ck(cudaMalloc(&m->ctr, 2 * sizeof(int)), "seeder alloc");
    ck(cudaMemset(m->ctr, 0, 2 * sizeof(int)), "seeder alloc");
  }
  if (m->c12.n < 2 * (size_t)nb) m->c12.alloc(2 * (size_t)nb);
  // One training step: the batch of step ctr[0] normalised, forward, MSE,
  // backward, Adam with the step's bias corrections, ctr[0] + 1. Its launches
  // read every varying value from device memory, so the step is captured once
  // into a CUDA graph and replayed (the first step of a call runs eagerly:
  // it sizes the GEMM workspace before the capture).
  auto train_step = [&]() {
    k_norm_rows_step<<<grid_for((size_t)B * ni), 256, 0, s>>>(m->Xs.p, m->idx, m->ctr, B, ni, m->fmean.p,
                                                              m->fistd.p, m->act[0].p);
    k_norm_rows_step<<<grid_for((size_t)B * no), 256, 0, s>>>(m->Ys.p, m->idx, m->ctr, B, no, m->tmean.p,
                                                              m->tistd.p, m->tgt.p);
    forward(m, B, s);
    float* gc = m->g1.p;
    float* gn = m->g2.p;
    k_mse<<<grid_for((size_t)B * no), 256, 0, s>>>(m->pre[m->L].p, m->tgt.p, gc, B, no, m->loss.p);
    for (int l = m->L; l >= 1; --l) {
      const int K = m->dims[l - 1], N = m->dims[l];
      gemm(K, N, B, m->act[l - 1].p, K, 1, gc, N, 0, m->gW[l - 1].p, N, 0, m->ws, s);
      k_colsum<<<(N + 127) / 128, 128, 0, s>>>(gc, B, N, m->gb[l - 1].p);
      if (l > 1) {
        gemm(B, K, N, gc, N, 0, m->W[l - 1].p, N, 1, gn, K, 0, m->ws, s);
        k_gelu_bwd<<<grid_for((size_t)B * K), 256, 0, s>>>(gn, m->pre[l - 1].p, B, K);
        std::swap(gc, gn);
      }
    }
    for (int l = 0; l < m->L; ++l) {
      const int nw = m->dims[l] * m->dims[l + 1], nbias = m->dims[l + 1];
      k_adam_step<<<(nw + 255) / 256, 256, 0, s>>>(m->W[l].p, m->gW[l].p, m->mW[l].p, m->vW[l].p, nw, lr,
                                                   m->c12.p, m->ctr);
      k_adam_step<<<(nbias + 255) / 256, 256, 0, s>>>(m->b[l].p, m->gb[l].p, m->mb[l].p, m->vb[l].p, nbias,
                                                      lr, m->c12.p, m->ctr);
    }
    k_step_advance<<<1, 32, 0, s>>>(m->ctr);
  };
  struct GraphGuard {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~GraphGuard() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
    }
  } graph;
  std::mt19937_64 rng(shuffle_seed);
  std::vector<int> perm(m->ns);
  std::vector<float> c12(2 * (size_t)nb);
  float last = 0.0f;
  for (int ep = 0; ep < epochs; ++ep) {
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    for (int q = 0; q < nb; ++q) {  // Adam's bias corrections of the epoch's steps
      const long st = m->step + 1 + q;
      c12[2 * q] = 1.0f - std::pow(0.9f, (float)st);
      c12[2 * q + 1] = 1.0f - std::pow(0.999f, (float)st);
    }
    ck(cudaMemcpyAsync(m->idx, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, s), "seeder idx");
    ck(cudaMemcpyAsync(m->c12.p, c12.data(), c12.size() * sizeof(float), cudaMemcpyHostToDevice, s),
       "seeder adam table");
    ck(cudaMemsetAsync(m->ctr, 0, sizeof(int), s), "seeder step");
    ck(cudaMemsetAsync(m->loss.p, 0, sizeof(float), s), "seeder loss");
    int q = 0;
    if (!graph.e) {
      train_step();  // eager: sizes the workspace
      ck(cudaGetLastError(), "seeder train launch");
      q = 1;
      if (nb > 1) {
        ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "seeder capture");
        train_step();
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(s, &graph.g);
        ck(le, "seeder step launch in capture");
        ck(ce, "seeder end capture");
        ck(cudaGraphInstantiate(&graph.e, graph.g, 0), "seeder graph instantiate");
      }
    }
    for (; q < nb; ++q) ck(cudaGraphLaunch(graph.e, s), "seeder graph launch");
    m->step += nb;
    // the host copies above read pageable buffers that the next epoch rewrites
    ck(cudaStreamSynchronize(s), "seeder epoch sync");
    if (ep == epochs - 1) {
      ck(cudaMemcpy(&last, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost), "seeder loss");
      last /= (float)std::max(1, nb);
    }
  }
  ck(cudaGetLastError(), "seeder train launch");
  check_gemm(m->ws, s);
  return last;
}

// Inference: the first layer's input normalised straight into BF16, then one
// tcgen05 GEMM per layer whose epilogue adds the bias and applies GELU while
// writing the next layer's BF16 operand (the last layer writes FP32). The
// values are those of the training forward pass (the same FP32 bias add and
// GELU, rounded to BF16 where that pass converts its activations).
void mlp_predict(Mlp* m, const float* dX, int n, double* out, int out_ld, cudaStream_t s) {
  if (!m->normed) throw std::runtime_error("seeder: not trained");
  const int ni = m->dims.front(), no = m->dims.back(), L = m->L;
  const int chunk = std::max(m->bcap, std::min(n, 4096));
  ensure_batch(m, chunk);
  if ((int)m->wbf.size() != L) {
    m->wbf.clear();
    m->abf.clear();
    for (int l = 0; l < L; ++l) {
      m->wbf.emplace_back();
      m->abf.emplace_back();
    }
    m->wbf_step = -1;
  }
  if (m->wbf_step != m->step) {
    for (int l = 0; l < L; ++l) {
      const int K = m->dims[l], N = m->dims[l + 1];
      m->wbf[l].need((size_t)N * pad8(K));
      to_bf16(m->W[l].p, N, 1, N, K, m->wbf[l].p, pad8(K), s);  // B[n][k] = W[k][n]
    }
    m->wbf_step = m->step;
  }
  for (int l = 0; l < L; ++l) m->abf[l].need((size_t)chunk * pad8(m->dims[l]));
  for (int r0 = 0; r0 < n; r0 += chunk) {
    const int B = std::min(chunk, n - r0);
    k_norm_rows_bf16<<<grid_for((size_t)B * ni), 256, 0, s>>>(dX + (size_t)r0 * ni, B, ni, m->fmean.p,
                                                              m->fistd.p, m->abf[0].p, pad8(ni));
    for (int l = 1; l <= L; ++l) {
      const int K = m->dims[l - 1], N = m->dims[l];
      TcEpilogue ep;
      ep.bias = m->b[l - 1].p;
      if (l < L) {
        ep.gelu = 1;
        ep.out_bf16 = m->abf[l].p;
        ep.ld_out = pad8(N);
      }
      ck(tc_gemm_bf16(B, N, K, m->abf[l - 1].p, pad8(K), m->wbf[l - 1].p, pad8(K),
                      l < L ? nullptr : m->pre[L].p, N, 0, m->ws.err_flag(), s, &ep),
         "tcgen05 gemm launch");
    }
    double* o = out_ld > 0 ? out + r0 : out + (size_t)r0 * no;
    k_denorm<<<grid_for((size_t)B * no), 256, 0, s>>>(m->pre[L].p, B, no, m->tmean.p, m->tsd.p, o, out_ld);
  }
  ck(cudaGetLastError(), "seeder predict launch");
}

void mlp_gemm(int M, int N, int K, const float* A, int lda, int transA, const float* B, int ldb,
              int transB, float* C, int ldc, int accumulate, cudaStream_t s) {
  static std::mutex mu;
  static GemmWs* ws = new GemmWs;  // kept for the process: the standalone entry point's workspace
  std::lock_guard<std::mutex> lock(mu);
  gemm(M, N, K, A, lda, transA, B, ldb, transB, C, ldc, accumulate, *ws, s);
  ck(cudaGetLastError(), "gemm launch");
  check_gemm(*ws, s);
}

}  // namespace karam

// ---------------------------------------------------------------------------
// features and targets of a problem's instances
// ---------------------------------------------------------------------------
namespace karam {

namespace {

// Row r describes instance g = idx ? idx[r] : r: X[r] = (VTO per MOSFET,
// KP per MOSFET, DC value per source), Y[r] = node voltages (permuted order).
__global__ void k_features(DevTopo T, DevInst I, const int* idx, int rows, float* X, float* Y) {
  const int nm = T.n_mos, nf = 2 * T.n_mos + T.n_vs;
  const size_t ld = I.ld;
  const size_t nx = (size_t)rows * nf;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nx;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / nf), j = (int)(e - (size_t)r * nf);
    const int g = idx ? idx[r] : r;
    float v;
    if (j < nm)
      v = I.vth ? I.vth[(size_t)j * ld + g] : (float)T.mos_card[j].y;
    else if (j < 2 * nm)
      v = I.kp ? I.kp[(size_t)(j - nm) * ld + g] : (float)T.mos_card[j - nm].x;
    else
      v = (float)I.vs_dc[(size_t)(j - 2 * nm) * ld + g];
    X[e] = v;
  }
  if (!Y) return;
  const size_t ny = (size_t)rows * T.n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ny;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / T.n), i = (int)(e - (size_t)r * T.n);
    const int g = idx ? idx[r] : r;
    Y[e] = (float)I.v[(size_t)i * ld + g];
  }
}

}  // namespace

void seeder_features(const DevTopo& T, const DevInst& I, const int* idx, int rows, float* X,
                     float* Y, cudaStream_t s) {
  const size_t n = (size_t)rows * (2 * T.n_mos + T.n_vs);
  k_features<<<grid_for(n), 256, 0, s>>>(T, I, idx, rows, X, Y);
  ck(cudaGetLastError(), "seeder features launch");
}

}  // namespace karam
