// kernels.cu -- sm_100a kernels (nr_device.cuh) and their launchers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <vector>

#include "../../include/karam.h"
#include "device.hpp"
#include "nr_device.cuh"

namespace karam {

using namespace knr;

namespace {

// the opt-in shared-memory limit of one CTA on sm_100 (227 KiB)
constexpr int kSmemOptin = 232448;

// Raises a kernel's dynamic shared-memory limit to what the opt-in maximum
// leaves beside its static shared memory. The limit is process-wide state of
// the kernel: setting it to this one value for every problem keeps problems
// planned from several threads from undoing each other's limits.
cudaError_t open_smem_limit(const void* kern, int max_smem) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              max_smem - (int)fa.sharedSizeBytes);
}

// Level schedule: ND slots + right-hand side of L instances; else value slots
// + right-hand side of L instances, then the packed pivot records.
size_t round_smem(const DevTopo& T, int L, size_t es, bool nd) {
  if (nd)
    return ((es * ((size_t)T.nd_S + (size_t)T.nd_SY) * (size_t)L + 15) & ~size_t(15)) +
           sizeof(int) * (size_t)T.nd_prog_len;
  size_t b = es * ((size_t)T.nv + (size_t)T.n) * (size_t)L;
  if (T.lu_rec) b = ((b + 15) & ~size_t(15)) + (2 * sizeof(int4) + sizeof(int2)) * (size_t)T.n;
  return b;
}

int grid_for(size_t total, int threads) {
  size_t b = (total + threads - 1) / threads;
  return (int)std::max<size_t>(1, std::min<size_t>(b, 1u << 20));
}

}  // namespace

namespace {

// The factor/solve kernel of a candidate schedule.
const void* lu_kernel(bool mixed, bool nd, int big) {
  if (big == 1)
    return mixed ? (const void*)k_lu_big<float, false, false> : (const void*)k_lu_big<double, false, false>;
  if (big == 2)
    return mixed ? (const void*)k_lu_big<float, true, false> : (const void*)k_lu_big<double, true, false>;
  if (big == 3)
    return mixed ? (const void*)k_lu_big<float, false, true> : (const void*)k_lu_big<double, false, true>;
  if (big == 5)
    return mixed ? (const void*)k_lu_big<float, true, false, true>
                 : (const void*)k_lu_big<double, true, false, true>;
  if (nd) return mixed ? (const void*)k_lu_nd<float> : (const void*)k_lu_nd<double>;
  return mixed ? (const void*)k_lu<float> : (const void*)k_lu<double>;
}

}  // namespace

RoundLaunch plan_round(const DevTopo& T, int ni, int prec, int max_smem, int num_sms,
                       int want_lanes) {
  const bool mixed = prec == KARAM_PREC_MIXED;
  const size_t es = mixed ? sizeof(float) : sizeof(double);
  RoundLaunch best;
  long best_waves = -1;
  int best_rank = -1;
  // candidates: the level-scheduled kernel with L instance warps (any L up to
  // its thread limit), the block-per-instance kernel on the level schedule
  // (ND slots in shared memory, or in a global workspace), then the
  // pivot-program kernel with power-of-two L
  struct Cand {
    int L;
    bool nd;
    int big;
    int rank;  // preference among candidates with as few waves
  };
  std::vector<Cand> cands;
  if (T.nd_prog_len > 0)
    for (int L = (mixed ? 32 : 16); L >= 1; --L) cands.push_back({L, true, 0, 3});
  if (T.nd_levels > 0) {
    if (T.nd_prog_len > 0) cands.push_back({1, false, 3, 2});
    cands.push_back({1, false, 1, 2});
    cands.push_back({1, false, 2, 1});
    cands.push_back({1, false, 5, 1});  // taken only where kind 2 does not fit
  }
  for (int L = kMaxLanes; L >= 1; L >>= 1) cands.push_back({L, false, 0, 0});
  bool big2_fits = false;
  for (const Cand& c : cands) {
    const int L = c.L;
    if (want_lanes > 0 && (c.big || L != want_lanes)) continue;
    if (want_lanes < 0 && c.big != -want_lanes) continue;
    if (c.big == 5 && want_lanes == 0 && big2_fits) continue;
    const void* kern = lu_kernel(mixed, c.nd, c.big);
    const int threads = c.big ? kBigThreads : c.nd ? 32 * L : kRoundThreads;
    size_t sm;
    if (c.big == 1)
      sm = es * ((size_t)T.nd_SY + (size_t)T.nd_S);
    else if (c.big == 3)
      sm = ((es * ((size_t)T.nd_SY + (size_t)T.nd_S) + 15) & ~size_t(15)) +
           sizeof(int) * (((size_t)T.nd_prog_len + 3) & ~size_t(3));
    else if (c.big == 2)
      sm = (es * (size_t)T.nd_SY + 15) & ~size_t(15);
    else if (c.big == 5)
      sm = 0;
    else
      sm = round_smem(T, L, es, c.nd);
    auto reject = [&](const char* what) {
      snprintf(best.why, sizeof(best.why), "%s: %s (kind %d, L %d, %zu B shared)",
               c.big ? "block per instance" : c.nd ? "warp per instance" : "pivot program", what,
               c.big, L, sm);
    };
    if (sm > (size_t)max_smem) {
      reject("shared memory");
      continue;
    }
    if (const cudaError_t e = open_smem_limit(kern, max_smem); e != cudaSuccess) {
      reject(cudaGetErrorString(e));
      cudaGetLastError();
      continue;
    }
    int per_sm = 0;
    if (const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, sm);
        e != cudaSuccess || per_sm < 1) {
      reject(e != cudaSuccess ? cudaGetErrorString(e) : "no CTA fits an SM");
      cudaGetLastError();
      continue;
    }
    if (c.big == 2) big2_fits = true;
    const int grid = (ni + L - 1) / L;
    const long slots = (long)per_sm * std::max(1, num_sms);
    const long waves = (grid + slots - 1) / slots;
    // fewest waves; among equals the preferred kind, then a grid that
    // reaches every SM (the streaming phases spread wider)
    const bool fills = grid >= num_sms, best_fills = best.grid >= num_sms;
    bool better = best_waves < 0 || waves < best_waves;
    if (!better && waves == best_waves) {
      if (c.rank != best_rank)
        better = c.rank > best_rank;
      else
        better = fills && !best_fills;
    }
    if (better) {
      best_waves = waves;
      best_rank = c.rank;
      best.L = L;
      best.grid = grid;
      best.smem = sm;
      best.ctas_per_sm = per_sm;
      best.threads = threads;
      best.nd = c.nd;
      best.big = c.big;
    }
  }
  open_smem_limit((const void*)k_rescue<float>, max_smem);
  open_smem_limit((const void*)k_rescue<double>, max_smem);
  return best;
}

void launch_live_list(const DevInst& I, int* list, int* count, cudaStream_t s) {
  k_live_list<<<(I.ni + 255) / 256, 256, 0, s>>>(I, list, count);
}

void launch_init(const DevTopo& T, const DevInst& I, const JobParams& P, cudaStream_t s) {
  k_init<<<(I.ni + 127) / 128, 128, 0, s>>>(T, I, P);
}

void launch_ema_seed(const DevTopo& T, const DevInst& I, int W, double* seed, int* ok,
                     cudaStream_t s) {
  k_ema_seed<<<1, 256, 0, s>>>(T, I, W, seed, ok);
}

void launch_tran_start(const DevTopo& T, const DevInst& I, const JobParams& P, int init_caps,
                       cudaStream_t s) {
  k_tran_start<<<(I.ni + 127) / 128, 128, 0, s>>>(T, I, P, init_caps);
}

void launch_eval_stamp(const DevTopo& T, const DevInst& I, const JobParams& P,
                       const RoundLaunch& L, int prec, cudaStream_t s) {
  if (L.es_one) {  // tail rounds: one CTA per listed live instance
    const size_t sm =
        sizeof(double) * (3 * (size_t)(T.n_mos + T.n_dio) + (size_t)T.n_ft_terms + (size_t)T.n_hub_slot_terms);
    if (prec == KARAM_PREC_MIXED)
      k_es_one<float><<<L.grid, kBigThreads, sm, s>>>(T, I, P);
    else
      k_es_one<double><<<L.grid, kBigThreads, sm, s>>>(T, I, P);
    return;
  }
  const dim3 grid((I.ni + 31) / 32, T.n_es_blocks);
  if (prec == KARAM_PREC_MIXED)
    (P.lte_rel > 0.0 ? k_es<float, true> : k_es<float, false>)<<<grid, 256, 0, s>>>(T, I, P);
  else
    (P.lte_rel > 0.0 ? k_es<double, true> : k_es<double, false>)<<<grid, 256, 0, s>>>(T, I, P);
}

void launch_lu(const DevTopo& T, const DevInst& I, const JobParams& P, const RoundLaunch& L,
               int prec, int* active, cudaStream_t s) {
  if (L.big == 1) {
    if (prec == KARAM_PREC_MIXED)
      k_lu_big<float, false, false><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
    else
      k_lu_big<double, false, false><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
  } else if (L.big == 2) {
    if (prec == KARAM_PREC_MIXED)
      k_lu_big<float, true, false><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
    else
      k_lu_big<double, true, false><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
  } else if (L.big == 3) {
    if (prec == KARAM_PREC_MIXED)
      k_lu_big<float, false, true><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
    else
      k_lu_big<double, false, true><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
  } else if (L.big == 5) {
    if (prec == KARAM_PREC_MIXED)
      k_lu_big<float, true, false, true><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
    else
      k_lu_big<double, true, false, true><<<L.grid, L.threads, L.smem, s>>>(T, I, P, active);
  } else if (L.nd) {
    if (prec == KARAM_PREC_MIXED)
      k_lu_nd<float><<<L.grid, L.threads, L.smem, s>>>(T, I, P, L.L, active);
    else
      k_lu_nd<double><<<L.grid, L.threads, L.smem, s>>>(T, I, P, L.L, active);
  } else if (prec == KARAM_PREC_MIXED) {
    k_lu<float><<<L.grid, kRoundThreads, L.smem, s>>>(T, I, P, L.L, active);
  } else {
    k_lu<double><<<L.grid, kRoundThreads, L.smem, s>>>(T, I, P, L.L, active);
  }
}

RescuePlan plan_rescue(const DevTopo& T) {
  const size_t limit = kSmemOptin;
  const size_t rec = (T.lu_rec ? rescue_rec_bytes(T.n) : 0) + rescue_tab_bytes(T.n, T.nv);
  RescuePlan R;
  for (int K = 2; K >= 0; --K) {
    if (K > T.n) continue;
    const size_t wb = rescue_warp_bytes(T.n, T.nv, K);
    if (rec + wb > limit) continue;
    R.K = K;
    R.warps = (int)std::min<size_t>(8, (limit - rec) / wb);
    R.smem = rec + (size_t)R.warps * wb;
    break;
  }
  return R;
}

int rescue_ctas_per_sm(const DevTopo& T, const RescuePlan& R) {
  if (R.warps <= 0) return 0;
  open_smem_limit((const void*)k_rescue<float>, kSmemOptin);
  open_smem_limit((const void*)k_rescue<double>, kSmemOptin);
  int a = 0, b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_rescue<float>, 32 * R.warps, R.smem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_rescue<double>, 32 * R.warps, R.smem) !=
          cudaSuccess)
    return 0;
  return std::min(a, b);
}

void launch_rescue(const DevTopo& T, const DevInst& I, const JobParams& P, const RescuePlan& R,
                   cudaStream_t s) {
  const int grid = (I.rescue_slots + R.warps - 1) / R.warps;
  if (P.precision == KARAM_PREC_MIXED)
    k_rescue<float><<<grid, 32 * R.warps, R.smem, s>>>(T, I, P, R.K);
  else
    k_rescue<double><<<grid, 32 * R.warps, R.smem, s>>>(T, I, P, R.K);
}

// The persistent plan's shared memory beyond the phases' minimum sm (lu, rs:
// the factor/solve's and the rescue's needs): the slot-term values of the
// evaluation and the instance's resident state, each when it fits, the
// values first.
static void fill_persist_smem(PersistPlan& plan, const DevTopo& T, size_t es, size_t sm, size_t lu, size_t rs,
                       size_t static_smem, int max_smem) {
  const size_t room = (size_t)max_smem - static_smem;
  const size_t ev_jv = sizeof(double) * (3 * (size_t)(T.n_mos + T.n_dio) + (size_t)T.n_ft_terms +
                                         (size_t)T.n_hub_slot_terms + (size_t)T.n_jt_terms);
  const size_t sm_jv = (std::max({ev_jv, lu, rs, size_t(16)}) + 15) & ~size_t(15);
  const size_t res = resident_layout(T, es).total;
  plan.slot_values = 0;
  plan.resident_at = 0;
  plan.smem = sm;
  if (sm_jv + res <= room) {
    plan.slot_values = 1;
    plan.resident_at = (int)sm_jv;
    plan.smem = sm_jv + res;
  } else if (sm + res <= room) {
    plan.resident_at = (int)sm;
    plan.smem = sm + res;
  } else if (sm_jv <= room) {
    plan.slot_values = 1;
    plan.smem = sm_jv;
  }
}

PersistPlan plan_persist(const DevTopo& T, int prec, const RescuePlan& R, int max_smem) {
  PersistPlan plan;
  if (T.nd_prog_len <= 0 || T.nd_levels <= 0) return plan;
  const size_t es = prec == KARAM_PREC_MIXED ? sizeof(float) : sizeof(double);
  const size_t ev = sizeof(double) * (3 * (size_t)(T.n_mos + T.n_dio) + (size_t)T.n_ft_terms +
                                      (size_t)T.n_hub_slot_terms);
  const size_t lu = ((es * ((size_t)T.nd_SY + (size_t)T.nd_S) + 15) & ~size_t(15)) +
                    sizeof(int) * (((size_t)T.nd_prog_len + 3) & ~size_t(3));
  const size_t rs = R.warps > 0 ? (T.lu_rec ? rescue_rec_bytes(T.n) : 0) + rescue_tab_bytes(T.n, T.nv) +
                                      rescue_warp_bytes(T.n, T.nv, R.K)
                                : 0;
  const size_t sm = (std::max({ev, lu, rs, size_t(16)}) + 15) & ~size_t(15);
  const void* kern = prec == KARAM_PREC_MIXED ? (const void*)k_persist<float> : (const void*)k_persist<double>;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) {
    cudaGetLastError();
    return plan;
  }
  if (sm + fa.sharedSizeBytes > (size_t)max_smem) return plan;
  if (open_smem_limit(kern, max_smem) != cudaSuccess) {
    cudaGetLastError();
    return plan;
  }
  plan.variant = 0;
  fill_persist_smem(plan, T, es, sm, lu, rs, fa.sharedSizeBytes, max_smem);
  return plan;
}

void launch_persist(const DevTopo& T, const DevInst& I, const JobParams& P, int prec, int grid,
                    const PersistPlan& plan, int max_rounds, int K, int* active, int* rounds_max,
                    cudaStream_t s) {
  if (prec == KARAM_PREC_MIXED)
    k_persist<float><<<grid, kPersistThreads, plan.smem, s>>>(T, I, P, max_rounds, K, active, rounds_max,
                                                              plan.resident_at, plan.slot_values);
  else
    k_persist<double><<<grid, kPersistThreads, plan.smem, s>>>(T, I, P, max_rounds, K, active, rounds_max,
                                                               plan.resident_at, plan.slot_values);
}

PersistPlan plan_persist_job(const DevTopo& T, int prec, const RescuePlan& R, int max_smem) {
  PersistPlan plan;
  if (T.nd_levels <= 0) return plan;
  const bool mixed = prec == KARAM_PREC_MIXED;
  const size_t es = mixed ? sizeof(float) : sizeof(double);
  const size_t ev = sizeof(double) * (3 * (size_t)(T.n_mos + T.n_dio) + (size_t)T.n_ft_terms +
                                      (size_t)T.n_hub_slot_terms);
  const size_t rs = R.warps > 0 ? (T.lu_rec ? rescue_rec_bytes(T.n) : 0) + rescue_tab_bytes(T.n, T.nv) +
                                      rescue_warp_bytes(T.n, T.nv, R.K)
                                : 0;
  const void* kern = mixed ? (const void*)k_persist_multi<float> : (const void*)k_persist_multi<double>;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) {
    cudaGetLastError();
    return plan;
  }
  const size_t slots = es * ((size_t)T.nd_SY + (size_t)T.nd_S);
  for (int v = 0; v < 3; ++v) {
    size_t lu;
    if (v == 0) {
      if (T.nd_prog_len <= 0) continue;
      lu = ((slots + 15) & ~size_t(15)) + sizeof(int) * (((size_t)T.nd_prog_len + 3) & ~size_t(3));
    } else if (v == 1) {
      lu = slots;
    } else {
      lu = (es * (size_t)T.nd_SY + 15) & ~size_t(15);
    }
    const size_t sm = (std::max({ev, lu, rs, size_t(16)}) + 15) & ~size_t(15);
    if (sm + fa.sharedSizeBytes > (size_t)max_smem) continue;
    if (open_smem_limit(kern, max_smem) != cudaSuccess) {
      cudaGetLastError();
      return plan;
    }
    plan.variant = v;
    fill_persist_smem(plan, T, es, sm, lu, rs, fa.sharedSizeBytes, max_smem);
    return plan;
  }
  return plan;
}

void launch_persist_multi(const PersistJob* jobs, int n_jobs, int prec, int grid, size_t smem,
                          int max_rounds, int* active, int* rounds_max, int* slot_timeouts,
                          cudaStream_t s) {
  if (prec == KARAM_PREC_MIXED)
    k_persist_multi<float><<<grid, kPersistThreads, smem, s>>>(jobs, n_jobs, max_rounds, active,
                                                               rounds_max, slot_timeouts);
  else
    k_persist_multi<double><<<grid, kPersistThreads, smem, s>>>(jobs, n_jobs, max_rounds, active,
                                                                rounds_max, slot_timeouts);
}

size_t plan_ac(const DevTopo& T, int max_smem, int* stage_prog) {
  *stage_prog = 0;
  if (T.nd_prog_len <= 0 || T.nd_levels <= 0) return 0;
  const size_t slots = sizeof(double2) * ((size_t)T.nd_SY + (size_t)T.nd_S);
  const size_t prog = sizeof(int) * (((size_t)T.nd_prog_len + 3) & ~size_t(3));
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k_ac) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const size_t room = (size_t)max_smem - fa.sharedSizeBytes;
  if (slots > room) return 0;
  if (open_smem_limit((const void*)k_ac, max_smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (slots + prog <= room) {
    *stage_prog = 1;
    return slots + prog;
  }
  return std::max<size_t>(slots, 16);
}

void launch_ac(const DevTopo& T, const DevInst& I, const AcParams& A, size_t smem, cudaStream_t s) {
  k_ac<<<dim3(A.n_points, I.ni), 256, smem, s>>>(T, I, A);
}

void unpermute(const double* v_perm, const int* perm, double* out, int ni, int ld, int n,
               cudaStream_t s) {
  k_unpermute<<<grid_for((size_t)n * ld, 256), 256, 0, s>>>(v_perm, perm, out, ni, ld, n);
}

void interleave_f(const float* src, const int* order, float* dst, int ni, int ld, int n,
                  cudaStream_t s) {
  k_interleave_f<<<grid_for((size_t)n * ld, 256), 256, 0, s>>>(src, order, dst, ni, ld, n);
}

void interleave(const double* src, const int* perm, double* dst, int ni, int ld, int n,
                cudaStream_t s) {
  k_interleave<<<grid_for((size_t)n * ld, 256), 256, 0, s>>>(src, perm, dst, ni, ld, n);
}

}  // namespace karam
