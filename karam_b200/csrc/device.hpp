// device.hpp -- host-side declarations of the kernel launchers. The data
// layout the kernels share with the host is in nr_types.h.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "nr_types.h"

namespace karam {

// Launch geometry of the factor/solve kernel of an NR round: one CTA per tile
// of L instances.
struct RoundLaunch {
  int L = 0;          // instances per CTA (a power of two <= 32 for the pivot program;
                      // any count <= 32 for the level schedule, one warp each)
  int grid = 0;       // CTAs
  size_t smem = 0;    // dynamic shared memory bytes
  int ctas_per_sm = 0;
  int threads = 0;    // CTA size
  bool nd = false;    // the level-scheduled kernel (k_lu_nd)
  int big = 0;        // block per instance on the level schedule (k_lu_big): 1 with the
                      // ND slots in shared memory, 2 in a global workspace
  bool es_one = false; // evaluation + stamping by k_es_one, one CTA per listed instance
  char why[192] = {};  // when no candidate fits: why the last ones were rejected
};

// Lane stride of the instance-interleaved arrays for ni instances.
inline int lane_stride(int ni) { return (ni + 31) / 32 * 32; }

// Picks the factor/solve schedule: the kernel kind and L (instances per CTA)
// so the tiles fit shared memory and spread over the SMs in the fewest waves.
// want_lanes > 0 asks for that L (warp-per-instance level schedule or pivot
// program), -1 for the block-per-instance kernel with the ND slots in shared
// memory, -2 with them in a global workspace; 0 chooses. Sets the kernels'
// shared-memory limits (call outside stream capture).
RoundLaunch plan_round(const DevTopo& T, int ni, int prec, int max_smem, int num_sms,
                       int want_lanes);
void launch_init(const DevTopo& T, const DevInst& I, const JobParams& P, cudaStream_t s);
// Lists the instances not yet done into list[0..*count) (*count starts at 0).
void launch_live_list(const DevInst& I, int* list, int* count, cudaStream_t s);
// The batch statistical seed from the DC solutions of instances 0..W-1 (lane 0
// of `seed`); *ok = 1 when it is confident enough to use.
void launch_ema_seed(const DevTopo& T, const DevInst& I, int W, double* seed, int* ok,
                     cudaStream_t s);
// Moves every converged instance into the transient at step 1 (capacitor
// history from the accepted point when init_caps).
void launch_tran_start(const DevTopo& T, const DevInst& I, const JobParams& P, int init_caps,
                       cudaStream_t s);
// Device evaluation + stamping of every live instance at x (k_es): Jacobian
// value slots, KCL residual and the per-instance reductions.
void launch_eval_stamp(const DevTopo& T, const DevInst& I, const JobParams& P,
                       const RoundLaunch& L, int prec, cudaStream_t s);
// Control flow + static-pivot factor/solve of every live instance (k_lu).
void launch_lu(const DevTopo& T, const DevInst& I, const JobParams& P, const RoundLaunch& L,
               int prec, int* active, cudaStream_t s);
// Rescue of the solves whose static pivots failed (FP64 static pivots, then
// LU with partial pivoting): one warp per solve and workspace slot, `warps`
// warps per CTA with K dense row buffers each in shared memory.
struct RescuePlan {
  int K = 0;
  int warps = 0;        // 0: the problem is too large for the rescue kernel
  size_t smem = 0;      // dynamic shared memory per CTA
  int ctas_per_sm = 0;  // filled by the caller (occupancy)
};
RescuePlan plan_rescue(const DevTopo& T);
// CTAs of the rescue kernel that can be resident per SM (sets its
// shared-memory limit first; call outside stream capture).
int rescue_ctas_per_sm(const DevTopo& T, const RescuePlan& R);
void launch_rescue(const DevTopo& T, const DevInst& I, const JobParams& P, const RescuePlan& R,
                   cudaStream_t s);
// The persistent kernels' launch plan for one problem: variant = where the
// factor/solve keeps its data (0 packed level program and ND slots in shared
// memory, 1 slots in shared memory, 2 slots in a global workspace of
// ni * nd_S values; PersistJob::variant); resident_at > 0: the byte offset in
// dynamic shared memory from which each instance's state is kept there for
// the whole launch (resident_in), when it fits beside the phases;
// smem = the dynamic shared memory, 0 when nothing fits.
struct PersistPlan {
  size_t smem = 0;
  int variant = -1;
  int resident_at = 0;
  int slot_values = 0;  // 1: the evaluation keeps every slot term's value in shared memory
};
// The plan of the persistent per-instance kernel (k_persist) for precision
// prec and rescue plan R (smem 0 when the problem cannot use it): it needs
// the packed level program, and its phases (evaluation + stamping of one
// instance, the packed factor/solve, a rescue warp) must each fit one CTA's
// shared memory. Sets the kernel's shared-memory limit (call outside stream
// capture).
PersistPlan plan_persist(const DevTopo& T, int prec, const RescuePlan& R, int max_smem);
// Every remaining NR round of each listed instance (or of instances
// 0 .. grid - 1 when I.live_in is null) in one launch of `grid` CTAs, at most
// max_rounds rounds each; *active receives the instances still live and
// *rounds_max the most rounds one instance ran.
void launch_persist(const DevTopo& T, const DevInst& I, const JobParams& P, int prec, int grid,
                    const PersistPlan& plan, int max_rounds, int K, int* active, int* rounds_max,
                    cudaStream_t s);
// The first variant (0, 1, 2) whose phases each fit one CTA's shared memory
// next to the multi-problem kernel's static shared memory. Sets the kernel's
// shared-memory limit (call outside stream capture).
PersistPlan plan_persist_job(const DevTopo& T, int prec, const RescuePlan& R, int max_smem);
// Every remaining NR round of every instance of n_jobs problems (jobs: a
// device array sorted by cta0, the first at 0, the CTA ranges back to back
// and covering grid CTAs) in one launch, at most max_rounds rounds each, with
// smem bytes of dynamic shared memory (the largest job's PersistPlan::smem);
// *active and *rounds_max as for launch_persist, over all jobs;
// *slot_timeouts counts solves that found no free rescue slot in time.
void launch_persist_multi(const PersistJob* jobs, int n_jobs, int prec, int grid, size_t smem,
                          int max_rounds, int* active, int* rounds_max, int* slot_timeouts,
                          cudaStream_t s);
// Dynamic shared memory of the AC kernel (k_ac), or 0 when the problem has
// no packed level program or its complex ND slots do not fit one CTA;
// *stage_prog = 1 when the program fits beside them. Sets the kernel's
// shared-memory limit (call outside stream capture).
size_t plan_ac(const DevTopo& T, int max_smem, int* stage_prog);
// One CTA per (frequency, instance): grid A.n_points x I.ni.
void launch_ac(const DevTopo& T, const DevInst& I, const AcParams& A, size_t smem, cudaStream_t s);
void unpermute(const double* v_perm, const int* perm, double* out, int ni, int ld, int n,
               cudaStream_t s);
// [ni][n] FP32 per-device parameters (netlist order) into [n][ld] SoA order.
void interleave_f(const float* src, const int* order, float* dst, int ni, int ld, int n,
                  cudaStream_t s);
void interleave(const double* src, const int* perm, double* dst, int ni, int ld, int n,
                cudaStream_t s);

}  // namespace karam
