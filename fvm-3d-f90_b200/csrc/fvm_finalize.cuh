// fvm_finalize.cuh — the end of a time step for one case, as a CTA-wide
// device function: ClassIteration%reset_residual / compute_residual per
// block in block order / update (class_iteration.f90, file-local 195-259),
// time += dt, the stop checks of converged (:180-188) and the next step's dt.
// Run by finalize_kernel, one CTA per case. Every FP64 operation is an
// explicitly rounded intrinsic, so the result does not depend on the
// contraction or fast-math flags of the including translation unit.
#pragma once
#include <cuda_runtime.h>

#include "fvm_types.h"

namespace fvm {

// One warp per block reduces its task partials (lanes stride the tasks, then
// a butterfly) and its lane 0 turns the sums into the block's squared norms;
// thread 0 folds the blocks in order, as the reference accumulates them. The
// six folds are independent chains, so a block costs thread 0 one square
// root of latency. Any multiple of 32 threads gives the same sums (each
// block's reduction and the fold order do not depend on the warp count). The
// CTA of case 0 also zeroes the stage work-queue counters for the next step.
// The descriptors (case, block list, block sizes and task ranges) change only
// when the engine re-plans between steps, so they are read before `wait`
// (the programmatic-launch wait for the step's last kernel) and their memory
// round trips overlap that kernel's tail; partials, counters and the case
// state are touched only after it.
template <class Wait>
__device__ __forceinline__ void finalize_case(int c, const DevBlock* blocks, const DevCase* cases, const int* case_blk,
                                              DevCaseState* st, const double* partials, int* counters,
                                              int ncounters, Wait wait) {
  constexpr int kMaxW = 8;
  __shared__ double red[kMaxW][6];
  __shared__ double redm[kMaxW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NW = min(kMaxW, (int)(blockDim.x >> 5));
  const DevCase& C = cases[c];
  const int nblocks = C.nblocks, block0 = C.block0, ts_set = C.timestep_set;
  const double dt_fixed = C.dt_fixed, cfl = C.cfl;
  // the first block of this warp
  int pf_task0 = 0, pf_ntask = 0;
  double pf_npt = 1.0;
  if (warp < NW && warp < nblocks) {
    const DevBlock& B = blocks[case_blk[block0 + warp]];
    pf_task0 = B.task0;
    pf_ntask = B.ntask;
    pf_npt = (double)((int64_t)B.n[0] * B.n[1] * B.n[2]);
  }
  wait();
  if (c == 0)
    for (int i = tid; i < ncounters; i += blockDim.x) counters[i] = 0;
  if (nblocks == 0) return;  // removed case (uniform over the CTA)
  double res[6] = {0, 0, 0, 0, 0, 0};
  double wmax = 0.0;
  for (int b0 = 0; b0 < nblocks; b0 += NW) {
    const int bb = b0 + warp;
    if (warp < NW && bb < nblocks) {
      int task0 = pf_task0, ntask = pf_ntask;
      double npt = pf_npt;
      if (b0 > 0) {
        const DevBlock& B = blocks[case_blk[block0 + bb]];
        task0 = B.task0;
        ntask = B.ntask;
        npt = (double)((int64_t)B.n[0] * B.n[1] * B.n[2]);
      }
      // each lane loads kU partials before adding them (in a fixed order), so
      // a block of many tasks costs one memory round trip per 32 * kU tasks
      constexpr int kU = 8;
      double s[5] = {0, 0, 0, 0, 0}, m = 0.0;
      for (int t = lane; t < ntask; t += 32 * kU) {
        double q[kU][6];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const int tt = t + 32 * u;
          if (tt < ntask) {
            const double* p = partials + (int64_t)(task0 + tt) * kPartStride;
#pragma unroll
            for (int v = 0; v < 6; ++v) q[u][v] = p[v];
          } else {
#pragma unroll
            for (int v = 0; v < 6; ++v) q[u][v] = 0.0;  // adds nothing: same sums as task by task
          }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
#pragma unroll
          for (int v = 0; v < 5; ++v) s[v] = __dadd_rn(s[v], q[u][v]);
          m = fmax(m, q[u][5]);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int v = 0; v < 5; ++v) s[v] = __dadd_rn(s[v], __shfl_xor_sync(0xffffffffu, s[v], o));
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      }
      if (lane == 0) {
        double res2_t = 0.0;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const double r2 = __ddiv_rn(s[v], npt);
          red[warp][v] = r2;
          res2_t = __dadd_rn(res2_t, r2);
        }
        red[warp][5] = __ddiv_rn(res2_t, 5.0);
        redm[warp] = m;
      }
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 0; w < NW && b0 + w < nblocks; ++w) {
#pragma unroll
        for (int v = 0; v < 6; ++v) res[v] = __dsqrt_rn(__dadd_rn(__dmul_rn(res[v], res[v]), red[w][v]));
        wmax = fmax(wmax, redm[w]);
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    DevCaseState& S = st[c];
    S.step += 1;
    S.t = __dadd_rn(S.t, S.dt);
    S.dt_last = S.dt;
    for (int e = 0; e < 6; ++e) S.res_abs[e] = res[e];
    if (S.step == 1)
      for (int e = 0; e < 6; ++e) S.res_abs0[e] = res[e];
    for (int e = 0; e < 6; ++e) S.res_rel[e] = __ddiv_rn(S.res_abs[e], S.res_abs0[e]);
    if (isnan(res[5]))
      S.status = 4;  // FVM_ERR_NONFINITE
    else if (res[5] > 1.0E10)
      S.status = 5;  // FVM_ERR_DIVERGED
    S.dt = (ts_set == 0) ? dt_fixed : __ddiv_rn(cfl, wmax);
  }
}

}  // namespace fvm
