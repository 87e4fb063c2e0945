// fvm_step2d.cuh — persistent step kernel for small 2D engines.
//
// A 2D Euler case of a few hundred tiles (the reference's own 256 x 256
// case: 256 tasks of 32 x 8 cells) spends most of a time step in launch and
// ramp latency: each RK stage is a separate launch of a few microseconds of
// work, then the finalize. This kernel runs whole time steps in one
// cooperative launch instead: every CTA stays resident, runs the stage body
// of stage_kernel (stage_run, with loads that see the other CTAs' writes of
// the same launch), and the stages are separated by a grid-wide barrier; after
// the last stage the CTAs of the cases run the finalize (residual norms, time,
// next dt, queue counters) and a last barrier closes the step. Same tasks,
// same arithmetic and same reduction order as the launch-per-stage path, so
// the results are bit-identical to it.
//
// The barrier waits are bounded: a CTA that waits more than one second at a
// barrier sets the engine's error word and leaves the kernel; the others then
// time out as well, and the host reports FVM_ERR_TIMEOUT with the context
// still usable. (A cooperative launch guarantees that every CTA is resident,
// so a barrier only waits for CTAs that are running.)
#pragma once
#include "fvm_finalize.cuh"
#include "fvm_stage.cuh"

namespace fvm {

// Grid-wide barrier of a cooperative launch: thread 0 of every CTA arrives on
// a counter; the last one resets it and advances the generation, the others
// poll the generation (at most 1 s). The fences on both sides order every
// write before the barrier before every read after it, across CTAs.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, int32_t* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = bar + 1;
    const unsigned int g0 = *gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(bar, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = global_ns();
      for (int i = 0;; ++i) {
        if (*gen != g0) break;
        if ((i & 63) == 63 && global_ns() - t0 > 1000000000ull) {
          ok = 0;
          atomicExch(err, 2);
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int RECON, int FLUX, int PREC, bool TB, int TX, int TY, int MINB>
__global__ void __launch_bounds__(StageCfg<RECON, FLUX, PREC, TB, 2, TX, TY>::NT,
                                  (MINB > 0 ? MINB : (PREC == PREC_FP32 ? 512 : 384) / (TX * TY)))
    step2d_kernel(const Step2DArgs a) {
  for (int s = 0; s < a.nsteps; ++s) {
    for (int m = 0; m < a.nstages; ++m) {
      stage_run<RECON, FLUX, PREC, TB, 2, TX, TY, true>(a.st[m]);
      if (!grid_barrier(a.bar, a.err)) return;
    }
    for (int c = blockIdx.x; c < a.ncases; c += gridDim.x)
      finalize_case(c, a.blocks, a.cases, a.case_blk, a.state, a.st[0].partials, a.counters, a.ncounters);
    if (!grid_barrier(a.bar, a.err)) return;
  }
}

}  // namespace fvm
