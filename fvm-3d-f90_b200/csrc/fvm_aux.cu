// fvm_aux.cu — the kernels around the fused stage: ghost gather, state
// pack/unpack, primitive download, CFL wave-speed reduction, the per-step
// finalize (residual norms, time, next dt) and the exact-FP64 form of the
// viscous contribution.
// Compiled with -fmad=false: every FP64 expression here keeps the
// reference's rounding order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fvm_aux.h"
#include "fvm_finalize.cuh"
#include "fvm_schemes.cuh"
#include "fvm_types.h"
#include "fvm_visc.cuh"

namespace fvm {

// ---------------------------------------------------------------- gather
// Ghost cells of connected / periodic regions: dst[i] = src[i] for all five
// variables, offsets relative to a role slab (the block-to-block exchange the
// reference describes in defs_face_geom.f90:378-402 but never performs).
// Every source is a real cell (the host resolves ghost-to-ghost chains), so
// the pairs are independent. Each thread takes kGatherPer pairs a grid
// apart (a warp's pairs stay consecutive; each pair one 8-byte load of two
// 32-bit cell offsets) and issues all their loads before any store, so the
// index-then-data latency chain is paid once per thread. Capped at 64
// registers, four 256-thread CTAs fit on an SM, so the 576 CTAs of the 128^3
// vortex in 8 blocks (583 K ghost cells) run as one wave (at 68 registers,
// three per SM: 444 + 132).
constexpr int kGatherPer = 4;
__global__ void __launch_bounds__(256, 4) gather_kernel(double* __restrict__ base, int64_t vs, const int2* __restrict__ pairs,
                              int64_t npairs) {
  const int64_t G = (int64_t)gridDim.x * blockDim.x;
  // the pairs change only when the engine re-plans between steps: the first
  // round's are loaded before the wait for the stage kernel that wrote the
  // values, so their round trip overlaps its tail
  int2 p[kGatherPer];
  {
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kGatherPer; ++j) {
      const int64_t i = i0 + j * G;
      p[j] = i < npairs ? pairs[i] : make_int2(-1, -1);
    }
  }
  pdl_wait();
  pdl_trigger();
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < npairs; i0 += G * kGatherPer) {
    if (i0 != blockIdx.x * (int64_t)blockDim.x + threadIdx.x) {
#pragma unroll
      for (int j = 0; j < kGatherPer; ++j) {
        const int64_t i = i0 + j * G;
        p[j] = i < npairs ? pairs[i] : make_int2(-1, -1);
      }
    }
    double val[kGatherPer][5];
#pragma unroll
    for (int j = 0; j < kGatherPer; ++j)
      if (p[j].x >= 0)
#pragma unroll
        for (int v = 0; v < 5; ++v) val[j][v] = base[(int64_t)p[j].y + v * vs];
#pragma unroll
    for (int j = 0; j < kGatherPer; ++j)
      if (p[j].x >= 0)
#pragma unroll
        for (int v = 0; v < 5; ++v) base[(int64_t)p[j].x + v * vs] = val[j][v];
  }
}

// ---------------------------------------------------------------- pack / unpack
// Host layout: Fortran (ni,nj,nk,5) of the real range, get_q()
// (defs_block_data.f90:299-312).
__global__ void unpack_kernel(double* __restrict__ role_blk, int64_t vs, int sy, int sz, int ni, int nj, int nk,
                              const double* __restrict__ host_layout) {
  const int64_t nc = (int64_t)ni * nj * nk;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % ni);
    const int64_t r = c / ni;
    const int j = (int)(r % nj), k = (int)(r / nj);
    const int64_t o = i + (int64_t)j * sy + (int64_t)k * sz;
#pragma unroll
    for (int v = 0; v < 5; ++v) role_blk[o + v * vs] = host_layout[c + v * nc];
  }
}

__global__ void pack_kernel(const double* __restrict__ role_blk, int64_t vs, int sy, int sz, int ni, int nj,
                            int nk, double* __restrict__ host_layout, int prim, double gm1) {
  const int64_t nc = (int64_t)ni * nj * nk;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % ni);
    const int64_t r = c / ni;
    const int j = (int)(r % nj), k = (int)(r / nj);
    const int64_t o = i + (int64_t)j * sy + (int64_t)k * sz;
    double q[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v] = role_blk[o + v * vs];
    if (prim) {
      // convert_q_to_p_blk_sub (class_flow_field.f90:383-396)
      Prim5<double> p = cons2prim<double, true>(q[0], q[1], q[2], q[3], q[4], gm1);
      q[0] = p.r; q[1] = p.u; q[2] = p.v; q[3] = p.w; q[4] = p.p;
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) host_layout[c + v * nc] = q[v];
  }
}

// ---------------------------------------------------------------- CFL
__device__ __forceinline__ double cell_wavespeed(const double q[5], double gamma, double gm1, const double dr[3],
                                                 int idim) {
  Prim5<double> p = cons2prim<double, true>(q[0], q[1], q[2], q[3], q[4], gm1);
  const double c = sqrt(gamma * p.p / p.r);
  double s = (fabs(p.u) + c) / dr[0] + (fabs(p.v) + c) / dr[1];
  if (idim == 3) s = s + (fabs(p.w) + c) / dr[2];
  return s;
}

// Max wave-speed sum per case over role `role` (max is order-free, so the
// atomic on the non-negative bit pattern is deterministic).
__global__ void wavespeed_kernel(const DevBlock* blocks, const DevCase* cases, int role,
                                 unsigned long long* case_max) {
  const DevBlock B = blocks[blockIdx.y];
  const DevCase& C = cases[B.case_id];
  const int64_t nc = (int64_t)B.n[0] * B.n[1] * B.n[2];
  double m = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % B.n[0]);
    const int64_t r = c / B.n[0];
    const int j = (int)(r % B.n[1]), k = (int)(r / B.n[1]);
    const int64_t o = i + (int64_t)j * B.sy + (int64_t)k * B.sz;
    double q[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v] = B.q[role][o + v * B.vs];
    m = fmax(m, cell_wavespeed(q, C.gamma, C.gm1, B.dr, C.idim));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&case_max[B.case_id], (unsigned long long)__double_as_longlong(m));
}

// dt of the first step: fix_timestep, or cfl / max wave-speed sum.
__global__ void init_dt_kernel(const DevCase* cases, DevCaseState* st, const unsigned long long* case_max,
                               const int* mask, int ncases) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncases || !mask[c]) return;
  const DevCase& C = cases[c];
  st[c].dt = (C.timestep_set == 0) ? C.dt_fixed : C.cfl / __longlong_as_double((long long)case_max[c]);
}

// ---------------------------------------------------------------- finalize
// One CTA per case, after the last stage of a step (finalize_case in
// fvm_finalize.cuh).
__global__ void finalize_kernel(const DevBlock* blocks, const DevCase* cases, const int* case_blk, DevCaseState* st,
                                const double* partials, int* counters, int ncounters) {
  finalize_case(blockIdx.x, blocks, cases, case_blk, st, partials, counters, ncounters, [] {
    pdl_wait();
    pdl_trigger();
  });
}

// ---------------------------------------------------------------- launchers
static inline int grid_for(int64_t n, int bs) {
  int64_t g = (n + bs - 1) / bs;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t launch_gather(double* base, int64_t vs, const int32_t* pairs, int64_t npairs, cudaStream_t s,
                          bool pdl) {
  if (npairs == 0) return cudaSuccess;
  const int64_t threads = (npairs + kGatherPer - 1) / kGatherPer;
  LaunchCfg L(dim3(grid_for(threads, 256)), dim3(256), 0, s, pdl);
  return cudaLaunchKernelEx(&L.cfg, gather_kernel, base, vs, reinterpret_cast<const int2*>(pairs), npairs);
}

cudaError_t launch_unpack(double* role_blk, int64_t vs, int sy, int sz, int ni, int nj, int nk, const double* src,
                          cudaStream_t s) {
  unpack_kernel<<<grid_for((int64_t)ni * nj * nk, 256), 256, 0, s>>>(role_blk, vs, sy, sz, ni, nj, nk, src);
  return cudaGetLastError();
}

cudaError_t launch_pack(const double* role_blk, int64_t vs, int sy, int sz, int ni, int nj, int nk, double* dst,
                        int prim, double gm1, cudaStream_t s) {
  pack_kernel<<<grid_for((int64_t)ni * nj * nk, 256), 256, 0, s>>>(role_blk, vs, sy, sz, ni, nj, nk, dst, prim,
                                                                    gm1);
  return cudaGetLastError();
}

cudaError_t launch_init_dt(const DevBlock* blocks, int nblocks, const DevCase* cases, DevCaseState* st, int ncases,
                           unsigned long long* case_max, const int* mask, int role, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(case_max, 0, sizeof(unsigned long long) * ncases, s);
  if (e != cudaSuccess) return e;
  if (nblocks > 0) {
    dim3 g(64, nblocks);
    wavespeed_kernel<<<g, 256, 0, s>>>(blocks, cases, role, case_max);
  }
  init_dt_kernel<<<(ncases + 127) / 128, 128, 0, s>>>(cases, st, case_max, mask, ncases);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const DevBlock* blocks, const DevCase* cases, const int* case_blk, DevCaseState* st,
                            int ncases, const double* partials, int* counters, int ncounters, cudaStream_t s,
                            bool pdl) {
  LaunchCfg L(dim3(ncases), dim3(256), 0, s, pdl);
  return cudaLaunchKernelEx(&L.cfg, finalize_kernel, blocks, cases, case_blk, st, partials, counters, ncounters);
}

cudaError_t visc_occupancy(int prec, int* ctas_per_sm) {
  return prec == PREC_EXACT ? visc_occupancy_prec<PREC_EXACT>(ctas_per_sm) : visc_occupancy_fast(prec, ctas_per_sm);
}

// The non-exact forms' FP64 reciprocal and reciprocal square root over an
// array (a test hook: their error against the correctly rounded values).
__global__ void fast_math_probe_kernel(const double* x, int64_t n, double* r, double* rs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    r[i] = rcp_(x[i]);
    rs[i] = rsqrt_(x[i]);
  }
}

cudaError_t launch_fast_math_probe(const double* x, int64_t n, double* r, double* rs, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  fast_math_probe_kernel<<<grid_for(n, 256), 256, 0, s>>>(x, n, r, rs);
  return cudaGetLastError();
}

cudaError_t launch_visc(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int ntasks, int idim,
                        int prec, int role, cudaStream_t s, bool pdl) {
  if (prec == PREC_EXACT) return launch_visc_prec<PREC_EXACT>(blocks, cases, tasks, ntasks, idim, role, s, pdl);
  return launch_visc_fast(blocks, cases, tasks, ntasks, idim, prec, role, s, pdl);
}

}  // namespace fvm
