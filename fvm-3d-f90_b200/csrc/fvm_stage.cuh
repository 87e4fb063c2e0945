// fvm_stage.cuh — the fused Runge-Kutta stage kernel.
//
// One launch performs one RK stage over every tile of every block in a work
// list: the per-direction loops of ClassSpaceDiscret%inviscid_flux
// (class_space_discret.f90:120-176: reconstruct, flux, update_residual),
// TimeScheme%Runge_Kutta (scheme_Runge_Kutta.f90:30-63) and, on the last
// stage, the rhs^2 sums of ClassIteration%compute_residual and the wave-speed
// maximum the next CFL time step needs.
//
// A task is a TX x TY column tile of one block over a z range [z0, z1).
// The CTA marches the tile along z:
//   * the z stencil of each column lives in a register window (planes
//     k-1 .. k+H), refilled from the next plane each step;
//   * plane k with its x/y halo (H cells, no corners) sits in shared memory;
//     in 3D the next plane and the z window's next plane arrive as TMA
//     tensor boxes while the current plane is computed (the large FP64
//     tiles prefetch into registers instead);
//   * each face flux is computed once and kept in shared memory (x, y) or in
//     registers (z), and the cell's rhs is the reference's sum
//       rhs = ((0 - dFx/dx) - dFy/dy) - dFz/dz.
// CTAs pull tasks from an atomic counter (persistent work queue), so blocks
// of uneven size and independent cases share one launch.
//
// Halo cells outside a block are read with the region rule of the block:
// transmissive regions clamp the index to the boundary cell (the values
// update_ghost_cell_sub, defs_block_data.f90:226-256, copies there); connected
// and periodic regions read the ghost storage the gather kernel fills.
#pragma once
#include <cuda_pipeline.h>

#include <type_traits>

#include "fvm_schemes.cuh"
#include "fvm_types.h"

namespace fvm {

template <int RECON, int FLUX, int PREC, bool TB, int DIM, int TX, int TY>
struct StageCfg {
  using R = typename PrecT<PREC>::R;
  static constexpr bool EX = PrecT<PREC>::ex;
  static constexpr int H = RECON == RECON_WENO_ ? 3 : (RECON == RECON_MUSCL_ ? 2 : 1);
  static constexpr int NC = TX * TY;  // column threads: one z column (a cell of each plane) each
  // threads of the CTA: NC rounded up to one warp per scheduler; a tile
  // smaller than its launch leaves whole warps that take only x / y node and
  // face items
  static constexpr int NT = (NC + 127) / 128 * 128;
  static constexpr int PW = TX + 2 * H, PH = TY + 2 * H;
  // node values per x / y node item: WENO 5 (left-biased) or 10 (both
  // sides); MUSCL 10 (the cell's values at its right and left faces)
  // AUSM on per-node sides (ausm_side): the reference's WENO variant, whose
  // node value is the left state of one face and the right state of the
  // next, with AUSM in a non-exact form; a node then stores the seven values
  // of AusmSide instead of its five primitives
  static constexpr bool SP = RECON == RECON_WENO_ && !TB && FLUX == FLUX_AUSM_ && !EX;
  static constexpr int NODEV = RECON == RECON_WENO_ ? (TB ? 10 : (SP ? 7 : 5)) : (RECON == RECON_MUSCL_ ? 10 : 0);
  static constexpr int NXN = (TX + 2) * TY, NYN = TX * (TY + 2);
  static constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1);
  static constexpr int NW = 2 * H * (TX + TY);             // halo cells of a plane
  static constexpr int NPL = (DIM == 2 ? NC : 0) + NW;     // plane cells loaded from HBM
  static constexpr int NPS = (NPL + NT - 1) / NT;          // per-thread load slots
  static constexpr int WIN = H + 2;                        // z window: planes k-1 .. k+H
  static constexpr int WZ = RECON == RECON_SIMPLE_ ? 1 : 2;  // warm-up planes before z0
  // R arrays first, then the FP64 staging of the cell's q0 / q_in / acc
  // WENO and MUSCL read the plane only in phase A (their face states are
  // node values), so the face fluxes (phase B / C) share its storage; a
  // barrier then separates phase C from the refill
  static constexpr bool FAL = RECON != RECON_SIMPLE_;
  static constexpr size_t PF = FAL ? (5 * PH * PW > 5 * (NXF + NYF) ? 5 * PH * PW : 5 * (NXF + NYF))
                                   : 5 * PH * PW + 5 * (NXF + NYF);
  static constexpr size_t r_elems = (size_t)(PF + NODEV * (NXN + NYN));
  static constexpr size_t stage_off = (sizeof(R) * r_elems + 127) / 128 * 128;
  // The next plane's loads are prefetched asynchronously into shared memory
  // in the FP32 flux form and in small FP64 tiles; the large FP64 tiles,
  // whose shared arrays would then no longer fit twice on an SM, prefetch
  // into registers.
  static constexpr bool PSM = sizeof(R) == 4 || TX * TY <= 128;
  // FP64 arrays: [2][5][NC] RK operands (q0, then q_in or acc), [6][NT] the
  // column's residual sums and wave-speed maximum and, with PSM, the prefetch
  // of the next plane's loaded cells [5][NPL] and, in 3D, of the z window's
  // next plane [5][NC], both as loaded (conservative FP64)
  // In 3D the prefetch is two tensor-map (TMA) boxes per plane, issued by
  // one thread and completed on an mbarrier: the whole next plane with its
  // x / y halo, [5][PH][TW] with TW = TX + 2H + 1 rounded up to even (the
  // box starts on an even x, so its first coordinate is 16-byte aligned),
  // and the z window's next plane, [5][TY][TX]; both padded to 128 bytes.
  // These kernels also take the RK operands of plane k as [5][TY][TX] boxes
  // (the layout of the operand arrays), which keeps the per-thread copies
  // and their L1 lines out of the plane loop.
  static constexpr bool TMA = PSM && DIM == 3;
  // FP64 WENO tiles with tensor copies read their node stencils straight
  // from the plane's box (no copy into the plane array, one barrier less per
  // plane); the next plane's box is issued once the node phase is done
  static constexpr bool BOXA = TMA && RECON == RECON_WENO_ && sizeof(R) == 8;
  static constexpr int TW = (TX + 2 * H + 2) / 2 * 2;
  static constexpr int TPB = (5 * PH * TW + 15) / 16 * 16;
  static constexpr int TZB = (5 * TY * TX + 15) / 16 * 16;
  static constexpr int NPRE = TMA ? TPB + TZB : (PSM ? 5 * NPL + (DIM == 3 ? 5 * NC : 0) : 0);
  static constexpr size_t smem_bytes = stage_off + sizeof(double) * (2 * 5 * NC + 6 * NT + NPRE);
};

// ---------------------------------------------------------------- helpers
struct BGeo {
  int n0, n1, n2, sy, sz, mask;
};

__device__ __forceinline__ int64_t cell_off(const BGeo& g, int x, int y, int z) {
  x = max(x, -kGhost);
  x = min(x, g.n0 + kGhost - 1);
  y = max(y, -kGhost);
  y = min(y, g.n1 + kGhost - 1);
  z = max(z, -kGhost);
  z = min(z, g.n2 + kGhost - 1);
  if (x < 0 && !(g.mask & 1)) x = 0;
  if (x >= g.n0 && !(g.mask & 2)) x = g.n0 - 1;
  if (y < 0 && !(g.mask & 4)) y = 0;
  if (y >= g.n1 && !(g.mask & 8)) y = g.n1 - 1;
  if (z < 0 && !(g.mask & 16)) z = 0;
  if (z >= g.n2 && !(g.mask & 32)) z = g.n2 - 1;
  return (int64_t)x + (int64_t)y * g.sy + (int64_t)z * g.sz;
}

// The same rule split into its (x, y) part and its z part, so the loads of
// a z-marching tile clamp x and y once per task.
__device__ __forceinline__ int xy_off(const BGeo& g, int x, int y) {
  x = max(x, -kGhost);
  x = min(x, g.n0 + kGhost - 1);
  y = max(y, -kGhost);
  y = min(y, g.n1 + kGhost - 1);
  if (x < 0 && !(g.mask & 1)) x = 0;
  if (x >= g.n0 && !(g.mask & 2)) x = g.n0 - 1;
  if (y < 0 && !(g.mask & 4)) y = 0;
  if (y >= g.n1 && !(g.mask & 8)) y = g.n1 - 1;
  return x + y * g.sy;
}
// The same rule returning the clamped (x, y).
__device__ __forceinline__ void xy_clamp(const BGeo& g, int& x, int& y) {
  x = max(x, -kGhost);
  x = min(x, g.n0 + kGhost - 1);
  y = max(y, -kGhost);
  y = min(y, g.n1 + kGhost - 1);
  if (x < 0 && !(g.mask & 1)) x = 0;
  if (x >= g.n0 && !(g.mask & 2)) x = g.n0 - 1;
  if (y < 0 && !(g.mask & 4)) y = 0;
  if (y >= g.n1 && !(g.mask & 8)) y = g.n1 - 1;
}

// ---- tensor-map copies and mbarriers (sm_90+ PTX; no cluster multicast)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the phase `parity` of b to complete; gives up one second after
// *issued (the globaltimer stamp the issuing thread took when it issued the
// copies of this plane, read only when the phase is not complete at once)
// and returns false. With one deadline for the whole CTA, every thread takes
// the same decision: a copy that lands before the deadline is seen by every
// waiting thread, and one that has not landed by then fails every thread
// still waiting (a thread could only differ by starting its wait after the
// copy landed, more than a second after the issue, while the CTA's threads
// meet at a barrier in every phase).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, const volatile uint64_t* issued) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t deadline = *issued + 1000000000ull;
  for (int i = 0; i < (1 << 26); ++i) {
    if (mbar_try_wait(b, parity)) return true;
    if (global_ns() > deadline) return false;
  }
  return false;
}
// Leaving the stage after a tensor copy timed out (every thread of the CTA,
// each after its own failed wait, which the common deadline makes the same
// decision): thread 0 reports it and then waits 200 ms more before it exits,
// so that any copy of this plane still in flight has landed (or will never
// land) before the CTA's shared memory is released. Out of line: the error
// path stays out of the plane loop's code.
static __device__ __noinline__ void leave_after_timeout(int tid, int32_t* err) {
  if (tid != 0) return;
  atomicExch(err, 1);
  const uint64_t t0 = global_ns();
  for (int i = 0; i < (1 << 26) && global_ns() - t0 < 200000000ull; ++i) __nanosleep(1000);
}
// 4D tiled tensor copy global -> this CTA's shared memory, completing on b.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(b))
      : "memory");
}

__device__ __forceinline__ int z_clamp(const BGeo& g, int z) {
  z = max(z, -kGhost);
  z = min(z, g.n2 + kGhost - 1);
  if (z < 0 && !(g.mask & 16)) z = 0;
  if (z >= g.n2 && !(g.mask & 32)) z = g.n2 - 1;
  return z;
}

__device__ __forceinline__ void ld5(const double* __restrict__ base, int64_t off, int64_t vs, double q[5]) {
#pragma unroll
  for (int v = 0; v < 5; ++v) q[v] = __ldg(base + off + v * vs);
}
__device__ __forceinline__ void cpy8(double* dst_smem, const double* src) {
  __pipeline_memcpy_async(dst_smem, src, sizeof(double));
}

// Stencil value stored for reconstruction: conservative for WENO (the
// reference reconstructs q, scheme_WENO.f90:28-72), primitive otherwise
// (MUSCL / simple reconstruct p, scheme_reconstruct_MUSCL.f90:47-104).
template <int RECON, class R, bool EX>
__device__ __forceinline__ void to_stencil(const double q[5], R s[5], double gm1d, R gm1) {
  if constexpr (RECON == RECON_WENO_) {
#pragma unroll
    for (int v = 0; v < 5; ++v) s[v] = (R)q[v];
  } else {
    if constexpr (sizeof(R) == 8) {
      Prim5<double> p = cons2prim<double, EX>(q[0], q[1], q[2], q[3], q[4], gm1d);
      s[0] = p.r; s[1] = p.u; s[2] = p.v; s[3] = p.w; s[4] = p.p;
    } else {
      Prim5<R> p = cons2prim<R, false>((R)q[0], (R)q[1], (R)q[2], (R)q[3], (R)q[4], gm1);
      s[0] = p.r; s[1] = p.u; s[2] = p.v; s[3] = p.w; s[4] = p.p;
    }
  }
}

// TEXTBOOK compat only: a reconstructed face state with non-positive density
// or pressure is replaced by the first-order state (the cell's own value).
template <class R> __device__ __forceinline__ bool admissible(const Prim5<R>& p) {
  return p.r > R(0) && p.p > R(0);
}

template <class R> __device__ __forceinline__ Prim5<R> mkprim(const R s[5]) {
  Prim5<R> p;
  p.r = s[0]; p.u = s[1]; p.v = s[2]; p.w = s[3]; p.p = s[4];
  return p;
}

// Wave-speed sum of one cell, sum_d (|u_d| + c) / dr_d, from conservative
// values, exact FP64 (the CFL time step of the host runtime).
// EX: divisions and the IEEE square root; the other forms the reciprocal,
// reciprocal square root and reciprocal cell sizes (idr).
template <bool EX>
__device__ __forceinline__ double wavespeed(const double q[5], double gamma, double gm1, const double dr[3],
                                            const double idr[3], int idim) {
  Prim5<double> p = cons2prim<double, EX>(q[0], q[1], q[2], q[3], q[4], gm1);
  if constexpr (EX) {
    const double c = sqrt(gamma * p.p / p.r);
    double s = (fabs(p.u) + c) / dr[0] + (fabs(p.v) + c) / dr[1];
    if (idim == 3) s = s + (fabs(p.w) + c) / dr[2];
    return s;
  } else {
    const double c = nsqrt_(gamma * p.p * rcp_(p.r));
    double s = (fabs(p.u) + c) * idr[0] + (fabs(p.v) + c) * idr[1];
    if (idim == 3) s = s + (fabs(p.w) + c) * idr[2];
    return s;
  }
}

// Deterministic CTA reduction of the column accumulators sS[6][NT] (5 sums,
// 1 max) into partials[slot].
template <int NT>
__device__ __forceinline__ void cta_reduce_store(const double* sS, double* red, double* dst) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NWARP = NT / 32;
  double ss[5], wm = sS[5 * NT + threadIdx.x];
#pragma unroll
  for (int v = 0; v < 5; ++v) ss[v] = sS[v * NT + threadIdx.x];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int v = 0; v < 5; ++v) ss[v] += __shfl_xor_sync(0xffffffffu, ss[v], o);
    wm = fmax(wm, __shfl_xor_sync(0xffffffffu, wm, o));
  }
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < 5; ++v) red[v * NWARP + warp] = ss[v];
    red[5 * NWARP + warp] = wm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[5] = {0, 0, 0, 0, 0}, m = 0.0;
    for (int w = 0; w < NWARP; ++w) {
#pragma unroll
      for (int v = 0; v < 5; ++v) t[v] += red[v * NWARP + w];
      m = fmax(m, red[5 * NWARP + w]);
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) dst[v] = t[v];
    dst[5] = m;
  }
  __syncthreads();
}

// Map a plane-load index w to shared-memory plane coordinates (xx, yy).
template <int TX, int TY, int H, int DIM>
__device__ __forceinline__ void plane_cell(int w, int& xx, int& yy) {
  if (DIM == 2) {
    if (w < TX * TY) {
      xx = H + w % TX;
      yy = H + w / TX;
      return;
    }
    w -= TX * TY;
  }
  if (w < 2 * H * TY) {
    const int side = w / (H * TY), r = w % (H * TY);
    xx = (side ? H + TX : 0) + r % H;
    yy = H + r / H;
  } else {
    w -= 2 * H * TY;
    const int side = w / (H * TX), r = w % (H * TX);
    xx = H + r % TX;
    yy = (side ? H + TY : 0) + r / TX;
  }
}

// ---------------------------------------------------------------- kernel
// One RK stage over the work list of `a`: the CTA takes tasks from the queue
// until it is empty (or, with tensor copies, until a copy times out).
template <int RECON, int FLUX, int PREC, bool TB, int DIM, int TX, int TY>
__device__ __forceinline__ void stage_run(const StageArgs& a) {
  using C = StageCfg<RECON, FLUX, PREC, TB, DIM, TX, TY>;
  using R = typename C::R;
  constexpr bool EX = C::EX;
  constexpr int H = C::H, NT = C::NT, NC = C::NC, PW = C::PW, PH = C::PH;
  constexpr int PLANE = PH * PW;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* sP = reinterpret_cast<R*>(smem_raw);   // [5][PH][PW]   plane k + halo
  R* sN = sP + (C::FAL ? C::PF : 5 * PLANE);  // [NODEV][NXN+NYN] x/y WENO nodes
  R* sF = C::FAL ? sP : sN + C::NODEV * (C::NXN + C::NYN);  // [5][NXF+NYF]  x/y face fluxes
  double* sQ = reinterpret_cast<double*>(smem_raw + C::stage_off);  // [2][5][NC] q0, q_in | acc
  double* sS = sQ + 2 * 5 * NC;                                       // [6][NT] residual / wave speed
  double* sX = sS + 6 * NT;                                           // [5][NPL] next plane's loads
  double* sZ = sX + 5 * C::NPL;                                       // [5][NC] z window's next plane (3D)
  double* sTP = sS + 6 * NT;                                          // TMA: [5][PH][TW] next plane
  double* sTZ = sTP + C::TPB;                                         // TMA: [5][TY][TX] z window's next plane
  __shared__ double s_red[6 * (NT / 32)];
  __shared__ int s_task;
  __shared__ __align__(8) uint64_t s_mbar[3];  // TMA: plane box, z box, RK operands
  __shared__ uint64_t s_issued;                  // TMA: globaltimer when this plane's copies were issued
  __shared__ uint64_t s_issp;                    // BOXA: globaltimer when the plane box was issued
  uint32_t ph_p = 0, ph_z = 0, ph_q = 0;       // TMA: expected phase parity of each mbarrier

  const int tid = threadIdx.x;
  // column threads own a z column; the others (whole warps) skip all z work
  const bool colt = (NC == NT) || tid < NC;
  const int tx = tid % TX, ty = tid / TX;
  if constexpr (C::TMA) {
    if (tid == 0) {
      mbar_init(&s_mbar[0], 1);
      mbar_init(&s_mbar[1], 1);
      mbar_init(&s_mbar[2], 1);
      mbar_fence_init();
    }
    __syncthreads();
  }
  // no early pdl_trigger here: the gather launched behind this kernel would
  // place its CTAs on the first SMs to free up and run unbalanced
  pdl_wait();

  for (;;) {
    if (tid == 0) s_task = atomicAdd(a.counter, 1);
    __syncthreads();
    const int ti = s_task;
    __syncthreads();
    if (ti >= a.ntasks) break;

    const Task T = a.tasks[ti];
    const DevBlock& B = a.blocks[T.blk];
    const DevCase& CS = a.cases[B.case_id];
    const double dtg = a.cstate[B.case_id].dt;
    const double* __restrict__ qin = B.q[a.rin];
    double* qout = B.q[a.rout];
    const double* q0p = B.q[a.rq0];
    double* accp = B.q[a.racc];
    const int64_t vs = B.vs;
    const double gm1d = CS.gm1;

    SchemeConst<R> K;
    K.gamma = (R)CS.gamma;
    K.gm1 = (R)CS.gm1;
    K.goverg1 = (R)(CS.gamma / CS.gm1);
    K.two_g2m1 = (R)(2.0 * (CS.gamma * CS.gamma - 1.0));
    K.fix = (R)CS.entropy_fix;
    K.kappa = (R)CS.kappa;
    K.omk = (R)(1.0 - CS.kappa);
    K.opk = (R)(1.0 + CS.kappa);
    K.limiter = CS.limiter;
    K.textbook = CS.compat;
    BGeo G;
    G.n0 = B.n[0]; G.n1 = B.n[1]; G.n2 = B.n[2];
    G.sy = B.sy; G.sz = B.sz; G.mask = B.ghost_mask;
    const double dr0 = B.dr[0], dr1 = B.dr[1], dr2 = B.dr[2];
    const double idr0 = B.inv_dr[0], idr1 = B.inv_dr[1], idr2 = B.inv_dr[2];
    const double drv[3] = {dr0, dr1, dr2};
    const double idrv[3] = {idr0, idr1, idr2};
    const int rk_stages = CS.rk_stages, ts_set = CS.timestep_set, idim = CS.idim;
    const double cfl = CS.cfl, gammad = CS.gamma;
    const double* visc = B.visc;
    double* rhs_out = a.last ? B.rhs : nullptr;
    const bool need_um = (rk_stages == 3 && a.m >= 2);
    const bool need_acc = (rk_stages == 4 && a.m >= 2);
    // RK4 folds q0 into its accumulator, so stage 4 reads no q0 (local time
    // steps still need it: the cell's dt comes from its q0)
    const bool need_u0 = !(rk_stages == 4 && a.m == 4) || ts_set == 2;

    const int nxt = min(TX, G.n0 - T.x0), nyt = min(TY, G.n1 - T.y0);
    const bool act = colt && tx < nxt && ty < nyt;
    const int gx = T.x0 + tx, gy = T.y0 + ty;

    if (a.last)
#pragma unroll
      for (int v = 0; v < 6; ++v) sS[v * NT + tid] = 0.0;

    // loop-invariant (x, y) parts of this thread's plane loads: the global
    // offset, or with TMA the index of the (clamped) cell in the plane box
    int lxy[C::NPS], lsp[C::NPS];
    // TMA: the plane box starts at padded x = xs (even), padded y = T.y0 + kGhost - H
    const int xs = (T.x0 + kPadX - H) & ~1;
#pragma unroll
    for (int sidx = 0; sidx < C::NPS; ++sidx) {
      const int w = tid + sidx * NT;
      lsp[sidx] = -1;
      lxy[sidx] = 0;
      if (w < C::NPL) {
        int xx, yy;
        plane_cell<TX, TY, H, DIM>(w, xx, yy);
        lsp[sidx] = yy * PW + xx;
        if constexpr (C::TMA) {
          int x = T.x0 + xx - H, y = T.y0 + yy - H;
          xy_clamp(G, x, y);
          lxy[sidx] = (y - T.y0 + H) * C::TW + (x + kPadX - xs);
        } else {
          lxy[sidx] = xy_off(G, T.x0 + xx - H, T.y0 + yy - H);
        }
      }
    }
    const int cxy = xy_off(G, gx, gy);
    // TMA: index of this column's (clamped) cell in the z box
    int zsrc = 0;
    if constexpr (C::TMA) {
      int x = gx, y = gy;
      xy_clamp(G, x, y);
      zsrc = (y - T.y0) * TX + (x - T.x0);
    }
    // BOXA: plane cell (xx, yy) is box element yy * TW + xx + xoff. The box
    // holds ghost storage where the clamped rule gives other values (halo
    // cells of transmissive faces) and, past a partial tile's block edge,
    // where the z window holds the clamped values: such a task fixes those
    // cells up in the box after each plane lands.
    const int xoff = (T.x0 + kPadX - H) - xs;
    bool fixt = false;
    if constexpr (C::BOXA)
      fixt = (!(G.mask & 1) && T.x0 < H) || (!(G.mask & 2) && T.x0 + nxt + H > G.n0) ||
             (!(G.mask & 4) && T.y0 < H) || (!(G.mask & 8) && T.y0 + nyt + H > G.n1) || nxt < TX || nyt < TY;
    // tensor maps of this block: [role][plane box, z-shaped box]
    const CUtensorMap* tmb = nullptr;
    const CUtensorMap* tmp = nullptr;
    if constexpr (C::TMA) {
      tmb = a.tmap + (int64_t)T.blk * NROLE * 2;
      tmp = tmb + a.rin * 2;
    }

    // ---- z window (3D) --------------------------------------------------
    R zw[C::WIN][5];
    // a node's face state: primitives, or with SP the AUSM side values
    using NodeT = std::conditional_t<C::SP, AusmSide<R>, Prim5<R>>;
    NodeT zWprev;          // WENO: node value of plane k (ref: left-biased; TB: minus side)
    R zFprev[5] = {0, 0, 0, 0, 0};
    const int kstart = (DIM == 3) ? T.z0 - C::WZ : T.z0;
    if constexpr (DIM == 3) {
      if (colt)
#pragma unroll
      for (int s = 0; s < C::WIN; ++s) {
        double q[5];
        ld5(qin, (int64_t)cxy + (int64_t)z_clamp(G, kstart - 1 + s) * G.sz, vs, q);
        to_stencil<RECON, R, EX>(q, zw[s], gm1d, K.gm1);
      }
    } else {
      // 2D: plane z0 into shared memory up front
#pragma unroll
      for (int sidx = 0; sidx < C::NPS; ++sidx) {
        if (lsp[sidx] >= 0) {
          double q[5];
          R s[5];
          ld5(qin, (int64_t)lxy[sidx] + (int64_t)T.z0 * G.sz, vs, q);
          to_stencil<RECON, R, EX>(q, s, gm1d, K.gm1);
#pragma unroll
          for (int v = 0; v < 5; ++v) sP[v * PLANE + lsp[sidx]] = s[v];
        }
      }
      __syncthreads();
    }

    for (int k = kstart; k < T.z1; ++k) {
      const bool do_xy = (k >= T.z0);
      const bool more = (k + 1 < T.z1);
      const bool more_xy = more && (k + 1 >= T.z0);  // plane k+1 lies in [z0, z1)

      // ---- prefetch the next plane's loaded cells (and the z window's next
      // plane): into shared memory with PSM (each thread later reads only its
      // own copies), else into registers.
      double pre[C::PSM ? 1 : C::NPS][5];
      double zpre[5];
      if constexpr (C::TMA) {
        if (tid == 0) {
          s_issued = global_ns();  // the deadline of this plane's waits is one second later
          // (BOXA: a node plane's box for plane k+1 is issued after its node phase)
          if (more_xy && !(C::BOXA && do_xy)) {
            if constexpr (C::BOXA) s_issp = s_issued;
            mbar_expect_tx(&s_mbar[0], sizeof(double) * 5 * PH * C::TW);
            // a.drop_copies (a test of the timeout path): the barrier is armed
            // but the copy never issued, so the wait below runs out
            if (!a.drop_copies) tma_load_4d(sTP, tmp, xs, T.y0 + kGhost - H, k + 1 + kGhost, 0, &s_mbar[0]);
          }
          if (more) {
            mbar_expect_tx(&s_mbar[1], sizeof(double) * 5 * TY * TX);
            tma_load_4d(sTZ, tmp + 1, T.x0 + kPadX, T.y0 + kGhost, z_clamp(G, k + H + 1) + kGhost, 0, &s_mbar[1]);
          }
        }
      } else if (more_xy) {
#pragma unroll
        for (int sidx = 0; sidx < C::NPS; ++sidx) {
          if (lsp[sidx] >= 0) {
            const double* src = qin + (int64_t)lxy[sidx] + (int64_t)(k + 1) * G.sz;
            if constexpr (C::PSM) {
              const int w = tid + sidx * NT;
#pragma unroll
              for (int v = 0; v < 5; ++v) cpy8(sX + v * C::NPL + w, src + v * vs);
            } else {
              ld5(src, 0, vs, pre[sidx]);
            }
          }
        }
      }
      if constexpr (DIM == 3 && !C::TMA) {
        if (more && colt) {
          const double* src = qin + (int64_t)cxy + (int64_t)z_clamp(G, k + H + 1) * G.sz;
          if constexpr (C::PSM) {
#pragma unroll
            for (int v = 0; v < 5; ++v) cpy8(sZ + v * NC + tid, src + v * vs);
          } else {
            ld5(src, 0, vs, zpre);
          }
        }
      }
      if constexpr (C::PSM && !C::TMA) __pipeline_commit();

      // ---- the cell's RK operands of plane k, copied asynchronously into
      // shared memory (TMA boxes, or per-thread copies of which phase C
      // waits for this thread's own only)
      const int64_t off_k = (int64_t)gx + (int64_t)gy * G.sy + (int64_t)k * G.sz;
      if constexpr (C::TMA) {
        // TMA kernels: the operands of the whole tile as [5][TY][TX] boxes of
        // plane k (the layout of sQ), straight into shared memory
        if (do_xy && tid == 0) {
          const int nb = (need_u0 ? 1 : 0) + ((need_um || need_acc) ? 1 : 0);
          mbar_expect_tx(&s_mbar[2], sizeof(double) * 5 * TY * TX * nb);
          const int bx = T.x0 + kPadX, by = T.y0 + kGhost, bz = k + kGhost;
          if (need_u0) tma_load_4d(sQ, tmb + a.rq0 * 2 + 1, bx, by, bz, 0, &s_mbar[2]);
          if (need_um) tma_load_4d(sQ + 5 * NC, tmb + a.rin * 2 + 1, bx, by, bz, 0, &s_mbar[2]);
          if (need_acc) tma_load_4d(sQ + 5 * NC, tmb + a.racc * 2 + 1, bx, by, bz, 0, &s_mbar[2]);
        }
      } else if (do_xy && act) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          if (need_u0) cpy8(sQ + (0 * 5 + v) * NC + tid, q0p + off_k + v * vs);
          if (need_um) cpy8(sQ + (1 * 5 + v) * NC + tid, qin + off_k + v * vs);
          if (need_acc) cpy8(sQ + (1 * 5 + v) * NC + tid, accp + off_k + v * vs);
        }
        __pipeline_commit();
      }

      // ---- phase A: WENO nodes --------------------------------------------
      NodeT zWcur, zWm_cur;
      constexpr int NNODE = C::NXN + C::NYN;
      // SP: the side values of x / y node w from its primitives and 1 / rho
      auto store_side = [&](int w, const Prim5<R>& pm, R ir, R E) {
        const AusmSide<R> sd = ausm_side<R>(pm, ir, E, w < C::NXN ? pm.u : pm.v, K);
        sN[0 * NNODE + w] = sd.u;
        sN[1 * NNODE + w] = sd.v;
        sN[2 * NNODE + w] = sd.w;
        sN[3 * NNODE + w] = sd.p;
        sN[4 * NNODE + w] = sd.H;
        sN[5 * NNODE + w] = sd.M;
        sN[6 * NNODE + w] = sd.rc;
      };
      if constexpr (RECON == RECON_WENO_) {
        if constexpr (sizeof(R) == 4 && !TB) {
          // FP32, left-biased nodes only. A node's five variables fill two and
          // a half f32x2 pairs, so nodes are taken in twos and their fifth
          // variables share a pair: the thread's first two x / y nodes, and
          // its third one with the z node of its column (or each alone).
          constexpr int NN = C::NXN + C::NYN;
          static_assert(NN >= NT && NN <= 3 * NT, "x/y node items per thread");
          auto load_node = [&](int w, R (&u)[5][5]) {
            if (w < C::NXN) {
              const int c = w % (TX + 2) - 1, row = w / (TX + 2);
              const int base = (H + row) * PW + (H + c - 2);
#pragma unroll
              for (int v = 0; v < 5; ++v)
#pragma unroll
                for (int s = 0; s < 5; ++s) u[v][s] = sP[v * PLANE + base + s];
            } else {
              const int w2 = w - C::NXN;
              const int col = w2 % TX, c = w2 / TX - 1;
              const int base = (H + c - 2) * PW + (H + col);
#pragma unroll
              for (int v = 0; v < 5; ++v)
#pragma unroll
                for (int s = 0; s < 5; ++s) u[v][s] = sP[v * PLANE + base + s * PW];
            }
          };
          auto pair = [&](const R (&x)[5], const R (&y)[5]) {
            return weno5x2(make_float2(x[0], y[0]), make_float2(x[1], y[1]), make_float2(x[2], y[2]),
                           make_float2(x[3], y[3]), make_float2(x[4], y[4]), K.textbook);
          };
          auto first4 = [&](const R (&u)[5][5], R (&wm)[5]) {
            const float2 r01 = pair(u[0], u[1]), r23 = pair(u[2], u[3]);
            wm[0] = r01.x;
            wm[1] = r01.y;
            wm[2] = r23.x;
            wm[3] = r23.y;
          };
          auto finish = [&](int w, const R (&u)[5][5], const R (&wm)[5]) {
            if constexpr (C::SP) {
              R ir;
              const Prim5<R> pm = cons2prim_ir<R>(wm[0], wm[1], wm[2], wm[3], wm[4], K.gm1, ir);
              store_side(w, pm, ir, wm[4]);
              return;
            }
            Prim5<R> pm = cons2prim<R, EX>(wm[0], wm[1], wm[2], wm[3], wm[4], K.gm1);
            if (K.textbook && !admissible(pm))
              pm = cons2prim<R, EX>(u[0][2], u[1][2], u[2][2], u[3][2], u[4][2], K.gm1);
            sN[0 * NN + w] = pm.r;
            sN[1 * NN + w] = pm.u;
            sN[2 * NN + w] = pm.v;
            sN[3 * NN + w] = pm.w;
            sN[4 * NN + w] = pm.p;
          };
          // z node of plane k+1 from planes k-1 .. k+3 (window slots 0..4)
          const bool hz = DIM == 3 && colt;
          R uz4[5], wz[5];
          bool zpaired = false;
          if (hz) {
            R uz[5][5];
#pragma unroll
            for (int v = 0; v < 5; ++v)
#pragma unroll
              for (int s = 0; s < 5; ++s) uz[v][s] = zw[s][v];
            first4(uz, wz);
#pragma unroll
            for (int s = 0; s < 5; ++s) uz4[s] = uz[4][s];
          }
          if (do_xy) {
            const int wa = tid, wb = tid + NT, wc = tid + 2 * NT;
            {
              R ua[5][5], va[5];
              load_node(wa, ua);
              first4(ua, va);
              if (wb < NN) {
                R ub[5][5], vb[5];
                load_node(wb, ub);
                first4(ub, vb);
                const float2 r4 = pair(ua[4], ub[4]);
                va[4] = r4.x;
                vb[4] = r4.y;
                finish(wa, ua, va);
                finish(wb, ub, vb);
              } else {
                va[4] = pair(ua[4], ua[4]).x;
                finish(wa, ua, va);
              }
            }
            if (wc < NN) {
              R uc[5][5], vc[5];
              load_node(wc, uc);
              first4(uc, vc);
              if (hz) {
                const float2 r4 = pair(uz4, uc[4]);
                wz[4] = r4.x;
                vc[4] = r4.y;
                zpaired = true;
              } else {
                vc[4] = pair(uc[4], uc[4]).x;
              }
              finish(wc, uc, vc);
            }
          }
          if (hz) {
            if (!zpaired) wz[4] = pair(uz4, uz4).x;
            if constexpr (C::SP) {
              R ir;
              const Prim5<R> pz = cons2prim_ir<R>(wz[0], wz[1], wz[2], wz[3], wz[4], K.gm1, ir);
              zWm_cur = ausm_side<R>(pz, ir, wz[4], pz.w, K);
              zWcur = zWm_cur;
            } else {
              zWm_cur = cons2prim<R, EX>(wz[0], wz[1], wz[2], wz[3], wz[4], K.gm1);
              zWcur = zWm_cur;
              if (K.textbook && !admissible(zWm_cur)) {
                zWm_cur = cons2prim<R, EX>(zw[2][0], zw[2][1], zw[2][2], zw[2][3], zw[2][4], K.gm1);
                zWcur = zWm_cur;
              }
            }
          }
          if (do_xy) __syncthreads();
        } else {
        if (DIM == 3 && colt) {
          // node of plane k+1 from planes k-1 .. k+3 (window slots 0..4)
          R wm[5], wp[5], u[5][5];
#pragma unroll
          for (int v = 0; v < 5; ++v)
#pragma unroll
            for (int s = 0; s < 5; ++s) u[v][s] = zw[s][v];
          weno5_node<R, EX, TB>(u, K.textbook, wm, wp);
          if constexpr (C::SP) {
            R ir;
            const Prim5<R> pz = cons2prim_ir<R>(wm[0], wm[1], wm[2], wm[3], wm[4], K.gm1, ir);
            zWm_cur = ausm_side<R>(pz, ir, wm[4], pz.w, K);
            zWcur = zWm_cur;
          } else {
          zWm_cur = cons2prim<R, EX>(wm[0], wm[1], wm[2], wm[3], wm[4], K.gm1);
          if (TB)
            zWcur = cons2prim<R, EX>(wp[0], wp[1], wp[2], wp[3], wp[4], K.gm1);
          else
            zWcur = zWm_cur;
          if (K.textbook && !(admissible(zWm_cur) && admissible(zWcur))) {
            const Prim5<R> pc = cons2prim<R, EX>(zw[2][0], zw[2][1], zw[2][2], zw[2][3], zw[2][4], K.gm1);
            if (!admissible(zWm_cur)) zWm_cur = pc;
            if (!admissible(zWcur)) zWcur = pc;
          }
          }
        }
        if constexpr (C::BOXA) {
          if (do_xy) {
            // the plane's box (issued after the last plane's node phase)
            if (!mbar_wait(&s_mbar[0], ph_p, &s_issp)) {
              leave_after_timeout(tid, a.err);
              return;
            }
            ph_p ^= 1;
            if (fixt) {
#pragma unroll
              for (int sidx = 0; sidx < C::NPS; ++sidx) {
                if (lsp[sidx] >= 0) {
                  const int nat = (lsp[sidx] / PW) * C::TW + lsp[sidx] % PW + xoff;
                  if (nat != lxy[sidx])
#pragma unroll
                    for (int v = 0; v < 5; ++v) sTP[v * (PH * C::TW) + nat] = sTP[v * (PH * C::TW) + lxy[sidx]];
                }
              }
              if (colt && (tx >= nxt || ty >= nyt))
#pragma unroll
                for (int v = 0; v < 5; ++v) sTP[v * (PH * C::TW) + (H + ty) * C::TW + H + tx + xoff] = zw[1][v];
              __syncthreads();
            }
          }
        }
        if (do_xy) {
          // node stencils from the plane array, or with BOXA from the box
          const R* pl = sP;
          if constexpr (C::BOXA) pl = reinterpret_cast<const R*>(sTP) + xoff;
          constexpr int PLS = C::BOXA ? PH * C::TW : PLANE, PWS = C::BOXA ? C::TW : PW;
          for (int w = tid; w < C::NXN + C::NYN; w += NT) {
            R u[5][5];
            if (w < C::NXN) {
              const int c = w % (TX + 2) - 1, row = w / (TX + 2);
              const int base = (H + row) * PWS + (H + c - 2);
#pragma unroll
              for (int v = 0; v < 5; ++v)
#pragma unroll
                for (int s = 0; s < 5; ++s) u[v][s] = pl[v * PLS + base + s];
            } else {
              const int w2 = w - C::NXN;
              const int col = w2 % TX, c = w2 / TX - 1;
              const int base = (H + c - 2) * PWS + (H + col);
#pragma unroll
              for (int v = 0; v < 5; ++v)
#pragma unroll
                for (int s = 0; s < 5; ++s) u[v][s] = pl[v * PLS + base + s * PWS];
            }
            R wm[5], wp[5];
            weno5_node<R, EX, TB>(u, K.textbook, wm, wp);
            if constexpr (C::SP) {
              R ir;
              const Prim5<R> pm = cons2prim_ir<R>(wm[0], wm[1], wm[2], wm[3], wm[4], K.gm1, ir);
              store_side(w, pm, ir, wm[4]);
              continue;
            }
            Prim5<R> pm = cons2prim<R, EX>(wm[0], wm[1], wm[2], wm[3], wm[4], K.gm1);
            if (K.textbook && !admissible(pm))
              pm = cons2prim<R, EX>(u[0][2], u[1][2], u[2][2], u[3][2], u[4][2], K.gm1);
            constexpr int NN = C::NXN + C::NYN;
            sN[0 * NN + w] = pm.r;
            sN[1 * NN + w] = pm.u;
            sN[2 * NN + w] = pm.v;
            sN[3 * NN + w] = pm.w;
            sN[4 * NN + w] = pm.p;
            if (TB) {
              Prim5<R> pp = cons2prim<R, EX>(wp[0], wp[1], wp[2], wp[3], wp[4], K.gm1);
              if (!admissible(pp)) pp = cons2prim<R, EX>(u[0][2], u[1][2], u[2][2], u[3][2], u[4][2], K.gm1);
              sN[5 * NN + w] = pp.r;
              sN[6 * NN + w] = pp.u;
              sN[7 * NN + w] = pp.v;
              sN[8 * NN + w] = pp.w;
              sN[9 * NN + w] = pp.p;
            }
          }
          __syncthreads();
          if constexpr (C::BOXA) {
            // the box is free: the next plane's copy goes out now and lands
            // while the fluxes and the update of this plane run
            if (tid == 0 && more_xy) {
              s_issp = global_ns();
              mbar_expect_tx(&s_mbar[0], sizeof(double) * 5 * PH * C::TW);
              if (!a.drop_copies) tma_load_4d(sTP, tmp, xs, T.y0 + kGhost - H, k + 1 + kGhost, 0, &s_mbar[0]);
            }
          }
        }
        }
      }

      if constexpr (RECON == RECON_MUSCL_) {
        // MUSCL node of a cell: its values at its right face (qR, the left
        // state of that face) and at its left face (qL), one limited slope
        // pair per cell (scheme_reconstruct_MUSCL.f90:114-226); TEXTBOOK
        // falls back to the cell value where a state is not admissible
        auto node = [&](const R (&p)[5][3], R (&qr)[5], R (&ql)[5]) {
#pragma unroll
          for (int v = 0; v < 5; ++v) {
            R Dbm, Dbp;
            muscl_slopes<R, EX>(p[v][0], p[v][1], p[v][2], K.limiter, Dbm, Dbp);
            qr[v] = p[v][1] + R(0.25) * (K.omk * Dbm + K.opk * Dbp);
            ql[v] = p[v][1] - R(0.25) * (K.omk * Dbp + K.opk * Dbm);
          }
          if (K.textbook) {
            if (!admissible(mkprim(qr)))
#pragma unroll
              for (int v = 0; v < 5; ++v) qr[v] = p[v][1];
            if (!admissible(mkprim(ql)))
#pragma unroll
              for (int v = 0; v < 5; ++v) ql[v] = p[v][1];
          }
        };
        if (DIM == 3 && colt) {
          // node of plane k+1 from planes k .. k+2 (window slots 1..3)
          R p[5][3], qr[5], ql[5];
#pragma unroll
          for (int v = 0; v < 5; ++v)
#pragma unroll
            for (int s = 0; s < 3; ++s) p[v][s] = zw[s + 1][v];
          node(p, qr, ql);
          zWm_cur = mkprim(qr);  // left state of face k+3/2, carried
          zWcur = mkprim(ql);    // right state of face k+1/2
        }
        if (do_xy) {
          constexpr int NN = C::NXN + C::NYN;
          // x node c (-1..TX) of tile row `row`, y node c (-1..TY) of tile
          // column `col`: stencil and node-array index
          auto xnode = [&](int c, int row, R (&p)[5][3]) {
            const int base = (H + row) * PW + (H + c);
#pragma unroll
            for (int v = 0; v < 5; ++v)
#pragma unroll
              for (int s = 0; s < 3; ++s) p[v][s] = sP[v * PLANE + base + s - 1];
            return row * (TX + 2) + c + 1;
          };
          auto ynode = [&](int c, int col, R (&p)[5][3]) {
            const int base = (H + c) * PW + (H + col);
#pragma unroll
            for (int v = 0; v < 5; ++v)
#pragma unroll
              for (int s = 0; s < 3; ++s) p[v][s] = sP[v * PLANE + base + (s - 1) * PW];
            return C::NXN + (c + 1) * TX + col;
          };
          auto put = [&](int w, const R (&qr)[5], const R (&ql)[5]) {
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              sN[v * NN + w] = qr[v];
              sN[(5 + v) * NN + w] = ql[v];
            }
          };
          // each column thread: the x node and the y node of its own cell in
          // one straight-line block (independent chains); then the tile's
          // edge nodes (x nodes -1 and TX of each row, y nodes -1 and TY of
          // each column) on 2 (TX + TY) threads
          static_assert(2 * (TX + TY) <= NT && NC <= NT, "edge nodes need 2 (TX + TY) threads");
          if (tid < NC) {
            R px[5][3], py[5][3], qrx[5], qlx[5], qry[5], qly[5];
            const int wx = xnode(tx, ty, px), wy = ynode(ty, tx, py);
            node(px, qrx, qlx);
            node(py, qry, qly);
            put(wx, qrx, qlx);
            put(wy, qry, qly);
          }
          if (tid < 2 * (TX + TY)) {
            R p[5][3], qr[5], ql[5];
            int w;
            if (tid < 2 * TY)
              w = xnode(tid < TY ? -1 : TX, tid % TY, p);
            else
              w = ynode(tid < 2 * TY + TX ? -1 : TY, (tid - 2 * TY) % TX, p);
            node(p, qr, ql);
            put(w, qr, ql);
          }
          __syncthreads();
        }
      }

      // ---- phase B: fluxes ---------------------------------------------------
      R zF[5] = {0, 0, 0, 0, 0};
      if constexpr (DIM == 3) {
        if (colt && k >= T.z0 - 1) {
          if constexpr (C::SP) {
            flux_ausm_sides<2, R>(zWprev, zWcur, zF);
          } else {
            Prim5<R> L, Rr;
            if constexpr (RECON == RECON_WENO_ || RECON == RECON_MUSCL_) {
              L = zWprev;
              Rr = zWcur;
            } else {
              L = mkprim(zw[1]);
              Rr = mkprim(zw[2]);
            }
            face_flux<FLUX, 2, R, EX>(L, Rr, K, zF);
          }
        }
      }
      if (do_xy) {
        constexpr int NN = C::NXN + C::NYN;
        constexpr int NF = C::NXF + C::NYF;
        auto load_side = [&](int n) {
          AusmSide<R> sd;
          sd.u = sN[0 * NN + n];
          sd.v = sN[1 * NN + n];
          sd.w = sN[2 * NN + n];
          sd.p = sN[3 * NN + n];
          sd.H = sN[4 * NN + n];
          sd.M = sN[5 * NN + n];
          sd.rc = sN[6 * NN + n];
          return sd;
        };
        // face states: x face f (cell f on its right) of tile row `row`, and
        // y face f (cell row f above it) of tile column `col`
        auto xstates = [&](int f, int row, Prim5<R>& L, Prim5<R>& Rr) {
          if constexpr (RECON == RECON_WENO_ || RECON == RECON_MUSCL_) {
            const int nl = row * (TX + 2) + f, nr = nl + 1;
            L.r = sN[0 * NN + nl]; L.u = sN[1 * NN + nl]; L.v = sN[2 * NN + nl];
            L.w = sN[3 * NN + nl]; L.p = sN[4 * NN + nl];
            const int o = (TB || RECON == RECON_MUSCL_) ? 5 : 0;
            Rr.r = sN[(o + 0) * NN + nr]; Rr.u = sN[(o + 1) * NN + nr]; Rr.v = sN[(o + 2) * NN + nr];
            Rr.w = sN[(o + 3) * NN + nr]; Rr.p = sN[(o + 4) * NN + nr];
          } else {
            const int base = (H + row) * PW + (H + f);  // cell f (right of the face)
            R l[5], r[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              l[v] = sP[v * PLANE + base - 1];
              r[v] = sP[v * PLANE + base];
            }
            L = mkprim(l);
            Rr = mkprim(r);
          }
        };
        auto ystates = [&](int f, int col, Prim5<R>& L, Prim5<R>& Rr) {
          if constexpr (RECON == RECON_WENO_ || RECON == RECON_MUSCL_) {
            const int nl = C::NXN + f * TX + col, nr = nl + TX;
            L.r = sN[0 * NN + nl]; L.u = sN[1 * NN + nl]; L.v = sN[2 * NN + nl];
            L.w = sN[3 * NN + nl]; L.p = sN[4 * NN + nl];
            const int o = (TB || RECON == RECON_MUSCL_) ? 5 : 0;
            Rr.r = sN[(o + 0) * NN + nr]; Rr.u = sN[(o + 1) * NN + nr]; Rr.v = sN[(o + 2) * NN + nr];
            Rr.w = sN[(o + 3) * NN + nr]; Rr.p = sN[(o + 4) * NN + nr];
          } else {
            const int base = (H + f) * PW + (H + col);
            R l[5], r[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              l[v] = sP[v * PLANE + base - PW];
              r[v] = sP[v * PLANE + base];
            }
            L = mkprim(l);
            Rr = mkprim(r);
          }
        };
        if constexpr (C::SP) {
          // as below: the cell's low x and y faces together, then the edges
          if (tid < NC) {
            const int cx = tid % TX, cy = tid / TX;
            R Fx[5], Fy[5];
            const int nlx = cy * (TX + 2) + cx, nly = C::NXN + cy * TX + cx;
            flux_ausm_sides<0, R>(load_side(nlx), load_side(nlx + 1), Fx);
            flux_ausm_sides<1, R>(load_side(nly), load_side(nly + TX), Fy);
            const int wx = cy * (TX + 1) + cx, wy = C::NXF + cy * TX + cx;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              sF[v * NF + wx] = Fx[v];
              sF[v * NF + wy] = Fy[v];
            }
          }
          if (tid < TY + TX) {
            R F[5];
            int w;
            if (tid < TY) {
              const int nl = tid * (TX + 2) + TX;
              flux_ausm_sides<0, R>(load_side(nl), load_side(nl + 1), F);
              w = tid * (TX + 1) + TX;
            } else {
              const int nl = C::NXN + TY * TX + (tid - TY);
              flux_ausm_sides<1, R>(load_side(nl), load_side(nl + TX), F);
              w = C::NXF + TY * TX + (tid - TY);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) sF[v * NF + w] = F[v];
          }
        } else {
          // each column thread computes the low x face and the low y face of
          // its cell in one straight-line block, so the two flux chains
          // interleave; the tile's high-edge faces (TY x faces, TX y faces)
          // follow on TY + TX threads
          if (tid < NC) {
            const int cx = tid % TX, cy = tid / TX;
            Prim5<R> Lx, Rx, Ly, Ry;
            R Fx[5], Fy[5];
            xstates(cx, cy, Lx, Rx);
            ystates(cy, cx, Ly, Ry);
            face_flux<FLUX, 0, R, EX>(Lx, Rx, K, Fx);
            face_flux<FLUX, 1, R, EX>(Ly, Ry, K, Fy);
            const int wx = cy * (TX + 1) + cx, wy = C::NXF + cy * TX + cx;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              sF[v * NF + wx] = Fx[v];
              sF[v * NF + wy] = Fy[v];
            }
          }
          static_assert(TY + TX <= NT && NC <= NT, "edge faces need TY + TX threads");
          if (tid < TY + TX) {
            R F[5];
            Prim5<R> L, Rr;
            int w;
            if (tid < TY) {
              xstates(TX, tid, L, Rr);
              face_flux<FLUX, 0, R, EX>(L, Rr, K, F);
              w = tid * (TX + 1) + TX;
            } else {
              ystates(TY, tid - TY, L, Rr);
              face_flux<FLUX, 1, R, EX>(L, Rr, K, F);
              w = C::NXF + TY * TX + (tid - TY);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) sF[v * NF + w] = F[v];
          }
        }
      }
      __syncthreads();

      // ---- phase C: rhs, RK update, reductions -------------------------------
      // Tensor copies: every thread waits (bounded, one deadline for the CTA)
      // for the boxes issued at the top of this plane; a failed wait makes the
      // thread skip its work and leave before the plane's closing barrier.
      // (A decision taken after that barrier instead, from a shared flag or a
      // reducing barrier, measured 0.6 % slower on the FP64 vortex step and
      // 2.4 % on the FP32 one.)
      bool fail = false;
      if constexpr (C::TMA) {
        if (do_xy) {
          fail = !mbar_wait(&s_mbar[2], ph_q, &s_issued);
          ph_q ^= 1;
        }
      }
      if (do_xy && act && !fail) {
        constexpr int NF = C::NXF + C::NYF;
        const int fxl = ty * (TX + 1) + tx;
        const int fyl = C::NXF + ty * TX + tx;
        const int64_t off = off_k;
        double rhs[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          if constexpr (sizeof(R) == 4) {
            // FP32 flux form: difference and scale in FP32, one conversion
            R d = (sF[v * NF + fxl] - sF[v * NF + fxl + 1]) * (R)idr0;
            d = d + (sF[v * NF + fyl] - sF[v * NF + fyl + TX]) * (R)idr1;
            if constexpr (DIM == 3) d = d + (zFprev[v] - zF[v]) * (R)idr2;
            rhs[v] = (double)d;
            continue;
          }
          const double fxr = (double)sF[v * NF + fxl + 1], fxL = (double)sF[v * NF + fxl];
          const double fyr = (double)sF[v * NF + fyl + TX], fyL = (double)sF[v * NF + fyl];
          double r;
          if constexpr (EX) {
            r = 0.0 - (fxr - fxL) / dr0;
            r = r - (fyr - fyL) / dr1;
            if constexpr (DIM == 3) r = r - ((double)zF[v] - (double)zFprev[v]) / dr2;
          } else {
            r = -(fxr - fxL) * idr0;
            r = r - (fyr - fyL) * idr1;
            if constexpr (DIM == 3) r = r - ((double)zF[v] - (double)zFprev[v]) * idr2;
          }
          rhs[v] = r;
        }
        if (visc) {
#pragma unroll
          for (int v = 0; v < 5; ++v) rhs[v] = rhs[v] + visc[off + v * vs];
        }
        // RK update (scheme_Runge_Kutta.f90:30-63; classic RK4 for 4 stages)
        double u0[5], um[5], ac[5];
        if constexpr (!C::TMA) __pipeline_wait_prior(0);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          u0[v] = sQ[(0 * 5 + v) * NC + tid];
          um[v] = need_um ? sQ[(1 * 5 + v) * NC + tid] : 0.0;
          ac[v] = need_acc ? sQ[(1 * 5 + v) * NC + tid] : 0.0;
        }
        double h = dtg;
        if (ts_set == 2) h = cfl / wavespeed<EX>(u0, gammad, gm1d, drv, idrv, idim);
        double out[5];
        if (rk_stages == 3) {
          if (a.m == 1) {
#pragma unroll
            for (int v = 0; v < 5; ++v) out[v] = u0[v] + h * rhs[v];
          } else if (a.m == 2) {
            const double c3 = 1.0 / 4.0 * h;
#pragma unroll
            for (int v = 0; v < 5; ++v) out[v] = 3.0 / 4.0 * u0[v] + 1.0 / 4.0 * um[v] + c3 * rhs[v];
          } else {
            const double c3 = 2.0 / 3.0 * h;
#pragma unroll
            for (int v = 0; v < 5; ++v) out[v] = 1.0 / 3.0 * u0[v] + 2.0 / 3.0 * um[v] + c3 * rhs[v];
          }
        } else {
          // classic RK4 with q0 folded into the accumulator:
          //   acc = q0 + h/6 k1, acc += h/3 k2, acc += h/3 k3, q = acc + h/6 k4
          // so the last stage reads the accumulator alone (3, 5, 5, 3 state
          // arrays per stage)
          if (a.m == 1) {
            const double h2 = 0.5 * h, h6 = h / 6.0;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              accp[off + v * vs] = u0[v] + h6 * rhs[v];
              out[v] = u0[v] + h2 * rhs[v];
            }
          } else if (a.m == 2 || a.m == 3) {
            const double hc = (a.m == 2) ? 0.5 * h : h, h3 = h / 3.0;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              accp[off + v * vs] = ac[v] + h3 * rhs[v];
              out[v] = u0[v] + hc * rhs[v];
            }
          } else {
            const double h6 = h / 6.0;
#pragma unroll
            for (int v = 0; v < 5; ++v) out[v] = ac[v] + h6 * rhs[v];
          }
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) qout[off + v * vs] = out[v];
        if (a.last) {
#pragma unroll
          for (int v = 0; v < 5; ++v) sS[v * NT + tid] += rhs[v] * rhs[v];
          if (ts_set != 0) sS[5 * NT + tid] = fmax(sS[5 * NT + tid], wavespeed<EX>(out, gammad, gm1d, drv, idrv, idim));
          if (rhs_out) {
            const int64_t nc = (int64_t)G.n0 * G.n1 * G.n2;
            const int64_t r0 = gx + (int64_t)G.n0 * (gy + (int64_t)G.n1 * k);
#pragma unroll
            for (int v = 0; v < 5; ++v) rhs_out[r0 + v * nc] = rhs[v];
          }
        }
      }

      // ---- carry, window shift and shared-memory refill ----------------------
      if constexpr (C::FAL && !C::BOXA) __syncthreads();
      if constexpr (C::PSM && !C::TMA) __pipeline_wait_prior(0);
      if constexpr (C::TMA) {
        if (more) {
          fail |= !mbar_wait(&s_mbar[1], ph_z, &s_issued);
          ph_z ^= 1;
        }
        if (more_xy && !C::BOXA) {
          fail |= !mbar_wait(&s_mbar[0], ph_p, &s_issued);
          ph_p ^= 1;
        }
      }
      if (DIM == 3 && colt) {
#pragma unroll
        for (int v = 0; v < 5; ++v) zFprev[v] = zF[v];
        if constexpr (RECON == RECON_WENO_ || RECON == RECON_MUSCL_) zWprev = zWm_cur;
#pragma unroll
        for (int s = 0; s + 1 < C::WIN; ++s)
#pragma unroll
          for (int v = 0; v < 5; ++v) zw[s][v] = zw[s + 1][v];
        if (more) {
          if constexpr (C::TMA) {
#pragma unroll
            for (int v = 0; v < 5; ++v) zpre[v] = sTZ[v * (TX * TY) + zsrc];
          } else if constexpr (C::PSM) {
#pragma unroll
            for (int v = 0; v < 5; ++v) zpre[v] = sZ[v * NC + tid];
          }
          to_stencil<RECON, R, EX>(zpre, zw[C::WIN - 1], gm1d, K.gm1);
        }
        if (more_xy && !C::BOXA) {
          // centre of plane k+1 is window slot 1 after the shift
#pragma unroll
          for (int v = 0; v < 5; ++v) sP[v * PLANE + (H + ty) * PW + (H + tx)] = zw[1][v];
        }
      }
      if (more_xy && !C::BOXA) {
#pragma unroll
        for (int sidx = 0; sidx < C::NPS; ++sidx) {
          if (lsp[sidx] >= 0) {
            double q[5];
            if constexpr (C::TMA) {
#pragma unroll
              for (int v = 0; v < 5; ++v) q[v] = sTP[v * (PH * C::TW) + lxy[sidx]];
            } else if constexpr (C::PSM) {
              const int w = tid + sidx * NT;
#pragma unroll
              for (int v = 0; v < 5; ++v) q[v] = sX[v * C::NPL + w];
            } else {
#pragma unroll
              for (int v = 0; v < 5; ++v) q[v] = pre[sidx][v];
            }
            R s[5];
            to_stencil<RECON, R, EX>(q, s, gm1d, K.gm1);
#pragma unroll
            for (int v = 0; v < 5; ++v) sP[v * PLANE + lsp[sidx]] = s[v];
          }
        }
      }
      if constexpr (C::TMA) {
        if (fail) {
          leave_after_timeout(tid, a.err);
          return;
        }
      }
      __syncthreads();
    }

    if (a.last) cta_reduce_store<NT>(sS, s_red, a.partials + (int64_t)T.slot * kPartStride);
  }
}

template <int RECON, int FLUX, int PREC, bool TB, int DIM, int TX, int TY, int MINB>
__global__ void __launch_bounds__(StageCfg<RECON, FLUX, PREC, TB, DIM, TX, TY>::NT,
                                  (MINB > 0 ? MINB : (PREC == PREC_FP32 ? 512 : 384) / (TX * TY)))
    stage_kernel(const StageArgs a) {
  stage_run<RECON, FLUX, PREC, TB, DIM, TX, TY>(a);
}

}  // namespace fvm
