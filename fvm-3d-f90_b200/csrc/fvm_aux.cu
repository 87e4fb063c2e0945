// fvm_aux.cu — the kernels around the fused stage: ghost gather, state
// pack/unpack, primitive download, CFL wave-speed reduction, the per-step
// finalize (residual norms, time, next dt) and the viscous contribution.
// Compiled with -fmad=false: every FP64 expression here keeps the
// reference's rounding order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fvm_aux.h"
#include "fvm_schemes.cuh"
#include "fvm_types.h"

namespace fvm {

// ---------------------------------------------------------------- gather
// Ghost cells of connected / periodic regions: dst[i] = src[i] for all five
// variables, offsets relative to a role slab (the block-to-block exchange the
// reference describes in defs_face_geom.f90:378-402 but never performs).
__global__ void gather_kernel(double* __restrict__ base, int64_t vs, const int64_t* __restrict__ pairs,
                              int64_t npairs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npairs;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = pairs[2 * i], s = pairs[2 * i + 1];
#pragma unroll
    for (int v = 0; v < 5; ++v) base[d + v * vs] = base[s + v * vs];
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
                               int ncases) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncases) return;
  const DevCase& C = cases[c];
  st[c].dt = (C.timestep_set == 0) ? C.dt_fixed : C.cfl / __longlong_as_double((long long)case_max[c]);
}

// ---------------------------------------------------------------- finalize
// One CTA per case, after the last stage of a step:
// ClassIteration%reset_residual / compute_residual per block in block order /
// update (class_iteration.f90, file-local 195-259), time += dt, the stop
// checks of converged (:180-188) and the next step's dt.
__global__ void finalize_kernel(const DevBlock* blocks, const DevCase* cases, const int* case_blk, DevCaseState* st,
                                const double* partials, int* counters, int ncounters) {
  // one warp per block reduces its task partials (lanes stride the tasks,
  // then a butterfly); thread 0 folds the blocks in order, as the reference
  // accumulates them (class_iteration.f90:195-259)
  constexpr int NW = 8;
  __shared__ double red[NW][6];
  const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const DevCase& C = cases[c];
  if (c == 0)
    for (int i = tid; i < ncounters; i += blockDim.x) counters[i] = 0;
  if (C.nblocks == 0) return;  // removed case
  double res[6] = {0, 0, 0, 0, 0, 0};
  double wmax = 0.0;
  for (int b0 = 0; b0 < C.nblocks; b0 += NW) {
    const int bb = b0 + warp;
    if (warp < NW && bb < C.nblocks) {
      const DevBlock& B = blocks[case_blk[C.block0 + bb]];
      double s[5] = {0, 0, 0, 0, 0}, m = 0.0;
      for (int t = lane; t < B.ntask; t += 32) {
        const double* p = partials + (int64_t)(B.task0 + t) * kPartStride;
#pragma unroll
        for (int v = 0; v < 5; ++v) s[v] += p[v];
        m = fmax(m, p[5]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int v = 0; v < 5; ++v) s[v] += __shfl_xor_sync(0xffffffffu, s[v], o);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      }
      if (lane == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) red[warp][v] = s[v];
        red[warp][5] = m;
      }
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 0; w < NW && b0 + w < C.nblocks; ++w) {
        const DevBlock& B = blocks[case_blk[C.block0 + b0 + w]];
        const double npt = (double)((int64_t)B.n[0] * B.n[1] * B.n[2]);
        double res2[5], res2_t = 0.0;
        for (int v = 0; v < 5; ++v) {
          res2[v] = red[w][v] / npt;
          res2_t = res2_t + res2[v];
        }
        res2_t = res2_t / 5.0;
        for (int v = 0; v < 5; ++v) res[v] = sqrt(res[v] * res[v] + res2[v]);
        res[5] = sqrt(res[5] * res[5] + res2_t);
        wmax = fmax(wmax, red[w][5]);
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    DevCaseState& S = st[c];
    S.step += 1;
    S.t = S.t + S.dt;
    S.dt_last = S.dt;
    for (int e = 0; e < 6; ++e) S.res_abs[e] = res[e];
    if (S.step == 1)
      for (int e = 0; e < 6; ++e) S.res_abs0[e] = res[e];
    for (int e = 0; e < 6; ++e) S.res_rel[e] = S.res_abs[e] / S.res_abs0[e];
    if (isnan(res[5]))
      S.status = 4;  // FVM_ERR_NONFINITE
    else if (res[5] > 1.0E10)
      S.status = 5;  // FVM_ERR_DIVERGED
    S.dt = (C.timestep_set == 0) ? C.dt_fixed : C.cfl / wmax;
  }
}

// ---------------------------------------------------------------- viscous
// Central second-order viscous contribution (the reference's
// viscous_flux_sub, class_space_discret.f90:671-675, is empty; this is the
// textbook form): V = (dGx + dGy) + dGz with dG = (G(i+1/2) - G(i-1/2)) / dr.
// Cell primitives the viscous stencil reads, in the arithmetic type R of the
// case's precision form (FP64, or FP32 for the FP32 flux form).
template <class R>
struct VPrimT {
  R u, v, w, th;
};

__device__ __forceinline__ int64_t vcell(const DevBlock& B, int x, int y, int z) {
  const int m = B.ghost_mask;
  if (x < 0 && !(m & 1)) x = 0;
  if (x >= B.n[0] && !(m & 2)) x = B.n[0] - 1;
  if (y < 0 && !(m & 4)) y = 0;
  if (y >= B.n[1] && !(m & 8)) y = B.n[1] - 1;
  if (z < 0 && !(m & 16)) z = 0;
  if (z >= B.n[2] && !(m & 32)) z = B.n[2] - 1;
  return x + (int64_t)y * B.sy + (int64_t)z * B.sz;
}

// EX: the exact expression trees (divisions); otherwise one reciprocal (in
// FP64, stored in R).
template <bool EX, class R>
__device__ __forceinline__ VPrimT<R> vprim(const double* q, int64_t o, int64_t vs, double gm1) {
  VPrimT<R> r;
  if constexpr (EX) {
    Prim5<double> p = cons2prim<double, true>(q[o], q[o + vs], q[o + 2 * vs], q[o + 3 * vs], q[o + 4 * vs], gm1);
    r.u = p.u;
    r.v = p.v;
    r.w = p.w;
    r.th = p.p / p.r;
  } else {
    const double q0 = q[o], q1 = q[o + vs], q2 = q[o + 2 * vs], q3 = q[o + 3 * vs], q4 = q[o + 4 * vs];
    const double ir = 1.0 / q0;
    const double u = q1 * ir, v = q2 * ir, w = q3 * ir;
    r.u = (R)u;
    r.v = (R)v;
    r.w = (R)w;
    r.th = (R)(gm1 * (q4 - 0.5 * (q1 * u + q2 * v + q3 * w)) * ir);
  }
  return r;
}

template <class R>
__device__ __forceinline__ R vcomp(const VPrimT<R>& p, int m) {
  return m == 0 ? p.u : (m == 1 ? p.v : (m == 2 ? p.w : p.th));
}

// Viscous flux G[1..4] (G[0] = 0) through a face normal to `dir` between
// cells L and R. tg[d] holds, for each tangential axis d != dir, the cells
// L + e_d, L - e_d, R + e_d, R - e_d; the tangential gradient is the mean of
// the two central differences.
// EX divides by the cell sizes; otherwise multiplies by their reciprocals.
template <bool EX, class T>
__device__ __forceinline__ void visc_flux(const VPrimT<T>& L, const VPrimT<T>& R, const VPrimT<T> (*tg)[4], int dir,
                                          const T dr[3], const T idr[3], T mu, T kq, int idim, T G[5]) {
  T grad[4][3];
  for (int m = 0; m < 4; ++m)
    for (int d = 0; d < 3; ++d) grad[m][d] = T(0);
  for (int m = 0; m < 4; ++m)
    grad[m][dir] = EX ? (vcomp(R, m) - vcomp(L, m)) / dr[dir] : (vcomp(R, m) - vcomp(L, m)) * idr[dir];
  for (int d = 0; d < idim; ++d) {
    if (d == dir) continue;
    const VPrimT<T>& lp = tg[d][0];
    const VPrimT<T>& lm = tg[d][1];
    const VPrimT<T>& rp = tg[d][2];
    const VPrimT<T>& rm = tg[d][3];
    for (int m = 0; m < 4; ++m) {
      const T s = (vcomp(lp, m) - vcomp(lm, m)) + (vcomp(rp, m) - vcomp(rm, m));
      grad[m][d] = EX ? s / (T(4.0) * dr[d]) : s * (T(0.25) * idr[d]);
    }
  }
  const T div = grad[0][0] + grad[1][1] + grad[2][2];
  const T uf[3] = {T(0.5) * (L.u + R.u), T(0.5) * (L.v + R.v), T(0.5) * (L.w + R.w)};
  T tau[3];
  for (int m = 0; m < 3; ++m) {
    tau[m] = mu * (grad[m][dir] + grad[dir][m]);
    if (m == dir) tau[m] = tau[m] - T(2.0 / 3.0) * mu * div;
  }
  G[0] = T(0);
  G[1] = tau[0];
  G[2] = tau[1];
  G[3] = tau[2];
  G[4] = uf[0] * tau[0] + uf[1] * tau[1] + uf[2] * tau[2] + kq * grad[3][dir];
}

// Tiled viscous kernel: one CTA per task (a TX x TY column tile over a z
// range). The cell primitives (u, v, w, p/rho) of planes k-1, k, k+1 with a
// one-cell halo sit in a shared-memory ring; each x / y face flux of plane k
// is computed once into shared memory, each z face once per column (the lower
// one carried in registers). V = (dGx + dGy) + dGz as in the per-cell form.
// EX: the exact form the exact-FP64 cases need for parity with the oracle;
// the other precision forms multiply by reciprocals instead of dividing.
template <int TX, int TY, int IDIM, bool EX, class R>
__device__ __forceinline__ void visc_tile_body(const DevBlock& B, const DevCase& C, const Task& T, int role,
                                               unsigned char* smem) {
  using VPrim = VPrimT<R>;
  constexpr int NT = TX * TY, PX = TX + 2;
  constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1), NF = NXF + NYF;
  constexpr int PL = (TX + 2) * (TY + 2);
  constexpr int NR = IDIM == 3 ? 3 : 1;
  VPrim (*sp)[PL] = reinterpret_cast<VPrim (*)[PL]>(smem);
  R (*sg)[NF] = reinterpret_cast<R (*)[NF]>(smem + sizeof(VPrim) * NR * PL);
  const double* q = B.q[role];
  const int64_t vs = B.vs;
  const double gm1 = C.gm1;
  const R mu = (R)C.mu, kq = (R)C.kq;
  const R dr[3] = {(R)B.dr[0], (R)B.dr[1], (R)B.dr[2]};
  const R idr[3] = {(R)B.inv_dr[0], (R)B.inv_dr[1], (R)B.inv_dr[2]};
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const bool act = (T.x0 + tx < B.n[0]) && (T.y0 + ty < B.n[1]);
  auto slot = [](int z) { return IDIM == 3 ? ((z % 3) + 3) % 3 : 0; };
  // cell primitives of plane z, halo included; positions stay within the
  // first ghost layer (partial tiles clamp onto it)
  auto fill = [&](int z) {
    VPrim* dst = sp[slot(z)];
    for (int w = tid; w < PL; w += NT) {
      const int x = min(max(T.x0 + w % PX - 1, -1), B.n[0]);
      const int y = min(max(T.y0 + w / PX - 1, -1), B.n[1]);
      dst[w] = vprim<EX, R>(q, vcell(B, x, y, z), vs, gm1);
    }
  };
  auto P = [&](int z, int x, int y) -> const VPrim& { return sp[slot(z)][(y + 1) * PX + (x + 1)]; };
  // z face between planes z and z+1 of this thread's column
  auto zface = [&](int z, R G[5]) {
    VPrim tg[3][4];
    tg[0][0] = P(z, tx + 1, ty);
    tg[0][1] = P(z, tx - 1, ty);
    tg[0][2] = P(z + 1, tx + 1, ty);
    tg[0][3] = P(z + 1, tx - 1, ty);
    tg[1][0] = P(z, tx, ty + 1);
    tg[1][1] = P(z, tx, ty - 1);
    tg[1][2] = P(z + 1, tx, ty + 1);
    tg[1][3] = P(z + 1, tx, ty - 1);
    visc_flux<EX>(P(z, tx, ty), P(z + 1, tx, ty), tg, 2, dr, idr, mu, kq, 3, G);
  };

  R Gzl[5] = {0, 0, 0, 0, 0}, Gzr[5] = {0, 0, 0, 0, 0};
  if (IDIM == 3) {
    fill(T.z0 - 1);
    fill(T.z0);
  }
  for (int k = T.z0; k < T.z1; ++k) {
    fill(IDIM == 3 ? k + 1 : k);
    __syncthreads();
    for (int w = tid; w < NF; w += NT) {
      VPrim tg[3][4];
      R G[5];
      if (w < NXF) {
        const int f = w % (TX + 1), row = w / (TX + 1);  // face between cells f-1 and f
        tg[1][0] = P(k, f - 1, row + 1);
        tg[1][1] = P(k, f - 1, row - 1);
        tg[1][2] = P(k, f, row + 1);
        tg[1][3] = P(k, f, row - 1);
        if (IDIM == 3) {
          tg[2][0] = P(k + 1, f - 1, row);
          tg[2][1] = P(k - 1, f - 1, row);
          tg[2][2] = P(k + 1, f, row);
          tg[2][3] = P(k - 1, f, row);
        }
        visc_flux<EX>(P(k, f - 1, row), P(k, f, row), tg, 0, dr, idr, mu, kq, IDIM, G);
      } else {
        const int w2 = w - NXF, col = w2 % TX, f = w2 / TX;  // face between rows f-1 and f
        tg[0][0] = P(k, col + 1, f - 1);
        tg[0][1] = P(k, col - 1, f - 1);
        tg[0][2] = P(k, col + 1, f);
        tg[0][3] = P(k, col - 1, f);
        if (IDIM == 3) {
          tg[2][0] = P(k + 1, col, f - 1);
          tg[2][1] = P(k - 1, col, f - 1);
          tg[2][2] = P(k + 1, col, f);
          tg[2][3] = P(k - 1, col, f);
        }
        visc_flux<EX>(P(k, col, f - 1), P(k, col, f), tg, 1, dr, idr, mu, kq, IDIM, G);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) sg[v][w] = G[v + 1];
    }
    if (IDIM == 3) {
      if (k == T.z0) zface(k - 1, Gzl);
      zface(k, Gzr);
    }
    __syncthreads();
    if (act) {
      const int fxl = ty * (TX + 1) + tx, fyl = NXF + ty * TX + tx;
      R V[5] = {0, 0, 0, 0, 0};
      for (int v = 1; v < 5; ++v) {
        if constexpr (EX) {
          V[v] = V[v] + (sg[v - 1][fxl + 1] - sg[v - 1][fxl]) / dr[0];
          V[v] = V[v] + (sg[v - 1][fyl + TX] - sg[v - 1][fyl]) / dr[1];
          if (IDIM == 3) V[v] = V[v] + (Gzr[v] - Gzl[v]) / dr[2];
        } else {
          V[v] = (sg[v - 1][fxl + 1] - sg[v - 1][fxl]) * idr[0] + (sg[v - 1][fyl + TX] - sg[v - 1][fyl]) * idr[1];
          if (IDIM == 3) V[v] = V[v] + (Gzr[v] - Gzl[v]) * idr[2];
        }
      }
      V[0] = R(0);
      const int64_t o = (T.x0 + tx) + (int64_t)(T.y0 + ty) * B.sy + (int64_t)k * B.sz;
      for (int v = 0; v < 5; ++v) B.visc[o + v * vs] = (double)V[v];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) Gzl[v] = Gzr[v];
  }
}

template <int TX, int TY, int IDIM>
__global__ void __launch_bounds__(TX* TY) visc_tile_kernel(const DevBlock* blocks, const DevCase* cases,
                                                          const Task* tasks, int role) {
  constexpr int NR = IDIM == 3 ? 3 : 1;
  // storage of the FP64 forms; the FP32 form uses the first half
  __shared__ __align__(16) unsigned char smem[sizeof(VPrimT<double>) * NR * (TX + 2) * (TY + 2) +
                                              sizeof(double) * 4 * ((TX + 1) * TY + TX * (TY + 1))];
  const Task T = tasks[blockIdx.x];
  const DevBlock& B = blocks[T.blk];
  const DevCase& C = cases[B.case_id];
  if (C.precision == PREC_EXACT)
    visc_tile_body<TX, TY, IDIM, true, double>(B, C, T, role, smem);
  else if (C.precision == PREC_FP32)
    visc_tile_body<TX, TY, IDIM, false, float>(B, C, T, role, smem);
  else
    visc_tile_body<TX, TY, IDIM, false, double>(B, C, T, role, smem);
}

// ---------------------------------------------------------------- launchers
static inline int grid_for(int64_t n, int bs) {
  int64_t g = (n + bs - 1) / bs;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t launch_gather(double* base, int64_t vs, const int64_t* pairs, int64_t npairs, cudaStream_t s) {
  if (npairs == 0) return cudaSuccess;
  gather_kernel<<<grid_for(npairs, 256), 256, 0, s>>>(base, vs, pairs, npairs);
  return cudaGetLastError();
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
                           unsigned long long* case_max, int role, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(case_max, 0, sizeof(unsigned long long) * ncases, s);
  if (e != cudaSuccess) return e;
  if (nblocks > 0) {
    dim3 g(64, nblocks);
    wavespeed_kernel<<<g, 256, 0, s>>>(blocks, cases, role, case_max);
  }
  init_dt_kernel<<<(ncases + 127) / 128, 128, 0, s>>>(cases, st, case_max, ncases);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const DevBlock* blocks, const DevCase* cases, const int* case_blk, DevCaseState* st,
                            int ncases, const double* partials, int* counters, int ncounters, cudaStream_t s) {
  finalize_kernel<<<ncases, 256, 0, s>>>(blocks, cases, case_blk, st, partials, counters, ncounters);
  return cudaGetLastError();
}

cudaError_t launch_visc(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int ntasks, int idim,
                        int role, cudaStream_t s) {
  if (ntasks == 0) return cudaSuccess;
  if (idim == 3)
    visc_tile_kernel<kViscTX, kViscTY, 3><<<ntasks, kViscTX * kViscTY, 0, s>>>(blocks, cases, tasks, role);
  else
    visc_tile_kernel<kViscTX, kViscTY, 2><<<ntasks, kViscTX * kViscTY, 0, s>>>(blocks, cases, tasks, role);
  return cudaGetLastError();
}

}  // namespace fvm
