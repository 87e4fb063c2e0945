// fvm_visc.cuh — the viscous contribution of the Navier-Stokes blocks:
// central second-order face fluxes on a column tile marched along z. Shared
// by the exact-FP64 instantiation (fvm_aux.cu, compiled without FMA
// contraction) and the FP64 / FP32 ones (fvm_visc.cu, contracted).
#pragma once
#include <cuda_pipeline.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fvm_aux.h"
#include "fvm_schemes.cuh"
#include "fvm_types.h"

namespace fvm {

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

// EX: the exact expression trees (divisions); otherwise one reciprocal, in
// the arithmetic type R.
template <bool EX, class R>
__device__ __forceinline__ VPrimT<R> vprim(double q0, double q1, double q2, double q3, double q4, double gm1) {
  VPrimT<R> r;
  if constexpr (EX) {
    Prim5<double> p = cons2prim<double, true>(q0, q1, q2, q3, q4, gm1);
    r.u = p.u;
    r.v = p.v;
    r.w = p.w;
    r.th = p.p / p.r;
  } else {
    // in R: the FP32 form converts the conserved values first
    const R f0 = (R)q0, f1 = (R)q1, f2 = (R)q2, f3 = (R)q3, f4 = (R)q4;
    const R ir = rcp_(f0);
    r.u = f1 * ir;
    r.v = f2 * ir;
    r.w = f3 * ir;
    r.th = (R)gm1 * (f4 - R(0.5) * (f1 * r.u + f2 * r.v + f3 * r.w)) * ir;
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
// range), one thread per column. The cell primitives (u, v, w, p/rho) of
// planes k-1, k, k+1 with a one-cell halo sit in a shared-memory ring, one
// array per component (a warp reading one component of 32 cells touches
// consecutive words). Each thread computes the faces on the low side of its
// cell (x face, y face) and the z face above it; its own column's primitives
// stay in registers, and the neighbour values the three faces share are read
// once. The faces on the high edges of the tile (x = TX, y = TY) are
// computed by the first TX + TY threads. x / y face fluxes meet in shared memory, the
// z face below is carried in registers. The conserved values of the next
// two planes are copied asynchronously into two staging buffers while the
// current plane's faces are computed; each thread converts the cells it
// copied itself, so the staging buffers need no barrier.
// V = (dGx + dGy) + dGz as in the per-cell form. EX: the exact form the
// exact-FP64 cases need for parity with the oracle; the other precision
// forms multiply by reciprocals instead of dividing.
template <int TX, int TY, int IDIM>
struct ViscCfg {
  static constexpr int NT = TX * TY, PX = TX + 2, PL = (TX + 2) * (TY + 2);
  static constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1), NF = NXF + NYF;
  static constexpr int NR = IDIM == 3 ? 3 : 1;      // primitive planes in the ring
  static constexpr int NPT = (PL + NT - 1) / NT;    // staged cells per thread
  static_assert(TX + TY <= NT, "one high-edge face per thread");
  // bytes for arithmetic type R of RB bytes: primitive ring, face fluxes,
  // two staging planes of FP64 conserved values
  template <int RB>
  struct Smem {
    static constexpr int v = RB * (NR * 4 * PL + 4 * NF) + 8 * 2 * 5 * PL;
  };
};

template <int TX, int TY, int IDIM, bool EX, class R>
__device__ __forceinline__ void visc_tile_body(const DevBlock& B, const DevCase& C, const Task& T, int role,
                                               unsigned char* smem) {
  using VPrim = VPrimT<R>;
  using Cf = ViscCfg<TX, TY, IDIM>;
  constexpr int NT = Cf::NT, PX = Cf::PX, PL = Cf::PL, NXF = Cf::NXF, NF = Cf::NF, NR = Cf::NR, NPT = Cf::NPT;
  R (*sp)[4][PL] = reinterpret_cast<R (*)[4][PL]>(smem);
  // face fluxes: x faces [row][0..TX], then y faces [0..TY][col]
  R (*sg)[NF] = reinterpret_cast<R (*)[NF]>(smem + sizeof(R) * NR * 4 * PL);
  double (*raw)[5][PL] = reinterpret_cast<double (*)[5][PL]>(smem + sizeof(R) * (NR * 4 * PL + 4 * NF));
  const double* q = B.q[role];
  const int64_t vs = B.vs;
  const double gm1 = C.gm1;
  const R mu = (R)C.mu, kq = (R)C.kq;
  const R dr[3] = {(R)B.dr[0], (R)B.dr[1], (R)B.dr[2]};
  const R idr[3] = {(R)B.inv_dr[0], (R)B.inv_dr[1], (R)B.inv_dr[2]};
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const bool act = (T.x0 + tx < B.n[0]) && (T.y0 + ty < B.n[1]);
  auto slot = [](int z) { return IDIM == 3 ? ((z % 3) + 3) % 3 : 0; };
  // staging offsets of this thread's cells (same x / y in every plane);
  // positions stay within the first ghost layer (partial tiles clamp onto it)
  int cx[NPT], cy[NPT];
#pragma unroll
  for (int j = 0; j < NPT; ++j) {
    const int w = tid + j * NT;
    cx[j] = min(max(T.x0 + w % PX - 1, -1), B.n[0]);
    cy[j] = min(max(T.y0 + w / PX - 1, -1), B.n[1]);
  }
  // copy the conserved values of plane z into its staging buffer (planes
  // beyond zlast commit an empty group, so the group count stays uniform)
  const int zlast = IDIM == 3 ? T.z1 : T.z1 - 1;
  auto issue = [&](int z) {
    if (z <= zlast) {
      double(*st)[PL] = raw[(z + 2) & 1];
#pragma unroll
      for (int j = 0; j < NPT; ++j) {
        const int w = tid + j * NT;
        if (w < PL) {
          const double* src = q + vcell(B, cx[j], cy[j], z);
#pragma unroll
          for (int v = 0; v < 5; ++v) __pipeline_memcpy_async(&st[v][w], src + v * vs, sizeof(double));
        }
      }
    }
    __pipeline_commit();
  };
  // primitives of staged plane z (the older of the two groups in flight)
  // into its ring slot
  auto convert = [&](int z) {
    __pipeline_wait_prior(1);
    R(*dst)[PL] = sp[slot(z)];
    double(*st)[PL] = raw[(z + 2) & 1];
#pragma unroll
    for (int j = 0; j < NPT; ++j) {
      const int w = tid + j * NT;
      if (w < PL) {
        const VPrim p = vprim<EX, R>(st[0][w], st[1][w], st[2][w], st[3][w], st[4][w], gm1);
        dst[0][w] = p.u;
        dst[1][w] = p.v;
        dst[2][w] = p.w;
        dst[3][w] = p.th;
      }
    }
  };
  // cell (x, y) of plane z, tile coordinates (-1 .. TX / TY)
  auto P = [&](int z, int x, int y) -> VPrim {
    const int s = slot(z), i = (y + 1) * PX + (x + 1);
    return VPrim{sp[s][0][i], sp[s][1][i], sp[s][2][i], sp[s][3][i]};
  };
  auto store_face = [&](int idx, const R G[5]) {
#pragma unroll
    for (int v = 0; v < 4; ++v) sg[v][idx] = G[v + 1];
  };

  R Gzl[5] = {0, 0, 0, 0, 0}, Gzr[5] = {0, 0, 0, 0, 0};
  VPrim cm{}, c0{};  // this column's cells at k-1 and k (3D)
  // two planes in flight: convert plane z, then issue plane z + 2 into the
  // staging buffer just read
  const int zf = IDIM == 3 ? T.z0 - 1 : T.z0;
  issue(zf);
  issue(zf + 1);
  if (IDIM == 3) {
    convert(T.z0 - 1);
    issue(T.z0 + 1);
    convert(T.z0);
    issue(T.z0 + 2);
  }
  for (int k = T.z0; k < T.z1; ++k) {
    // plane k + 1 (3D) / k (2D) from the staging buffer, then the next copy
    const int zc = IDIM == 3 ? k + 1 : k;
    convert(zc);
    issue(zc + 2);
    __syncthreads();
    if (IDIM == 3 && k == T.z0) {
      cm = P(k - 1, tx, ty);
      c0 = P(k, tx, ty);
    }
    if (IDIM != 3) c0 = P(k, tx, ty);
    // neighbours in plane k shared by the three faces
    const VPrim xm = P(k, tx - 1, ty), xp = P(k, tx + 1, ty);
    const VPrim ym = P(k, tx, ty - 1), yp = P(k, tx, ty + 1);
    const VPrim xmym = P(k, tx - 1, ty - 1);
    VPrim cp{}, xm_p{}, ym_p{};
    R Gx[5], Gy[5];
    {
      // x face between (tx-1, ty) and (tx, ty)
      VPrim tg[3][4];
      tg[1][0] = P(k, tx - 1, ty + 1);
      tg[1][1] = xmym;
      tg[1][2] = yp;
      tg[1][3] = ym;
      if (IDIM == 3) {
        xm_p = P(k + 1, tx - 1, ty);
        cp = P(k + 1, tx, ty);
        tg[2][0] = xm_p;
        tg[2][1] = P(k - 1, tx - 1, ty);
        tg[2][2] = cp;
        tg[2][3] = cm;
      }
      visc_flux<EX>(xm, c0, tg, 0, dr, idr, mu, kq, IDIM, Gx);
    }
    {
      // y face between (tx, ty-1) and (tx, ty)
      VPrim tg[3][4];
      tg[0][0] = P(k, tx + 1, ty - 1);
      tg[0][1] = xmym;
      tg[0][2] = xp;
      tg[0][3] = xm;
      if (IDIM == 3) {
        ym_p = P(k + 1, tx, ty - 1);
        tg[2][0] = ym_p;
        tg[2][1] = P(k - 1, tx, ty - 1);
        tg[2][2] = cp;
        tg[2][3] = cm;
      }
      visc_flux<EX>(ym, c0, tg, 1, dr, idr, mu, kq, IDIM, Gy);
    }
    store_face(ty * (TX + 1) + tx, Gx);
    store_face(NXF + ty * TX + tx, Gy);
    if (IDIM == 3) {
      // z face between planes k and k+1 (and k-1 / k once per task)
      if (k == T.z0) {
        VPrim tg[3][4];
        tg[0][0] = P(k - 1, tx + 1, ty);
        tg[0][1] = P(k - 1, tx - 1, ty);
        tg[0][2] = xp;
        tg[0][3] = xm;
        tg[1][0] = P(k - 1, tx, ty + 1);
        tg[1][1] = P(k - 1, tx, ty - 1);
        tg[1][2] = yp;
        tg[1][3] = ym;
        visc_flux<EX>(cm, c0, tg, 2, dr, idr, mu, kq, 3, Gzl);
      }
      VPrim tg[3][4];
      tg[0][0] = xp;
      tg[0][1] = xm;
      tg[0][2] = P(k + 1, tx + 1, ty);
      tg[0][3] = xm_p;
      tg[1][0] = yp;
      tg[1][1] = ym;
      tg[1][2] = P(k + 1, tx, ty + 1);
      tg[1][3] = ym_p;
      visc_flux<EX>(c0, cp, tg, 2, dr, idr, mu, kq, 3, Gzr);
    }
    // faces on the high x / y edges of the tile
    if (tid < TY + TX) {
      VPrim tg[3][4];
      R G[5];
      if (tid < TY) {
        const int row = tid;  // x face between (TX-1, row) and (TX, row)
        tg[1][0] = P(k, TX - 1, row + 1);
        tg[1][1] = P(k, TX - 1, row - 1);
        tg[1][2] = P(k, TX, row + 1);
        tg[1][3] = P(k, TX, row - 1);
        if (IDIM == 3) {
          tg[2][0] = P(k + 1, TX - 1, row);
          tg[2][1] = P(k - 1, TX - 1, row);
          tg[2][2] = P(k + 1, TX, row);
          tg[2][3] = P(k - 1, TX, row);
        }
        visc_flux<EX>(P(k, TX - 1, row), P(k, TX, row), tg, 0, dr, idr, mu, kq, IDIM, G);
        store_face(row * (TX + 1) + TX, G);
      } else {
        const int col = tid - TY;  // y face between (col, TY-1) and (col, TY)
        tg[0][0] = P(k, col + 1, TY - 1);
        tg[0][1] = P(k, col - 1, TY - 1);
        tg[0][2] = P(k, col + 1, TY);
        tg[0][3] = P(k, col - 1, TY);
        if (IDIM == 3) {
          tg[2][0] = P(k + 1, col, TY - 1);
          tg[2][1] = P(k - 1, col, TY - 1);
          tg[2][2] = P(k + 1, col, TY);
          tg[2][3] = P(k - 1, col, TY);
        }
        visc_flux<EX>(P(k, col, TY - 1), P(k, col, TY), tg, 1, dr, idr, mu, kq, IDIM, G);
        store_face(NXF + TY * TX + col, G);
      }
    }
    __syncthreads();
    if (act) {
      const int fxr = ty * (TX + 1) + tx + 1, fyr = NXF + (ty + 1) * TX + tx;
      R V[5] = {0, 0, 0, 0, 0};
      for (int v = 1; v < 5; ++v) {
        if constexpr (EX) {
          V[v] = V[v] + (sg[v - 1][fxr] - Gx[v]) / dr[0];
          V[v] = V[v] + (sg[v - 1][fyr] - Gy[v]) / dr[1];
          if (IDIM == 3) V[v] = V[v] + (Gzr[v] - Gzl[v]) / dr[2];
        } else {
          V[v] = (sg[v - 1][fxr] - Gx[v]) * idr[0] + (sg[v - 1][fyr] - Gy[v]) * idr[1];
          if (IDIM == 3) V[v] = V[v] + (Gzr[v] - Gzl[v]) * idr[2];
        }
      }
      V[0] = R(0);
      const int64_t o = (T.x0 + tx) + (int64_t)(T.y0 + ty) * B.sy + (int64_t)k * B.sz;
      for (int v = 0; v < 5; ++v) B.visc[o + v * vs] = (double)V[v];
    }
    if (IDIM == 3) {
#pragma unroll
      for (int v = 0; v < 5; ++v) Gzl[v] = Gzr[v];
      cm = c0;
      c0 = cp;
    }
  }
}

// One precision form of the tiled viscous kernel. Register budgets: the
// exact form keeps its division chains unspilled at 3 CTAs per SM, the
// others run 4 (FP64) and 5 (FP32) CTAs per SM.
template <int PREC>
struct ViscMinBlocks {
  static constexpr int v = PREC == PREC_EXACT ? 4 : (PREC == PREC_FP64 ? 4 : 6);
};

template <int TX, int TY, int IDIM, int PREC>
__global__ void __launch_bounds__(TX* TY, ViscMinBlocks<PREC>::v)
    visc_tile_kernel(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int role) {
  using PT = PrecT<PREC>;
  __shared__ __align__(16)
      unsigned char smem[ViscCfg<TX, TY, IDIM>::template Smem<(int)sizeof(typename PT::R)>::v];
  pdl_wait();  // no early trigger (see stage_kernel)
  const Task T = tasks[blockIdx.x];
  const DevBlock& B = blocks[T.blk];
  visc_tile_body<TX, TY, IDIM, PT::ex, typename PT::R>(B, cases[B.case_id], T, role, smem);
}

template <int PREC>
cudaError_t launch_visc_prec(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int ntasks, int idim,
                             int role, cudaStream_t s, bool pdl) {
  constexpr int TX = visc_tx(PREC), TY = visc_ty(PREC);
  if (ntasks == 0) return cudaSuccess;
  LaunchCfg L(dim3(ntasks), dim3(TX * TY), 0, s, pdl);
  if (idim == 3) return cudaLaunchKernelEx(&L.cfg, visc_tile_kernel<TX, TY, 3, PREC>, blocks, cases, tasks, role);
  return cudaLaunchKernelEx(&L.cfg, visc_tile_kernel<TX, TY, 2, PREC>, blocks, cases, tasks, role);
}

template <int PREC>
cudaError_t visc_occupancy_prec(int* ctas_per_sm) {
  constexpr int TX = visc_tx(PREC), TY = visc_ty(PREC);
  int occ = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, visc_tile_kernel<TX, TY, 3, PREC>, TX * TY, 0);
  *ctas_per_sm = occ < 1 ? 1 : occ;
  return e;
}

}  // namespace fvm
