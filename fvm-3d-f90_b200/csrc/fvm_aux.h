// fvm_aux.h — launchers of the auxiliary kernels (fvm_aux.cu) and the
// lookup of fused stage-kernel instantiations (fvm_stage_inst.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fvm_types.h"

namespace fvm {

// A launch configuration, with programmatic stream serialization when pdl is
// set (the kernel must call pdl_wait() first). Used in place: cfg.attrs
// points into the object.
struct LaunchCfg {
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1]{};
  LaunchCfg(dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl) {
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
  }
  LaunchCfg(const LaunchCfg&) = delete;
  LaunchCfg& operator=(const LaunchCfg&) = delete;
};

// gather, finalize and visc take pdl: launch with programmatic stream
// serialization (inside the step graphs).
cudaError_t launch_gather(double* base, int64_t vs, const int32_t* pairs, int64_t npairs, cudaStream_t s,
                          bool pdl = false);
cudaError_t launch_unpack(double* role_blk, int64_t vs, int sy, int sz, int ni, int nj, int nk, const double* src,
                          cudaStream_t s);
cudaError_t launch_pack(const double* role_blk, int64_t vs, int sy, int sz, int ni, int nj, int nk, double* dst,
                        int prim, double gm1, cudaStream_t s);
cudaError_t launch_init_dt(const DevBlock* blocks, int nblocks, const DevCase* cases, DevCaseState* st, int ncases,
                           unsigned long long* case_max, const int* mask, int role, cudaStream_t s);
cudaError_t launch_finalize(const DevBlock* blocks, const DevCase* cases, const int* case_blk, DevCaseState* st,
                            int ncases, const double* partials, int* counters, int ncounters, cudaStream_t s,
                            bool pdl = false);
// Viscous contribution of the Navier-Stokes blocks: one CTA per task of a
// viscous task list (column tiles over z ranges), all of dimension idim and
// precision form prec (PREC_*). The tile is 16 x 8 for the FP64 forms and
// 32 x 4 for the FP32 form, whose warps then read one row of 32 floats
// (bank-conflict free; two 16-float rows 18 floats apart share two banks).
// visc_occupancy: CTAs of the 3D kernel of that form resident on one SM. The
// *_fast entry points serve the FP64 and FP32 forms.
constexpr int visc_tx(int prec) { return prec == 2 ? 32 : 16; }
constexpr int visc_ty(int prec) { return prec == 2 ? 4 : 8; }
cudaError_t launch_visc(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int ntasks, int idim,
                        int prec, int role, cudaStream_t s, bool pdl = false);
cudaError_t visc_occupancy(int prec, int* ctas_per_sm);
cudaError_t launch_visc_fast(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int ntasks, int idim,
                             int prec, int role, cudaStream_t s, bool pdl);
cudaError_t visc_occupancy_fast(int prec, int* ctas_per_sm);
// rcp_ / rsqrt_ of the non-exact FP64 forms over x[0..n) (device arrays).
cudaError_t launch_fast_math_probe(const double* x, int64_t n, double* r, double* rs, cudaStream_t s);

// One compiled instantiation of the fused stage kernel.
struct StageKernelInfo {
  const void* fn = nullptr;
  size_t smem = 0;
  int threads = 0;
  int tx = 0, ty = 0;
  // tensor-map prefetch: the plane box is box_w x box_h cells (x, y), the z
  // box tx x ty; the kernel expects StageArgs::tmap (0 = no tensor maps)
  int tma = 0, box_w = 0, box_h = 0, halo = 0;
};

// Tile shapes compiled for every scheme (index -> TX x TY, minimum resident
// CTAs per SM the register allocation is capped for; 0 = 16 warps per SM for
// the FP32 flux form, 12 for FP64 (rounded down to whole CTAs)).
constexpr int kNumTiles = 4;
constexpr int kTileTX[kNumTiles] = {32, 16, 32, 16};
constexpr int kTileTY[kNumTiles] = {8, 16, 8, 8};
constexpr int kTileMinB[kNumTiles] = {0, 0, 2, 0};

// prec: 0 exact FP64, 1 FP64, 2 FP32 flux; dim 2|3; recon 200..202;
// flux 300|301|303; tb: textbook WENO (mirrored right state); tile 0..kNumTiles-1.
bool lookup_stage_kernel(int prec, int dim, int recon, int flux, bool tb, int tile, StageKernelInfo* out);

}  // namespace fvm
