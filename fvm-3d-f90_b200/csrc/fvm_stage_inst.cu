// fvm_stage_inst.cu — explicit instantiations of the fused stage kernel for
// one precision and one reconstruction, selected by -DFVM_PREC / -DFVM_RECON
// (the build compiles this file once per pair, so the exact-FP64 objects can
// be built with -fmad=false and the FP32 objects with fast single math).
#include "fvm_aux.h"
#include "fvm_stage.cuh"

#ifndef FVM_PREC
#error "FVM_PREC not defined"
#endif
#ifndef FVM_RECON
#error "FVM_RECON not defined"
#endif

#define FVM_CAT2(a, b) a##b
#define FVM_CAT(a, b) FVM_CAT2(a, b)
#define FVM_LOOKUP_NAME FVM_CAT(FVM_CAT(lookup_stage_p, FVM_PREC), FVM_CAT(_r, FVM_RECON))

namespace fvm {

template <int FLUX, bool TB, int DIM, int TX, int TY, int MINB>
static bool fill(StageKernelInfo* out) {
  using Cfg = StageCfg<FVM_RECON, FLUX, FVM_PREC, TB, DIM, TX, TY>;
  out->fn = reinterpret_cast<const void*>(&stage_kernel<FVM_RECON, FLUX, FVM_PREC, TB, DIM, TX, TY, MINB>);
  out->smem = Cfg::smem_bytes;
  out->threads = Cfg::NT;
  out->tx = TX;
  out->ty = TY;
  out->tma = Cfg::TMA ? 1 : 0;
  out->box_w = Cfg::TW;
  out->box_h = Cfg::PH;
  out->halo = Cfg::H;
  return true;
}

template <int FLUX, bool TB, int DIM>
static bool by_tile(int tile, StageKernelInfo* out) {
  switch (tile) {
    case 0: return fill<FLUX, TB, DIM, kTileTX[0], kTileTY[0], kTileMinB[0]>(out);
    case 1: return fill<FLUX, TB, DIM, kTileTX[1], kTileTY[1], kTileMinB[1]>(out);
    case 2: return fill<FLUX, TB, DIM, kTileTX[2], kTileTY[2], kTileMinB[2]>(out);
    case 3: return fill<FLUX, TB, DIM, kTileTX[3], kTileTY[3], kTileMinB[3]>(out);
    default: return false;
  }
}

template <int FLUX, bool TB>
static bool by_dim(int dim, int tile, StageKernelInfo* out) {
  if (dim == 2) return by_tile<FLUX, TB, 2>(tile, out);
  if (dim == 3) return by_tile<FLUX, TB, 3>(tile, out);
  return false;
}

template <bool TB>
static bool by_flux(int flux, int dim, int tile, StageKernelInfo* out) {
  switch (flux) {
    case FLUX_ROE_: return by_dim<FLUX_ROE_, TB>(dim, tile, out);
    case FLUX_VANLEER_: return by_dim<FLUX_VANLEER_, TB>(dim, tile, out);
    case FLUX_AUSM_: return by_dim<FLUX_AUSM_, TB>(dim, tile, out);
    default: return false;
  }
}

bool FVM_LOOKUP_NAME(int dim, int flux, bool tb, int tile, StageKernelInfo* out) {
#if FVM_RECON == 202
  if (tb) return by_flux<true>(flux, dim, tile, out);
#else
  if (tb) return false;
#endif
  return by_flux<false>(flux, dim, tile, out);
}

}  // namespace fvm
