// fvm_resid.cu — residual norms of one block's rhs held in device memory.
//
// Restates ClassIteration%compute_residual_sub (class_iteration.f90,
// file-local 210-248) for a caller that keeps rhs on the device:
//   res2(e) = sum(rhs(:,:,:,e)^2) / (ni*nj*nk),  res2_t = sum_e res2(e) / neq
//   R(e)    = sqrt(R(e)^2 + res2(e)),            R_t = sqrt(R_t^2 + res2_t)
// so repeated calls over the blocks of a case accumulate exactly as the
// reference does. The sum is deterministic: one CTA per piece of a k plane
// (its row ranges depend only on the block's shape) writes the piece's five
// sums (fixed-order tree inside the CTA), then one CTA adds the pieces in a
// fixed order.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/fvm3d.h"

namespace fvm {

constexpr int kResidThreads = 256;
constexpr int64_t kResidMaxParts = 4096;  // partial slots of one call (5 doubles each)

// Pieces each k plane is cut into (row ranges): enough CTAs to fill the GPU
// (about four per SM), at most one per row, and at most kResidMaxParts slots
// in all when the block has no more planes than that. A function of the
// block's shape only, so the summation order (and the result) is too.
int64_t resid_chunks(const int64_t nvert[3]) {
  const int64_t nk = nvert[2];
  int64_t c = (600 + nk - 1) / nk;
  c = std::min<int64_t>(c, nvert[1]);
  if (nk <= kResidMaxParts) c = std::min<int64_t>(c, kResidMaxParts / nk);
  return std::max<int64_t>(c, 1);
}

// One CTA per (plane k, row range): the five sums of rhs^2 over its cells,
// a fixed-order tree inside the CTA, into parts[(k * chunks + c) * 5 + e].
__global__ void resid_plane_kernel(const double* __restrict__ rhs, int64_t ni, int64_t nj, int64_t nk,
                                   int64_t chunks, double* __restrict__ parts) {
  __shared__ double red[5][kResidThreads];
  const int64_t b = blockIdx.x, k = b / chunks, c = b % chunks;
  const int64_t j0 = c * nj / chunks, j1 = (c + 1) * nj / chunks;
  const int64_t nc = ni * nj * nk;
  const double* base = rhs + k * ni * nj + j0 * ni;
  const int64_t n = (j1 - j0) * ni;
  double s[5] = {0, 0, 0, 0, 0};
  for (int64_t i = threadIdx.x; i < n; i += kResidThreads) {
#pragma unroll
    for (int e = 0; e < 5; ++e) {
      const double v = base[i + e * nc];
      s[e] += v * v;
    }
  }
#pragma unroll
  for (int e = 0; e < 5; ++e) red[e][threadIdx.x] = s[e];
  __syncthreads();
  for (int w = kResidThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int e = 0; e < 5; ++e) red[e][threadIdx.x] += red[e][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int e = 0; e < 5; ++e) parts[b * 5 + e] = red[e][0];
}

// One CTA: thread t adds the pieces t, t + 256, ... in order, then a
// fixed-order tree; thread 0 turns the sums into the norms and folds them
// into res (R = sqrt(R^2 + res2), class_iteration.f90's accumulation).
__global__ void resid_finalize_kernel(const double* __restrict__ parts, int64_t nparts, int64_t ncells,
                                      double* __restrict__ res) {
  __shared__ double red[5][kResidThreads];
  double s[5] = {0, 0, 0, 0, 0};
  for (int64_t b = threadIdx.x; b < nparts; b += kResidThreads)
#pragma unroll
    for (int e = 0; e < 5; ++e) s[e] += parts[b * 5 + e];
#pragma unroll
  for (int e = 0; e < 5; ++e) red[e][threadIdx.x] = s[e];
  __syncthreads();
  for (int w = kResidThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int e = 0; e < 5; ++e) red[e][threadIdx.x] += red[e][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double res2[5], res2_t = 0.0;
  for (int e = 0; e < 5; ++e) {
    res2[e] = red[e][0] / (double)ncells;
    res2_t = res2_t + res2[e];
  }
  res2_t = res2_t / 5.0;
  for (int e = 0; e < 5; ++e) res[e] = sqrt(res[e] * res[e] + res2[e]);
  res[5] = sqrt(res[5] * res[5] + res2_t);
}

int residual_launch(const double* rhs, const int64_t nvert[3], double* res, double* scratch, cudaStream_t s) {
  (void)cudaGetLastError();  // report only the errors of these launches
  const int64_t chunks = resid_chunks(nvert);
  const int64_t nparts = nvert[2] * chunks;
  resid_plane_kernel<<<(unsigned)nparts, kResidThreads, 0, s>>>(rhs, nvert[0], nvert[1], nvert[2], chunks, scratch);
  resid_finalize_kernel<<<1, kResidThreads, 0, s>>>(scratch, nparts, nvert[0] * nvert[1] * nvert[2], res);
  return cudaGetLastError() == cudaSuccess ? FVM_OK : FVM_ERR_CUDA;
}

}  // namespace fvm

void fvm_internal_set_global_error(const char* msg);

extern "C" int fvm_residual_norms(const double* rhs_dev, const int64_t nvert[3], double* res_dev, void* stream) {
  if (!rhs_dev || !nvert || !res_dev) {
    fvm_internal_set_global_error("fvm_residual_norms: null argument");
    return FVM_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d)
    if (nvert[d] < 1) {
      fvm_internal_set_global_error("fvm_residual_norms: nvert must be >= 1");
      return FVM_ERR_INVALID;
    }
  if (nvert[2] > 0x7fffffff) {
    fvm_internal_set_global_error("fvm_residual_norms: nvert[2] above 2^31-1 planes");
    return FVM_ERR_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  if (cudaMalloc(&scratch, sizeof(double) * 5 * nvert[2] * fvm::resid_chunks(nvert)) != cudaSuccess) {
    (void)cudaGetLastError();
    fvm_internal_set_global_error("fvm_residual_norms: cudaMalloc of the per-plane scratch failed");
    return FVM_ERR_NOMEM;
  }
  int rc = fvm::residual_launch(rhs_dev, nvert, res_dev, scratch, s);
  if (rc) fvm_internal_set_global_error("fvm_residual_norms: kernel launch failed");
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    rc = FVM_ERR_CUDA;
    fvm_internal_set_global_error("fvm_residual_norms: the stream reported an error");
  }
  cudaFree(scratch);
  return rc;
}

// ---------------------------------------------------------------- no allocation
// fvm_residual_norms_noalloc: the same two kernels, with the per-plane sums in
// a fixed array that is part of the library image, for callers that may not
// allocate device memory themselves (their device memory belongs to an
// allocator they do not control: a host code that reserves the whole GPU
// budget for its own pool at start-up, or a runtime that forbids new
// allocations once a simulation runs). The array holds 4096 five-double
// partials (pieces of k planes, at most 4096 in all for blocks of up to
// kNoAllocMaxPlanes planes); every GPU that loads the library keeps these
// 160 KiB until the process exits.
namespace {

constexpr int64_t kNoAllocMaxPlanes = 4096;

static_assert(kNoAllocMaxPlanes <= fvm::kResidMaxParts, "every block the array accepts splits into at most its slots");
static __device__ __align__(256) double g_noalloc_plane_sums[fvm::kResidMaxParts * 5];

}  // namespace

extern "C" int fvm_residual_norms_noalloc(const double* rhs_dev, const int64_t nvert[3], double* res_dev,
                                          void* stream) {
  if (!rhs_dev || !nvert || !res_dev) {
    fvm_internal_set_global_error("fvm_residual_norms_noalloc: null argument");
    return FVM_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d)
    if (nvert[d] < 1) {
      fvm_internal_set_global_error("fvm_residual_norms_noalloc: nvert must be >= 1");
      return FVM_ERR_INVALID;
    }
  if (nvert[2] > kNoAllocMaxPlanes) {
    fvm_internal_set_global_error(
        "fvm_residual_norms_noalloc: nvert[2] exceeds 4096, the planes its fixed scratch array holds; "
        "use fvm_residual_norms");
    return FVM_ERR_INVALID;
  }
  // The array's device address on the current device. Its name in host code
  // is only a host-side stand-in, so the address is looked up here, with the
  // caller's device current, on every call: a host-side query that allocates
  // nothing and so never goes stale (after a cudaDeviceReset the module is
  // loaded again at a new address). The first call on a device loads the
  // library's device code there, which is why it belongs before any capture.
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_plane_sums);
  if (e != cudaSuccess || !p) {
    (void)cudaGetLastError();
    fvm_internal_set_global_error("fvm_residual_norms_noalloc: cudaGetSymbolAddress failed on the current device");
    return FVM_ERR_CUDA;
  }
  double* scratch = static_cast<double*>(p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = fvm::residual_launch(rhs_dev, nvert, res_dev, scratch, s);
  if (rc) fvm_internal_set_global_error("fvm_residual_norms_noalloc: kernel launch failed");
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    rc = FVM_ERR_CUDA;
    fvm_internal_set_global_error("fvm_residual_norms_noalloc: the stream reported an error");
  }
  return rc;
}
