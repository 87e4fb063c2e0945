// fvm_resid.cu — residual norms of one block's rhs held in device memory.
//
// Restates ClassIteration%compute_residual_sub (class_iteration.f90,
// file-local 210-248) for a caller that keeps rhs on the device:
//   res2(e) = sum(rhs(:,:,:,e)^2) / (ni*nj*nk),  res2_t = sum_e res2(e) / neq
//   R(e)    = sqrt(R(e)^2 + res2(e)),            R_t = sqrt(R_t^2 + res2_t)
// so repeated calls over the blocks of a case accumulate exactly as the
// reference does. The sum is deterministic: one CTA per k plane writes the
// plane's five sums (fixed-order tree inside the CTA), then one CTA adds the
// planes in k order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fvm3d.h"

namespace fvm {

constexpr int kResidThreads = 256;

__global__ void resid_plane_kernel(const double* __restrict__ rhs, int64_t ni, int64_t nj, int64_t nk,
                                   double* __restrict__ plane_sums) {
  __shared__ double red[5][kResidThreads];
  const int64_t k = blockIdx.x;
  const int64_t nplane = ni * nj;
  const int64_t nc = nplane * nk;
  double s[5] = {0, 0, 0, 0, 0};
  for (int64_t c = threadIdx.x; c < nplane; c += kResidThreads) {
#pragma unroll
    for (int e = 0; e < 5; ++e) {
      const double v = rhs[k * nplane + c + e * nc];
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
    for (int e = 0; e < 5; ++e) plane_sums[k * 5 + e] = red[e][0];
}

__global__ void resid_finalize_kernel(const double* __restrict__ plane_sums, int64_t ni, int64_t nj, int64_t nk,
                                      double* __restrict__ res) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double res2[5] = {0, 0, 0, 0, 0}, res2_t = 0.0;
  for (int e = 0; e < 5; ++e) {
    for (int64_t k = 0; k < nk; ++k) res2[e] = res2[e] + plane_sums[k * 5 + e];
    res2[e] = res2[e] / (double)(ni * nj * nk);
    res2_t = res2_t + res2[e];
  }
  res2_t = res2_t / 5.0;
  for (int e = 0; e < 5; ++e) res[e] = sqrt(res[e] * res[e] + res2[e]);
  res[5] = sqrt(res[5] * res[5] + res2_t);
}

int residual_launch(const double* rhs, const int64_t nvert[3], double* res, double* scratch, cudaStream_t s) {
  (void)cudaGetLastError();  // report only the errors of these launches
  resid_plane_kernel<<<(unsigned)nvert[2], kResidThreads, 0, s>>>(rhs, nvert[0], nvert[1], nvert[2], scratch);
  resid_finalize_kernel<<<1, 32, 0, s>>>(scratch, nvert[0], nvert[1], nvert[2], res);
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
  if (cudaMalloc(&scratch, sizeof(double) * 5 * nvert[2]) != cudaSuccess) {
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
// allocations once a simulation runs). The array holds one 5-double partial
// per k plane, so blocks up to kNoAllocMaxPlanes planes fit; every GPU that
// loads the library keeps these 160 KiB until the process exits.
namespace {

constexpr int64_t kNoAllocMaxPlanes = 4096;

static __device__ __align__(256) double g_noalloc_plane_sums[kNoAllocMaxPlanes * 5];

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
