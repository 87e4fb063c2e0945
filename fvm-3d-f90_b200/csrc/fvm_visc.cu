// fvm_visc.cu — the FP64 and FP32 forms of the viscous kernel (fvm_visc.cuh),
// compiled with FMA contraction; the exact form lives in fvm_aux.cu.
#include "fvm_visc.cuh"

namespace fvm {

cudaError_t launch_visc_fast(const DevBlock* blocks, const DevCase* cases, const Task* tasks, int ntasks, int idim,
                             int prec, int role, cudaStream_t s, bool pdl) {
  if (prec == PREC_FP32) return launch_visc_prec<PREC_FP32>(blocks, cases, tasks, ntasks, idim, role, s, pdl);
  return launch_visc_prec<PREC_FP64>(blocks, cases, tasks, ntasks, idim, role, s, pdl);
}

cudaError_t visc_occupancy_fast(int prec, int* ctas_per_sm) {
  return prec == PREC_FP32 ? visc_occupancy_prec<PREC_FP32>(ctas_per_sm) : visc_occupancy_prec<PREC_FP64>(ctas_per_sm);
}

}  // namespace fvm
