// fvm_registry.cpp — maps (precision, reconstruction) to the instantiation
// objects built from fvm_stage_inst.cu.
#include "fvm_aux.h"

namespace fvm {

#define FVM_DECL(P, R) bool lookup_stage_p##P##_r##R(int dim, int flux, bool tb, int tile, StageKernelInfo* out);
FVM_DECL(0, 200) FVM_DECL(0, 201) FVM_DECL(0, 202)
FVM_DECL(1, 200) FVM_DECL(1, 201) FVM_DECL(1, 202)
FVM_DECL(2, 200) FVM_DECL(2, 201) FVM_DECL(2, 202)
#undef FVM_DECL

bool lookup_stage_kernel(int prec, int dim, int recon, int flux, bool tb, int tile, StageKernelInfo* out) {
#define FVM_CASE(P, R) \
  if (prec == P && recon == R) return lookup_stage_p##P##_r##R(dim, flux, tb, tile, out);
  FVM_CASE(0, 200) FVM_CASE(0, 201) FVM_CASE(0, 202)
  FVM_CASE(1, 200) FVM_CASE(1, 201) FVM_CASE(1, 202)
  FVM_CASE(2, 200) FVM_CASE(2, 201) FVM_CASE(2, 202)
#undef FVM_CASE
  return false;
}

}  // namespace fvm
