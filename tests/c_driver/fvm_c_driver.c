/* A plain-C host of the library (test infrastructure): builds a 3D oblique
 * shock tube in one transmissive block and a periodic pressure pulse in a
 * second context, advances each a few steps through the C ABI, and prints
 * the initial state, the time, the residuals and every final state value as
 * exact hexadecimal floats,
 * so that a test can compare them with the same run made through the Python
 * bindings. It is what a C, C++ or Fortran host linking -lfvm3d does. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "fvm3d.h"

#define CHECK(call)                                                   \
  do {                                                                \
    int rc_ = (call);                                                 \
    if (rc_ != FVM_OK) {                                              \
      char msg_[512];                                                 \
      fvm_last_error(ctx, msg_, sizeof msg_);                         \
      fprintf(stderr, "%s failed: %d %s\n", #call, rc_, msg_);        \
      return 1;                                                       \
    }                                                                 \
  } while (0)

static void initial_state(int ni, int nj, int nk, int pulse, double* q) {
  const double g = 1.4;
  const size_t n = (size_t)ni * nj * nk;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const double x = (i + 0.5) / ni, y = (j + 0.5) / nj, z = (k + 0.5) / nk;
        double rho, p;
        if (pulse) {
          const double r2 = (x - 0.4) * (x - 0.4) + (y - 0.5) * (y - 0.5) + (z - 0.6) * (z - 0.6);
          rho = 1.0;
          p = 1.0 + 0.3 * exp(-40.0 * r2);
        } else {
          const int left = 0.6 * x + 0.3 * y + 0.1 * z < 0.5;
          rho = left ? 1.0 : 0.125;
          p = left ? 1.0 : 0.1;
        }
        const size_t c = i + (size_t)ni * (j + (size_t)nj * k);
        q[c + 0 * n] = rho;
        q[c + 1 * n] = 0.0;
        q[c + 2 * n] = 0.0;
        q[c + 3 * n] = 0.0;
        q[c + 4 * n] = p / (g - 1.0);
      }
}

static int run(int pulse) {
  fvm_ctx* ctx = NULL;
  fvm_config cfg;
  if (fvm_config_default(&cfg) != FVM_OK) return 1;
  cfg.idimension = 3;
  cfg.reconstruct = pulse ? FVM_RECON_WENO : FVM_RECON_MUSCL;
  cfg.limiter = FVM_LIMITER_MINMOD;
  cfg.flux_split = pulse ? FVM_FLUX_AUSM : FVM_FLUX_ROE;
  cfg.rk_stages = pulse ? 4 : 3;
  cfg.timestep_set = FVM_DT_CFL;
  cfg.cfl = 0.4;
  cfg.precision = FVM_PREC_FP64_EXACT;
  if (fvm_create(&cfg, &ctx) != FVM_OK) return 1;
  const int64_t nv[3] = {20, 12, 9};
  const double dr[3] = {1.0 / 20, 1.0 / 12, 1.0 / 9};
  int blk = -1;
  CHECK(fvm_add_block(ctx, nv, dr, &blk));
  if (pulse)
    for (int r = 1; r <= 6; ++r) CHECK(fvm_set_boundary(ctx, blk, r, FVM_BC_PERIODIC));
  const size_t n = 20 * 12 * 9;
  double* q = (double*)malloc(sizeof(double) * 5 * n);
  initial_state(20, 12, 9, pulse, q);
  printf("case %d init\n", pulse);
  for (size_t c = 0; c < 5 * n; ++c) printf("%a\n", q[c]);
  CHECK(fvm_set_state(ctx, blk, q));
  double t = 0.0, ra[6], rr[6];
  CHECK(fvm_step(ctx, 4, &t, ra, rr));
  CHECK(fvm_get_state(ctx, blk, q));
  printf("case %d t %a\n", pulse, t);
  for (int e = 0; e < 6; ++e) printf("res %a\n", ra[e]);
  for (size_t c = 0; c < 5 * n; ++c) printf("%a\n", q[c]);
  free(q);
  fvm_destroy(ctx);
  return 0;
}

int main(void) {
  if (fvm_abi_version() != FVM3D_ABI_VERSION) {
    fprintf(stderr, "ABI version mismatch\n");
    return 1;
  }
  if (run(0)) return 1;
  if (run(1)) return 1;
  return 0;
}
