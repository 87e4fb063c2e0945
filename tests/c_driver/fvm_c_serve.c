/* A plain-C host of the library's server (test infrastructure): submits three
 * requests at once through fvm_case_submit (an oblique shock tube, MUSCL +
 * Roe, SSP-RK3, transmissive faces; a periodic pressure pulse, WENO5 + AUSM,
 * classic RK4; the same pulse as a Navier-Stokes case, SSP-RK3), waits for
 * each with fvm_wait, reads the results with fvm_fetch_state, and compares
 * each, bit for bit, with the same case run alone through fvm_create /
 * fvm_step. Then it checks the error codes of the serving calls. Exit status
 * 0 means every check passed. This is the loop a C or Fortran host runs in
 * place of one solve_process per case. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fvm3d.h"

#define NI 20
#define NJ 12
#define NK 9
#define NV (5 * NI * NJ * NK)

static void initial_state(int kind, double* q) {
  const double g = 1.4;
  const size_t n = (size_t)NI * NJ * NK;
  for (int k = 0; k < NK; ++k)
    for (int j = 0; j < NJ; ++j)
      for (int i = 0; i < NI; ++i) {
        const double x = (i + 0.5) / NI, y = (j + 0.5) / NJ, z = (k + 0.5) / NK;
        double rho, p;
        if (kind) {
          const double r2 = (x - 0.4) * (x - 0.4) + (y - 0.5) * (y - 0.5) + (z - 0.6) * (z - 0.6);
          rho = 1.0;
          p = 1.0 + 0.3 * exp(-40.0 * r2);
        } else {
          const int left = 0.6 * x + 0.3 * y + 0.1 * z < 0.5;
          rho = left ? 1.0 : 0.125;
          p = left ? 1.0 : 0.1;
        }
        const size_t c = i + (size_t)NI * (j + (size_t)NJ * k);
        q[c + 0 * n] = rho;
        q[c + 1 * n] = 0.0;
        q[c + 2 * n] = 0.0;
        q[c + 3 * n] = 0.0;
        q[c + 4 * n] = p / (g - 1.0);
      }
}

static void make_config(int which, fvm_config* cfg) {
  fvm_config_default(cfg);
  cfg->idimension = 3;
  cfg->limiter = FVM_LIMITER_MINMOD;
  cfg->timestep_set = FVM_DT_CFL;
  cfg->cfl = 0.4;
  cfg->precision = FVM_PREC_FP64_EXACT;
  if (which == 0) {
    cfg->reconstruct = FVM_RECON_MUSCL;
    cfg->flux_split = FVM_FLUX_ROE;
    cfg->rk_stages = 3;
  } else if (which == 1) {
    cfg->reconstruct = FVM_RECON_WENO;
    cfg->flux_split = FVM_FLUX_AUSM;
    cfg->rk_stages = 4;
  } else {
    cfg->reconstruct = FVM_RECON_MUSCL;
    cfg->limiter = FVM_LIMITER_VANALBADA;
    cfg->flux_split = FVM_FLUX_ROE;
    cfg->rk_stages = 3;
    cfg->equation = FVM_EQ_NAVIER_STOKES;
    cfg->mu = 0.01;
  }
}

static const int64_t kSteps[3] = {5, 4, 6};

/* the case run alone through a context */
static int run_alone(int which, const double* q0, double* out) {
  fvm_ctx* ctx = NULL;
  fvm_config cfg;
  make_config(which, &cfg);
  const int64_t nv[3] = {NI, NJ, NK};
  const double dr[3] = {1.0 / NI, 1.0 / NJ, 1.0 / NK};
  int blk = -1;
  if (fvm_create(&cfg, &ctx) != FVM_OK) return 1;
  int rc = fvm_add_block(ctx, nv, dr, &blk);
  for (int region = 1; region <= 6 && !rc && which; ++region) rc = fvm_set_boundary(ctx, blk, region, FVM_BC_PERIODIC);
  if (!rc) rc = fvm_set_state(ctx, blk, q0);
  if (!rc) rc = fvm_step(ctx, (int)kSteps[which], NULL, NULL, NULL);
  if (!rc) rc = fvm_get_state(ctx, blk, out);
  fvm_destroy(ctx);
  return rc;
}

#define FAIL(...)                     \
  do {                                \
    fprintf(stderr, __VA_ARGS__);     \
    return 1;                         \
  } while (0)

int main(void) {
  static double q0[3][NV], served[3][NV], alone[3][NV];
  fvm_config cfg[3];
  int32_t bc[6][3];
  for (int r = 0; r < 6; ++r) {
    bc[r][0] = 0;
    bc[r][1] = r + 1;
    bc[r][2] = FVM_BC_PERIODIC;
  }
  const int64_t nv[3] = {NI, NJ, NK};
  const double dr[3] = {1.0 / NI, 1.0 / NJ, 1.0 / NK};

  fvm_server_config sc;
  if (fvm_server_config_default(&sc) != FVM_OK) FAIL("fvm_server_config_default\n");
  int64_t cells = 0;
  if (fvm_block_cells(3, nv, &cells) != FVM_OK) FAIL("fvm_block_cells\n");
  sc.budget_cells = 3 * cells;
  sc.chunk_steps = 2;
  fvm_server* srv = NULL;
  if (fvm_server_create(&sc, &srv) != FVM_OK) FAIL("fvm_server_create\n");

  int64_t id[3];
  for (int w = 0; w < 3; ++w) {
    initial_state(w != 0, q0[w]);
    make_config(w, &cfg[w]);
    const double* qp[1] = {q0[w]};
    fvm_request req;
    memset(&req, 0, sizeof req);
    req.struct_size = (int32_t)sizeof req;
    req.nblocks = 1;
    req.cfg = &cfg[w];
    req.nvert = nv;
    req.dr = dr;
    req.q = qp;
    req.nbc = w ? 6 : 0;
    req.bc = w ? &bc[0][0] : NULL;
    req.steps = kSteps[w];
    if (fvm_case_submit(srv, &req, &id[w]) != FVM_OK) FAIL("fvm_case_submit %d\n", w);
  }
  for (int w = 0; w < 3; ++w) {
    int state = -1, status = -1;
    int64_t done = 0;
    double t = 0.0, lat = 0.0;
    if (fvm_wait(srv, id[w], 120.0, &state) != FVM_OK) FAIL("fvm_wait %d\n", w);
    if (fvm_poll(srv, id[w], &state, &done, &t, &lat, &status) != FVM_OK) FAIL("fvm_poll %d\n", w);
    if (state != FVM_REQ_DONE || status != FVM_OK || done != kSteps[w] || !(t > 0.0) || !(lat > 0.0))
      FAIL("request %d: state %d status %d steps %lld\n", w, state, status, (long long)done);
    if (fvm_fetch_state(srv, id[w], 0, served[w]) != FVM_OK) FAIL("fvm_fetch_state %d\n", w);
    if (fvm_release(srv, id[w]) != FVM_OK) FAIL("fvm_release %d\n", w);
    if (run_alone(w, q0[w], alone[w]) != FVM_OK) FAIL("run alone %d\n", w);
    if (memcmp(served[w], alone[w], sizeof served[w]) != 0) FAIL("request %d differs from its run alone\n", w);
  }

  /* error codes: a released id is unknown, a request larger than the budget
   * is invalid, fetching an unfinished request is refused */
  if (fvm_poll(srv, id[0], NULL, NULL, NULL, NULL, NULL) != FVM_ERR_NOT_FOUND) FAIL("poll of a released id\n");
  if (fvm_release(srv, 12345) != FVM_ERR_NOT_FOUND) FAIL("release of an unknown id\n");
  {
    const int64_t big[3] = {64, 64, 64};
    static double qb[5 * 64 * 64 * 64];
    const double* qp[1] = {qb};
    fvm_request req;
    memset(&req, 0, sizeof req);
    req.struct_size = (int32_t)sizeof req;
    req.nblocks = 1;
    req.cfg = &cfg[0];
    req.nvert = big;
    req.dr = dr;
    req.q = qp;
    req.steps = 1;
    int64_t bid = -1;
    if (fvm_case_submit(srv, &req, &bid) != FVM_ERR_INVALID) FAIL("a request above the budget was accepted\n");
  }
  if (fvm_server_destroy(srv) != FVM_OK) FAIL("fvm_server_destroy\n");
  printf("served 3 requests, each equal to its run alone\n");
  return 0;
}
