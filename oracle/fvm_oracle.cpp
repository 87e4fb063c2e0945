// fvm_oracle.cpp — CPU oracle for the FVM-3D-F90 explicit residual-and-update path.
//
// TEST INFRASTRUCTURE ONLY. This is the checker the CUDA product is compared
// against (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg).
// The product library never links, loads or calls it.
//
// It restates, function by function and in the reference's operation order,
// the Fortran of the reference's hot path (paths relative to the reference
// project):
//   src/scheme/scheme_reconstruct_simple.f90:42-85     reconstruct_simple
//   src/scheme/scheme_reconstruct_MUSCL.f90:47-226     MUSCL + limiters
//   src/scheme/scheme_WENO.f90:28-121                  WENO_JS (as written)
//   src/scheme/scheme_FDS_Roe.f90:25-177               Roe + Harten fix
//   src/scheme/scheme_FVS_VanLeer.f90:25-126           Van Leer FVS
//   src/scheme/scheme_AUSM.f90:27-171                  AUSM
//   src/scheme/scheme_Runge_Kutta.f90:30-63            3-stage RK
//   src/solve/class_space_discret.f90:120-732          per-block, per-direction,
//                                                      per-line drivers + update_residual
//   src/solve/class_time_discret.f90:125-196           solve / Runge_Kutta
//   src/solve/class_flow_field.f90:328-474             q<->p, reset_q0, reset_rhs
//   src/base/defs_block_data.f90:204-256               reset_pool, update_ghost_cell
//   src/base/defs_ghost_cell.f90:79-227                ghost / real index maps
//   src/solve/class_iteration.f90 (file-local 195-259) residual norms
// The reference is built with -fdefault-real-8 (CMakeLists.txt:45), so every
// default-real literal there (0.5, 3.0/4.0, 1.0/3.0, AUSM's 0.1) is FP64 here.
// gfortran's sign(1.0,-0.0) = -1 is copysign. Build with -ffp-contract=off so
// every expression keeps the reference's left-to-right rounding order.
//
// PARITY UNPINNED against the reference binary: no Fortran compiler exists on
// this image or on the GPU hosts, and the reference's own tests hold no
// numbers (src/test/ is Fortran-language experiments only). The restatement is
// pinned instead by analytic known-answer tests (tests/test_oracle_kat.py).
//
// Features the reference does not implement (their oracle is a textbook
// restatement, marked EXTENSION below): CFL and local time steps, classic RK4,
// Navier-Stokes central viscous flux, periodic and block-to-block ghost
// exchange, TEXTBOOK compat (WENO5-JS as published, Van Leer FVS supersonic
// branches).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/fvm3d.h"

namespace {

struct Prim {  // defs_fluid_props.f90:64-70 (Primitive_Variable)
  double rho = 0.0, u = 0.0, v = 0.0, w = 0.0, press = 0.0;
};

inline double fsign1(double x) { return std::copysign(1.0, x); }
inline double fmin2(double a, double b) { return (b < a) ? b : a; }

// ---------------------------------------------------------------- limiters
// scheme_reconstruct_MUSCL.f90:177-184
double minmod(double x, double y, double b) {
  return 0.5 * (fsign1(x) + fsign1(y)) * fmin2(std::fabs(x), std::fabs(b * y));
}
// scheme_reconstruct_MUSCL.f90:198-205
double vanleer_lim(double x, double y) {
  const double eps = 1.0E-6;
  return (fsign1(x) + fsign1(y)) * x * y / (std::fabs(x) + std::fabs(y) + eps);
}
// scheme_reconstruct_MUSCL.f90:219-226
double vanalbada_lim(double x, double y) {
  const double eps = 1.0E-6;
  return (x * (y * y + eps) + y * (x * x + eps)) / (x * x + y * y + eps);
}

// scheme_reconstruct_MUSCL.f90:114-159 (MUSCL function)
double muscl(double p1, double p2, double p3, int wind, int limiter, double kappa) {
  double D_m = p2 - p1;
  double D_p = p3 - p2;
  double Db_m = 0.0, Db_p = 0.0;
  if (limiter == FVM_LIMITER_NONE || limiter == FVM_SCHEME_NULL) {
    Db_m = D_m;
    Db_p = D_p;
  } else if (limiter == FVM_LIMITER_MINMOD) {
    double b = 1.0;
    Db_m = minmod(D_m, D_p, b);
    Db_p = minmod(D_p, D_m, b);
  } else if (limiter == FVM_LIMITER_VANLEER) {
    Db_m = vanleer_lim(D_m, D_p);
    Db_p = Db_m;
  } else if (limiter == FVM_LIMITER_VANALBADA) {
    Db_m = vanalbada_lim(D_m, D_p);
    Db_p = Db_m;
  }
  if (wind == -1) return p2 + 0.25 * ((1.0 - kappa) * Db_m + (1.0 + kappa) * Db_p);
  return p2 - 0.25 * ((1.0 - kappa) * Db_p + (1.0 + kappa) * Db_m);
}

// scheme_WENO.f90:87-121 (WENO_JS). compat REFERENCE keeps IS_1's (u2+u4)^2
// (:107-108); TEXTBOOK uses Jiang & Shu's (u2-u4)^2.
double weno_js(const double* u, int compat) {
  const double c_0 = 0.1, c_1 = 0.6, c_2 = 0.3, eps = 1.0e-6;
  double q0 = 1.0 / 3.0 * u[0] - 7.0 / 6.0 * u[1] + 11.0 / 6.0 * u[2];
  double q1 = -1.0 / 6.0 * u[1] + 5.0 / 6.0 * u[2] + 1.0 / 3.0 * u[3];
  double q2 = 1.0 / 3.0 * u[2] + 5.0 / 6.0 * u[3] - 1.0 / 6.0 * u[4];
  double a0 = u[0] - 2.0 * u[1] + u[2];
  double b0 = u[0] - 4.0 * u[1] + 3.0 * u[2];
  double IS_0 = 13.0 / 12.0 * (a0 * a0) + 1.0 / 4.0 * (b0 * b0);
  double a1 = u[1] - 2.0 * u[2] + u[3];
  double b1 = (compat == FVM_COMPAT_REFERENCE) ? (u[1] + u[3]) : (u[1] - u[3]);
  double IS_1 = 13.0 / 12.0 * (a1 * a1) + 1.0 / 4.0 * (b1 * b1);
  double a2 = u[2] - 2.0 * u[3] + u[4];
  double b2 = 3.0 * u[2] - 4.0 * u[3] + u[4];
  double IS_2 = 13.0 / 12.0 * (a2 * a2) + 1.0 / 4.0 * (b2 * b2);
  double e0 = IS_0 + eps, e1 = IS_1 + eps, e2 = IS_2 + eps;
  double alpha_0 = c_0 / (e0 * e0);
  double alpha_1 = c_1 / (e1 * e1);
  double alpha_2 = c_2 / (e2 * e2);
  double alpha_sum = alpha_0 + alpha_1 + alpha_2;
  double omega_0 = alpha_0 / alpha_sum;
  double omega_1 = alpha_1 / alpha_sum;
  double omega_2 = alpha_2 / alpha_sum;
  return omega_0 * q0 + omega_1 * q1 + omega_2 * q2;
}

// ---------------------------------------------------------------- fluxes
// All three receive the face normal as the axis unit vector the drivers build
// (class_space_discret.f90:458-461: norm = 0, norm(:,dir) = 1).

// scheme_FDS_Roe.f90:151-159
inline double roe_avg(double rho_l, double rho_b, double q_r, double q_l) {
  return (rho_l * q_l + rho_b * q_r) / (rho_l + rho_b);
}
// scheme_FDS_Roe.f90:167-177
inline double entropy_correct(double lambda, double delta) {
  if (lambda > delta) return lambda;
  return 0.5 * (lambda * lambda + delta * delta) / delta;
}

// scheme_FDS_Roe.f90:25-138, one face.
void roe_face(double gamma, const double* n, const Prim& L, const Prim& R, double fix, double* F) {
  double rho_l = L.rho, u_l = L.u, v_l = L.v, w_l = L.w, p_l = L.press;
  double rho_r = R.rho, u_r = R.u, v_r = R.v, w_r = R.w, p_r = R.press;
  double Vc_l = u_l * n[0] + v_l * n[1] + w_l * n[2];
  double Vc_r = u_r * n[0] + v_r * n[1] + w_r * n[2];
  double H_l = gamma / (gamma - 1.0) * p_l / rho_l + 0.5 * (u_l * u_l + v_l * v_l + w_l * w_l);
  double H_r = gamma / (gamma - 1.0) * p_r / rho_r + 0.5 * (u_r * u_r + v_r * v_r + w_r * w_r);
  double drho = rho_r - rho_l, du = u_r - u_l, dv = v_r - v_l, dw = w_r - w_l;
  double dpress = p_r - p_l, dVl = Vc_r - Vc_l;
  double rho_b = std::sqrt(rho_l * rho_r);
  double u_b = roe_avg(rho_l, rho_b, u_r, u_l);
  double v_b = roe_avg(rho_l, rho_b, v_r, v_l);
  double w_b = roe_avg(rho_l, rho_b, w_r, w_l);
  double H_b = roe_avg(rho_l, rho_b, H_r, H_l);
  double Vl_b = u_b * n[0] + v_b * n[1] + w_b * n[2];
  double q2_b = u_b * u_b + v_b * v_b + w_b * w_b;
  double c_b = std::sqrt((gamma - 1.0) * (H_b - 0.5 * q2_b));
  double delta = fix * std::fabs(Vl_b + c_b);
  double lam1 = entropy_correct(std::fabs(Vl_b - c_b), delta);
  double lam2 = entropy_correct(std::fabs(Vl_b), delta);
  double lam5 = entropy_correct(std::fabs(Vl_b + c_b), delta);
  double d1[5], d234[5], d5[5], fl[5], fr[5];
  d1[0] = lam1 * (dpress - rho_b * c_b * dVl) / (2.0 * c_b * c_b);
  d1[1] = d1[0] * (u_b - c_b * n[0]);
  d1[2] = d1[0] * (v_b - c_b * n[1]);
  d1[3] = d1[0] * (w_b - c_b * n[2]);
  d1[4] = d1[0] * (H_b - c_b * Vl_b);
  d234[0] = lam2 * (drho - dpress / (c_b * c_b));
  d234[1] = d234[0] * u_b + lam2 * rho_b * (du - dVl * n[0]);
  d234[2] = d234[0] * v_b + lam2 * rho_b * (dv - dVl * n[1]);
  d234[3] = d234[0] * w_b + lam2 * rho_b * (dw - dVl * n[2]);
  d234[4] = d234[0] * 0.5 * q2_b + lam2 * rho_b * (u_b * du + v_b * dv + w_b * dw - Vl_b * dVl);
  d5[0] = lam5 * (dpress + rho_b * c_b * dVl) / (2.0 * c_b * c_b);
  d5[1] = d5[0] * (u_b + c_b * n[0]);
  d5[2] = d5[0] * (v_b + c_b * n[1]);
  d5[3] = d5[0] * (w_b + c_b * n[2]);
  d5[4] = d5[0] * (H_b + c_b * Vl_b);
  fl[0] = rho_l * Vc_l;
  fl[1] = rho_l * u_l * Vc_l + p_l * n[0];
  fl[2] = rho_l * v_l * Vc_l + p_l * n[1];
  fl[3] = rho_l * w_l * Vc_l + p_l * n[2];
  fl[4] = rho_l * H_l * Vc_l;
  fr[0] = rho_r * Vc_r;
  fr[1] = rho_r * u_r * Vc_r + p_r * n[0];
  fr[2] = rho_r * v_r * Vc_r + p_r * n[1];
  fr[3] = rho_r * w_r * Vc_r + p_r * n[2];
  fr[4] = rho_r * H_r * Vc_r;
  for (int e = 0; e < 5; ++e) F[e] = 0.5 * ((fl[e] + fr[e]) - (d1[e] + d234[e] + d5[e]));
}

// scheme_FVS_VanLeer.f90:101-126
double vanleer_mach_split(double Ma, double Mn, int wind) {
  if (wind == -1) {
    if (Mn >= 1.0) return Ma;
    if (Mn <= -1.0) return 0.0;
    return 0.25 * (Ma + 1.0) * (Ma + 1.0);
  }
  if (Mn >= 1.0) return 0.0;
  if (Mn <= -1.0) return Ma;
  return -(0.25 * (Ma - 1.0) * (Ma - 1.0));
}

// Physical Euler flux along n (used by the TEXTBOOK Van Leer supersonic branches).
void euler_flux(double gamma, const double* n, const Prim& s, double* F) {
  double Vc = s.u * n[0] + s.v * n[1] + s.w * n[2];
  double H = gamma / (gamma - 1.0) * s.press / s.rho + 0.5 * (s.u * s.u + s.v * s.v + s.w * s.w);
  F[0] = s.rho * Vc;
  F[1] = s.rho * s.u * Vc + s.press * n[0];
  F[2] = s.rho * s.v * Vc + s.press * n[1];
  F[3] = s.rho * s.w * Vc + s.press * n[2];
  F[4] = s.rho * H * Vc;
}

// scheme_FVS_VanLeer.f90:25-98, one face. REFERENCE keeps the subsonic
// momentum / energy factors in the supersonic branches (:84-95);
// TEXTBOOK switches to the full / zero flux there (EXTENSION).
void vanleer_face(double gamma, const double* n, const Prim& L, const Prim& R, int compat, double* F) {
  double rho_l = L.rho, u_l = L.u, v_l = L.v, w_l = L.w, p_l = L.press;
  double rho_r = R.rho, u_r = R.u, v_r = R.v, w_r = R.w, p_r = R.press;
  double Vc_l = u_l * n[0] + v_l * n[1] + w_l * n[2];
  double Vc_r = u_r * n[0] + v_r * n[1] + w_r * n[2];
  double q2_l = u_l * u_l + v_l * v_l + w_l * w_l;
  double q2_r = u_r * u_r + v_r * v_r + w_r * w_r;
  double c_l = std::sqrt(gamma * p_l / rho_l);
  double c_r = std::sqrt(gamma * p_r / rho_r);
  double M_l = Vc_l / c_l;
  double M_r = Vc_r / c_r;
  double fp[5], fm[5];
  if (compat == FVM_COMPAT_TEXTBOOK && M_l >= 1.0) {
    euler_flux(gamma, n, L, fp);
  } else if (compat == FVM_COMPAT_TEXTBOOK && M_l <= -1.0) {
    for (int e = 0; e < 5; ++e) fp[e] = 0.0;
  } else {
    double Ms = vanleer_mach_split(M_l, M_l, -1);
    fp[0] = rho_l * c_l * Ms;
    fp[1] = fp[0] * (n[0] * (-Vc_l + 2.0 * c_l) / gamma + u_l);
    fp[2] = fp[0] * (n[1] * (-Vc_l + 2.0 * c_l) / gamma + v_l);
    fp[3] = fp[0] * (n[2] * (-Vc_l + 2.0 * c_l) / gamma + w_l);
    double t = (gamma - 1.0) * Vc_l + 2.0 * c_l;
    fp[4] = fp[0] * (t * t / (2.0 * (gamma * gamma - 1.0)) + (q2_l - Vc_l * Vc_l) / 2.0);
  }
  if (compat == FVM_COMPAT_TEXTBOOK && M_r <= -1.0) {
    euler_flux(gamma, n, R, fm);
  } else if (compat == FVM_COMPAT_TEXTBOOK && M_r >= 1.0) {
    for (int e = 0; e < 5; ++e) fm[e] = 0.0;
  } else {
    double Ms = vanleer_mach_split(M_r, M_r, 1);
    fm[0] = rho_r * c_r * Ms;
    fm[1] = fm[0] * (n[0] * (-Vc_r - 2.0 * c_r) / gamma + u_r);
    fm[2] = fm[0] * (n[1] * (-Vc_r - 2.0 * c_r) / gamma + v_r);
    fm[3] = fm[0] * (n[2] * (-Vc_r - 2.0 * c_r) / gamma + w_r);
    double t = (gamma - 1.0) * Vc_r - 2.0 * c_r;
    fm[4] = fm[0] * (t * t / (2.0 * (gamma * gamma - 1.0)) + (q2_r - Vc_r * Vc_r) / 2.0);
  }
  for (int e = 0; e < 5; ++e) F[e] = fp[e] + fm[e];
}

// scheme_AUSM.f90:123-139 (beta = 0)
double mach_split_ausm(double Ma, int wind_) {
  const double beta = 0.0;
  double wind = (double)wind_;
  if (std::fabs(Ma) >= 1.0) return 0.5 * (Ma + wind * std::fabs(Ma));
  return wind * (0.25 * ((Ma + wind) * (Ma + wind)) + beta * ((Ma * Ma - 1.0) * (Ma * Ma - 1.0)));
}
// scheme_AUSM.f90:140-158 (alpha = 0)
double pressure_split_ausm(double p, double Ma, int wind_) {
  const double alpha = 0.0;
  double wind = (double)wind_;
  double p_s;
  if (std::fabs(Ma) >= 1.0) {
    p_s = 0.5 * (1.0 + wind * fsign1(Ma));
  } else {
    p_s = 0.25 * ((Ma + wind) * (Ma + wind)) * (2.0 - wind * Ma) +
          wind * alpha * Ma * ((Ma * Ma - 1.0) * (Ma * Ma - 1.0));
  }
  return p_s * p;
}
// scheme_AUSM.f90:160-171
double artificial_dissipation_ausm(double Mn_abs) {
  const double delta = 0.1;
  if (Mn_abs > delta) return Mn_abs;
  return 0.5 * (Mn_abs * Mn_abs + delta * delta) / delta;
}

// scheme_AUSM.f90:27-112, one face.
void ausm_face(double gamma, const double* n, const Prim& L, const Prim& R, double* F) {
  double rho_l = L.rho, u_l = L.u, v_l = L.v, w_l = L.w, p_l = L.press;
  double rho_r = R.rho, u_r = R.u, v_r = R.v, w_r = R.w, p_r = R.press;
  double Vc_l = u_l * n[0] + v_l * n[1] + w_l * n[2];
  double Vc_r = u_r * n[0] + v_r * n[1] + w_r * n[2];
  double H_l = gamma / (gamma - 1.0) * p_l / rho_l + 0.5 * (u_l * u_l + v_l * v_l + w_l * w_l);
  double H_r = gamma / (gamma - 1.0) * p_r / rho_r + 0.5 * (u_r * u_r + v_r * v_r + w_r * w_r);
  double c_l = std::sqrt(gamma * p_l / rho_l);
  double c_r = std::sqrt(gamma * p_r / rho_r);
  double M_l = Vc_l / c_l;
  double M_r = Vc_r / c_r;
  double Mn = mach_split_ausm(M_l, 1) + mach_split_ausm(M_r, -1);
  double Mn_abs = artificial_dissipation_ausm(std::fabs(Mn));
  double Phi_l[5], Phi_r[5];
  Phi_l[0] = rho_l * c_l;
  Phi_l[1] = Phi_l[0] * u_l;
  Phi_l[2] = Phi_l[0] * v_l;
  Phi_l[3] = Phi_l[0] * w_l;
  Phi_l[4] = Phi_l[0] * H_l;
  Phi_r[0] = rho_r * c_r;
  Phi_r[1] = Phi_r[0] * u_r;
  Phi_r[2] = Phi_r[0] * v_r;
  Phi_r[3] = Phi_r[0] * w_r;
  Phi_r[4] = Phi_r[0] * H_r;
  double p_ = pressure_split_ausm(p_l, M_l, 1) + pressure_split_ausm(p_r, M_r, -1);
  double norm_[5] = {0.0, n[0], n[1], n[2], 0.0};
  for (int e = 0; e < 5; ++e)
    F[e] = 0.5 * (Mn + Mn_abs) * Phi_l[e] + 0.5 * (Mn - Mn_abs) * Phi_r[e] + p_ * norm_[e];
}

// class_flow_field.f90:383-396 / 415-444 (convert_q_to_p_*)
inline Prim q_to_p(double gamma, const double* q, int64_t s) {
  Prim p;
  p.rho = q[0];
  p.u = q[s] / p.rho;
  p.v = q[2 * s] / p.rho;
  p.w = q[3 * s] / p.rho;
  p.press = (gamma - 1.0) * (q[4 * s] - 0.5 * p.rho * (p.u * p.u + p.v * p.v + p.w * p.w));
  return p;
}

// ---------------------------------------------------------------- blocks
struct Conn {  // one fvm_connect call
  int64_t range[3][2];
  int donor;
  int64_t drange[3][2];
  int dtype[3];
};

struct Block {
  int64_t n[3] = {1, 1, 1};  // real nvert
  int64_t g[3] = {7, 7, 7};  // ghost nvert = n + 6 (defs_ghost_cell.f90:79-90)
  double dr[3] = {1.0, 1.0, 1.0};
  int bc[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> q;     // q(g0,g1,g2,5), ghost mesh (defs_block_data.f90:141)
  std::vector<Prim> p;       // p(g0,g1,g2), ghost mesh (defs_block_data.f90:144)
  std::vector<double> q0;    // q0(n0,n1,n2,5) (defs_block_data.f90:127)
  std::vector<double> rhs;   // rhs(n0,n1,n2,5) (defs_block_data.f90:130)
  std::vector<double> acc;   // RK4 accumulator (EXTENSION)
  std::vector<double> dtl;   // local time step per real cell (EXTENSION)
  std::vector<Conn> conns;
  int64_t gvol() const { return g[0] * g[1] * g[2]; }
  int64_t rvol() const { return n[0] * n[1] * n[2]; }
  // 0-based real-cell indices (may be -3..n+2) -> ghost-mesh linear index
  int64_t gidx(int64_t i, int64_t j, int64_t k) const {
    return (i + 3) + g[0] * ((j + 3) + g[1] * (k + 3));
  }
  int64_t ridx(int64_t i, int64_t j, int64_t k) const { return i + n[0] * (j + n[1] * k); }
};

}  // namespace

struct orc_ctx {
  fvm_config cfg;
  std::vector<Block> blocks;
  double time = 0.0;
  double dt_last = 0.0;
  int64_t step = 0;
  double res_abs[6] = {0, 0, 0, 0, 0, 0};
  double res_abs0[6] = {0, 0, 0, 0, 0, 0};
  double res_rel[6] = {0, 0, 0, 0, 0, 0};
  std::string err;
};

namespace {

int fail(orc_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

// ---------------------------------------------------------------- ghosts
// defs_block_data.f90:226-256 (update_ghost_cell_sub) restricted to the
// regions whose kind is transmissive, with the layer ranges of
// defs_ghost_cell.f90:122-166.
void ghost_transmissive(Block& b) {
  for (int region = 1; region <= 6; ++region) {
    if (b.bc[region - 1] != FVM_BC_TRANSMISSIVE) continue;
    for (int ilayer = 1; ilayer <= 3; ++ilayer) {
      // layer(:,1..2) = real range in ghost-mesh 1-based numbering
      int64_t lo[3], hi[3], nrm[3] = {0, 0, 0};
      for (int d = 0; d < 3; ++d) {
        lo[d] = 1 + 3;
        hi[d] = b.g[d] - 3;
      }
      int ax = (region - 1) / 2;
      if ((region - 1) % 2 == 0) {
        lo[ax] = 1 + 3 - ilayer;
        hi[ax] = lo[ax];
        nrm[ax] = -1;
      } else {
        hi[ax] = b.g[ax] - 3 + ilayer;
        lo[ax] = hi[ax];
        nrm[ax] = 1;
      }
      for (int64_t k = lo[2]; k <= hi[2]; ++k)
        for (int64_t j = lo[1]; j <= hi[1]; ++j)
          for (int64_t i = lo[0]; i <= hi[0]; ++i) {
            // this%p(i,j,k) = this%p(i-di,j-dj,k-dk), d* = layer(:,3)*ilayer:
            // every layer copies the real boundary cell.
            int64_t si = i - nrm[0] * ilayer, sj = j - nrm[1] * ilayer, sk = k - nrm[2] * ilayer;
            int64_t dst = (i - 1) + b.g[0] * ((j - 1) + b.g[1] * (k - 1));
            int64_t src = (si - 1) + b.g[0] * ((sj - 1) + b.g[1] * (sk - 1));
            b.p[dst] = b.p[src];
            for (int e = 0; e < 5; ++e) b.q[dst + e * b.gvol()] = b.q[src + e * b.gvol()];
          }
    }
  }
}

// Block-to-block / periodic ghost fill (EXTENSION: the reference keeps the
// connection metadata, defs_face_geom.f90:378-402, but moves no data).
void ghost_connections(std::vector<Block>& blocks) {
  for (auto& b : blocks) {
    for (const auto& c : b.conns) {
      const Block& d = blocks[c.donor];
      for (int64_t k = c.range[2][0]; k <= c.range[2][1]; ++k)
        for (int64_t j = c.range[1][0]; j <= c.range[1][1]; ++j)
          for (int64_t i = c.range[0][0]; i <= c.range[0][1]; ++i) {
            int64_t x[3] = {i, j, k}, y[3];
            for (int a = 0; a < 3; ++a) {
              int da = std::abs(c.dtype[a]) - 1;
              int64_t s = c.dtype[a] > 0 ? 1 : -1;
              y[da] = c.drange[a][0] + s * (x[a] - c.range[a][0]);
            }
            int64_t dst = b.gidx(i, j, k), src = d.gidx(y[0], y[1], y[2]);
            b.p[dst] = d.p[src];
            for (int e = 0; e < 5; ++e) b.q[dst + e * b.gvol()] = d.q[src + e * d.gvol()];
          }
    }
  }
}

// Layer-1 edge ghosts, needed by the viscous stencil only (EXTENSION).
// An edge cell outside the block along axes a < b is copied, after the face
// ghosts are in place, from the cell the face-a rule maps it to.
void ghost_edges(std::vector<Block>& blocks) {
  for (size_t bi = 0; bi < blocks.size(); ++bi) {
    Block& b = blocks[bi];
    for (int a = 0; a < 3; ++a)
      for (int bb = a + 1; bb < 3; ++bb) {
        int c3 = 3 - a - bb;
        for (int sa = 0; sa < 2; ++sa)
          for (int sb = 0; sb < 2; ++sb)
            for (int64_t t = 0; t < b.n[c3]; ++t) {
              int64_t x[3];
              x[a] = sa ? b.n[a] : -1;
              x[bb] = sb ? b.n[bb] : -1;
              x[c3] = t;
              int region = 2 * a + sa + 1;
              int src_blk = (int)bi;
              int64_t y[3] = {x[0], x[1], x[2]};
              if (b.bc[region - 1] == FVM_BC_TRANSMISSIVE) {
                y[a] = sa ? b.n[a] - 1 : 0;
              } else {
                // the connection on this region whose box holds x when x[bb]
                // is clamped into the block
                int64_t xc[3] = {x[0], x[1], x[2]};
                xc[bb] = std::min<int64_t>(std::max<int64_t>(xc[bb], 0), b.n[bb] - 1);
                const Conn* hit = nullptr;
                for (const auto& c : b.conns) {
                  bool in = true;
                  for (int d = 0; d < 3; ++d) in = in && xc[d] >= c.range[d][0] && xc[d] <= c.range[d][1];
                  if (in) {
                    hit = &c;
                    break;
                  }
                }
                if (!hit) continue;
                for (int d = 0; d < 3; ++d) {
                  int dd = std::abs(hit->dtype[d]) - 1;
                  int64_t s = hit->dtype[d] > 0 ? 1 : -1;
                  y[dd] = hit->drange[d][0] + s * (x[d] - hit->range[d][0]);
                }
                src_blk = hit->donor;
              }
              const Block& d = blocks[src_blk];
              int64_t dst = b.gidx(x[0], x[1], x[2]), src = d.gidx(y[0], y[1], y[2]);
              b.p[dst] = d.p[src];
              for (int e = 0; e < 5; ++e) b.q[dst + e * b.gvol()] = d.q[src + e * d.gvol()];
            }
      }
  }
}

// class_flow_field.f90:328-340 (update_primitive_sub): q->p on the real
// range of every block, then the ghost layers.
void flow_update(orc_ctx* c) {
  const double gamma = c->cfg.gamma;
  for (auto& b : c->blocks) {
    const int64_t gv = b.gvol();
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t k = 0; k < b.n[2]; ++k)
      for (int64_t j = 0; j < b.n[1]; ++j)
        for (int64_t i = 0; i < b.n[0]; ++i) {
          int64_t g = b.gidx(i, j, k);
          b.p[g] = q_to_p(gamma, &b.q[g], gv);
        }
  }
  for (auto& b : c->blocks) ghost_transmissive(b);
  ghost_connections(c->blocks);
  if (c->cfg.equation == FVM_EQ_NAVIER_STOKES) ghost_edges(c->blocks);
}

// ---------------------------------------------------------------- space discretisation
// One direction of one block: per line, reconstruct (class_space_discret.f90:
// 179-424 + scheme_*), flux (:427-668 + scheme_*), then update_residual
// (:678-732) for the cells of that line. The reference runs recon for all
// lines, then flux for all lines, then update_residual; every step is
// line-local, so the per-line order gives the same numbers.
void inviscid_dir(orc_ctx* c, Block& b, int dir) {
  const fvm_config& cfg = c->cfg;
  const int64_t nd = b.n[dir];
  const int64_t nface = nd + 1;           // defs_ghost_cell.f90:198-204
  const int64_t dghost = 3;               // map_ijk (defs_ghost_cell.f90:221-227)
  const int t1 = (dir == 0) ? 1 : 0;
  const int t2 = (dir == 2) ? 1 : 2;
  const int64_t gv = b.gvol();
  const int64_t rv = b.rvol();
  double norm[3] = {0.0, 0.0, 0.0};
  norm[dir] = 1.0;
  int64_t gstride[3] = {1, b.g[0], b.g[0] * b.g[1]};
  const double drd = b.dr[dir];
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t l2 = 0; l2 < b.n[t2]; ++l2)
    for (int64_t l1 = 0; l1 < b.n[t1]; ++l1) {
      int64_t x[3];
      x[dir] = -3;
      x[t1] = l1;
      x[t2] = l2;
      const int64_t g0 = b.gidx(x[0], x[1], x[2]);  // ghost index 1 of the line
      const int64_t gs = gstride[dir];
      const int64_t ng = nd + 6;
      std::vector<Prim> pm(nface), pp(nface);
      if (cfg.reconstruct == FVM_RECON_SIMPLE) {
        // scheme_reconstruct_simple.f90:42-85: p_r(iface) = p_ghost(iface+dghost+dw)
        for (int64_t f = 1; f <= nface; ++f) {
          pm[f - 1] = b.p[g0 + (f + dghost - 1 - 1) * gs];
          pp[f - 1] = b.p[g0 + (f + dghost - 1) * gs];
        }
      } else if (cfg.reconstruct == FVM_RECON_MUSCL) {
        // scheme_reconstruct_MUSCL.f90:47-104
        for (int wind = -1; wind <= 1; wind += 2) {
          int64_t st0 = (wind == -1) ? -1 : 0;
          std::vector<Prim>& out = (wind == -1) ? pm : pp;
          for (int64_t f = 1; f <= nface; ++f) {
            int64_t ig = f + dghost - 1;
            const Prim& a = b.p[g0 + (ig + st0 - 1) * gs];
            const Prim& m = b.p[g0 + (ig + st0 + 1 - 1) * gs];
            const Prim& z = b.p[g0 + (ig + st0 + 2 - 1) * gs];
            Prim r;
            r.rho = muscl(a.rho, m.rho, z.rho, wind, cfg.limiter, cfg.kappa);
            r.u = muscl(a.u, m.u, z.u, wind, cfg.limiter, cfg.kappa);
            r.v = muscl(a.v, m.v, z.v, wind, cfg.limiter, cfg.kappa);
            r.w = muscl(a.w, m.w, z.w, wind, cfg.limiter, cfg.kappa);
            r.press = muscl(a.press, m.press, z.press, wind, cfg.limiter, cfg.kappa);
            out[f - 1] = r;
          }
        }
      } else {
        // scheme_WENO.f90:28-72 on the conservative line, then
        // convert_q_to_p_line_sub (class_flow_field.f90:415-428)
        std::vector<double> line(ng * 5);
        for (int e = 0; e < 5; ++e)
          for (int64_t i = 0; i < ng; ++i) line[e * ng + i] = b.q[g0 + i * gs + e * gv];
        double qr[5];
        for (int wind = -1; wind <= 1; wind += 2) {
          std::vector<Prim>& out = (wind == -1) ? pm : pp;
          for (int64_t f = 1; f <= nface; ++f) {
            int64_t ig = f + dghost - 1;
            for (int e = 0; e < 5; ++e) {
              double u[5];
              if (wind == -1 || cfg.compat == FVM_COMPAT_REFERENCE) {
                // stencil (-2,2) / (-1,3), same left-biased formula
                int64_t lo = ig + ((wind == -1) ? -2 : -1);
                for (int s = 0; s < 5; ++s) u[s] = line[e * ng + (lo + s - 1)];
              } else {
                // TEXTBOOK: mirror image for the right state of face f
                for (int s = 0; s < 5; ++s) u[s] = line[e * ng + (ig + 3 - s - 1)];
              }
              qr[e] = weno_js(u, cfg.compat);
            }
            out[f - 1] = q_to_p(cfg.gamma, qr, 1);
          }
        }
      }
      // TEXTBOOK only (EXTENSION): a reconstructed state with non-positive
      // density or pressure falls back to the first-order state of its cell
      if (cfg.compat == FVM_COMPAT_TEXTBOOK && cfg.reconstruct != FVM_RECON_SIMPLE) {
        for (int64_t f = 1; f <= nface; ++f) {
          if (!(pm[f - 1].rho > 0.0 && pm[f - 1].press > 0.0)) pm[f - 1] = b.p[g0 + (f + dghost - 1 - 1) * gs];
          if (!(pp[f - 1].rho > 0.0 && pp[f - 1].press > 0.0)) pp[f - 1] = b.p[g0 + (f + dghost - 1) * gs];
        }
      }
      // flux (scheme_FDS_Roe / scheme_FVS_VanLeer / scheme_AUSM)
      std::vector<double> flux(nface * 5);
      for (int64_t f = 0; f < nface; ++f) {
        double F[5];
        if (cfg.flux_split == FVM_FLUX_ROE)
          roe_face(cfg.gamma, norm, pm[f], pp[f], cfg.entropy_fix, F);
        else if (cfg.flux_split == FVM_FLUX_VANLEER)
          vanleer_face(cfg.gamma, norm, pm[f], pp[f], cfg.compat, F);
        else
          ausm_face(cfg.gamma, norm, pm[f], pp[f], F);
        for (int e = 0; e < 5; ++e) flux[f * 5 + e] = F[e];
      }
      // update_residual (class_space_discret.f90:704-723)
      for (int64_t i = 0; i < nd; ++i) {
        int64_t y[3];
        y[dir] = i;
        y[t1] = l1;
        y[t2] = l2;
        int64_t r = b.ridx(y[0], y[1], y[2]);
        for (int e = 0; e < 5; ++e)
          b.rhs[r + e * rv] = b.rhs[r + e * rv] - (flux[(i + 1) * 5 + e] - flux[i * 5 + e]) / drd;
      }
    }
}

// Central second-order viscous flux (EXTENSION; the reference's
// viscous_flux_sub, class_space_discret.f90:671-675, is empty). The per-cell
// contribution V = (dGx + dGy) + dGz is summed first and then added to the
// inviscid rhs, rhs = rhs + V. Face gradients:
// normal derivative from the two adjacent cells, tangential derivatives as
// the mean of the two cells' central differences. tau with Stokes'
// hypothesis; heat flux k dT/dx = mu*gamma/(Pr*(gamma-1)) d(p/rho)/dx.
void viscous_dir(orc_ctx* c, Block& b, int dir, std::vector<double>& V) {
  const fvm_config& cfg = c->cfg;
  const int idim = cfg.idimension;
  const int64_t nd = b.n[dir];
  const int64_t rv = b.rvol();
  const int t1 = (dir == 0) ? 1 : 0;
  const int t2 = (dir == 2) ? 1 : 2;
  const double mu = cfg.mu;
  const double kq = cfg.mu * cfg.gamma / (cfg.prandtl * (cfg.gamma - 1.0));
  int64_t gstride[3] = {1, b.g[0], b.g[0] * b.g[1]};
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t l2 = 0; l2 < b.n[t2]; ++l2)
    for (int64_t l1 = 0; l1 < b.n[t1]; ++l1) {
      std::vector<double> fv((nd + 1) * 5);
      for (int64_t f = 0; f <= nd; ++f) {
        int64_t x[3];
        x[dir] = f - 1;
        x[t1] = l1;
        x[t2] = l2;
        const int64_t gL = b.gidx(x[0], x[1], x[2]);
        const int64_t gR = gL + gstride[dir];
        const Prim& L = b.p[gL];
        const Prim& R = b.p[gR];
        // gradient[m][d] of (u,v,w,theta) at the face
        double grad[4][3];
        double vl[4] = {L.u, L.v, L.w, L.press / L.rho};
        double vr[4] = {R.u, R.v, R.w, R.press / R.rho};
        for (int m = 0; m < 4; ++m)
          for (int d = 0; d < 3; ++d) grad[m][d] = 0.0;
        for (int m = 0; m < 4; ++m) grad[m][dir] = (vr[m] - vl[m]) / b.dr[dir];
        for (int d = 0; d < idim; ++d) {
          if (d == dir) continue;
          const int64_t s = gstride[d];
          const Prim& Lp = b.p[gL + s];
          const Prim& Lm = b.p[gL - s];
          const Prim& Rp = b.p[gR + s];
          const Prim& Rm = b.p[gR - s];
          double lp[4] = {Lp.u, Lp.v, Lp.w, Lp.press / Lp.rho};
          double lm[4] = {Lm.u, Lm.v, Lm.w, Lm.press / Lm.rho};
          double rp[4] = {Rp.u, Rp.v, Rp.w, Rp.press / Rp.rho};
          double rm[4] = {Rm.u, Rm.v, Rm.w, Rm.press / Rm.rho};
          for (int m = 0; m < 4; ++m)
            grad[m][d] = ((lp[m] - lm[m]) + (rp[m] - rm[m])) / (4.0 * b.dr[d]);
        }
        double div = grad[0][0] + grad[1][1] + grad[2][2];
        double uf[3] = {0.5 * (L.u + R.u), 0.5 * (L.v + R.v), 0.5 * (L.w + R.w)};
        double tau[3];
        for (int m = 0; m < 3; ++m) {
          tau[m] = mu * (grad[m][dir] + grad[dir][m]);
          if (m == dir) tau[m] = tau[m] - 2.0 / 3.0 * mu * div;
        }
        fv[f * 5 + 0] = 0.0;
        fv[f * 5 + 1] = tau[0];
        fv[f * 5 + 2] = tau[1];
        fv[f * 5 + 3] = tau[2];
        fv[f * 5 + 4] = uf[0] * tau[0] + uf[1] * tau[1] + uf[2] * tau[2] + kq * grad[3][dir];
      }
      for (int64_t i = 0; i < nd; ++i) {
        int64_t y[3];
        y[dir] = i;
        y[t1] = l1;
        y[t2] = l2;
        int64_t r = b.ridx(y[0], y[1], y[2]);
        for (int e = 0; e < 5; ++e) V[r + e * rv] = V[r + e * rv] + (fv[(i + 1) * 5 + e] - fv[i * 5 + e]) / b.dr[dir];
      }
    }
}

// Max over real cells of sum_d (|u_d| + c) / dr_d (EXTENSION: CFL time step,
// "Not implemented yet" in class_time_discret.f90:101-104).
double cell_wavespeed(const fvm_config& cfg, const Block& b, const Prim& p) {
  double c = std::sqrt(cfg.gamma * p.press / p.rho);
  double s = (std::fabs(p.u) + c) / b.dr[0] + (std::fabs(p.v) + c) / b.dr[1];
  if (cfg.idimension == 3) s = s + (std::fabs(p.w) + c) / b.dr[2];
  return s;
}

// class_time_discret.f90:111-122 (timestep_fun) + EXTENSION CFL modes.
double timestep(orc_ctx* c) {
  const fvm_config& cfg = c->cfg;
  if (cfg.timestep_set == FVM_DT_FIXED) return cfg.dt;
  double smax = 0.0;
  for (auto& b : c->blocks) {
    if (cfg.timestep_set == FVM_DT_CFL_LOCAL) b.dtl.assign(b.rvol(), 0.0);
    for (int64_t k = 0; k < b.n[2]; ++k)
      for (int64_t j = 0; j < b.n[1]; ++j)
        for (int64_t i = 0; i < b.n[0]; ++i) {
          double s = cell_wavespeed(cfg, b, b.p[b.gidx(i, j, k)]);
          smax = std::max(smax, s);
          if (cfg.timestep_set == FVM_DT_CFL_LOCAL) b.dtl[b.ridx(i, j, k)] = cfg.cfl / s;
        }
  }
  return cfg.cfl / smax;
}

// scheme_Runge_Kutta.f90:30-63 (3 stages) and classic RK4 (EXTENSION) for
// one block. dt is the global step or, for local stepping, dtl per cell.
void rk_update(orc_ctx* c, Block& b, int m, double dt) {
  const fvm_config& cfg = c->cfg;
  const int64_t rv = b.rvol();
  const int64_t gv = b.gvol();
  const bool local = cfg.timestep_set == FVM_DT_CFL_LOCAL;
  const double a2_1 = 3.0 / 4.0, a2_2 = 1.0 / 4.0, a2_3 = 1.0 / 4.0;
  const double a3_1 = 1.0 / 3.0, a3_2 = 2.0 / 3.0, a3_3 = 2.0 / 3.0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = 0; k < b.n[2]; ++k)
    for (int64_t j = 0; j < b.n[1]; ++j)
      for (int64_t i = 0; i < b.n[0]; ++i) {
        const int64_t r = b.ridx(i, j, k);
        const int64_t g = b.gidx(i, j, k);
        const double h = local ? b.dtl[r] : dt;
        for (int e = 0; e < 5; ++e) {
          double u0 = b.q0[r + e * rv];
          double um = b.q[g + e * gv];
          double rm = b.rhs[r + e * rv];
          double out;
          if (cfg.rk_stages == 3) {
            if (m == 1)
              out = u0 + h * rm;
            else if (m == 2)
              out = a2_1 * u0 + a2_2 * um + a2_3 * h * rm;
            else
              out = a3_1 * u0 + a3_2 * um + a3_3 * h * rm;
          } else {
            // classic RK4, q0 folded into the accumulator (low storage: the
            // last stage reads acc, not q0)
            double& acc = b.acc[r + e * rv];
            if (m == 1) {
              acc = u0 + h / 6.0 * rm;
              out = u0 + 0.5 * h * rm;
            } else if (m == 2) {
              acc = acc + h / 3.0 * rm;
              out = u0 + 0.5 * h * rm;
            } else if (m == 3) {
              acc = acc + h / 3.0 * rm;
              out = u0 + h * rm;
            } else {
              out = acc + h / 6.0 * rm;
            }
          }
          b.q[g + e * gv] = out;
        }
      }
}

// class_iteration.f90 (file-local 195-259): reset_residual, compute_residual
// per block in block order, update (relative to step 1).
void residual(orc_ctx* c) {
  for (int e = 0; e < 6; ++e) c->res_abs[e] = 0.0;
  for (auto& b : c->blocks) {
    const int64_t rv = b.rvol();
    double res2[5] = {0, 0, 0, 0, 0};
    double res2_t = 0.0;
    for (int e = 0; e < 5; ++e) {
      for (int64_t k = 0; k < b.n[2]; ++k)
        for (int64_t j = 0; j < b.n[1]; ++j)
          for (int64_t i = 0; i < b.n[0]; ++i) {
            double v = b.rhs[b.ridx(i, j, k) + e * rv];
            res2[e] = res2[e] + v * v;
          }
      res2[e] = res2[e] / (double)rv;
      res2_t = res2_t + res2[e];
    }
    res2_t = res2_t / 5.0;
    for (int e = 0; e < 5; ++e) c->res_abs[e] = std::sqrt(c->res_abs[e] * c->res_abs[e] + res2[e]);
    c->res_abs[5] = std::sqrt(c->res_abs[5] * c->res_abs[5] + res2_t);
  }
  if (c->step == 1)
    for (int e = 0; e < 6; ++e) c->res_abs0[e] = c->res_abs[e];
  for (int e = 0; e < 6; ++e) c->res_rel[e] = c->res_abs[e] / c->res_abs0[e];
}

// class_time_discret.f90:125-196 (solve_sub + Runge_Kutta_sub).
void solve_one(orc_ctx* c) {
  const fvm_config& cfg = c->cfg;
  c->step += 1;
  double dt = timestep(c);
  c->dt_last = dt;
  c->time = c->time + dt;
  // reset_q0 (class_flow_field.f90:447-460)
  for (auto& b : c->blocks) {
    const int64_t rv = b.rvol(), gv = b.gvol();
    for (int e = 0; e < 5; ++e)
      for (int64_t k = 0; k < b.n[2]; ++k)
        for (int64_t j = 0; j < b.n[1]; ++j)
          for (int64_t i = 0; i < b.n[0]; ++i)
            b.q0[b.ridx(i, j, k) + e * rv] = b.q[b.gidx(i, j, k) + e * gv];
  }
  for (int m = 1; m <= cfg.rk_stages; ++m) {
    for (auto& b : c->blocks) std::fill(b.rhs.begin(), b.rhs.end(), 0.0);  // reset_rhs
    for (auto& b : c->blocks)
      for (int dir = 0; dir < cfg.idimension; ++dir) inviscid_dir(c, b, dir);
    if (cfg.equation == FVM_EQ_NAVIER_STOKES)
      for (auto& b : c->blocks) {
        std::vector<double> V(b.rhs.size(), 0.0);
        for (int dir = 0; dir < cfg.idimension; ++dir) viscous_dir(c, b, dir, V);
        for (size_t i = 0; i < V.size(); ++i) b.rhs[i] = b.rhs[i] + V[i];
      }
    for (auto& b : c->blocks) rk_update(c, b, m, dt);
    flow_update(c);
  }
  residual(c);
}

bool valid_perm(const int32_t* t) {
  int seen = 0;
  for (int a = 0; a < 3; ++a) {
    int d = std::abs(t[a]);
    if (d < 1 || d > 3) return false;
    seen |= 1 << (d - 1);
  }
  return seen == 7;
}

}  // namespace

// ---------------------------------------------------------------- C API
extern "C" {

orc_ctx* orc_create(const fvm_config* cfg) {
  if (!cfg) return nullptr;
  orc_ctx* c = new orc_ctx();
  c->cfg = *cfg;
  return c;
}

void orc_destroy(orc_ctx* c) { delete c; }

const char* orc_last_error(orc_ctx* c) { return c ? c->err.c_str() : ""; }

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_add_block(orc_ctx* c, const int64_t* n, const double* dr) {
  Block b;
  for (int d = 0; d < 3; ++d) {
    if (n[d] < 1) return -fail(c, FVM_ERR_INVALID, "nvert < 1");
    b.n[d] = n[d];
    b.g[d] = n[d] + 6;
    b.dr[d] = dr[d];
  }
  b.q.assign(b.gvol() * 5, 0.0);
  b.p.assign(b.gvol(), Prim());
  b.q0.assign(b.rvol() * 5, 0.0);
  b.rhs.assign(b.rvol() * 5, 0.0);
  if (c->cfg.rk_stages == 4) b.acc.assign(b.rvol() * 5, 0.0);
  c->blocks.push_back(std::move(b));
  return (int)c->blocks.size() - 1;
}

int orc_set_boundary(orc_ctx* c, int blk, int region, int kind) {
  if (blk < 0 || blk >= (int)c->blocks.size() || region < 1 || region > 6)
    return fail(c, FVM_ERR_INVALID, "bad block or region");
  Block& b = c->blocks[blk];
  // drop earlier connections of this region
  int ax = (region - 1) / 2;
  bool hi = (region - 1) % 2 == 1;
  std::vector<Conn> keep;
  for (auto& cn : b.conns) {
    bool same = hi ? (cn.range[ax][0] >= b.n[ax]) : (cn.range[ax][1] < 0);
    if (!same) keep.push_back(cn);
  }
  b.conns = keep;
  b.bc[region - 1] = kind;
  if (kind == FVM_BC_PERIODIC) {
    Conn cn;
    for (int d = 0; d < 3; ++d) {
      cn.range[d][0] = 0;
      cn.range[d][1] = b.n[d] - 1;
      cn.drange[d][0] = 0;
      cn.drange[d][1] = b.n[d] - 1;
      cn.dtype[d] = d + 1;
    }
    if (hi) {
      cn.range[ax][0] = b.n[ax];
      cn.range[ax][1] = b.n[ax] + 2;
      cn.drange[ax][0] = 0;
      cn.drange[ax][1] = 2;
    } else {
      cn.range[ax][0] = -3;
      cn.range[ax][1] = -1;
      cn.drange[ax][0] = b.n[ax] - 3;
      cn.drange[ax][1] = b.n[ax] - 1;
    }
    cn.donor = blk;
    b.conns.push_back(cn);
  }
  return FVM_OK;
}

int orc_connect(orc_ctx* c, int blk, const int64_t* range, int donor, const int64_t* drange,
                const int32_t* dtype) {
  if (blk < 0 || blk >= (int)c->blocks.size() || donor < 0 || donor >= (int)c->blocks.size())
    return fail(c, FVM_ERR_INVALID, "bad block id");
  if (!valid_perm(dtype)) return fail(c, FVM_ERR_INVALID, "donor_type is not a signed permutation");
  Block& b = c->blocks[blk];
  Conn cn;
  cn.donor = donor;
  int out_axis = -1;
  for (int a = 0; a < 3; ++a) {
    cn.range[a][0] = range[2 * a];
    cn.range[a][1] = range[2 * a + 1];
    cn.drange[a][0] = drange[2 * a];
    cn.drange[a][1] = drange[2 * a + 1];
    cn.dtype[a] = dtype[a];
    if (cn.range[a][1] < cn.range[a][0]) return fail(c, FVM_ERR_INVALID, "empty range");
    int64_t s = dtype[a] > 0 ? 1 : -1;
    if (cn.drange[a][1] - cn.drange[a][0] != s * (cn.range[a][1] - cn.range[a][0]))
      return fail(c, FVM_ERR_INVALID, "donor range extent does not match");
    bool out = cn.range[a][1] < 0 || cn.range[a][0] >= b.n[a];
    bool in = cn.range[a][0] >= 0 && cn.range[a][1] < b.n[a];
    if (out) {
      if (out_axis >= 0) return fail(c, FVM_ERR_INVALID, "range is not a face ghost box");
      out_axis = a;
      if (cn.range[a][0] < -3 || cn.range[a][1] > b.n[a] + 2)
        return fail(c, FVM_ERR_INVALID, "range beyond the 3 ghost layers");
    } else if (!in) {
      return fail(c, FVM_ERR_INVALID, "range straddles the block boundary");
    }
  }
  if (out_axis < 0) return fail(c, FVM_ERR_INVALID, "range holds no ghost cells");
  const Block& d = c->blocks[donor];
  for (int a = 0; a < 3; ++a) {
    int da = std::abs(dtype[a]) - 1;
    for (int s = 0; s < 2; ++s)
      if (cn.drange[a][s] < 0 || cn.drange[a][s] >= d.n[da])
        return fail(c, FVM_ERR_INVALID, "donor range outside the donor's real cells");
  }
  int region = 2 * out_axis + (cn.range[out_axis][0] >= b.n[out_axis] ? 2 : 1);
  b.bc[region - 1] = FVM_BC_CONNECTED;
  b.conns.push_back(cn);
  return FVM_OK;
}

int orc_set_state(orc_ctx* c, int blk, const double* q) {
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(c, FVM_ERR_INVALID, "bad block");
  Block& b = c->blocks[blk];
  const int64_t rv = b.rvol(), gv = b.gvol();
  for (int e = 0; e < 5; ++e)
    for (int64_t k = 0; k < b.n[2]; ++k)
      for (int64_t j = 0; j < b.n[1]; ++j)
        for (int64_t i = 0; i < b.n[0]; ++i)
          b.q[b.gidx(i, j, k) + e * gv] = q[b.ridx(i, j, k) + e * rv];
  return FVM_OK;
}

// After every block's state is set: q->p and ghosts (class_flow_field.f90:244-253).
int orc_prepare(orc_ctx* c) {
  flow_update(c);
  return FVM_OK;
}

int orc_get_state(orc_ctx* c, int blk, double* q) {
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(c, FVM_ERR_INVALID, "bad block");
  Block& b = c->blocks[blk];
  const int64_t rv = b.rvol(), gv = b.gvol();
  for (int e = 0; e < 5; ++e)
    for (int64_t k = 0; k < b.n[2]; ++k)
      for (int64_t j = 0; j < b.n[1]; ++j)
        for (int64_t i = 0; i < b.n[0]; ++i)
          q[b.ridx(i, j, k) + e * rv] = b.q[b.gidx(i, j, k) + e * gv];
  return FVM_OK;
}

// Ghost-mesh q including ghosts: (n0+6, n1+6, n2+6, 5) column-major.
int orc_get_ghost_state(orc_ctx* c, int blk, double* q) {
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(c, FVM_ERR_INVALID, "bad block");
  Block& b = c->blocks[blk];
  std::memcpy(q, b.q.data(), sizeof(double) * b.q.size());
  return FVM_OK;
}

int orc_get_rhs(orc_ctx* c, int blk, double* rhs) {
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(c, FVM_ERR_INVALID, "bad block");
  Block& b = c->blocks[blk];
  std::memcpy(rhs, b.rhs.data(), sizeof(double) * b.rhs.size());
  return FVM_OK;
}

int orc_get_primitive(orc_ctx* c, int blk, double* p) {
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(c, FVM_ERR_INVALID, "bad block");
  Block& b = c->blocks[blk];
  const int64_t rv = b.rvol();
  for (int64_t k = 0; k < b.n[2]; ++k)
    for (int64_t j = 0; j < b.n[1]; ++j)
      for (int64_t i = 0; i < b.n[0]; ++i) {
        const Prim& s = b.p[b.gidx(i, j, k)];
        int64_t r = b.ridx(i, j, k);
        p[r] = s.rho;
        p[r + rv] = s.u;
        p[r + 2 * rv] = s.v;
        p[r + 3 * rv] = s.w;
        p[r + 4 * rv] = s.press;
      }
  return FVM_OK;
}

int orc_step(orc_ctx* c, int nsteps, double* t, double* res_abs, double* res_rel, double* dt) {
  for (int s = 0; s < nsteps; ++s) solve_one(c);
  if (t) *t = c->time;
  if (dt) *dt = c->dt_last;
  if (res_abs) std::memcpy(res_abs, c->res_abs, sizeof(c->res_abs));
  if (res_rel) std::memcpy(res_rel, c->res_rel, sizeof(c->res_rel));
  return FVM_OK;
}

// ---- point-wise entries for the known-answer tests --------------------------
double orc_muscl_point(double p1, double p2, double p3, int wind, int limiter, double kappa) {
  return muscl(p1, p2, p3, wind, limiter, kappa);
}

double orc_weno_point(const double* u, int compat) { return weno_js(u, compat); }

// prim L/R = (rho,u,v,w,p); dir 0..2
void orc_flux_point(int flux, int dir, double gamma, double fix, int compat, const double* Lp,
                    const double* Rp, double* F) {
  double n[3] = {0, 0, 0};
  n[dir] = 1.0;
  Prim L{Lp[0], Lp[1], Lp[2], Lp[3], Lp[4]}, R{Rp[0], Rp[1], Rp[2], Rp[3], Rp[4]};
  if (flux == FVM_FLUX_ROE)
    roe_face(gamma, n, L, R, fix, F);
  else if (flux == FVM_FLUX_VANLEER)
    vanleer_face(gamma, n, L, R, compat, F);
  else
    ausm_face(gamma, n, L, R, F);
}

}  // extern "C"
