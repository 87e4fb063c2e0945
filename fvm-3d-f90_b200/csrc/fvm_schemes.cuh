// fvm_schemes.cuh — point-wise reconstruction and flux functions of the fused
// sweep, templated on the arithmetic type R and on EX (exact mode).
//
// EX = true reproduces the reference's expression trees operation by
// operation (the translation unit is compiled with -fmad=false), so results
// are bit-identical to the CPU oracle. EX = false keeps the same mathematics
// but shares reciprocals, uses the division-free WENO weights and lets the
// compiler contract to FMA.
//
// The face normal is always an axis vector (class_space_discret.f90:458-461),
// so every term multiplied by a zero normal component is dropped: x + y*0 and
// x - y*0 equal x as numbers (only the sign of a zero can differ), and x*1 is
// exact. DIR is the sweep axis 0..2.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fvm {

enum ReconId { RECON_SIMPLE_ = 200, RECON_MUSCL_ = 201, RECON_WENO_ = 202 };
enum FluxId { FLUX_ROE_ = 300, FLUX_VANLEER_ = 301, FLUX_AUSM_ = 303 };
enum LimiterId { LIM_NONE_ = 250, LIM_MINMOD_ = 251, LIM_VANLEER_ = 252, LIM_VANALBADA_ = 253 };
enum PrecId { PREC_EXACT = 0, PREC_FP64 = 1, PREC_FP32 = 2 };

template <int P> struct PrecT { using R = double; static constexpr bool ex = true; };
template <> struct PrecT<PREC_FP64> { using R = double; static constexpr bool ex = false; };
template <> struct PrecT<PREC_FP32> { using R = float; static constexpr bool ex = false; };

template <class R> struct Prim5 { R r, u, v, w, p; };

// Case constants in the arithmetic type of the sweep.
template <class R> struct SchemeConst {
  R gamma, gm1, goverg1, two_g2m1, fix, kappa, omk, opk;
  int limiter;
  int textbook;
};

// rcp_ / rsqrt_ / nsqrt_ serve the non-exact forms only (the exact form
// divides and takes IEEE square roots in the reference's order). In FP64
// they start from the hardware approximation (rcp / rsqrt .approx.ftz.f64)
// and take one third-order correction: with e = 1 - x r (reciprocal) or
// e = 1 - x y^2 (reciprocal square root), r (1 + e + e^2) = (1 - e^3) / x
// and y (1 + e/2 + 3e^2/8) = x^(-1/2) (1 + O(e^3)), so the approximation's
// relative error is cubed in three (reciprocal) or five (reciprocal square
// root) FP64 operations, and the result is within a couple of ulp of the
// correctly rounded one with no special-case branch. Arguments are positive
// normal numbers (densities, pressures, squared sound speeds, limiter and
// entropy-fix denominators); a zero argument gives a non-finite result, as
// the exact division does.
__device__ __forceinline__ double rcp_(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  const double e = fma(-x, r, 1.0);
  return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ float rcp_(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double rsqrt_(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-(x * y), y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}
__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
__device__ __forceinline__ double nsqrt_(double x) { return x * rsqrt_(x); }
__device__ __forceinline__ float nsqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double abs_(double x) { return fabs(x); }
__device__ __forceinline__ float abs_(float x) { return fabsf(x); }
__device__ __forceinline__ double sgn1_(double x) { return copysign(1.0, x); }
__device__ __forceinline__ float sgn1_(float x) { return copysignf(1.0f, x); }
template <class R> __device__ __forceinline__ R min2_(R a, R b) { return (b < a) ? b : a; }

template <int DIR, class R> __device__ __forceinline__ R nrm_(R u, R v, R w) {
  return DIR == 0 ? u : (DIR == 1 ? v : w);
}

// ------------------------------------------------------------ q -> p
// convert_q_to_p_* (class_flow_field.f90:383-444)
template <class R, bool EX>
__device__ __forceinline__ Prim5<R> cons2prim(R q0, R q1, R q2, R q3, R q4, R gm1) {
  Prim5<R> s;
  s.r = q0;
  if constexpr (EX) {
    s.u = q1 / q0;
    s.v = q2 / q0;
    s.w = q3 / q0;
    s.p = gm1 * (q4 - R(0.5) * q0 * (s.u * s.u + s.v * s.v + s.w * s.w));
  } else {
    const R ir = rcp_(q0);
    s.u = q1 * ir;
    s.v = q2 * ir;
    s.w = q3 * ir;
    s.p = gm1 * (q4 - R(0.5) * (q1 * s.u + q2 * s.v + q3 * s.w));
  }
  return s;
}
// The non-exact conversion that also returns 1 / rho.
template <class R>
__device__ __forceinline__ Prim5<R> cons2prim_ir(R q0, R q1, R q2, R q3, R q4, R gm1, R& ir) {
  Prim5<R> s;
  s.r = q0;
  ir = rcp_(q0);
  s.u = q1 * ir;
  s.v = q2 * ir;
  s.w = q3 * ir;
  s.p = gm1 * (q4 - R(0.5) * (q1 * s.u + q2 * s.v + q3 * s.w));
  return s;
}

// ------------------------------------------------------------ MUSCL
// scheme_reconstruct_MUSCL.f90:114-226. Limited differences of the centre
// p2 of the stencil (p1, p2, p3).
// EX divides as the reference does; the other forms multiply by rcp_.
template <class R, bool EX>
__device__ __forceinline__ void muscl_slopes(R p1, R p2, R p3, int lim, R& Dbm, R& Dbp) {
  const R Dm = p2 - p1;
  const R Dp = p3 - p2;
  if (lim == LIM_MINMOD_) {
    // minmod(x, y, b=1) = 0.5*(sign(x)+sign(y))*min(|x|,|b*y|)
    Dbm = R(0.5) * (sgn1_(Dm) + sgn1_(Dp)) * min2_(abs_(Dm), abs_(Dp));
    Dbp = R(0.5) * (sgn1_(Dp) + sgn1_(Dm)) * min2_(abs_(Dp), abs_(Dm));
  } else if (lim == LIM_VANLEER_) {
    if constexpr (EX)
      Dbm = (sgn1_(Dm) + sgn1_(Dp)) * Dm * Dp / (abs_(Dm) + abs_(Dp) + R(1.0E-6));
    else
      Dbm = (sgn1_(Dm) + sgn1_(Dp)) * Dm * Dp * rcp_(abs_(Dm) + abs_(Dp) + R(1.0E-6));
    Dbp = Dbm;
  } else if (lim == LIM_VANALBADA_) {
    const R num = Dm * (Dp * Dp + R(1.0E-6)) + Dp * (Dm * Dm + R(1.0E-6));
    if constexpr (EX)
      Dbm = num / (Dm * Dm + Dp * Dp + R(1.0E-6));
    else
      Dbm = num * rcp_(Dm * Dm + Dp * Dp + R(1.0E-6));
    Dbp = Dbm;
  } else {  // none_ / NULL
    Dbm = Dm;
    Dbp = Dp;
  }
}

// ------------------------------------------------------------ WENO
// scheme_WENO.f90:87-121 (WENO_JS on u0..u4, value at the right face of u2).
// textbook != 0: IS_1 with (u1-u3)^2 (Jiang & Shu); 0: (u1+u3)^2 as written.
template <class R, bool EX>
__device__ __forceinline__ R weno5(R u0, R u1, R u2, R u3, R u4, int textbook) {
  if constexpr (EX) {
    const R q0 = R(1.0 / 3.0) * u0 - R(7.0 / 6.0) * u1 + R(11.0 / 6.0) * u2;
    const R q1 = R(-1.0 / 6.0) * u1 + R(5.0 / 6.0) * u2 + R(1.0 / 3.0) * u3;
    const R q2 = R(1.0 / 3.0) * u2 + R(5.0 / 6.0) * u3 - R(1.0 / 6.0) * u4;
    const R a0 = u0 - R(2.0) * u1 + u2;
    const R b0 = u0 - R(4.0) * u1 + R(3.0) * u2;
    const R a1 = u1 - R(2.0) * u2 + u3;
    const R b1 = textbook ? (u1 - u3) : (u1 + u3);
    const R a2 = u2 - R(2.0) * u3 + u4;
    const R b2 = R(3.0) * u2 - R(4.0) * u3 + u4;
    const R IS0 = R(13.0 / 12.0) * (a0 * a0) + R(1.0 / 4.0) * (b0 * b0);
    const R IS1 = R(13.0 / 12.0) * (a1 * a1) + R(1.0 / 4.0) * (b1 * b1);
    const R IS2 = R(13.0 / 12.0) * (a2 * a2) + R(1.0 / 4.0) * (b2 * b2);
    const R e0 = IS0 + R(1.0e-6), e1 = IS1 + R(1.0e-6), e2 = IS2 + R(1.0e-6);
    const R al0 = R(0.1) / (e0 * e0);
    const R al1 = R(0.6) / (e1 * e1);
    const R al2 = R(0.3) / (e2 * e2);
    const R as = al0 + al1 + al2;
    const R w0 = al0 / as, w1 = al1 / as, w2 = al2 / as;
    return w0 * q0 + w1 * q1 + w2 * q2;
  } else {
    // The same mathematics in fewer operations. With the first differences
    // Dij = uj - ui: q_k = u2 + delta_k (delta_0 = (5 D12 - 2 D01)/6,
    // delta_1 = (D12 + 2 D23)/6, delta_2 = (4 D23 - D34)/6); a_k are the
    // second differences, b_0 = 2 D12 + a_0, b_2 = a_2 - 2 D23. The
    // smoothness indicators and eps are scaled by 4 (the weights only see
    // their ratios): 4 (IS_k + eps) = 13/3 a_k^2 + b_k^2 + 4e-6. The weights
    // are division-free, omega_k = c_k prod_{j!=k} d_j / D with d = e^2, and
    // the result is u2 + sum omega_k delta_k. With P0 = d1 d2, P1 = d0 d2
    // and P2 = d0 d1 / 2 the weights are (P0, 6 P1, 6 P2) / (P0 + 6 (P1 + P2)),
    // so the constants of the linear weights fold into 6 delta_1 =
    // D12 + 2 D23 and 6 delta_2 = 4 D23 - D34 (one operation each).
    const R D01 = u1 - u0, D12 = u2 - u1, D23 = u3 - u2, D34 = u4 - u3;
    const R a0 = D12 - D01, a1 = D23 - D12, a2 = D34 - D23;
    const R b0 = R(2.0) * D12 + a0;
    const R b1 = textbook ? (D12 + D23) : (u1 + u3);
    const R b2 = a2 - R(2.0) * D23;
    const R e0 = (R(13.0 / 3.0) * a0) * a0 + (b0 * b0 + R(4.0e-6));
    const R e1 = (R(13.0 / 3.0) * a1) * a1 + (b1 * b1 + R(4.0e-6));
    const R e2 = (R(13.0 / 3.0) * a2) * a2 + (b2 * b2 + R(4.0e-6));
    const R d0 = e0 * e0, d1 = e1 * e1, d2 = e2 * e2;
    const R P0 = d1 * d2, P1 = d0 * d2, P2 = (R(0.5) * d0) * d1;
    const R s0 = R(1.0 / 3.0) * b0 + R(-1.0 / 6.0) * D12;  // delta_0 = (2 b0 - D12) / 6
    const R S1 = R(2.0) * D23 + D12;
    const R S2 = R(4.0) * D23 - D34;
    return (P0 * s0 + (P1 * S1 + P2 * S2)) * rcp_(R(6.0) * (P1 + P2) + P0) + u2;
  }
}

// Two WENO5 evaluations at once in packed FP32 (sm_100 f32x2 FMA / add /
// multiply: one instruction per pair), for the FP32 flux form: the
// difference form of weno5<R, false>; the pair shares `textbook`.
__device__ __forceinline__ float2 f2_(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 weno5x2(float2 u0, float2 u1, float2 u2, float2 u3, float2 u4, int textbook) {
  const float2 m1 = f2_(-1.0f);
  const float2 D01 = __ffma2_rn(m1, u0, u1), D12 = __ffma2_rn(m1, u1, u2);
  const float2 D23 = __ffma2_rn(m1, u2, u3), D34 = __ffma2_rn(m1, u3, u4);
  const float2 a0 = __ffma2_rn(m1, D01, D12), a1 = __ffma2_rn(m1, D12, D23), a2 = __ffma2_rn(m1, D23, D34);
  const float2 b0 = __ffma2_rn(f2_(2.0f), D12, a0);
  const float2 b1 = textbook ? __fadd2_rn(D12, D23) : __fadd2_rn(u1, u3);
  const float2 b2 = __ffma2_rn(f2_(-2.0f), D23, a2);
  // 4 (IS_k + eps) = 13/3 a_k^2 + b_k^2 + 4e-6
  const float2 c = f2_(13.0f / 3.0f), eps = f2_(4.0e-6f);
  const float2 e0 = __ffma2_rn(__fmul2_rn(c, a0), a0, __ffma2_rn(b0, b0, eps));
  const float2 e1 = __ffma2_rn(__fmul2_rn(c, a1), a1, __ffma2_rn(b1, b1, eps));
  const float2 e2 = __ffma2_rn(__fmul2_rn(c, a2), a2, __ffma2_rn(b2, b2, eps));
  const float2 d0 = __fmul2_rn(e0, e0), d1 = __fmul2_rn(e1, e1), d2 = __fmul2_rn(e2, e2);
  // weights c_k / d_k normalised by 1 / c_0, with the constants of c_1 and
  // c_2 folded into the differences (the FP64 form's P0, P1, P2, S1, S2)
  const float2 P0 = __fmul2_rn(d1, d2);
  const float2 P1 = __fmul2_rn(d0, d2);
  const float2 P2 = __fmul2_rn(__fmul2_rn(f2_(0.5f), d0), d1);
  const float2 s0 = __ffma2_rn(f2_(1.0f / 3.0f), b0, __fmul2_rn(f2_(-1.0f / 6.0f), D12));
  const float2 S1 = __ffma2_rn(f2_(2.0f), D23, D12);
  const float2 S2 = __ffma2_rn(m1, b2, D23);  // 4 D23 - D34
  const float2 num = __ffma2_rn(P0, s0, __ffma2_rn(P1, S1, __fmul2_rn(P2, S2)));
  const float2 den = __ffma2_rn(f2_(6.0f), __fadd2_rn(P1, P2), P0);
  return __ffma2_rn(num, make_float2(rcp_(den.x), rcp_(den.y)), u2);
}

// The WENO node values of one stencil u[var][0..4]: wm (left-biased, value
// at the right face of u[.][2]) and, with TB, wp (mirrored, value at its left
// face, always the textbook form). The FP32 flux form evaluates them in pairs.
template <class R, bool EX, bool TB>
__device__ __forceinline__ void weno5_node(const R (&u)[5][5], int textbook, R wm[5], R wp[5]) {
  if constexpr (sizeof(R) == 4) {
    if constexpr (TB) {
      // TB implies TEXTBOOK compat, so both sides take the textbook form
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const float2 r = weno5x2(make_float2(u[v][0], u[v][4]), make_float2(u[v][1], u[v][3]),
                                 make_float2(u[v][2], u[v][2]), make_float2(u[v][3], u[v][1]),
                                 make_float2(u[v][4], u[v][0]), 1);
        wm[v] = r.x;
        wp[v] = r.y;
      }
    } else {
#pragma unroll
      for (int v = 0; v < 5; v += 2) {
        const int w = v + 1 < 5 ? v + 1 : v;
        const float2 r = weno5x2(make_float2(u[v][0], u[w][0]), make_float2(u[v][1], u[w][1]),
                                 make_float2(u[v][2], u[w][2]), make_float2(u[v][3], u[w][3]),
                                 make_float2(u[v][4], u[w][4]), textbook);
        wm[v] = r.x;
        if (v + 1 < 5) wm[v + 1] = r.y;
      }
    }
  } else {
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      wm[v] = weno5<R, EX>(u[v][0], u[v][1], u[v][2], u[v][3], u[v][4], textbook);
      if (TB) wp[v] = weno5<R, EX>(u[v][4], u[v][3], u[v][2], u[v][1], u[v][0], 1);
    }
  }
}

// ------------------------------------------------------------ Roe
// scheme_FDS_Roe.f90:25-177
template <class R, bool EX> __device__ __forceinline__ R entropy_fix_(R lam, R delta) {
  if constexpr (EX)
    return (lam > delta) ? lam : R(0.5) * (lam * lam + delta * delta) / delta;
  else
    return (lam > delta) ? lam : R(0.5) * (lam * lam + delta * delta) * rcp_(delta);
}

template <int DIR, class R, bool EX>
__device__ __forceinline__ void flux_roe(const Prim5<R>& L, const Prim5<R>& Rs, const SchemeConst<R>& k,
                                         R F[5]) {
  const R Vc_l = nrm_<DIR>(L.u, L.v, L.w);
  const R Vc_r = nrm_<DIR>(Rs.u, Rs.v, Rs.w);
  R H_l, H_r, rho_b, u_b, v_b, w_b, H_b;
  if constexpr (EX) {
    H_l = k.goverg1 * L.p / L.r + R(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w);
    H_r = k.goverg1 * Rs.p / Rs.r + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v + Rs.w * Rs.w);
    rho_b = sqrt_(L.r * Rs.r);
    u_b = (L.r * L.u + rho_b * Rs.u) / (L.r + rho_b);
    v_b = (L.r * L.v + rho_b * Rs.v) / (L.r + rho_b);
    w_b = (L.r * L.w + rho_b * Rs.w) / (L.r + rho_b);
    H_b = (L.r * H_l + rho_b * H_r) / (L.r + rho_b);
  } else {
    H_l = k.goverg1 * L.p * rcp_(L.r) + R(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w);
    H_r = k.goverg1 * Rs.p * rcp_(Rs.r) + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v + Rs.w * Rs.w);
    rho_b = nsqrt_(L.r * Rs.r);
    const R id = rcp_(L.r + rho_b);
    u_b = (L.r * L.u + rho_b * Rs.u) * id;
    v_b = (L.r * L.v + rho_b * Rs.v) * id;
    w_b = (L.r * L.w + rho_b * Rs.w) * id;
    H_b = (L.r * H_l + rho_b * H_r) * id;
  }
  const R drho = Rs.r - L.r, du = Rs.u - L.u, dv = Rs.v - L.v, dw = Rs.w - L.w;
  const R dp = Rs.p - L.p, dVl = Vc_r - Vc_l;
  const R Vl_b = nrm_<DIR>(u_b, v_b, w_b);
  const R q2_b = u_b * u_b + v_b * v_b + w_b * w_b;
  R c_b, ic2 = R(0);
  if constexpr (EX) {
    c_b = sqrt_(k.gm1 * (H_b - R(0.5) * q2_b));
  } else {
    const R a2 = k.gm1 * (H_b - R(0.5) * q2_b);
    const R rs = rsqrt_(a2);
    c_b = a2 * rs;
    ic2 = rs * rs;
  }
  const R delta = k.fix * abs_(Vl_b + c_b);
  const R lam1 = entropy_fix_<R, EX>(abs_(Vl_b - c_b), delta);
  const R lam2 = entropy_fix_<R, EX>(abs_(Vl_b), delta);
  const R lam5 = entropy_fix_<R, EX>(abs_(Vl_b + c_b), delta);
  R d1_0, d234_0, d5_0;
  if constexpr (EX) {
    d1_0 = lam1 * (dp - rho_b * c_b * dVl) / (R(2.0) * c_b * c_b);
    d234_0 = lam2 * (drho - dp / (c_b * c_b));
    d5_0 = lam5 * (dp + rho_b * c_b * dVl) / (R(2.0) * c_b * c_b);
  } else {
    d1_0 = lam1 * (dp - rho_b * c_b * dVl) * (R(0.5) * ic2);
    d234_0 = lam2 * (drho - dp * ic2);
    d5_0 = lam5 * (dp + rho_b * c_b * dVl) * (R(0.5) * ic2);
  }
  const R ub[3] = {u_b, v_b, w_b};
  const R dd[3] = {du, dv, dw};
  const R ul[3] = {L.u, L.v, L.w};
  const R ur[3] = {Rs.u, Rs.v, Rs.w};
  const R l2r = lam2 * rho_b;
  if constexpr (!EX) {
    // the same flux with the wave sums collected: sum_k d_k r_k has
    // momentum (d1+d234+d5) u_b + lam2 rho_b du (+ (d5-d1) c_b - lam2 rho_b dV
    // along the normal) and energy (d1+d5) H_b + (d5-d1) c_b V_b
    // + d234 q2_b / 2 + lam2 rho_b (u_b . du - V_b dV)
    // Along the normal the velocity jump is dVl itself, so lam2 rho_b (du_n
    // - dVl) and u_b,n du_n - V_b dVl vanish: the normal momentum's
    // dissipation is dsum u_b,n + ddif and u_b . du - V_b dV sums the two
    // tangential terms.
    const R dsum = d1_0 + d234_0 + d5_0;
    const R ddif = (d5_0 - d1_0) * c_b;
    const R ml = L.r * Vc_l, mr = Rs.r * Vc_r;
    F[0] = R(0.5) * ((ml + mr) - dsum);
    R ud = R(0);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      R diss, phys = ml * ul[m] + mr * ur[m];
      if (m == DIR) {
        diss = dsum * ub[m] + ddif;
        phys = phys + (L.p + Rs.p);
      } else {
        diss = dsum * ub[m] + l2r * dd[m];
        ud = ud + ub[m] * dd[m];
      }
      F[1 + m] = R(0.5) * (phys - diss);
    }
    const R de = (d1_0 + d5_0) * H_b + ddif * Vl_b + d234_0 * (R(0.5) * q2_b) + l2r * ud;
    F[4] = R(0.5) * ((ml * H_l + mr * H_r) - de);
    return;
  }
  // mass
  F[0] = R(0.5) * ((L.r * Vc_l + Rs.r * Vc_r) - (d1_0 + d234_0 + d5_0));
  // momentum
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const R d1m = d1_0 * (m == DIR ? ub[m] - c_b : ub[m]);
    const R d234m = d234_0 * ub[m] + l2r * (m == DIR ? dd[m] - dVl : dd[m]);
    const R d5m = d5_0 * (m == DIR ? ub[m] + c_b : ub[m]);
    const R flm = (m == DIR) ? L.r * ul[m] * Vc_l + L.p : L.r * ul[m] * Vc_l;
    const R frm = (m == DIR) ? Rs.r * ur[m] * Vc_r + Rs.p : Rs.r * ur[m] * Vc_r;
    F[1 + m] = R(0.5) * ((flm + frm) - (d1m + d234m + d5m));
  }
  // energy
  {
    const R d1e = d1_0 * (H_b - c_b * Vl_b);
    const R d234e = d234_0 * R(0.5) * q2_b + l2r * (u_b * du + v_b * dv + w_b * dw - Vl_b * dVl);
    const R d5e = d5_0 * (H_b + c_b * Vl_b);
    F[4] = R(0.5) * ((L.r * H_l * Vc_l + Rs.r * H_r * Vc_r) - (d1e + d234e + d5e));
  }
}

// ------------------------------------------------------------ Van Leer FVS
// scheme_FVS_VanLeer.f90:25-126; textbook: supersonic sides carry the full or
// no flux.
template <int DIR, class R, bool EX>
__device__ __forceinline__ void euler_flux_(const Prim5<R>& s, const SchemeConst<R>& k, R F[5]) {
  const R Vc = nrm_<DIR>(s.u, s.v, s.w);
  R H;
  if constexpr (EX)
    H = k.goverg1 * s.p / s.r + R(0.5) * (s.u * s.u + s.v * s.v + s.w * s.w);
  else
    H = k.goverg1 * s.p * rcp_(s.r) + R(0.5) * (s.u * s.u + s.v * s.v + s.w * s.w);
  const R uu[3] = {s.u, s.v, s.w};
  F[0] = s.r * Vc;
#pragma unroll
  for (int m = 0; m < 3; ++m) F[1 + m] = (m == DIR) ? s.r * uu[m] * Vc + s.p : s.r * uu[m] * Vc;
  F[4] = s.r * H * Vc;
}

template <int DIR, class R, bool EX, int SIDE /* +1 left/plus, -1 right/minus */>
__device__ __forceinline__ void vanleer_half(const Prim5<R>& s, const SchemeConst<R>& k, R F[5]) {
  const R Vc = nrm_<DIR>(s.u, s.v, s.w);
  const R q2 = s.u * s.u + s.v * s.v + s.w * s.w;
  R c, M;
  if constexpr (EX) {
    c = sqrt_(k.gamma * s.p / s.r);
    M = Vc / c;
  } else {
    const R a2 = k.gamma * s.p * rcp_(s.r);
    const R rs = rsqrt_(a2);
    c = a2 * rs;
    M = Vc * rs;
  }
  if (k.textbook) {
    if ((SIDE > 0 && M >= R(1.0)) || (SIDE < 0 && M <= R(-1.0))) {
      euler_flux_<DIR, R, EX>(s, k, F);
      return;
    }
    if ((SIDE > 0 && M <= R(-1.0)) || (SIDE < 0 && M >= R(1.0))) {
      F[0] = F[1] = F[2] = F[3] = F[4] = R(0.0);
      return;
    }
  }
  R Ms;
  if (SIDE > 0)
    Ms = (M >= R(1.0)) ? M : ((M <= R(-1.0)) ? R(0.0) : R(0.25) * (M + R(1.0)) * (M + R(1.0)));
  else
    Ms = (M >= R(1.0)) ? R(0.0) : ((M <= R(-1.0)) ? M : -(R(0.25) * (M - R(1.0)) * (M - R(1.0))));
  const R f0 = s.r * c * Ms;
  const R uu[3] = {s.u, s.v, s.w};
  R tn, t;
  if (SIDE > 0) {
    t = k.gm1 * Vc + R(2.0) * c;
    tn = EX ? (-Vc + R(2.0) * c) / k.gamma : (-Vc + R(2.0) * c) * rcp_(k.gamma);
  } else {
    t = k.gm1 * Vc - R(2.0) * c;
    tn = EX ? (-Vc - R(2.0) * c) / k.gamma : (-Vc - R(2.0) * c) * rcp_(k.gamma);
  }
  F[0] = f0;
#pragma unroll
  for (int m = 0; m < 3; ++m) F[1 + m] = f0 * ((m == DIR) ? tn + uu[m] : uu[m]);
  if constexpr (EX)
    F[4] = f0 * (t * t / k.two_g2m1 + (q2 - Vc * Vc) / R(2.0));
  else
    F[4] = f0 * (t * t * rcp_(k.two_g2m1) + (q2 - Vc * Vc) * R(0.5));
}

template <int DIR, class R, bool EX>
__device__ __forceinline__ void flux_vanleer(const Prim5<R>& L, const Prim5<R>& Rs, const SchemeConst<R>& k,
                                             R F[5]) {
  R fp[5], fm[5];
  vanleer_half<DIR, R, EX, +1>(L, k, fp);
  vanleer_half<DIR, R, EX, -1>(Rs, k, fm);
#pragma unroll
  for (int e = 0; e < 5; ++e) F[e] = fp[e] + fm[e];
}

// ------------------------------------------------------------ AUSM
// scheme_AUSM.f90:27-171 (beta = alpha = 0; Harten-type |M| fix, delta 0.1)
template <int DIR, class R, bool EX>
__device__ __forceinline__ void flux_ausm(const Prim5<R>& L, const Prim5<R>& Rs, const SchemeConst<R>& k,
                                          R F[5]) {
  const R Vc_l = nrm_<DIR>(L.u, L.v, L.w);
  const R Vc_r = nrm_<DIR>(Rs.u, Rs.v, Rs.w);
  R H_l, H_r, c_l, c_r, M_l, M_r;
  if constexpr (EX) {
    H_l = k.goverg1 * L.p / L.r + R(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w);
    H_r = k.goverg1 * Rs.p / Rs.r + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v + Rs.w * Rs.w);
    c_l = sqrt_(k.gamma * L.p / L.r);
    c_r = sqrt_(k.gamma * Rs.p / Rs.r);
    M_l = Vc_l / c_l;
    M_r = Vc_r / c_r;
  } else {
    const R irl = rcp_(L.r), irr = rcp_(Rs.r);
    const R pl = L.p * irl, pr = Rs.p * irr;
    H_l = k.goverg1 * pl + R(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w);
    H_r = k.goverg1 * pr + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v + Rs.w * Rs.w);
    const R al = k.gamma * pl, ar = k.gamma * pr;
    const R rsl = rsqrt_(al), rsr = rsqrt_(ar);
    c_l = al * rsl;
    c_r = ar * rsr;
    M_l = Vc_l * rsl;
    M_r = Vc_r * rsr;
  }
  if constexpr (!EX) {
    // the same fluxes in fewer operations: the supersonic split Mach numbers
    // 0.5 (M +- |M|) are max / min (M, 0) and the supersonic pressure splits
    // 0.5 (1 +- sign M) are 0 or 1 (both exact); the subsonic pressure split
    // reuses the subsonic Mach split, 1/4 (M +- 1)^2 (2 -+ M); the mass flux
    // factors w rho c are formed once per side
    const bool sup_l = abs_(M_l) >= R(1.0), sup_r = abs_(M_r) >= R(1.0);
    const R hl = M_l + R(1.0), hr = M_r - R(1.0);
    const R msub_l = (R(0.25) * hl) * hl, msub_r = (R(0.25) * hr) * hr;
    const R ms_l = sup_l ? fmax(M_l, R(0)) : msub_l;
    const R ms_r = sup_r ? fmin(M_r, R(0)) : -msub_r;
    const R ps_l = sup_l ? (M_l > R(0) ? R(1) : R(0)) : msub_l * (R(2.0) - M_l);
    const R ps_r = sup_r ? (M_r < R(0) ? R(1) : R(0)) : msub_r * (R(2.0) + M_r);
    const R Mn = ms_l + ms_r;
    const R am = abs_(Mn);
    const R Mabs = (am > R(0.1)) ? am : (am * am + R(0.01)) * R(5.0);
    const R p_ = ps_l * L.p + ps_r * Rs.p;
    const R gl = (R(0.5) * (Mn + Mabs)) * (L.r * c_l);
    const R gr = (R(0.5) * (Mn - Mabs)) * (Rs.r * c_r);
    F[0] = gl + gr;
    F[1] = gl * L.u + gr * Rs.u;
    F[2] = gl * L.v + gr * Rs.v;
    F[3] = gl * L.w + gr * Rs.w;
    F[1 + DIR] = F[1 + DIR] + p_;
    F[4] = gl * H_l + gr * H_r;
    return;
  }
  // Mach_Split_AUSM(M_l, +1) + Mach_Split_AUSM(M_r, -1)
  const R ms_l = (abs_(M_l) >= R(1.0)) ? R(0.5) * (M_l + abs_(M_l)) : R(0.25) * ((M_l + R(1.0)) * (M_l + R(1.0)));
  const R ms_r = (abs_(M_r) >= R(1.0)) ? R(0.5) * (M_r - abs_(M_r))
                                       : -(R(0.25) * ((M_r - R(1.0)) * (M_r - R(1.0))));
  const R Mn = ms_l + ms_r;
  const R am = abs_(Mn);
  const R dlt = R(0.1);
  R Mabs;
  if constexpr (EX)
    Mabs = (am > dlt) ? am : R(0.5) * (am * am + dlt * dlt) / dlt;
  else
    Mabs = (am > dlt) ? am : (am * am + dlt * dlt) * R(5.0);
  // Pressure_Split_AUSM(p_l, M_l, +1) + Pressure_Split_AUSM(p_r, M_r, -1)
  const R ps_l = (abs_(M_l) >= R(1.0)) ? R(0.5) * (R(1.0) + sgn1_(M_l))
                                       : R(0.25) * ((M_l + R(1.0)) * (M_l + R(1.0))) * (R(2.0) - M_l);
  const R ps_r = (abs_(M_r) >= R(1.0)) ? R(0.5) * (R(1.0) - sgn1_(M_r))
                                       : R(0.25) * ((M_r - R(1.0)) * (M_r - R(1.0))) * (R(2.0) + M_r);
  const R p_ = ps_l * L.p + ps_r * Rs.p;
  const R wl = R(0.5) * (Mn + Mabs), wr = R(0.5) * (Mn - Mabs);
  const R phl = L.r * c_l, phr = Rs.r * c_r;
  F[0] = wl * phl + wr * phr;
  F[1] = wl * (phl * L.u) + wr * (phr * Rs.u);
  F[2] = wl * (phl * L.v) + wr * (phr * Rs.v);
  F[3] = wl * (phl * L.w) + wr * (phr * Rs.w);
  F[1 + DIR] = F[1 + DIR] + p_;
  F[4] = wl * (phl * H_l) + wr * (phr * H_r);
}

// AUSM on precomputed sides (non-exact forms). In the reference's WENO
// variant a node's reconstructed state is the left state of one face and the
// right state of the next, so what AUSM derives from one side alone (1/rho,
// H, c, the normal Mach number, rho c) is formed once per node by ausm_side
// instead of once per face and side; flux_ausm_sides is then the !EX branch
// of flux_ausm with those values, operation for operation.
template <class R> struct AusmSide { R u, v, w, p, H, M, rc; };

// s: the node's primitive state, ir = 1 / s.r (as cons2prim formed it),
// E: its total energy per volume (the reconstructed q5), Vc: its velocity
// along the face normal. H = (E + p) / rho and rho c = gamma p / c are the
// same quantities as the flux's gamma/(gamma-1) p/rho + |u|^2/2 and
// rho sqrt(gamma p / rho), in fewer operations.
template <class R>
__device__ __forceinline__ AusmSide<R> ausm_side(const Prim5<R>& s, R ir, R E, R Vc, const SchemeConst<R>& k) {
  AusmSide<R> o;
  o.u = s.u;
  o.v = s.v;
  o.w = s.w;
  o.p = s.p;
  o.H = (E + s.p) * ir;
  const R gp = k.gamma * s.p;
  const R rs = rsqrt_(gp * ir);
  o.M = Vc * rs;
  o.rc = gp * rs;
  return o;
}

template <int DIR, class R>
__device__ __forceinline__ void flux_ausm_sides(const AusmSide<R>& L, const AusmSide<R>& Rs, R F[5]) {
  const R M_l = L.M, M_r = Rs.M;
  const bool sup_l = abs_(M_l) >= R(1.0), sup_r = abs_(M_r) >= R(1.0);
  const R hl = M_l + R(1.0), hr = M_r - R(1.0);
  const R msub_l = (R(0.25) * hl) * hl, msub_r = (R(0.25) * hr) * hr;
  const R ms_l = sup_l ? fmax(M_l, R(0)) : msub_l;
  const R ms_r = sup_r ? fmin(M_r, R(0)) : -msub_r;
  const R ps_l = sup_l ? (M_l > R(0) ? R(1) : R(0)) : msub_l * (R(2.0) - M_l);
  const R ps_r = sup_r ? (M_r < R(0) ? R(1) : R(0)) : msub_r * (R(2.0) + M_r);
  const R Mn = ms_l + ms_r;
  const R am = abs_(Mn);
  const R Mabs = (am > R(0.1)) ? am : (am * am + R(0.01)) * R(5.0);
  const R p_ = ps_l * L.p + ps_r * Rs.p;
  const R gl = (R(0.5) * (Mn + Mabs)) * L.rc;
  const R gr = (R(0.5) * (Mn - Mabs)) * Rs.rc;
  F[0] = gl + gr;
  F[1] = gl * L.u + gr * Rs.u;
  F[2] = gl * L.v + gr * Rs.v;
  F[3] = gl * L.w + gr * Rs.w;
  F[1 + DIR] = F[1 + DIR] + p_;
  F[4] = gl * L.H + gr * Rs.H;
}

template <int FLUX, int DIR, class R, bool EX>
__device__ __forceinline__ void face_flux(const Prim5<R>& L, const Prim5<R>& Rs, const SchemeConst<R>& k,
                                          R F[5]) {
  if constexpr (FLUX == FLUX_ROE_)
    flux_roe<DIR, R, EX>(L, Rs, k, F);
  else if constexpr (FLUX == FLUX_VANLEER_)
    flux_vanleer<DIR, R, EX>(L, Rs, k, F);
  else
    flux_ausm<DIR, R, EX>(L, Rs, k, F);
}

}  // namespace fvm
