// fk_device.cuh -- device-side Fenton-Karma model for sm_100a.
//
// Data layout in HBM (every state, adjoint state and trajectory slot):
//   three planes u, v, w of a padded grid, plane = rows_alloc * ld doubles,
//   logical cell (i, j) at offset (i + HALO) * ld + (j + HALO);
//   a ring of HALO NaN cells surrounds the grid and holes hold NaN.
// With a NaN ring the reference's edge rule (mirror the inner neighbour,
// src/cuda/fk_forward_Et_mono_PARAMETERS.cu:319-361) and its hole rule (a NaN
// neighbour is replaced by the opposite one, :348-358) are the same rule, and
// the adjoint stencil's off-grid and hole cases coincide too, so the kernels
// have no boundary branches and tile loads never leave the allocation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

// Build switches (compile-time; the defaults are the tuned choices).
#ifndef FKADJ_HOLE_BRANCH
#define FKADJ_HOLE_BRANCH 1
#endif
#ifndef FKADJ_SHARED_EXP
#define FKADJ_SHARED_EXP 1
#endif
#ifndef FKADJ_OWN_RCP
#define FKADJ_OWN_RCP 1
#endif
// 1/tau_v-(q) from q's exponential with one reciprocal (see tvm_rcp)
#ifndef FKADJ_MERGED_TVM
#define FKADJ_MERGED_TVM 1
#endif
// Smoothed steps without their overflow tests (see step_of_exp); the same
// bits in the model's range, and the forward step 2 % faster at 512^2
#ifndef FKADJ_FAST_STEPS
#define FKADJ_FAST_STEPS 1
#endif
// Mirrored neighbours of v and w read at offsets chosen from u's NaN tests
// (1), u's too (2), instead of selected among all four (0; see rhs_at): the
// same values summed in the same order, and 1.5 % off the forward step
#ifndef FKADJ_MIRROR_OFFSETS
#define FKADJ_MIRROR_OFFSETS 1
#endif

namespace fkadj {

constexpr int HALO = 4;

// Model constants as the kernels use them: reciprocals replace the divisions
// by constant time scales of the reference's F_ion / jacT (cu-F:29-45,
// cu-G:1160-1184); this moves results by at most an ulp per operation.
struct DevModel {
    double u_c, u_v, ksm, k_fk, u_csi;
    double r_tau_d, r_tau_0, r_tau_r, r_2tau_si;
    double tau_v1m, tau_v2m, r_tau_vp, r_tau_wm, r_tau_wp;
    double r_tau_v2m;  // 1 / tau_v2_minus
    double m2ksm, m2kfk;  // -2 ksm, -2 k_fk: -2 (k x) = (-2 k) x exactly
    double dv12;  // tau_v2_minus - tau_v1_minus
    double eq;    // exp(-2 ksm (u_c - u_v)): e^{-2ksm(u-u_v)} = eq * e^{-2ksm(u-u_c)}
    double cu, cv, cw;  // D / h^2
    double dt;
    // constant factors of the factored Jacobian (fk_jacT, FKADJ_JAC_FACTORED)
    double two_ksm;    // 2 ksm: dp/du = 2 ksm p (1 - p)
    double kfk_r2tsi;  // k_fk / (2 tau_si)
    double hksm_dv12;  // ksm (tau_v2- - tau_v1-) / 2
};

struct DevGrid {
    int nrows, ncols, ld, rows_alloc;
    long long plane;  // doubles per field plane
    // Forward stencil code per padded cell (null: the NaN tests decide).
    const uint8_t* fcode;
};

// Forward stencil codes: which neighbour the 5-point Laplacian takes in each
// direction, fixed by the geometry.  The reference replaces a missing (NaN)
// neighbour by the opposite one (cu-F:319-420); these bits say so ahead of
// time, so the stencil reads the right neighbours without testing values:
//   FC_N  north missing: take the south neighbour for north
//   FC_S  south missing and north present: take the north neighbour for south
//   FC_W, FC_E  the same across
//   FC_HOLE  the cell is a hole or outside the grid (its result is NaN)
// (with north and south both missing both reads take the south neighbour,
// NaN, as the reference's rule does).  The codes equal the NaN tests as long
// as no active cell has two opposite holes: such a cell turns NaN after its
// first stage and its neighbours then mirror it, which no fixed code
// describes; problems with such cells keep the NaN tests (fcode null).
constexpr int FC_N = 1, FC_S = 2, FC_W = 4, FC_E = 8, FC_HOLE = 16;

// Refinement of the reciprocal estimate (own_rcp):
//   0: two Newton-Raphson steps r <- r + r (1 - x r), each squaring the
//      relative error (4 DFMA);
//   1: one third-order step r <- r (1 + e + e^2), e = 1 - x r, which cubes it
//      (3 DFMA): 1/x = r / (1 - e) = r (1 + e + e^2 + e^3 + ...).
// Both are within one ulp of the quotient; 1 (the default) took the forward
// step from 16.5 to 16.3 us at 512^2.
#ifndef FKADJ_RCP_CUBIC
#define FKADJ_RCP_CUBIC 1
#endif

// r refined towards 1/x from the estimate r (see FKADJ_RCP_CUBIC)
__device__ __forceinline__ double rcp_refine(double x, double r) {
#if FKADJ_RCP_CUBIC
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
#else
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
#endif
}

// 1/x for positive x or x = +inf without the division's branches: the hardware
// reciprocal estimate (rcp.approx.ftz.f64) refined by rcp_refine.  Within one
// ulp of the correctly rounded quotient (tests/test_gpu_mathfn.py); x = +inf,
// and x beyond 2^1022 (where the estimate flushes the subnormal quotient),
// give 0.  It takes the three logistic reciprocals and the 1/tau_v- of every
// vector-field and Jacobian evaluation; the IEEE division in their place
// (FKADJ_OWN_RCP=0) costs about 3 % of the gradient's time at 512 x 512.
__device__ __forceinline__ double own_rcp(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = rcp_refine(x, r);
    return isinf(x) ? 0.0 : r;  // the refinement turns inf * 0 into NaN
}

// 1/x for the positive denominators of the model (1 + e^{...}, tau_v-)
__device__ __forceinline__ double fk_rcp(double x) {
#if FKADJ_OWN_RCP
    return own_rcp(x);
#else
    return 1.0 / x;
#endif
}

// own_rcp for finite x in [1, 2^1001]: the same value, without the +inf test.
__device__ __forceinline__ double fk_rcp_finite(double x) {
#if FKADJ_OWN_RCP
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return rcp_refine(x, r);
#else
    return 1.0 / x;
#endif
}

// The exponential of the smoothed steps (FKADJ_OWN_EXP):
//   0: CUDA's exp;
//   1: own, by Cody and Waite's argument reduction (Software Manual for the
//      Elementary Functions, 1980): x = k ln2 + r with k = rint(x / ln2) and
//      ln2 split in two so that k ln2_hi is exact, |r| <= ln2 / 2, then e^x =
//      2^k p(r) with p the degree-11 Chebyshev fit of e^r on [-ln2/2, ln2/2]
//      (fit error 3.2e-18; coefficients computed with mpmath's chebyfit);
//   2: own, by Tang's table-driven method (ACM TOMS 15(2), 1989): x =
//      (16 m + j) ln2/16 + r with |r| <= ln2/32, e^x = 2^m 2^(j/16) (1 + p(r)),
//      p(r) = r + r^2 q(r) and q the degree-4 Chebyshev fit of
//      (e^r - 1 - r) / r^2 on [-ln2/32, ln2/32] (error of p 2.8e-17), the 16
//      values 2^(j/16) in shared memory (exp_table_init).
// Both own forms are within 1.3 ulp of e^x for x in [-707, 692] (measured
// against a long-double exp on 2e7 arguments; tests/test_gpu_mathfn.py checks
// them against CUDA's exp).  They saturate instead of overflowing: for
// |x| < 2^51 ln2 the result stays in [2^-1020, 2^1000) (k, resp. m, is
// clamped), so the smoothed steps need no cap of their own.  A NaN argument
// gives NaN; beyond |x| = 2^51 ln2 (|u| above 1e13, a state that has blown
// up) and at infinities the value is unspecified.  The rounding to an integer
// is the fma's own: adding 1.5 * 2^52 leaves rint(x / ln2) in the low bits of
// the sum.
// Measured at 512^2 x 2000 steps (sqrt store, one B200): forward step 16.5 us
// (CUDA's exp), 16.0 (form 1), 15.7 (form 2); 15.4 us with the cubic
// reciprocal, and the gradient 137.2 -> 132.0 ms.  Form 2 is the default.
#ifndef FKADJ_OWN_EXP
#define FKADJ_OWN_EXP 2
#endif

#if FKADJ_OWN_EXP == 2
// 2^(j/16), j = 0..15, as the kernels read them (one copy per CTA)
__shared__ double fk_exp2_tab[16];
__constant__ double kExp2Tab[16] = {
    0x1.0000000000000p+0, 0x1.0b5586cf9890fp+0, 0x1.172b83c7d517bp+0, 0x1.2387a6e756238p+0,
    0x1.306fe0a31b715p+0, 0x1.3dea64c123422p+0, 0x1.4bfdad5362a27p+0, 0x1.5ab07dd485429p+0,
    0x1.6a09e667f3bcdp+0, 0x1.7a11473eb0187p+0, 0x1.8ace5422aa0dbp+0, 0x1.9c49182a3f090p+0,
    0x1.ae89f995ad3adp+0, 0x1.c199bdd85529cp+0, 0x1.d5818dcfba487p+0, 0x1.ea4afa2a490dap+0};
#endif

// Every kernel that evaluates the model calls this before its first CTA
// barrier (the table form fills its shared table; the others do nothing).
__device__ __forceinline__ void exp_table_init() {
#if FKADJ_OWN_EXP == 2
    if (threadIdx.x < 16) fk_exp2_tab[threadIdx.x] = kExp2Tab[threadIdx.x];
#endif
}

__device__ __forceinline__ double fk_exp(double x) {
#if FKADJ_OWN_EXP == 1
    constexpr double kShift = 0x1.8p52;
    const double t = fma(x, 0x1.71547652b82fep+0, kShift);  // 1.5 2^52 + rint(x / ln2)
    const double kd = t - kShift;
    int k = __double2loint(t);
    double r = fma(kd, -0x1.62e42fefa3800p-1, x);  // exact: ln2_hi has 42 significant bits
    r = fma(kd, -0x1.ef35793c76730p-45, r);
    double p = 0x1.af631d0059becp-26;
    p = fma(p, r, 0x1.28b4057f44145p-22);
    p = fma(p, r, 0x1.71ddf5749d126p-19);
    p = fma(p, r, 0x1.a01991ac8730ap-16);
    p = fma(p, r, 0x1.a01a01b14378fp-13);
    p = fma(p, r, 0x1.6c16c187fbe02p-10);
    p = fma(p, r, 0x1.111111110f225p-7);
    p = fma(p, r, 0x1.555555554f0cfp-5);
    p = fma(p, r, 0x1.555555555555ap-3);
    p = fma(p, r, 0x1.0000000000011p-1);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    k = min(max(k, -1020), 999);
    return p * __hiloint2double((k + 1023) << 20, 0);  // times 2^k, exactly
#elif FKADJ_OWN_EXP == 2
    constexpr double kShift = 0x1.8p52;
    const double t = fma(x, 0x1.71547652b82fep+4, kShift);  // 1.5 2^52 + rint(16 x / ln2)
    const double kd = t - kShift;
    const int k = __double2loint(t);
    double r = fma(kd, -0x1.62e42fefa0000p-5, x);  // exact: (ln2/16)_hi has 36 significant bits
    r = fma(kd, -0x1.cf79abc9e3b3ap-44, r);
    double q = 0x1.6c17bb51f236dp-10;
    q = fma(q, r, 0x1.11120af701debp-7);
    q = fma(q, r, 0x1.55555555194d2p-5);
    q = fma(q, r, 0x1.55555554dd44dp-3);
    q = fma(q, r, 0.5);
    const double pm1 = fma(r * r, q, r);  // e^r - 1
    const int m = min(max(k >> 4, -1020), 998);  // k >> 4 = floor(k / 16)
    const double T = fk_exp2_tab[k & 15];
    // 2^m 2^(j/16): m added to the exponent field (T in [1, 2), m clamped)
    const double Ts = __hiloint2double(__double2hiint(T) + (m << 20), __double2loint(T));
    return fma(Ts, pm1, Ts);
#else
    return exp(x);
#endif
}

// Smoothed step s = (1 + tanh x)/2 written as the logistic 1/(1 + e^{-2x})
// (the same function; one exp and one reciprocal instead of a tanh) and its
// complement 1 - s = e^{-2x} s without cancellation.  e^{-2x} overflows to
// +inf for x < -354 and gives s = 0, 1 - s = 1 as tanh does.
struct Step {
    double s, c;  // s and 1 - s
};
//
// FKADJ_FAST_STEPS: e is capped at 2^1000 first, so 1 + e stays finite and s
// positive, and neither the reciprocal's +inf test nor the s = 0 test is
// needed.  Below the cap (|x| < 346, i.e. u more than 3.4 below u_c for the
// p step: far outside the model's range) the value is the same to the bit;
// above it s is 2^-1000 instead of 0 and 1 - s is 1.
__device__ __forceinline__ Step step_of_exp(double e) {
#if FKADJ_FAST_STEPS
#if FKADJ_OWN_EXP == 0
    e = fmin(e, 0x1p1000);  // the own exponentials stay below 2^1000 by themselves
#endif
    const double s = fk_rcp_finite(1.0 + e);
    return {s, e * s};
#else
    const double s = fk_rcp(1.0 + e);
    // s = 0 when 1 + e is +inf, or (own reciprocal) beyond 2^1022
    return {s, s == 0.0 ? 1.0 : e * s};
#endif
}
__device__ __forceinline__ Step smooth_step(double x) { return step_of_exp(fk_exp(-2.0 * x)); }

// e^{-2 k (u - u0)} as the smoothed steps take it; m2k = -2 k (the same product)
__device__ __forceinline__ double step_exp(double m2k, double k, double u, double u0) {
#if FKADJ_FAST_STEPS
    return fk_exp(m2k * (u - u0));
#else
    return fk_exp(-2.0 * (k * (u - u0)));
#endif
}

// p and q share the slope ksm, so q's exponential is p's times a constant:
// one exp for both.
__device__ __forceinline__ void steps_pq(const DevModel& P, double u, Step& sp, Step& sq) {
#if FKADJ_SHARED_EXP
    const double e = fk_exp(-2.0 * (P.ksm * (u - P.u_c)));
    sp = step_of_exp(e);
    sq = step_of_exp(e * P.eq);
#else
    sp = smooth_step(P.ksm * (u - P.u_c));
    sq = smooth_step(P.ksm * (u - P.u_v));
#endif
}

// The voltage-dependent time scale tau_v-(q) = q tau_v1- + (1 - q) tau_v2- of
// the v gate, with q = 1/(1 + eq), eq = e^{-2 ksm (u - u_v)}, only ever enters
// as its reciprocal (and, in the Jacobian, through dq/du): since
// tau_v- = (tau_v1- + eq tau_v2-) / (1 + eq),
//   1/tau_v- = (1 + eq) rT   and   4 q (1 - q) / tau_v-^2 = 4 eq rT^2,
// rT = 1 / (tau_v1- + eq tau_v2-): one reciprocal where q's logistic and the
// time scale took two.  Same function, rounding moved by about an ulp.  For
// eq beyond 1e300 (u < -3.4, far outside the model's range) the limits
// 1/tau_v2- and 0 are taken.
struct TvmRcp {
    double r;    // 1 / tau_v-
    double dqr;  // 4 q (1 - q) / tau_v-^2
};
__device__ __forceinline__ TvmRcp tvm_rcp(const DevModel& P, double eq) {
    if (eq > 1e300) return {P.r_tau_v2m, 0.0};
#if FKADJ_FAST_STEPS
    const double rT = fk_rcp_finite(fma(eq, P.tau_v2m, P.tau_v1m));  // finite: eq <= 1e300
#else
    const double rT = fk_rcp(fma(eq, P.tau_v2m, P.tau_v1m));
#endif
    return {(1.0 + eq) * rT, (4.0 * eq) * (rT * rT)};
}

// Ionic currents (formula of cu-F:29-45): p, q and (1 + tanh)/2 of the slow
// inward current are the three smoothed steps.
__device__ __forceinline__ void fk_ion(const DevModel& P, double u, double v, double w,
                                       double& ud, double& vd, double& wd) {
#if FKADJ_MERGED_TVM
    const double e = step_exp(P.m2ksm, P.ksm, u, P.u_c);
    const Step sp = step_of_exp(e);
    const double rtvm = tvm_rcp(P, e * P.eq).r;
#else
    Step sp, sq;
    steps_pq(P, u, sp, sq);
    const double q = sq.s;
    const double tvm = q * P.tau_v1m + sq.c * P.tau_v2m;
    const double rtvm = fk_rcp(tvm);
#endif
    const Step ss = step_of_exp(step_exp(P.m2kfk, P.k_fk, u, P.u_csi));
    const double p = sp.s;
    const double j_fi = -v * p * (1.0 - u) * (u - P.u_c) * P.r_tau_d;
    const double j_so = u * sp.c * P.r_tau_0 + p * P.r_tau_r;
    const double j_si = -w * (2.0 * ss.s) * P.r_2tau_si;
    ud = -(j_fi + j_so + j_si);
    vd = (sp.c * (1.0 - v)) * rtvm - (p * v) * P.r_tau_vp;
    wd = (sp.c * (1.0 - w)) * P.r_tau_wm - (p * w) * P.r_tau_wp;
}

// The seven non-zero entries of the transposed Jacobian of fk_ion
// (formula of cu-G:1160-1184): jt[0]=du'/du, jt[1]=dv'/du, jt[2]=dw'/du,
// jt[3]=du'/dv, jt[4]=dv'/dv, jt[5]=du'/dw, jt[6]=dw'/dw.
struct JacT {
    double a0, a1, a2, a3, a4, a5, a6;
};

// Jacobian entries as the reference writes them (0), or factored (1): the
// same derivatives with the common factors taken out and the constant
// products precomputed,
//   a0 = hk (v g r_d + u r_0 - r_r) + p v r_d ((1-u) - (u-u_c)) + k_fk r_2si w ds - (1-p) r_0,
//   a1 = (1-p)(1-v) (ksm dtau/2) dq/tau^2 - hk (v r_v+ + (1-v)/tau_v-),
//   a2 = -hk (w r_w+ + (1-w) r_w-),
// with hk = dp/du = 2 ksm p (1-p), g = (1-u)(u-u_c), ds = 4 s (1-s) of the
// slow inward step: about 20 FP64 instructions fewer per Jacobian, results
// moved by a few ulp (the gradient by 6e-16 relative).  Measured at 512^2 x
// 2000 steps: gradient 131.6 -> 131.0 ms (adjoint step 26.6 -> 26.1 us
// bracketed), so on by default.
#ifndef FKADJ_JAC_FACTORED
#define FKADJ_JAC_FACTORED 1
#endif

// 1 - tanh^2 = 4 s (1 - s) for the smoothed step s.
__device__ __forceinline__ JacT fk_jacT(const DevModel& P, double u, double v, double w) {
#if FKADJ_MERGED_TVM
    const double e = step_exp(P.m2ksm, P.ksm, u, P.u_c);
    const Step sp = step_of_exp(e);
    const TvmRcp tv = tvm_rcp(P, e * P.eq);
    const double rtvm = tv.r, dq_rtvm2 = tv.dqr;
#else
    Step sp, sq;
    steps_pq(P, u, sp, sq);
    const double q = sq.s;
    const double dq = 4.0 * sq.s * sq.c;
    const double tvm = q * P.tau_v1m + P.tau_v2m * sq.c;
    const double rtvm = fk_rcp(tvm);
    const double dq_rtvm2 = dq * (rtvm * rtvm);
#endif
    const Step ss = step_of_exp(step_exp(P.m2kfk, P.k_fk, u, P.u_csi));
#if FKADJ_JAC_FACTORED
    const double p = sp.s, cp = sp.c;
    const double hk = P.two_ksm * (p * cp);
    const double ds = 4.0 * (ss.s * ss.c);
    const double g1 = 1.0 - u, g2 = u - P.u_c;
    const double g12 = g1 * g2;
    const double pv = p * v;
    const double omv = 1.0 - v;
    JacT J;
    J.a3 = (p * g12) * P.r_tau_d;
    J.a5 = (2.0 * ss.s) * P.r_2tau_si;
    J.a0 = fma(hk, fma(v * g12, P.r_tau_d, fma(u, P.r_tau_0, -P.r_tau_r)),
               fma(pv * P.r_tau_d, g1 - g2, fma(P.kfk_r2tsi * w, ds, -(cp * P.r_tau_0))));
    J.a1 = fma((cp * omv) * P.hksm_dv12, dq_rtvm2, -(hk * fma(v, P.r_tau_vp, omv * rtvm)));
    J.a4 = -p * P.r_tau_vp - cp * rtvm;
    J.a2 = -(hk * fma(w, P.r_tau_wp, (1.0 - w) * P.r_tau_wm));
    J.a6 = -p * P.r_tau_wp - cp * P.r_tau_wm;
    return J;
#else
    const double p = sp.s;
    const double dp = 4.0 * sp.s * sp.c;
    const double ds = 4.0 * ss.s * ss.c;
    const double hk = 0.5 * dp * P.ksm;
    JacT J;
    J.a0 = -hk * P.r_tau_r + hk * v * (1.0 - u) * (u - P.u_c) * P.r_tau_d + hk * u * P.r_tau_0 +
           P.k_fk * w * ds * P.r_2tau_si + p * v * (1.0 - u) * P.r_tau_d -
           p * v * (u - P.u_c) * P.r_tau_d - sp.c * P.r_tau_0;
    J.a3 = p * (1.0 - u) * (u - P.u_c) * P.r_tau_d;
    J.a5 = (2.0 * ss.s) * P.r_2tau_si;
    J.a1 = -hk * v * P.r_tau_vp - hk * (1.0 - v) * rtvm + sp.c * (1.0 - v) * (0.5 * P.ksm * P.dv12) * dq_rtvm2;
    J.a4 = -p * P.r_tau_vp - sp.c * rtvm;
    J.a2 = -hk * w * P.r_tau_wp - hk * (1.0 - w) * P.r_tau_wm;
    J.a6 = -p * P.r_tau_wp - sp.c * P.r_tau_wm;
    return J;
#endif
}

// u as the exponentials see it.  Without the hole branch, holes (NaN) reach
// the ionic terms: they run on a finite u there, which keeps exp off its NaN
// path, and the Laplacian / adjoint-stencil terms still make the result NaN.
__device__ __forceinline__ double finite_u(double u) {
#if FKADJ_HOLE_BRANCH
    return u;
#else
    return isnan(u) ? 0.0 : u;
#endif
}

// NaN tests of the forward stencil (the hole test and the four mirrored
// neighbours): FP64 compares (0), or integer tests of the high word (1), which
// keep them off the FP64 pipe.  The integer test sees every NaN whose
// significand has a bit set in its high word, i.e. every NaN arithmetic or the
// NaN ring produces (quiet NaNs); a signalling NaN with only low-word payload
// bits would pass for an infinity, and none is ever stored.  Measured slower
// (forward step 15.6 against 15.4 us at 512^2: the integer tests take more
// issue slots than the compares take FP64 cycles), so off.
#ifndef FKADJ_INT_NAN
#define FKADJ_INT_NAN 0
#endif
__device__ __forceinline__ bool stencil_nan(double x) {
#if FKADJ_INT_NAN
    return ((unsigned)__double2hiint(x) << 1) > 0xffe00000u;
#else
    return isnan(x);
#endif
}

// Forward stencil codes (FC_*) in place of the NaN tests: measured slower on
// B200 (forward step 18.3 against 17.0 us at 512^2), so off by default.
#ifndef FKADJ_FWD_CODES
#define FKADJ_FWD_CODES 0
#endif

// Forward vector field at shared-memory cell q of a region W doubles wide with
// field planes RN apart: 5-point Laplacian with NaN mirroring + F_ion + E*gh.
// code: the cell's forward stencil code, or -1 to test the values for NaN.
template <int W, int RN>
__device__ __forceinline__ void rhs_at(const DevModel& P, const double* __restrict__ Y, int q,
                                       double Egh, double& fu, double& fv, double& fw, int code = -1) {
    const double u = Y[q];
#if FKADJ_FWD_CODES
    if (code >= 0) {
        if (code & FC_HOLE) {  // a hole or the NaN ring: its value is NaN, and so is the result
            fu = fv = fw = u;
            return;
        }
        const int oa = (code & FC_N) ? W : -W, ob = (code & FC_S) ? -W : W;
        const int oc = (code & FC_W) ? 1 : -1, od = (code & FC_E) ? -1 : 1;
        const double v = Y[RN + q], w = Y[2 * RN + q];
        const double* Yv = Y + RN;
        const double* Yw = Y + 2 * RN;
        const double lu = P.cu * ((((Y[q + oa] + Y[q + ob]) + Y[q + oc]) + Y[q + od]) - 4.0 * u);
        const double lv = P.cv * ((((Yv[q + oa] + Yv[q + ob]) + Yv[q + oc]) + Yv[q + od]) - 4.0 * v);
        const double lw = P.cw * ((((Yw[q + oa] + Yw[q + ob]) + Yw[q + oc]) + Yw[q + od]) - 4.0 * w);
        double ud, vd, wd;
        fk_ion(P, u, v, w, ud, vd, wd);
        fu = (lu + ud) + Egh;
        fv = lv + vd;
        fw = lw + wd;
        return;
    }
#endif
#if FKADJ_HOLE_BRANCH
    // holes and the NaN ring skip the arithmetic (their result is NaN either way)
    if (stencil_nan(u)) {
        fu = fv = fw = u;
        return;
    }
#endif
    const double v = Y[RN + q], w = Y[2 * RN + q];
    const double un = Y[q - W], us = Y[q + W], uw = Y[q - 1], ue = Y[q + 1];
    const bool nN = stencil_nan(un), nS = !nN && stencil_nan(us);
    const bool nW = stencil_nan(uw), nE = !nW && stencil_nan(ue);
#if FKADJ_MIRROR_OFFSETS
    // the same neighbours as the selects below, read where they are
    const int qa = nN ? q + W : q - W, qb = nS ? q - W : q + W;
    const int qc = nW ? q + 1 : q - 1, qd = nE ? q - 1 : q + 1;
#if FKADJ_MIRROR_OFFSETS == 2
    const double a_u = Y[qa], b_u = Y[qb], c_u = Y[qc], d_u = Y[qd];
#else
    const double a_u = nN ? us : un, b_u = nS ? un : us, c_u = nW ? ue : uw, d_u = nE ? uw : ue;
#endif
    const double* Yv = Y + RN;
    const double* Yw = Y + 2 * RN;
    const double lu = P.cu * ((((a_u + b_u) + c_u) + d_u) - 4.0 * u);
    const double lv = P.cv * ((((Yv[qa] + Yv[qb]) + Yv[qc]) + Yv[qd]) - 4.0 * v);
    const double lw = P.cw * ((((Yw[qa] + Yw[qb]) + Yw[qc]) + Yw[qd]) - 4.0 * w);
#else
    const double vn = Y[RN + q - W], vs = Y[RN + q + W], vw = Y[RN + q - 1], ve = Y[RN + q + 1];
    const double wn = Y[2 * RN + q - W], ws = Y[2 * RN + q + W], ww = Y[2 * RN + q - 1],
                 we = Y[2 * RN + q + 1];
    // neighbour pairs after mirroring (cu-F:319-420); selects, not a branch to
    // a plain sum away from holes, which measured 4 % slower on the forward step
    const double a_u = nN ? us : un, b_u = nS ? un : us, c_u = nW ? ue : uw, d_u = nE ? uw : ue;
    const double a_v = nN ? vs : vn, b_v = nS ? vn : vs, c_v = nW ? ve : vw, d_v = nE ? vw : ve;
    const double a_w = nN ? ws : wn, b_w = nS ? wn : ws, c_w = nW ? we : ww, d_w = nE ? ww : we;
    const double lu = P.cu * ((((a_u + b_u) + c_u) + d_u) - 4.0 * u);
    const double lv = P.cv * ((((a_v + b_v) + c_v) + d_v) - 4.0 * v);
    const double lw = P.cw * ((((a_w + b_w) + c_w) + d_w) - 4.0 * w);
#endif
    double ud, vd, wd;
    fk_ion(P, finite_u(u), v, w, ud, vd, wd);
    fu = (lu + ud) + Egh;
    fv = lv + vd;
    fw = lw + wd;
}

// Weight code of the transposed Laplacian at a cell: 2 bits per direction
// (north, south, west, east), value 0 (neighbour missing), 1, or 2 (the
// neighbour mirrored this cell); rule of cu-G:1004-1111.
__device__ __forceinline__ int wcode_n(int c) { return c & 3; }
__device__ __forceinline__ int wcode_s(int c) { return (c >> 2) & 3; }
__device__ __forceinline__ int wcode_w(int c) { return (c >> 4) & 3; }
__device__ __forceinline__ int wcode_e(int c) { return (c >> 6) & 3; }

// Adjoint vector field L^T z + J_F(y)^T z at shared-memory cell q.
template <int W, int RN>
__device__ __forceinline__ void adj_at(const DevModel& P, const double* __restrict__ Z, int q,
                                       int code, const JacT& J, double& gu, double& gv,
                                       double& gw) {
    const double z0 = Z[q], z1 = Z[RN + q], z2 = Z[2 * RN + q];
    const int cn = wcode_n(code), cs = wcode_s(code), cw = wcode_w(code), ce = wcode_e(code);
    const double pn = (double)cn, ps = (double)cs, pw = (double)cw, pe = (double)ce;
    double l[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        const double* Zf = Z + f * RN;
        const double vn = cn ? Zf[q - W] : 0.0;  // integer tests: no FP64 compares
        const double vs = cs ? Zf[q + W] : 0.0;
        const double vw = cw ? Zf[q - 1] : 0.0;
        const double ve = ce ? Zf[q + 1] : 0.0;
        const double c = f == 0 ? P.cu : (f == 1 ? P.cv : P.cw);
        l[f] = c * ((((pn * vn + ps * vs) + pw * vw) + pe * ve) - 4.0 * Zf[q]);
    }
    gu = l[0] + ((J.a0 * z0 + J.a1 * z1) + J.a2 * z2);
    gv = l[1] + (J.a3 * z0 + J.a4 * z1);
    gw = l[2] + (J.a5 * z0 + J.a6 * z2);
}

}  // namespace fkadj
