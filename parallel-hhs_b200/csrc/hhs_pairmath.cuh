// hhs_pairmath.cuh -- per-pair arithmetic of the timestep and kick, in two precisions.
//
// FP64 ("exact") forms follow the reference expressions operation by operation
// (src/timestep.cuh:27-57, src/kick.cuh:19-30) with explicit round-to-nearest
// intrinsics, so no multiply-add is ever contracted and results are bit-identical
// to an IEEE binary64 evaluation on the host.
//
// Mixed forms take FP64 relative coordinates through a double-single split
// (x = hi + lo, both FP32; dx = (hi_j - hi_i) + (lo_j - lo_i), where the hi
// difference is exact for nearby particles by Sterbenz's lemma) and evaluate the
// pair terms in FP32 with rsqrt refined by one Newton-Raphson step
// y1 = y0 * (3 - x*y0^2) / 2.
#pragma once
#include <cuda_runtime.h>

namespace hhs {

__device__ __forceinline__ double f64_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double f64_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double f64_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double f64_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double f64_sqrt(double a) { return __dsqrt_rn(a); }

// Pair timestep (src/timestep.cuh:27-57), dr = x_i - x_j, dv = v_i - v_j.
// eta_s2 = eta / M_SQRT2. Updates minval with both candidate timescales.
__device__ __forceinline__ void ts_pair_fp64(double drx, double dry, double drz, double dvx,
                                             double dvy, double dvz, double mi, double mj,
                                             double eta, double eta_s2, double& minval) {
    const double dr2 = f64_add(f64_add(f64_mul(drx, drx), f64_mul(dry, dry)), f64_mul(drz, drz));
    const double dv2 = f64_add(f64_add(f64_mul(dvx, dvx), f64_mul(dvy, dvy)), f64_mul(dvz, dvz));
    const double r = f64_sqrt(dr2);
    const double vdotdr2 =
        f64_div(f64_add(f64_add(f64_mul(dvx, drx), f64_mul(dvy, dry)), f64_mul(dvz, drz)), dr2);
    double tau = f64_mul(f64_mul(eta_s2, r), f64_sqrt(f64_div(r, f64_add(mj, mi))));
    double dtau = f64_mul(f64_mul(f64_mul(3.0, tau), vdotdr2), 0.5);
    dtau = (dtau < 1.0) ? dtau : 1.0;
    tau = f64_div(tau, f64_sub(1.0, f64_mul(dtau, 0.5)));
    if (tau < minval) minval = tau;
    tau = f64_div(f64_mul(eta, r), f64_sqrt(dv2));
    dtau = f64_mul(f64_mul(tau, vdotdr2), f64_add(1.0, f64_div(f64_add(mi, mj), f64_mul(dv2, r))));
    dtau = (dtau < 1.0) ? dtau : 1.0;
    tau = f64_div(tau, f64_sub(1.0, f64_mul(dtau, 0.5)));
    if (tau < minval) minval = tau;
}

// Pair acceleration (src/kick.cuh:19-30 with the attractive sign of
// tests/test_nbforce.cu:14-18): dx = x_j - x_i, skip d2 == 0, a += dx * (m_j/(d2*d)).
// eps2 is the squared softening length the reference stores but never applies
// (src/particle_system.cuh:16, TODOs at src/hold.cuh:136,141,157); with eps2 = 0 the
// result is unchanged bit for bit (d2 + 0 == d2).
__device__ __forceinline__ void kick_pair_fp64(double dx, double dy, double dz, double mj,
                                               double& ax, double& ay, double& az,
                                               double eps2 = 0.0) {
    const double d2 = f64_add(
        f64_add(f64_add(f64_mul(dx, dx), f64_mul(dy, dy)), f64_mul(dz, dz)), eps2);
    if (d2 == 0.0) return;
    const double d = f64_sqrt(d2);
    const double s = f64_mul(mj, f64_div(1.0, f64_mul(d2, d)));
    ax = f64_add(ax, f64_mul(dx, s));
    ay = f64_add(ay, f64_mul(dy, s));
    az = f64_add(az, f64_mul(dz, s));
}

// ---- mixed precision -------------------------------------------------------------

struct DS {  // double-single: value = hi + lo
    float hi, lo;
};

__device__ __forceinline__ DS ds_split(double v) {
    DS r;
    r.hi = __double2float_rn(v);
    r.lo = __double2float_rn(v - (double)r.hi);
    return r;
}

// (a - b) of two double-single numbers, rounded to FP32
__device__ __forceinline__ float ds_diff(float ahi, float alo, float bhi, float blo) {
    return __fadd_rn(__fsub_rn(ahi, bhi), __fsub_rn(alo, blo));
}

__device__ __forceinline__ float rsqrt_nr(float x) {
    const float y = rsqrtf(x);
    return y * fmaf(-0.5f * x, y * y, 1.5f);
}

// m / d^3 from rsqrtf(d2) with one Newton-Raphson correction folded into the cube:
// y^3 (2.5 - 1.5 d2 y^2), whose relative error is second order in rsqrtf's; 0 when d2 == 0
// (a particle and itself).
__device__ __forceinline__ float mr3_nr(float m, float d2) {
    const float y = rsqrtf(d2);
    const float y2 = y * y;
    const float c = fmaf(-1.5f, d2 * y2, 2.5f);
    return d2 > 0.0f ? m * (y2 * y) * c : 0.0f;
}

// Kahan-compensated accumulation s += t (c holds the running compensation).
__device__ __forceinline__ void kahan_add(float& s, float& c, float t) {
    const float y = __fsub_rn(t, c);
    const float u = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(u, s), y);
    s = u;
}

// Pair timestep as a rate (1/tau) in FP32; min over tau == max over rates.
// Free-fall: rate0 = sqrt(M/r^3)/eta_s2; the reference's correction
// tau/(1 - dtau/2) with dtau = 1.5*tau0*vdotdr2 clamped at 1 becomes
// rate0 - 0.75*vdotdr2 (or rate0/2 when clamped). Fly-by: rate0 = |dv|/(eta*r),
// dtau = vdotdr2*(1 + M/(dv2*r))/rate0, likewise. dr2 == 0 gives +inf (tau = 0 in
// the reference). dv2 == 0 makes the fly-by rate NaN (rsqrt(0) = inf times 0), which
// fmaxf discards: the pair's rate is then the free-fall one, as tau = inf for the
// fly-by term in the reference. The three reciprocal square roots are rsqrtf without a
// Newton step: its error (a few units in the last place, ~2e-7 relative) is far inside
// the timestep tolerance, and the timestep only selects the level of each particle.
__device__ __forceinline__ float ts_pair_rate_mixed(float drx, float dry, float drz, float dvx,
                                                    float dvy, float dvz, float msum,
                                                    float inv_eta_s2, float inv_eta) {
    const float dr2 = fmaf(drx, drx, fmaf(dry, dry, drz * drz));
    const float dv2 = fmaf(dvx, dvx, fmaf(dvy, dvy, dvz * dvz));
    const float rdv = fmaf(drx, dvx, fmaf(dry, dvy, drz * dvz));
    const float rinv = rsqrtf(dr2);
    const float rinv2 = rinv * rinv;
    const float vdr = rdv * rinv2;
    const float mr1 = msum * rinv;
    const float u = mr1 * rinv2;
    const float r0 = u * rsqrtf(u) * inv_eta_s2;
    const float b0 = 1.5f * vdr;
    // (b0 < r0) ? r0 - b0/2 : r0/2, as r0 - min(b0, r0)/2 (the same value: r0 - r0/2 is
    // exact, and fminf keeps r0 when b0 is NaN, as the comparison does)
    const float rate_ff = fmaf(-0.5f, fminf(b0, r0), r0);
    const float q = rsqrtf(dv2);
    const float r1 = dv2 * q * rinv * inv_eta;
    const float b1 = vdr * fmaf(mr1, q * q, 1.0f);
    const float rate_fb = fmaf(-0.5f, fminf(b1, r1), r1);
    const float rate = fmaxf(rate_ff, rate_fb);
    return dr2 == 0.0f ? __int_as_float(0x7f800000) : rate;
}

// ---- packed FP32 pairs (sm_100 f32x2) ----------------------------------------------
// A sink against two sources at once in f32x2 arithmetic: the sink's values come negated
// and duplicated, the sources' as pairs. Every lane runs the operations of
// ts_pair_rate_mixed in the same order on the negated offsets (source minus sink), whose
// squares and products are those of the scalar form, so each lane's rate equals it bit
// for bit.
struct TsSink2 {
    float2 nxh, nyh, nzh, nxl, nyl, nzl, nvx, nvy, nvz, m;
};

__device__ __forceinline__ float2 f2dup(float v) { return make_float2(v, v); }

__device__ __forceinline__ float2 ts_pair_rate_mixed2(float2 xh, float2 yh, float2 zh, float2 xl,
                                                      float2 yl, float2 zl, float2 vx, float2 vy,
                                                      float2 vz, float2 m, const TsSink2& s,
                                                      float inv_eta_s2, float inv_eta) {
    const float2 drx = __fadd2_rn(__fadd2_rn(xh, s.nxh), __fadd2_rn(xl, s.nxl));
    const float2 dry = __fadd2_rn(__fadd2_rn(yh, s.nyh), __fadd2_rn(yl, s.nyl));
    const float2 drz = __fadd2_rn(__fadd2_rn(zh, s.nzh), __fadd2_rn(zl, s.nzl));
    const float2 dvx = __fadd2_rn(vx, s.nvx), dvy = __fadd2_rn(vy, s.nvy),
                 dvz = __fadd2_rn(vz, s.nvz);
    const float2 dr2 = __ffma2_rn(drx, drx, __ffma2_rn(dry, dry, __fmul2_rn(drz, drz)));
    const float2 dv2 = __ffma2_rn(dvx, dvx, __ffma2_rn(dvy, dvy, __fmul2_rn(dvz, dvz)));
    const float2 rdv = __ffma2_rn(drx, dvx, __ffma2_rn(dry, dvy, __fmul2_rn(drz, dvz)));
    const float2 rinv = make_float2(rsqrtf(dr2.x), rsqrtf(dr2.y));
    const float2 rinv2 = __fmul2_rn(rinv, rinv);
    const float2 vdr = __fmul2_rn(rdv, rinv2);
    const float2 mr1 = __fmul2_rn(__fadd2_rn(s.m, m), rinv);
    const float2 u = __fmul2_rn(mr1, rinv2);
    const float2 ru = make_float2(rsqrtf(u.x), rsqrtf(u.y));
    const float2 r0 = __fmul2_rn(__fmul2_rn(u, ru), f2dup(inv_eta_s2));
    const float2 b0 = __fmul2_rn(f2dup(1.5f), vdr);
    const float2 rff =
        __ffma2_rn(f2dup(-0.5f), make_float2(fminf(b0.x, r0.x), fminf(b0.y, r0.y)), r0);
    const float2 q = make_float2(rsqrtf(dv2.x), rsqrtf(dv2.y));
    const float2 r1 = __fmul2_rn(__fmul2_rn(__fmul2_rn(dv2, q), rinv), f2dup(inv_eta));
    const float2 b1 = __fmul2_rn(vdr, __ffma2_rn(mr1, __fmul2_rn(q, q), f2dup(1.0f)));
    const float2 rfb =
        __ffma2_rn(f2dup(-0.5f), make_float2(fminf(b1.x, r1.x), fminf(b1.y, r1.y)), r1);
    const float inf = __int_as_float(0x7f800000);
    return make_float2(dr2.x == 0.0f ? inf : fmaxf(rff.x, rfb.x),
                       dr2.y == 0.0f ? inf : fmaxf(rff.y, rfb.y));
}

__device__ __forceinline__ float2 rsqrt_nr2(float2 x) {
    const float2 y = make_float2(rsqrtf(x.x), rsqrtf(x.y));
    return __fmul2_rn(y, __ffma2_rn(__fmul2_rn(x, make_float2(-0.5f, -0.5f)), __fmul2_rn(y, y),
                                    make_float2(1.5f, 1.5f)));
}

}  // namespace hhs
