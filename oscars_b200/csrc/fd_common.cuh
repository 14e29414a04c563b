// fd_common.cuh -- device pieces shared by the single-trajectory and the batched radiation kernels:
// the trajectory spline evaluation at a level time, the mixed-precision per-sample term, the
// complex 3-vector helpers of the stop rule and the lane-group reductions of the finalize kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace osc {
namespace dev {

constexpr double kCLight = 2.99792458e8;
constexpr double kPiD = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------------
// Trajectory spline at time T (TSpline1D3::GetValue, include/TOMATH.h:92-121) for the 9 components
// x y z bx by bz ax ay az.  `knots` is the SoA block t[n] | y[9][n] | ypp[9][n].  The interval
// search returns the reference bisection's result (largest k in [0, n-2] with t[k] <= T), started
// from the uniform-spacing estimate and corrected by local steps.  Round-to-nearest intrinsics keep
// the reference's association order, so values are bit-identical to the reference CPU build.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void spline_eval9(const double* __restrict__ knots, int64_t n, double T, double* v) {
  const double* t = knots;
  const double* y = knots + n;
  const double* ypp = knots + 10 * n;
  int64_t k = (int64_t)((T - t[0]) / (t[n - 1] - t[0]) * (double)(n - 1));
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  while (k > 0 && t[k] > T) --k;
  while (k < n - 2 && t[k + 1] <= T) ++k;
  const int64_t klo = k, khi = k + 1;
  const double h = __dsub_rn(t[khi], t[klo]);
  const double a = __ddiv_rn(__dsub_rn(t[khi], T), h);
  const double b = __ddiv_rn(__dsub_rn(T, t[klo]), h);
  const double ca = __dsub_rn(__dmul_rn(__dmul_rn(a, a), a), a);
  const double cb = __dsub_rn(__dmul_rn(__dmul_rn(b, b), b), b);
  const double hh = __dmul_rn(h, h);
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const double* Y = y + c * n;
    const double* P = ypp + c * n;
    const double lin = __dadd_rn(__dmul_rn(a, Y[klo]), __dmul_rn(b, Y[khi]));
    const double cur = __ddiv_rn(__dmul_rn(__dadd_rn(__dmul_rn(ca, P[klo]), __dmul_rn(cb, P[khi])), hh), 6.0);
    v[c] = __dadd_rn(lin, cur);
  }
}

// Time of sample s of the level ladder (level L = floor(log2 s), i = s - 2^L):
// tstart + T/2^(L+1) + i T/2^L  (src/TParticleTrajectoryInterpolated.cc:124-158).
__device__ __forceinline__ double level_time(double tstart, double tstop, int64_t s) {
  const int L = 63 - __clzll((unsigned long long)s);
  const int64_t i = s - ((int64_t)1 << L);
  const double ts = __dadd_rn(tstart, __ddiv_rn(__dsub_rn(tstop, tstart), ldexp(1.0, L + 1)));
  const double sp = __ddiv_rn(__dsub_rn(tstop, tstart), ldexp(1.0, L));
  return __dadd_rn(ts, __dmul_rn(sp, (double)i));
}

// ---------------------------------------------------------------------------------------------
// Mixed-precision per-sample term.  A sample is stored as 3 x float4 = 48 bytes in the particle
// frame (origin X0, third axis along the initial velocity):
//   r0 = (x, y, z, tau_s = t - t0/c - z/c)   r1 = (bx, by, 1-bz, 1-b^2)   r2 = (ax, ay, az, 0)
// With R = O - X, rho^2 = Rx^2 + Ry^2 and D = Rz + corr, corr = rho^2/(Rz + D) (series for
// |rho/D| < 1e-2), the retarded phase is -(w tau_s + (w/c) corr) up to the constant w Oz/c, and the
// amplitude (src/OSCARSSR.cc:4219) with u = n - b, om = 1 - n.b is
//   u (1/(D om^2)) ((1-b^2)/D + n.a) - a / (D om).
// Adds the term times exp(i phase) to s[6] (x re, x im, y re, y im, z re, z im); returns the phase.
// ---------------------------------------------------------------------------------------------
constexpr float kTwoPiHiF = 6.28318548202514648f;     // RN_f(2 pi)
constexpr float kTwoPiLoF = -1.7484556e-07f;         // RN_f(2 pi - kTwoPiHiF)
constexpr float kInvTwoPiF = 0.159154943f;

__device__ __forceinline__ float mixed_sample(const float4 r0, const float4 r1, const float4 r2, float Ox, float Oy,
                                              float Oz, float w, float wc, float* s) {
  const float rx = Ox - r0.x, ry = Oy - r0.y, rz = Oz - r0.z;
  const float rho2 = fmaf(rx, rx, ry * ry);
  const float d2 = fmaf(rz, rz, rho2);
  const float iD = rsqrtf(d2);
  const float q = rho2 * iD * iD;                                  // (rho/D)^2
  const float corr = rho2 * iD * fmaf(0.125f, q, 0.5f);           // rho^2/(Rz+D), |rho/D| < 1e-2
  const float ph = -fmaf(wc, corr, w * r0.w);                      // exp(-i w (t + D/c))
  const float k = rintf(ph * kInvTwoPiF);
  const float rr = fmaf(-k, kTwoPiLoF, fmaf(-k, kTwoPiHiF, ph));  // Cody-Waite reduction to [-pi, pi]
  float sn, cs;
  __sincosf(rr, &sn, &cs);
  const float nx = rx * iD, ny = ry * iD;
  const float en = corr * iD;                                      // 1 - n_z
  const float ux = nx - r1.x, uy = ny - r1.y, uz = r1.z - en;
  const float om = fmaf(-nx, r1.x, fmaf(-ny, r1.y, fmaf(-en, r1.z, en + r1.z)));
  const float io = __fdividef(1.f, om);
  const float na = fmaf(nx, r2.x, fmaf(ny, r2.y, (1.f - en) * r2.z));
  const float k1 = io * io * iD * fmaf(r1.w, iD, na);
  const float k2 = io * iD;
  const float ex = fmaf(k1, ux, -k2 * r2.x);
  const float ey = fmaf(k1, uy, -k2 * r2.y);
  const float ez = fmaf(k1, uz, -k2 * r2.z);
  s[0] = fmaf(ex, cs, s[0]); s[1] = fmaf(ex, sn, s[1]);
  s[2] = fmaf(ey, cs, s[2]); s[3] = fmaf(ey, sn, s[3]);
  s[4] = fmaf(ez, cs, s[4]); s[5] = fmaf(ez, sn, s[5]);
  return ph;
}

// Validity of the near-axis phase form for an observer at (fx, fy, fz) in the particle frame: small
// angle from the frame axis and a bounded correction phase; otherwise the FP64 path must be used.
__device__ __forceinline__ bool mixed_geometry_ok(double fx, double fy, double fz, double om, double xperp_max,
                                                  double z_max) {
  const double rho = sqrt(fx * fx + fy * fy) + xperp_max;
  const double rz = fz - z_max;
  return rz > 0 && rho < 1e-2 * rz && (om / kCLight) * rho * rho / (2 * rz) < 3e4;
}

// ---------------------------------------------------------------------------------------------
// Complex 3-vectors of the stop rule.
// ---------------------------------------------------------------------------------------------
struct C3 { double xr, xi, yr, yi, zr, zi; };

__device__ __forceinline__ C3 c3_scale(C3 a, double s) {
  return {a.xr * s, a.xi * s, a.yr * s, a.yi * s, a.zr * s, a.zi * s};
}
// (E . P) P with the complex (unconjugated) dot product of TVector3DC::Dot.
__device__ __forceinline__ C3 c3_project(C3 e, const double* P) {
  const double cr = (e.xr * P[0] - e.xi * P[1]) + (e.yr * P[2] - e.yi * P[3]) + (e.zr * P[4] - e.zi * P[5]);
  const double ci = (e.xr * P[1] + e.xi * P[0]) + (e.yr * P[3] + e.yi * P[2]) + (e.zr * P[5] + e.zi * P[4]);
  return {P[0] * cr - P[1] * ci, P[0] * ci + P[1] * cr, P[2] * cr - P[3] * ci,
          P[2] * ci + P[3] * cr, P[4] * cr - P[5] * ci, P[4] * ci + P[5] * cr};
}
__device__ __forceinline__ double c3_mag2(C3 a) {
  return (a.xr * a.xr + a.xi * a.xi) + (a.yr * a.yr + a.yi * a.yi) + (a.zr * a.zr + a.zi * a.zi);
}

// Span partials of one entry are reduced by a group of kFinLanes lanes: lane l sums the spans
// l, l + kFinLanes, ... in order, then a fixed shuffle tree combines the lanes (deterministic).
constexpr int kFinLanes = 8;

__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = kFinLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, kFinLanes);
  return v;
}
__device__ __forceinline__ double group_max(double v) {
#pragma unroll
  for (int o = kFinLanes / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o, kFinLanes));
  return v;
}

}  // namespace dev
}  // namespace osc
