// fd_common.cuh -- device pieces shared by the single-trajectory and the batched radiation kernels:
// the trajectory spline evaluation at a level time, the mixed-precision per-sample term, the
// complex 3-vector helpers of the stop rule and the lane-group reductions of the finalize kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

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
// tstart + T/2^(L+1) + i dt_L.  Levels up to ext_from are the ones the reference holds in memory,
// dt_L = T/2^L (src/TParticleTrajectoryInterpolated.cc:124-158); the levels above them are its
// extended levels, evaluated on the fly with dt_L = T/(2^L - 1) (TParticleTrajectoryInterpolatedPoints::Set
// and GetT, src/TParticleTrajectoryInterpolatedPoints.cc:32-55; GetDeltaTThisLevel,
// src/TParticleTrajectoryInterpolated.cc:242-251).  Extended levels do not nest with the lower ones and
// their last samples lie past tstop, where the spline continues its last interval's cubic, as the
// reference's does.
__device__ __forceinline__ double level_time(double tstart, double tstop, int64_t s, int ext_from) {
  const int L = 63 - __clzll((unsigned long long)s);
  const int64_t i = s - ((int64_t)1 << L);
  const double ts = __dadd_rn(tstart, __ddiv_rn(__dsub_rn(tstop, tstart), ldexp(1.0, L + 1)));
  const double sp = __ddiv_rn(__dsub_rn(tstop, tstart), L > ext_from ? __dsub_rn(ldexp(1.0, L), 1.0) : ldexp(1.0, L));
  return __dadd_rn(ts, __dmul_rn(sp, (double)i));
}

// ---------------------------------------------------------------------------------------------
// Mixed-precision sample term over pair records.
//
// Frame: origin X0 (the particle start), third axis e3 along the initial velocity, so observers
// downstream sit near the axis.  With R = O - X = (Rx, Ry, Rz) in that frame, rho^2 = Rx^2 + Ry^2,
//     D = |R| = Rz + corr,   corr = rho^2 / (Rz + D)                      (no cancellation)
//     w (t + D/c) = w tau_s + (w/c) corr + w Oz/c,   tau_s = t - t0/c - z/c
// The last term is a constant phase per (observer, energy) entry: it multiplies the whole sum by a
// unit complex number and drops out of |E|^2, of the polarization projection and of the phase steps
// of the stop rule, so it is not computed.  Phases are carried in turns (units of 2 pi).
//
// Phase of the pair's first sample, FP64.  corr is first formed in FP32 (relative error ~1e-7 -- a
// few 1e-3 rad when (w/c) corr reaches 1e4 rad, too much for a 1e-4 flux tolerance).  One Newton step
// on f(c) = c (c + 2 Rz) - rho^2, whose root is D - Rz, refines it in FP64 from the FP64 position:
//     c1 = c - f(c) / f'(c),   f'(c) = 2 (c + Rz) = 2 D,
// with 1/(2D) taken from the FP32 rsqrt (its 1e-7 error multiplies a correction that is itself 1e-7
// of c), so c1 is exact to ~1e-14 relative.  The phase in turns, (w/2pi) tau_s + (w/2pi c) c1, is
// accumulated onto 1.5 * 2^22: for |turns| < 2^21 the sum keeps the binade [2^22, 2^23), whose
// significand has 30 bits below the units place, so the fraction of a turn is read off the low
// word of the double (rounded to 2^-30 turns, then to the 23 bits of a float: < 4e-7 rad).
//
// Phase of the second sample, FP32 step from the first.  With dR = R1 - R0 = -(X1 - X0) and
// S = R1 + R0 (exact in FP64, stored as FP32 in the record),
//     corr1 - corr0 = (D1 - D0) - dRz = (dRx Sx + dRy Sy - dRz (corr0 + corr1)) / (D0 + D1)
// [D1^2 - D0^2 = dR . S and Sz - D0 - D1 = -(corr0 + corr1)], a quotient of small terms with no
// cancellation; the step (w/2pi) dtau_s + (w/2pi c)(corr1 - corr0) is then good to a few 1e-7 of
// its own size (a few rad at convergence, where the stop rule bounds the steps by pi), and each
// pair restarts from its FP64 anchor, so errors do not accumulate along the trajectory.
//
// Amplitude, FP32 (src/OSCARSSR.cc:4219), with u = n - b, om = 1 - n.b and |n| = 1:
//     (1-b^2) u / (D^2 om^2) + n x (u x a) / (D om^2)
//   = u (1/(D om^2)) ((1-b^2)/D + n.a) - a / (D om)        [n x (u x a) = u (n.a) - a (n.u), n.u = om]
// with the small differences formed without cancellation from per-sample FP64-exact inputs:
//     1 - n_z = corr / D,  u_z = (1 - b_z) - (1 - n_z),  om = (1-b_z) + (1-n_z) b_z - n_x b_x - n_y b_y.
// The FP32 phase P32 = w tau_s + (w/c) corr of the same operands gives the phase steps of the stop
// rule (|P_j - P_{j-1}| < pi), where its ~1e-3 rad rounding is immaterial.
//
// Pair records: samples 2p and 2p + 1 share 36 floats (144 bytes).  Floats 0..23 hold the FP32
// components, component c of sample 2p + b at float 4 (c / 2) + 2 (c % 2) + b, with
//   x, y, z, tau_s | -bx, -by, 1-bz, bz | 1-b^2, az, ax, ay
// so that every half of a loaded float4 is one component of both samples (the operand of one packed
// f32x2 instruction); floats 24..27 hold dRx, dRy, dRz, dtau_s (second sample minus first); bytes
// 112..143 hold the FP64 x, y, z, tau_s of the first sample.  Sample 0, the unused slot of the level
// ladder, holds a zero-amplitude record at the position and time of sample 1 (no contribution, no
// phase step), so every span is a whole number of pairs.
// ---------------------------------------------------------------------------------------------
// Hardware approximations (MUFU) with denormals flushed: the terms never see denormal operands
// (distances ~1..100 m, 1 - n.b ~ 1e-9..1e-4, reduced phases in [-pi, pi]).
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ void sincos_ftz(float x, float* s, float* c) {
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(*s) : "f"(x));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(*c) : "f"(x));
}

constexpr int kPairFloats = 36;                        // floats per pair record (144 bytes)
constexpr int kPairF4 = kPairFloats / 4;               // float4 per pair record
constexpr double kTwoPiD = 6.283185307179586;          // RN(2 pi)
constexpr float kTwoPiF = 6.28318548202514648f;        // RN_f(2 pi)
constexpr double kTurnBase = 6291456.0;                // 1.5 * 2^22 (see fp64_turns)
// Largest |phase| in turns the FP64 accumulation onto kTurnBase allows (2^21), with a factor 2 of
// margin; the host-side guard (mixed_geometry_ok) keeps every sample's phase below it.
constexpr double kMaxTurns = 1048576.0;

// Record of one level sample (FP64 values in the particle frame) at sample index s of pair record
// storage `rec` (s even-aligned with the level ladder).  zero_amplitude writes the record of sample 0
// (the position and time of sample 1 must be passed for it).  (xo, yo, zo, tauo) are the FP64 values
// of the pair's other sample: the odd sample writes the step from the even one, the even sample its
// FP64 values.
__device__ __forceinline__ void write_pair_record(float* __restrict__ rec, int64_t s, bool zero_amplitude, double x,
                                                  double y, double z, double taus, double px, double py, double pz,
                                                  double qx, double qy, double qz, double xo, double yo, double zo,
                                                  double tauo) {
  const double g2 = 1.0 - (px * px + py * py + pz * pz);       // 1 - b^2, ~1/gamma^2
  const double ebz = (g2 + px * px + py * py) / (1.0 + pz);     // 1 - b_z without cancellation
  float v[12] = {(float)x, (float)y, (float)z, (float)taus, (float)-px, (float)-py,
                 (float)ebz, (float)pz, (float)g2, (float)qz, (float)qx, (float)qy};
  if (zero_amplitude) {
    v[4] = v[5] = 0.f;
    v[6] = 1.f;
    v[7] = v[8] = v[9] = v[10] = v[11] = 0.f;
  }
  float* pr = rec + kPairFloats * (s >> 1);
  float* base = pr + (s & 1);
#pragma unroll
  for (int c = 0; c < 12; ++c) base[4 * (c >> 1) + 2 * (c & 1)] = v[c];
  if (s & 1) {  // dR = R1 - R0 = X0 - X1 and dtau = tau1 - tau0, the even sample's values in (xo .. tauo)
    pr[24] = (float)(xo - x);
    pr[25] = (float)(yo - y);
    pr[26] = (float)(zo - z);
    pr[27] = (float)(taus - tauo);
  } else {
    double* d = reinterpret_cast<double*>(pr + 28);
    d[0] = x;
    d[1] = y;
    d[2] = z;
    d[3] = taus;
  }
}

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// Per-entry constants: observer in the particle frame, w and w/c (radians) in FP32 (both lanes
// equal), w/2pi and w/(2pi c) (turns) in FP32 and FP64, the FP64 observer.
struct PairObs {
  float2 ox, oy, oz, w, wc;
  float wt, wct;
  double dox, doy, doz, dwt, dwct;
};

__device__ __forceinline__ PairObs make_pair_obs(double fx, double fy, double fz, double om) {
  PairObs o;
  o.ox = f2((float)fx);
  o.oy = f2((float)fy);
  o.oz = f2((float)fz);
  o.w = f2((float)om);
  o.wc = f2((float)(om / kCLight));
  o.dox = fx;
  o.doy = fy;
  o.doz = fz;
  o.dwt = om / kTwoPiD;
  o.dwct = om / (kTwoPiD * kCLight);
  o.wt = (float)o.dwt;
  o.wct = (float)o.dwct;
  return o;
}

// FP32 phase P32 of one sample with the per-lane operations of pair_sample (same value): the
// quantity whose steps the stop rule bounds.
__device__ __forceinline__ float pair_phase(float x, float y, float z, float tau, const PairObs& o) {
  const float rx = fmaf(x, -1.f, o.ox.x), ry = fmaf(y, -1.f, o.oy.x), rz = fmaf(z, -1.f, o.oz.x);
  const float rho2 = fmaf(rx, rx, __fmul_rn(ry, ry));
  const float d2 = fmaf(rz, rz, rho2);
  const float iD = rsqrt_ftz(d2);
  const float ri = __fmul_rn(rho2, iD);
  const float q = __fmul_rn(ri, iD);
  const float corr = __fmul_rn(ri, fmaf(0.125f, q, 0.5f));
  return fmaf(o.wc.x, corr, __fmul_rn(o.w.x, tau));
}

// P32 of sample b (0 or 1) of the pair record at `q` (shared or global memory).
__device__ __forceinline__ float pair_phase_at(const float* q, int b, const PairObs& o) {
  return pair_phase(q[b], q[2 + b], q[4 + b], q[6 + b], o);
}

// Exact float -> double of a non-negative normal float by assembling the bits on the integer pipe
// (the F2F conversion instructions share the slow XU pipe with sin, cos, rsqrt and rcp); +0 and
// denormals come out as ~6e-39 instead of their value, which no caller tells apart from 0.
__device__ __forceinline__ double nonneg_float_to_double(float x) {
  const unsigned u = __float_as_uint(x);
  return __hiloint2double((int)((u >> 3) + 0x38000000u), (int)(u << 29));
}

// FP64 retarded phase of one sample as a fraction of a turn in [-1/2, 1/2) (see the section
// comment), shifted by half a turn: a constant phase shared by every sample, which drops out of
// |E|^2.  corr_f and half_iD = 1 / (2 D) are the sample's FP32 values.  v = 1.5 * 2^22 + turns lies
// in [2^22, 2^23) (|turns| < 2^21), so bits 0..29 of its low word are the fraction of a turn in
// units of 2^-30; bits 7..29, rounded, become the significand of a float in [1, 2).
__device__ __forceinline__ float fp64_turns(double x, double y, double z, double tau, float corr_f, float half_iD,
                                            const PairObs& o) {
  const double Rx = o.dox - x, Ry = o.doy - y, Rz = o.doz - z;
  const double r2 = fma(Rx, Rx, Ry * Ry);
  const double c = nonneg_float_to_double(corr_f);
  const double f = fma(c, fma(2.0, Rz, c), -r2);
  const double c1 = fma(-f, nonneg_float_to_double(half_iD), c);
  const double v = fma(o.dwct, c1, fma(o.dwt, tau, kTurnBase));
  const unsigned lo = (unsigned)__double2loint(v) + 0x40u;  // round to 23 fraction bits (a carry wraps mod 1)
  return __uint_as_float(((lo >> 7) & 0x007FFFFFu) | 0x3F800000u) - 1.5f;
}

// Both samples of one pair record `q` for one entry: adds e (cos P, sin P) per lane to acc (x re,
// x im, y re, y im, z re, z im; the imaginary parts with the sign of +sin P) and returns P32 of both
// samples.  The sum uses exp(-i P): the caller negates the imaginary parts when it folds acc.
__device__ __forceinline__ float2 pair_sample(const float4* __restrict__ q, const PairObs& o, float2* acc) {
  const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
  const double2* dq = reinterpret_cast<const double2*>(q + 7);
  const double2 DXY = dq[0], DZT = dq[1];
  const float2 X = make_float2(q0.x, q0.y), Y = make_float2(q0.z, q0.w);
  const float2 Z = make_float2(q1.x, q1.y), T = make_float2(q1.z, q1.w);
  const float2 NBX = make_float2(q2.x, q2.y), NBY = make_float2(q2.z, q2.w);
  const float2 EB = make_float2(q3.x, q3.y), BZ = make_float2(q3.z, q3.w);
  const float2 G = make_float2(q4.x, q4.y), AZ = make_float2(q4.z, q4.w);
  const float2 AX = make_float2(q5.x, q5.y), AY = make_float2(q5.z, q5.w);
  const float2 M1 = f2(-1.f);
  const float2 rx = fma2(X, M1, o.ox), ry = fma2(Y, M1, o.oy), rz = fma2(Z, M1, o.oz);
  const float2 rho2 = fma2(rx, rx, mul2(ry, ry));
  const float2 d2 = fma2(rz, rz, rho2);
  const float2 iD = make_float2(rsqrt_ftz(d2.x), rsqrt_ftz(d2.y));
  const float2 ri = mul2(rho2, iD);
  const float2 qq = mul2(ri, iD);
  const float2 corr = mul2(ri, fma2(f2(0.125f), qq, f2(0.5f)));
  const float2 P = fma2(o.wc, corr, mul2(o.w, T));
  const float t0 = fp64_turns(DXY.x, DXY.y, DZT.x, DZT.y, corr.x, 0.5f * iD.x, o);
  // second sample: the FP32 step from the first (section comment)
  const float2 DD = mul2(d2, iD);  // D0, D1
  const float inv = rcp_ftz(DD.x + DD.y);
  const float num = fmaf(q6.x, rx.x + rx.y, fmaf(q6.y, ry.x + ry.y, -q6.z * (corr.x + corr.y)));
  const float t1 = t0 + fmaf(o.wct, num * inv, o.wt * q6.w);
  const float2 ph = mul2(make_float2(t0, t1), f2(kTwoPiF));
  float2 sn, cs;
  sincos_ftz(ph.x, &sn.x, &cs.x);
  sincos_ftz(ph.y, &sn.y, &cs.y);
  const float2 nx = mul2(rx, iD), ny = mul2(ry, iD), en = mul2(corr, iD);  // en = 1 - nz
  const float2 ux = add2(nx, NBX), uy = add2(ny, NBY), uz = fma2(en, M1, EB);
  const float2 om = fma2(ny, NBY, fma2(nx, NBX, fma2(en, BZ, EB)));
  // e = k2 (h u - a) with k2 = 1/(D om), h = ((1-b^2)/D + n.a)/om, formed from -1/om:
  // v = a + (-h) u = -(h u - a), e = (-k2) v.
  const float2 nio = make_float2(rcp_ftz(-om.x), rcp_ftz(-om.y));
  const float2 na = fma2(nx, AX, fma2(ny, AY, mul2(fma2(en, M1, f2(1.f)), AZ)));
  const float2 nh = mul2(nio, fma2(G, iD, na));
  const float2 vx = fma2(nh, ux, AX), vy = fma2(nh, uy, AY), vz = fma2(nh, uz, AZ);
  const float2 nk2 = mul2(nio, iD);
  const float2 kc = mul2(nk2, cs), ks = mul2(nk2, sn);
  acc[0] = fma2(vx, kc, acc[0]);
  acc[1] = fma2(vx, ks, acc[1]);
  acc[2] = fma2(vy, kc, acc[2]);
  acc[3] = fma2(vy, ks, acc[3]);
  acc[4] = fma2(vz, kc, acc[4]);
  acc[5] = fma2(vz, ks, acc[5]);
  return P;
}

// Validity of the mixed path for an observer at (fx, fy, fz) in the particle frame: within
// F.theta_max of the frame axis (trajectory extent included), downstream of the trajectory, a
// correction phase (w/c) rho^2 / (2 Rz) of at most 3e4 rad, and a phase w |tau_s| + correction below
// kMaxTurns turns (the range of fp64_turns).  theta_max = min(1e-2, 20 / gamma) (mixed_theta_max):
// beyond ~20 / gamma the flux is a deep cancellation of nearly equal terms (|sum| << sum |terms|)
// that FP32 amplitudes do not resolve to 1e-4.
__device__ __forceinline__ bool mixed_geometry_ok(double fx, double fy, double fz, double om, const MixedFrame& F) {
  const double rho = sqrt(fx * fx + fy * fy) + F.xperp_max;
  const double rz = fz - F.z_max;
  const double corr_phase = (om / kCLight) * rho * rho / (2 * rz);
  return rz > 0 && rho < F.theta_max * rz && corr_phase < 3e4 &&
         (om * F.tau_max + corr_phase) < kMaxTurns * kTwoPiD;
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

// ---------------------------------------------------------------------------------------------
// Finalize of the frequency-domain waves: span reduction, the stop rule of
// src/OSCARSSR.cc:4222-4238, finished entries' outputs (:4246-4267) and the survivor list.
// ---------------------------------------------------------------------------------------------
// Warp-aggregated bookkeeping: one atomic per warp for the survivor list and for each statistics
// counter, instead of one per entry on a single address.
// `level_max` (may be NULL) records the highest level at which an entry finished.
__device__ __forceinline__ void finalize_bookkeeping(bool finished, bool unconverged, bool survive, int64_t item,
                                                     int L, int* act_next, unsigned* n_next,
                                                     unsigned long long* not_converged, unsigned long long* samples,
                                                     unsigned* level_max) {
  const unsigned full = 0xffffffffu;
  const int lane32 = threadIdx.x & 31;
  const unsigned fin = __ballot_sync(full, finished);
  const unsigned unc = __ballot_sync(full, unconverged);
  const unsigned sur = __ballot_sync(full, survive);
  if (lane32 == 0) {
    if (fin) atomicAdd(samples, (unsigned long long)__popc(fin) * (unsigned long long)((2ll << L) - 1));
    if (unc) atomicAdd(not_converged, (unsigned long long)__popc(unc));
    if (fin && level_max) atomicMax(level_max, (unsigned)L);
  }
  unsigned base = 0;
  if (sur && lane32 == __ffs(sur) - 1) base = atomicAdd(n_next, (unsigned)__popc(sur));
  base = __shfl_sync(full, base, sur ? __ffs(sur) - 1 : 0);
  if (survive) act_next[base + __popc(sur & ((1u << lane32) - 1u))] = (int)item;
}

// One power-density entry after its sum up to level L (src/OSCARSSR.cc:2924-2952): finish it
// (converged or last level) or keep its state.
__device__ __forceinline__ void pd_entry_decide(const PdFinalArgs& A, int64_t item, double sum, double last_sum,
                                                bool& finished, bool& unconverged, bool& survive) {
  const int L = A.level;
  const int64_t N = A.n_items;
  const double this_sum = sum * A.dt_level;
  double prec = fabs(this_sum - last_sum) / last_sum;
  const double bd = A.bdmax_levels[L];
  int result_level = -1;
  bool stop = false;
  if ((L > 8 && prec < A.precision && bd < A.two_over_gamma) || (L > 8 && bd < A.two_over_gamma && this_sum == last_sum)) {
    stop = true;
    result_level = L;
  } else if (L > 8 && this_sum == last_sum) {
    stop = true;
    result_level = L;
    prec = 0;
  }
  if (stop || L >= A.max_level) {
    double sv = sum * (A.scale * A.dt_level);
    sv /= 1e6;
    if (!A.directional && sv < 0) sv *= -1;
    double v;
    if (A.quantity == 1) v = prec * A.weight;
    else if (A.quantity == 2) v = (double)result_level * A.weight;
    else v = sv * A.weight;
    A.out[item] = v;
    if (A.level_out) A.level_out[item] = result_level;
    finished = true;
    unconverged = !stop;
  } else {
    A.state[item] = sum;
    A.state[N + item] = this_sum;
    survive = true;
  }
}

// Fused finalize of one tile of the mixed power-density wave by warp 0 (TE entries, 32 at a time):
// each entry's span partials summed in span order from the tile-major layout
// [tile][segment][span][entry in tile], the stop rule of pd_entry_decide, survivors appended.
__device__ __forceinline__ void pd_tile_finalize(const PdFinalArgs& A, const WavePlan& P, int64_t tile, int64_t n_act,
                                                 int TE) {
  if (threadIdx.x >= 32) return;
  const int64_t N = A.n_items;
  for (int q0 = 0; q0 < TE; q0 += 32) {
    const int q = q0 + (int)threadIdx.x;
    const int64_t slot = tile * TE + q;
    const bool live = q < TE && slot < n_act;
    const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
    auto seg_sum = [&](int g) {
      double t = 0;
      for (int sp = 0; sp < P.spans; ++sp) t += __ldcg(A.part + ((tile * P.nseg + g) * P.spans + sp) * TE + q);
      return t;
    };
    bool finished = false, unconverged = false, survive = false;
    if (live) {
      double sum = 0, last_sum = -1;
      if (A.first) {
        if (P.nseg == 2) {
          sum += seg_sum(0);
          last_sum = sum * A.dt_prev;
        }
        sum += seg_sum(P.nseg - 1);
      } else {
        sum = A.state[item];
        last_sum = A.state[N + item];
        sum += seg_sum(0);
      }
      pd_entry_decide(A, item, sum, last_sum, finished, unconverged, survive);
    }
    finalize_bookkeeping(finished, unconverged, survive, item, A.level, A.act_next, A.n_next, A.not_converged,
                         A.samples, A.level_max);
  }
}

// One entry after its sum S up to level L: finish it (converged or last level) or keep its state.
__device__ __forceinline__ void fd_entry_decide(const FdFinalArgs& A, int64_t item, const C3& S, double last_mag,
                                                double dmax, bool& finished, bool& unconverged, bool& survive) {
  C3 t = c3_scale(S, A.dt_level);
  if (A.project) t = c3_project(t, A.pol);
  const double this_mag = c3_mag2(t);
  const double prec = fabs(this_mag - last_mag) / last_mag;
  const int L = A.level;
  const bool stop = (L > 8 && prec < A.precision && dmax < kPiD) || (L > 8 && dmax < kPiD && this_mag == last_mag);
  if (stop || L >= A.max_level) {
    const int result_level = stop ? L : -1;
    C3 E = c3_scale(S, A.c0 * A.dt_level);
    if (A.project) E = c3_project(E, A.pol);
    double v;
    if (A.quantity == 1) v = prec * A.weight;
    else if (A.quantity == 2) v = (double)result_level * A.weight;
    else v = A.c2 * c3_mag2(E) * A.weight;
    A.out[item] = v;
    if (A.level_out) A.level_out[item] = result_level;
    finished = true;
    unconverged = !stop;
  } else {
    const int64_t N = A.n_items;
    A.state[item] = S.xr; A.state[N + item] = S.xi; A.state[2 * N + item] = S.yr;
    A.state[3 * N + item] = S.yi; A.state[4 * N + item] = S.zr; A.state[5 * N + item] = S.zi;
    A.state[6 * N + item] = this_mag;
    survive = true;
  }
}

// Index of partial component k of (tile, segment g, span sp, entry q of the tile) in the fused,
// tile-major layout.
__device__ __forceinline__ int64_t fused_part_index(const WavePlan& P, int64_t tile, int g, int sp, int k, int q,
                                                    int tile_entries) {
  return ((((tile * P.nseg + g) * P.spans + sp) * kFdPartials) + k) * (int64_t)tile_entries + q;
}

// Fused finalize of one tile by all threads of the CTA that finished its last span; entry q of the
// tile is (e * THREADS + threadIdx.x) for q < TE.  Partials are read through L2 (other CTAs wrote
// them).  With A.dmax_spans_joined the stored maxima already include the step into each span.
template <int EPT, int THREADS>
__device__ void fd_tile_finalize(const FdFinalArgs& A, const WavePlan& P, int64_t tile, int64_t n_act, int TE) {
  for (int e = 0; e < EPT; ++e) {
    const int q = e * THREADS + (int)threadIdx.x;
    const int64_t slot = tile * TE + q;
    const bool live = q < TE && slot < n_act;
    const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
    auto seg_sum = [&](int g, C3& s, double& dmax) {
      for (int sp = 0; sp < P.spans; ++sp) {
        const double* p = A.part + fused_part_index(P, tile, g, sp, 0, q, TE);
        s.xr += __ldcg(p); s.xi += __ldcg(p + TE); s.yr += __ldcg(p + 2 * TE);
        s.yi += __ldcg(p + 3 * TE); s.zr += __ldcg(p + 4 * TE); s.zi += __ldcg(p + 5 * TE);
        const double dm = __ldcg(p + 8 * TE);
        if (dm >= 0) {  // non-empty span (empty spans only trail the segment)
          dmax = fmax(dmax, dm);
          if (sp > 0 && !A.dmax_spans_joined) {
            const double* pp = A.part + fused_part_index(P, tile, g, sp - 1, 0, q, TE);
            dmax = fmax(dmax, fabs(__dsub_rn(__ldcg(p + 6 * TE), __ldcg(pp + 7 * TE))));
          }
        }
      }
    };
    bool finished = false, unconverged = false, survive = false;
    if (live) {
      C3 S = {0, 0, 0, 0, 0, 0};
      double last_mag = -1, dmax = 0;
      if (A.first) {
        double unused = 0;
        if (P.nseg == 2) {
          seg_sum(0, S, unused);
          C3 t = c3_scale(S, A.dt_prev);
          if (A.project) t = c3_project(t, A.pol);
          last_mag = c3_mag2(t);
        }
        seg_sum(P.nseg - 1, S, dmax);
      } else {
        const int64_t N = A.n_items;
        S = {A.state[item], A.state[N + item], A.state[2 * N + item], A.state[3 * N + item], A.state[4 * N + item],
             A.state[5 * N + item]};
        last_mag = A.state[6 * N + item];
        seg_sum(0, S, dmax);
      }
      fd_entry_decide(A, item, S, last_mag, dmax, finished, unconverged, survive);
    }
    finalize_bookkeeping(finished, unconverged, survive, item, A.level, A.act_next, A.n_next, A.not_converged,
                         A.samples, A.level_max);
  }
}

// Fused finalize of one tile by all THREADS threads of the CTA, in G = THREADS / TE groups of TE
// threads (entry q = threadIdx.x % TE): group g sums the spans g, g + G, ... of its entry in order, the
// groups' sums are combined in group order through `red` ((G - 1) x 7 x TE doubles) and group 0
// applies the stop rule.  The span maxima include the step into each span (the mixed kernels).
template <int THREADS>
__device__ void fd_tile_finalize_grouped(const FdFinalArgs& A, const WavePlan& P, int64_t tile, int64_t n_act, int TE,
                                         double* red) {
  const int G = THREADS / TE;
  const int grp = (int)threadIdx.x / TE, q = (int)threadIdx.x % TE;
  const int64_t slot = tile * TE + q;
  const bool live = slot < n_act;
  const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
  // sum of segment g over all spans, complete in group 0 (all threads take part: it synchronises)
  auto seg_sum = [&](int g, C3& s, double& dmax) {
    double t[6] = {0, 0, 0, 0, 0, 0};
    double dm = 0;
    if (live) {
      for (int sp = grp; sp < P.spans; sp += G) {
        const double* p = A.part + fused_part_index(P, tile, g, sp, 0, q, TE);
#pragma unroll
        for (int k = 0; k < 6; ++k) t[k] += __ldcg(p + k * TE);
        const double d = __ldcg(p + 8 * TE);
        if (d >= 0) dm = fmax(dm, d);  // -1: an empty span (they only trail the segment)
      }
    }
    if (G > 1) {
      if (grp > 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) red[((grp - 1) * 7 + k) * TE + q] = t[k];
        red[((grp - 1) * 7 + 6) * TE + q] = dm;
      }
      __syncthreads();
      if (grp == 0) {
        for (int o = 0; o < G - 1; ++o) {
#pragma unroll
          for (int k = 0; k < 6; ++k) t[k] += red[(o * 7 + k) * TE + q];
          dm = fmax(dm, red[(o * 7 + 6) * TE + q]);
        }
      }
      __syncthreads();
    }
    s.xr += t[0]; s.xi += t[1]; s.yr += t[2]; s.yi += t[3]; s.zr += t[4]; s.zi += t[5];
    dmax = fmax(dmax, dm);
  };
  C3 S = {0, 0, 0, 0, 0, 0};
  double last_mag = -1, dmax = 0;
  if (A.first) {
    double unused = 0;
    if (P.nseg == 2) {
      seg_sum(0, S, unused);
      C3 t = c3_scale(S, A.dt_prev);
      if (A.project) t = c3_project(t, A.pol);
      last_mag = c3_mag2(t);
    }
    seg_sum(P.nseg - 1, S, dmax);
  } else {
    if (live && grp == 0) {
      const int64_t N = A.n_items;
      S = {A.state[item], A.state[N + item], A.state[2 * N + item], A.state[3 * N + item], A.state[4 * N + item],
           A.state[5 * N + item]};
      last_mag = A.state[6 * N + item];
    }
    seg_sum(0, S, dmax);
  }
  bool finished = false, unconverged = false, survive = false;
  if (live && grp == 0) fd_entry_decide(A, item, S, last_mag, dmax, finished, unconverged, survive);
  finalize_bookkeeping(finished, unconverged, survive, item, A.level, A.act_next, A.n_next, A.not_converged,
                       A.samples, A.level_max);
}

// End of a unit of a fused wave with the grouped finalize (the mixed kernels): as fused_unit_done.
template <int THREADS>
__device__ __forceinline__ void fused_unit_done_grouped(const FdWaveArgs& A, const WavePlan& P, int64_t tile,
                                                        int64_t n_act, int* s_last, int TE, double* red) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned done = atomicAdd(&A.tile_done[tile], 1u);
    *s_last = done == (unsigned)(P.spans - 1);
    if (*s_last) __threadfence();
  }
  __syncthreads();
  if (*s_last) {
    fd_tile_finalize_grouped<THREADS>(A.fin, P, tile, n_act, TE, red);
    if (threadIdx.x == 0) A.tile_done[tile] = 0;
  }
}

// End of a unit in a fused wave: publish this CTA's partials, count the tile's finished spans, and
// let the CTA that finished the last one finalize the tile.
template <int EPT, int THREADS>
__device__ __forceinline__ void fused_unit_done(const FdWaveArgs& A, const WavePlan& P, int64_t tile,
                                                int64_t n_act, int* s_last, int TE = EPT * THREADS) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned done = atomicAdd(&A.tile_done[tile], 1u);
    *s_last = done == (unsigned)(P.spans - 1);
    if (*s_last) __threadfence();
  }
  __syncthreads();
  if (*s_last) {
    fd_tile_finalize<EPT, THREADS>(A.fin, P, tile, n_act, TE);
    if (threadIdx.x == 0) A.tile_done[tile] = 0;
  }
}

}  // namespace dev
}  // namespace osc
