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
// Hardware approximations (MUFU) with denormals flushed: the mixed-precision terms never see
// denormal operands (distances ~1..100 m, 1 - n.b ~ 1e-9..1e-6, reduced phases in [-pi, pi]), so
// the flush-to-zero forms give the same values as rsqrtf / __fdividef(1, x) / __sincosf on every
// input they receive, without the extra instructions that handle denormal inputs.
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

constexpr float kTwoPiHiF = 6.28318548202514648f;     // RN_f(2 pi)
constexpr float kTwoPiLoF = -1.7484556e-07f;         // RN_f(2 pi - kTwoPiHiF)
constexpr float kInvTwoPiF = 0.159154943f;

__device__ __forceinline__ float mixed_sample(const float4 r0, const float4 r1, const float4 r2, float Ox, float Oy,
                                              float Oz, float w, float wc, float* s) {
  const float rx = Ox - r0.x, ry = Oy - r0.y, rz = Oz - r0.z;
  const float rho2 = fmaf(rx, rx, ry * ry);
  const float d2 = fmaf(rz, rz, rho2);
  const float iD = rsqrt_ftz(d2);
  const float q = rho2 * iD * iD;                                  // (rho/D)^2
  const float corr = rho2 * iD * fmaf(0.125f, q, 0.5f);           // rho^2/(Rz+D), |rho/D| < 1e-2
  const float ph = -fmaf(wc, corr, w * r0.w);                      // exp(-i w (t + D/c))
  const float k = rintf(ph * kInvTwoPiF);
  const float rr = fmaf(-k, kTwoPiLoF, fmaf(-k, kTwoPiHiF, ph));  // Cody-Waite reduction to [-pi, pi]
  float sn, cs;
  sincos_ftz(rr, &sn, &cs);
  const float nx = rx * iD, ny = ry * iD;
  const float en = corr * iD;                                      // 1 - n_z
  const float ux = nx - r1.x, uy = ny - r1.y, uz = r1.z - en;
  const float om = fmaf(-nx, r1.x, fmaf(-ny, r1.y, fmaf(-en, r1.z, en + r1.z)));
  const float io = rcp_ftz(om);
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

// The phase alone, with the operations of mixed_sample (same value).
__device__ __forceinline__ float mixed_phase(const float4 r0, float Ox, float Oy, float Oz, float w, float wc) {
  const float rx = Ox - r0.x, ry = Oy - r0.y, rz = Oz - r0.z;
  const float rho2 = fmaf(rx, rx, ry * ry);
  const float d2 = fmaf(rz, rz, rho2);
  const float iD = rsqrt_ftz(d2);
  const float q = rho2 * iD * iD;
  const float corr = rho2 * iD * fmaf(0.125f, q, 0.5f);
  return -fmaf(wc, corr, w * r0.w);
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

// ---------------------------------------------------------------------------------------------
// Finalize of the frequency-domain waves: span reduction, the stop rule of
// src/OSCARSSR.cc:4222-4238, finished entries' outputs (:4246-4267) and the survivor list.
// ---------------------------------------------------------------------------------------------
// Warp-aggregated bookkeeping: one atomic per warp for the survivor list and for each statistics
// counter, instead of one per entry on a single address.
__device__ __forceinline__ void finalize_bookkeeping(bool finished, bool unconverged, bool survive, int64_t item,
                                                     int L, int* act_next, unsigned* n_next,
                                                     unsigned long long* not_converged, unsigned long long* samples) {
  const unsigned full = 0xffffffffu;
  const int lane32 = threadIdx.x & 31;
  const unsigned fin = __ballot_sync(full, finished);
  const unsigned unc = __ballot_sync(full, unconverged);
  const unsigned sur = __ballot_sync(full, survive);
  if (lane32 == 0) {
    if (fin) atomicAdd(samples, (unsigned long long)__popc(fin) * (unsigned long long)((2ll << L) - 1));
    if (unc) atomicAdd(not_converged, (unsigned long long)__popc(unc));
  }
  unsigned base = 0;
  if (sur && lane32 == __ffs(sur) - 1) base = atomicAdd(n_next, (unsigned)__popc(sur));
  base = __shfl_sync(full, base, sur ? __ffs(sur) - 1 : 0);
  if (survive) act_next[base + __popc(sur & ((1u << lane32) - 1u))] = (int)item;
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
                         A.samples);
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
