// adjoint.cu -- gradient of a fixed-level flux with respect to the per-half-period amplitude factors
// of an undulator (reverse mode; the radiation part in FP64 or mixed precision, the trajectory part
// in FP64).
//
// Forward (what is differentiated): the RK4 trajectory through the fields (src/OSCARSSR.cc:910-1009),
// its clamped spline (include/TOMATH.h:141-203), the level samples s = 1 .. 2^(L+1)-1 of the fixed
// level L (src/TParticleTrajectoryInterpolated.cc:124-158), and per (observer, energy) entry the
// complex sum S = sum_s A_s exp(-i w (t_s + D_s/c)), F = C2 |C0 dT_L S|^2 (src/OSCARSSR.cc:4179-4268).
// Given dLoss/dF per entry, the reverse sweep is:
//   k_adj_sums          S and F per entry from the forward wave's partials (kept for the next call)
//   k_adj_weights       W = 2 C2 (C0 dT)^2 dLoss/dF conj(S) per entry
//   k_adj_samples       per level sample, sum over entries of d Re(W . A e^{i phi}) / d(X, beta, a/c);
//                       one thread per sample, entries staged through shared memory (FP64)
//   k_adj_samples_mixed the same over the mixed pair records, one thread per pair of samples (FP32
//                       with the FP64 phase of each pair)
//   k_adj_spline_eval   sample -> knot values and second derivatives (transpose of the evaluation)
//   k_adj_spline_solve  second derivatives -> knot values (transpose of the tridiagonal sweeps)
//   k_adj_rk4_recompute trajectory states recomputed from checkpoints every 256 steps
//   k_adj_rk4_segments  knots -> RK4 states -> field amplitudes, parallel in time: every 64-step
//                       segment of both integration chains runs its reverse pass at once (each
//                       step's stages recomputed and differentiated), once with the knot adjoints and
//                       once per unit adjoint entering it;
//   k_adj_rk4_lam       a sequential sweep of the 6 x 6 segment Jacobians joins the segments
//   k_adj_rk4_pgrad     the parameter gradients of the unit-adjoint passes, weighted by it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "batch.h"
#include "device_common.cuh"
#include "engine.h"
#include "fd_common.cuh"
#include "kernels.h"

namespace osc {
namespace dev {

// ---- 1. entry sums and weights ------------------------------------------------------------
// part: partials of a one-span first wave at level L (two segments: levels 0..L-1 and level L),
// entry-major [entry][segment][kFdPartials] (the FP64 wave, unfused) when tile_entries == 0, else
// tile-major [tile][segment][kFdPartials][entry in tile] (the mixed wave).  S: the 6 sums of every
// entry; flux: F = C2 |C0 dT S|^2.
__global__ void k_adj_sums(const double* __restrict__ part, int64_t n, int tile_entries, double c0dt, double c2,
                           double* __restrict__ S, double* __restrict__ flux) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int te = tile_entries;
  const double* p0 = te == 0 ? part + e * 2 * kFdPartials : part + (e / te) * 2 * kFdPartials * te + e % te;
  const int64_t seg = te == 0 ? kFdPartials : (int64_t)kFdPartials * te;  // segment 1 relative to segment 0
  const int64_t cs = te == 0 ? 1 : te;                                    // stride between components
  double m = 0;
  for (int k = 0; k < 6; ++k) {
    const double v = p0[k * cs] + p0[seg + k * cs];
    S[6 * e + k] = v;
    m += (c0dt * v) * (c0dt * v);
  }
  flux[e] = c2 * m;
}

// W = 2 C2 (C0 dT)^2 dLoss/dF conj(S) per entry, and the largest |W| component (bits of a positive
// double, folded with atomicMax) for the mixed samples kernel's scaling.
__global__ void k_adj_weights(const double* __restrict__ S, int64_t n, const double* __restrict__ grad_flux,
                              double c0dt, double c2, double* __restrict__ W,
                              unsigned long long* __restrict__ wmax_bits) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double w = 2.0 * c2 * c0dt * c0dt * grad_flux[e];
  double mx = 0;
  for (int k = 0; k < 3; ++k) {
    const double re = w * S[6 * e + 2 * k], im = -w * S[6 * e + 2 * k + 1];  // conj(S)
    W[6 * e + 2 * k] = re;
    W[6 * e + 2 * k + 1] = im;
    mx = fmax(mx, fmax(fabs(re), fabs(im)));
  }
  if (mx > 0) atomicMax(wmax_bits, (unsigned long long)__double_as_longlong(mx));
}

// ---- 2. per-sample gradients --------------------------------------------------------------
constexpr int kAdjThreads = 128;
constexpr int kAdjStage = 128;

struct AdjEntry {
  double o[3], w, wr[3], wi[3];
};

// Reverse mode of A = u k1 - a k2 (u = n - b, k2 = 1/(D om), k1 = k2 / om (g/D + n.a), om = 1 - n.b,
// g = 1 - b.b, n = R / D, R = O - X) and phi = -w (t + D/c), for J = Re(sum_c W_c A_c e^{i phi}).
__global__ void __launch_bounds__(kAdjThreads) k_adj_samples(const double* __restrict__ lev, int64_t cap,
                                                               int64_t s_end, const double* __restrict__ obs,
                                                               const double* __restrict__ omega, int64_t n_e,
                                                               const double* __restrict__ W, int64_t n_entries,
                                                               int64_t entries_per_cta, double* __restrict__ gs) {
  __shared__ AdjEntry se[kAdjStage];
  const int64_t s = 1 + (int64_t)blockIdx.x * kAdjThreads + threadIdx.x;
  const bool live = s < s_end;
  const int64_t si = live ? s : 1;
  const double T = lev[si];
  const double X = lev[cap + si], Y = lev[2 * cap + si], Z = lev[3 * cap + si];
  const double bx = lev[4 * cap + si], by = lev[5 * cap + si], bz = lev[6 * cap + si];
  const double ax = lev[7 * cap + si], ay = lev[8 * cap + si], az = lev[9 * cap + si];
  const double g = 1.0 - (bx * bx + by * by + bz * bz);
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t e0 = (int64_t)blockIdx.y * entries_per_cta;
  const int64_t e1 = min(n_entries, e0 + entries_per_cta);
  for (int64_t base = e0; base < e1; base += kAdjStage) {
    const int64_t e = base + threadIdx.x;
    if (threadIdx.x < kAdjStage && e < e1) {
      const int64_t io = e / n_e, ie = e % n_e;
      AdjEntry& E = se[threadIdx.x];
      E.o[0] = obs[3 * io]; E.o[1] = obs[3 * io + 1]; E.o[2] = obs[3 * io + 2];
      E.w = omega[ie];
      for (int k = 0; k < 3; ++k) { E.wr[k] = W[6 * e + 2 * k]; E.wi[k] = W[6 * e + 2 * k + 1]; }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kAdjStage, e1 - base);
    if (live) {
      for (int j = 0; j < cnt; ++j) {
        const AdjEntry& E = se[j];
        const double Rx = E.o[0] - X, Ry = E.o[1] - Y, Rz = E.o[2] - Z;
        const double D = sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
        const double iD = 1.0 / D;
        const double nx = Rx * iD, ny = Ry * iD, nz = Rz * iD;
        const double ux = nx - bx, uy = ny - by, uz = nz - bz;
        const double om = 1.0 - (nx * bx + ny * by + nz * bz);
        const double iom = 1.0 / om;
        const double na = nx * ax + ny * ay + nz * az;
        const double k2 = iD * iom;
        const double h = g * iD + na;
        const double k1 = k2 * iom * h;
        const double Ax = ux * k1 - ax * k2, Ay = uy * k1 - ay * k2, Az = uz * k1 - az * k2;
        double sn, cs;
        sincos(reduce_2pi(-E.w * (T + D / kCLight)), &sn, &cs);
        const double Px = E.wr[0] * cs - E.wi[0] * sn, Py = E.wr[1] * cs - E.wi[1] * sn, Pz = E.wr[2] * cs - E.wi[2] * sn;
        const double Qx = E.wr[0] * sn + E.wi[0] * cs, Qy = E.wr[1] * sn + E.wi[1] * cs, Qz = E.wr[2] * sn + E.wi[2] * cs;
        // reverse sweep
        const double phb = -(Qx * Ax + Qy * Ay + Qz * Az);
        double Db = -(E.w / kCLight) * phb;
        const double ubx = Px * k1, uby = Py * k1, ubz = Pz * k1;
        const double k1b = Px * ux + Py * uy + Pz * uz;
        double abx = -Px * k2, aby = -Py * k2, abz = -Pz * k2;
        double k2b = -(Px * ax + Py * ay + Pz * az);
        k2b += k1b * iom * h;
        double iomb = k1b * k2 * h;
        const double hb = k1b * k2 * iom;
        const double gb = hb * iD;
        double iDb = hb * g;
        const double nab = hb;
        iDb += k2b * iom;
        iomb += k2b * iD;
        const double omb = -iomb * iom * iom;
        Db += -iDb * iD * iD;
        double bbx = -2.0 * gb * bx, bby = -2.0 * gb * by, bbz = -2.0 * gb * bz;
        double nbx = nab * ax, nby = nab * ay, nbz = nab * az;
        abx += nab * nx; aby += nab * ny; abz += nab * nz;
        nbx += -omb * bx; nby += -omb * by; nbz += -omb * bz;
        bbx += -omb * nx; bby += -omb * ny; bbz += -omb * nz;
        nbx += ubx; nby += uby; nbz += ubz;
        bbx -= ubx; bby -= uby; bbz -= ubz;
        const double nbn = nbx * nx + nby * ny + nbz * nz;
        Db += -nbn * iD;
        const double Rbx = nbx * iD + Db * nx, Rby = nby * iD + Db * ny, Rbz = nbz * iD + Db * nz;
        acc[0] -= Rbx; acc[1] -= Rby; acc[2] -= Rbz;
        acc[3] += bbx; acc[4] += bby; acc[5] += bbz;
        acc[6] += abx; acc[7] += aby; acc[8] += abz;
      }
    }
    __syncthreads();
  }
  if (live)
    for (int c = 0; c < 9; ++c) atomicAdd(&gs[c * cap + s], acc[c]);
}

// ---- 2b. per-sample gradients, mixed precision -----------------------------------------------
// The same reverse sweep over the mixed pair records of levels 0..L (fd_common.cuh), one thread per
// pair of samples, in the particle frame: the phase of the pair's first sample in FP64 (fp64_turns),
// the second's as the FP32 step from it, amplitudes, sincos and the reverse sweep in FP32, the
// entries' contributions summed in FP32 over a staged chunk and folded into FP64 sums in shared
// memory.  The phase constant the frame drops (w (t_ref + O_z / c) and the half turn of fp64_turns,
// also absent from the mixed wave's sums S) cancels in Re(W A e^{i phi}) with W from conj(S).  W is
// scaled by 1 / max|W| into FP32 range and the sums by max|W| back; the gradients are rotated back
// to the lab frame (g = R^T g').
constexpr int kAdjMxThreads = 128;
constexpr int kAdjMxStage = 64;

struct AdjEntryMx {
  PairObs o;
  float wr[3], wi[3];
};

// Reverse sweep of both samples of a pair record for one entry, each f32x2 lane one sample (the
// operand layout of pair_sample): geometry and phases as the mixed forward kernel forms them (the
// first sample's phase in FP64, the second's as the FP32 step), the amplitude
// A = u k1 - a k2 (u = n - b, k2 = 1/(D om), k1 = k2 (g/D + n.a)/om, om = 1 - n.b, g = 1 - b.b) and
// the reverse sweep of J = Re(sum_c W_c A_c e^{i phi}), phi = -2 pi t.  acc: dJ/dX (3), dJ/dbeta (3),
// dJ/d(a/c) (3) of the two samples.
__device__ __forceinline__ void adj_pair_mx(const float4 q0, const float4 q1, const float4 q2, const float4 q3,
                                            const float4 q4, const float4 q5, const float4 q6, const double2 DXY,
                                            const double2 DZT, const PairObs& o, const float* wr, const float* wi,
                                            float2* acc) {
  const float2 X = make_float2(q0.x, q0.y), Y = make_float2(q0.z, q0.w), Z = make_float2(q1.x, q1.y);
  const float2 MBX = make_float2(q2.x, q2.y), MBY = make_float2(q2.z, q2.w);
  const float2 EB = make_float2(q3.x, q3.y), BZ = make_float2(q3.z, q3.w);
  const float2 G = make_float2(q4.x, q4.y), AZ = make_float2(q4.z, q4.w);
  const float2 AX = make_float2(q5.x, q5.y), AY = make_float2(q5.z, q5.w);
  const float2 M1 = f2(-1.f), ONE = f2(1.f);
  // geometry and phases (pair_sample)
  const float2 rx = fma2(X, M1, o.ox), ry = fma2(Y, M1, o.oy), rz = fma2(Z, M1, o.oz);
  const float2 rho2 = fma2(rx, rx, mul2(ry, ry));
  const float2 d2 = fma2(rz, rz, rho2);
  const float2 iD = make_float2(rsqrt_ftz(d2.x), rsqrt_ftz(d2.y));
  const float2 ri = mul2(rho2, iD);
  const float2 corr = mul2(ri, fma2(f2(0.125f), mul2(ri, iD), f2(0.5f)));
  const float t0 = fp64_turns(DXY.x, DXY.y, DZT.x, DZT.y, corr.x, 0.5f * iD.x, o);
  const float2 DD = mul2(d2, iD);
  const float inv = rcp_ftz(DD.x + DD.y);
  const float num = fmaf(q6.x, rx.x + rx.y, fmaf(q6.y, ry.x + ry.y, -q6.z * (corr.x + corr.y)));
  const float t1 = t0 + fmaf(o.wct, num * inv, o.wt * q6.w);
  const float2 ph = mul2(make_float2(t0, t1), f2(kTwoPiF));
  float2 sn, c;
  sincos_ftz(ph.x, &sn.x, &c.x);
  sincos_ftz(ph.y, &sn.y, &c.y);
  // amplitude
  const float2 nx = mul2(rx, iD), ny = mul2(ry, iD), en = mul2(corr, iD), nz = fma2(en, M1, ONE);
  const float2 ux = add2(nx, MBX), uy = add2(ny, MBY), uz = fma2(en, M1, EB);
  const float2 om = fma2(ny, MBY, fma2(nx, MBX, fma2(en, BZ, EB)));  // 1 - n.b without cancellation
  const float2 iom = make_float2(rcp_ftz(om.x), rcp_ftz(om.y));
  const float2 na = fma2(nx, AX, fma2(ny, AY, mul2(nz, AZ)));
  const float2 k2 = mul2(iD, iom), mk2 = mul2(k2, M1);
  const float2 h = fma2(G, iD, na);
  const float2 k1 = mul2(mul2(k2, iom), h);
  const float2 Ax = fma2(ux, k1, mul2(AX, mk2)), Ay = fma2(uy, k1, mul2(AY, mk2)), Az = fma2(uz, k1, mul2(AZ, mk2));
  // W e^{i phi} = (Wr + i Wi)(c - i sn): P its real part, Q its imaginary part
  const float2 Px = fma2(f2(wr[0]), c, mul2(f2(wi[0]), sn)), Py = fma2(f2(wr[1]), c, mul2(f2(wi[1]), sn)),
               Pz = fma2(f2(wr[2]), c, mul2(f2(wi[2]), sn));
  const float2 Qx = fma2(f2(wi[0]), c, mul2(f2(-wr[0]), sn)), Qy = fma2(f2(wi[1]), c, mul2(f2(-wr[1]), sn)),
               Qz = fma2(f2(wi[2]), c, mul2(f2(-wr[2]), sn));
  // reverse sweep (the FP64 kernel's, in FP32)
  float2 Db = mul2(o.wc, fma2(Qx, Ax, fma2(Qy, Ay, mul2(Qz, Az))));  // -(w/c) phib, phib = -Q.A
  const float2 ubx = mul2(Px, k1), uby = mul2(Py, k1), ubz = mul2(Pz, k1);
  const float2 k1b = fma2(Px, ux, fma2(Py, uy, mul2(Pz, uz)));
  const float2 pa = fma2(Px, AX, fma2(Py, AY, mul2(Pz, AZ)));
  const float2 k2b = fma2(mul2(k1b, iom), h, mul2(pa, M1));
  const float2 hb = mul2(mul2(k1b, k2), iom);
  const float2 gb2 = mul2(mul2(hb, iD), f2(-2.f));  // -2 gb
  const float2 iDb = fma2(hb, G, mul2(k2b, iom));
  const float2 iomb = fma2(mul2(k1b, k2), h, mul2(k2b, iD));
  const float2 momb = mul2(mul2(iomb, iom), iom);  // -omb
  Db = fma2(mul2(mul2(iDb, iD), M1), iD, Db);
  // b = (-MBX, -MBY, BZ): bb = -2 gb b - omb n - ub, nb = hb a - omb b + ub
  const float2 bbx = fma2(momb, nx, fma2(gb2, mul2(MBX, M1), mul2(ubx, M1)));
  const float2 bby = fma2(momb, ny, fma2(gb2, mul2(MBY, M1), mul2(uby, M1)));
  const float2 bbz = fma2(momb, nz, fma2(gb2, BZ, mul2(ubz, M1)));
  const float2 nbx = fma2(hb, AX, fma2(momb, mul2(MBX, M1), ubx));
  const float2 nby = fma2(hb, AY, fma2(momb, mul2(MBY, M1), uby));
  const float2 nbz = fma2(hb, AZ, fma2(momb, BZ, ubz));
  const float2 nbn = fma2(nbx, nx, fma2(nby, ny, mul2(nbz, nz)));
  Db = fma2(mul2(nbn, M1), iD, Db);
  acc[0] = fma2(fma2(nbx, iD, mul2(Db, nx)), M1, acc[0]);
  acc[1] = fma2(fma2(nby, iD, mul2(Db, ny)), M1, acc[1]);
  acc[2] = fma2(fma2(nbz, iD, mul2(Db, nz)), M1, acc[2]);
  acc[3] = add2(acc[3], bbx);
  acc[4] = add2(acc[4], bby);
  acc[5] = add2(acc[5], bbz);
  acc[6] = fma2(hb, nx, add2(acc[6], mul2(Px, mk2)));
  acc[7] = fma2(hb, ny, add2(acc[7], mul2(Py, mk2)));
  acc[8] = fma2(hb, nz, add2(acc[8], mul2(Pz, mk2)));
}

__global__ void __launch_bounds__(kAdjMxThreads, 3)
    k_adj_samples_mixed(const float4* __restrict__ rec, int64_t n_pairs, MixedFrame F, const double* __restrict__ obs,
                        const double* __restrict__ omega, int64_t n_e, const double* __restrict__ W,
                        const unsigned long long* __restrict__ wmax_bits, int64_t n_entries, int64_t entries_per_cta,
                        double* __restrict__ gs, int64_t gcap) {
  __shared__ AdjEntryMx se[kAdjMxStage];
  __shared__ double sacc[18][kAdjMxThreads];
  const int tid = threadIdx.x;
  const int64_t p = (int64_t)blockIdx.x * kAdjMxThreads + tid;
  const bool live = p < n_pairs;
  const float4* q = rec + kPairF4 * (live ? p : 0);
  const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
  const double2* dq = reinterpret_cast<const double2*>(q + 7);
  const double2 DXY = dq[0], DZT = dq[1];
  const double wmax = __longlong_as_double((long long)*wmax_bits);
  const double wscale = wmax > 0 ? 1.0 / wmax : 0.0;
#pragma unroll
  for (int k = 0; k < 18; ++k) sacc[k][tid] = 0.0;
  const int64_t e0 = (int64_t)blockIdx.y * entries_per_cta;
  const int64_t e1 = min(n_entries, e0 + entries_per_cta);
  for (int64_t base = e0; base < e1; base += kAdjMxStage) {
    const int64_t e = base + tid;
    if (tid < kAdjMxStage && e < e1) {
      const int64_t io = e / n_e, ie = e % n_e;
      const double* R = F.rot;
      const double ox = obs[3 * io] - F.x0[0], oy = obs[3 * io + 1] - F.x0[1], oz = obs[3 * io + 2] - F.x0[2];
      AdjEntryMx& E = se[tid];
      E.o = make_pair_obs(R[0] * ox + R[1] * oy + R[2] * oz, R[3] * ox + R[4] * oy + R[5] * oz,
                          R[6] * ox + R[7] * oy + R[8] * oz, omega[ie]);
      for (int k = 0; k < 3; ++k) {
        E.wr[k] = (float)(W[6 * e + 2 * k] * wscale);
        E.wi[k] = (float)(W[6 * e + 2 * k + 1] * wscale);
      }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kAdjMxStage, e1 - base);
    if (live) {
      float2 acc[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) acc[k] = f2(0.f);
      for (int j = 0; j < cnt; ++j)
        adj_pair_mx(q0, q1, q2, q3, q4, q5, q6, DXY, DZT, se[j].o, se[j].wr, se[j].wi, acc);
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        sacc[k][tid] += (double)acc[k].x;
        sacc[9 + k][tid] += (double)acc[k].y;
      }
    }
    __syncthreads();
  }
  if (!live) return;
  const double* R = F.rot;
  for (int b = 0; b < 2; ++b) {
    const int64_t smp = 2 * p + b;
    if (smp == 0) continue;  // the unused slot of the level ladder
    for (int v = 0; v < 3; ++v) {  // X, beta, a/c: g = R^T g'
      const double gx = sacc[9 * b + 3 * v][tid], gy = sacc[9 * b + 3 * v + 1][tid], gz = sacc[9 * b + 3 * v + 2][tid];
      for (int r = 0; r < 3; ++r)
        atomicAdd(&gs[(3 * v + r) * gcap + smp], wmax * (R[r] * gx + R[3 + r] * gy + R[6 + r] * gz));
    }
  }
}

// ---- 3. sample -> knots ---------------------------------------------------------------------
__global__ void k_adj_spline_eval(const double* __restrict__ knots, int64_t n, double tstart, double tstop,
                                  int64_t s_end, const double* __restrict__ gs, int64_t cap,
                                  double* __restrict__ ybar, double* __restrict__ pbar) {
  const int64_t s = 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= s_end) return;
  const double* t = knots;
  const double T = level_time(tstart, tstop, s, kMaxLevelMemory);  // fixed levels, all in memory
  int64_t k = (int64_t)((T - t[0]) / (t[n - 1] - t[0]) * (double)(n - 1));
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  while (k > 0 && t[k] > T) --k;
  while (k < n - 2 && t[k + 1] <= T) ++k;
  const double h = t[k + 1] - t[k];
  const double a = (t[k + 1] - T) / h, b = (T - t[k]) / h;
  const double ca = (a * a * a - a) * (h * h) / 6.0, cb = (b * b * b - b) * (h * h) / 6.0;
  for (int c = 0; c < 9; ++c) {
    const double v = gs[c * cap + s];
    if (v == 0) continue;
    atomicAdd(&ybar[c * n + k], a * v);
    atomicAdd(&ybar[c * n + k + 1], b * v);
    atomicAdd(&pbar[c * n + k], ca * v);
    atomicAdd(&pbar[c * n + k + 1], cb * v);
  }
}

// ---- 4. second derivatives -> knot values --------------------------------------------------
// Forward (linear in y): u_0 = 0, u_i = (6 ud_i / (X_{i+1} - X_{i-1}) - sig_i u_{i-1}) / p_i,
// ypp_{n-1} = -0.5 u_{n-2} / (0.5 diag_{n-2} + 1), ypp_k = diag_k ypp_{k+1} + u_k, with
// sig_i = (X_i - X_{i-1}) / (X_{i+1} - X_{i-1}), p_i = sig_i diag_{i-1} + 2.  Its transpose is two
// first-order linear recurrences, each evaluated as a block-wide scan of affine maps x -> a x + b
// (one block of kScanThreads per component), then a three-point gather.
constexpr int kScanThreads = 1024;

struct Affine { double a, b; };  // x -> a x + b
__device__ __forceinline__ Affine compose(Affine first, Affine then) {  // then(first(x))
  return {then.a * first.a, then.a * first.b + then.b};
}

// x_k = A(k) x_{k-1} + B(k) for k = 0 .. m-1 (x_{-1} = 0), in index order k or (reverse) m-1-k;
// A(k), B(k) are callables of the recurrence index, `out(k, x)` receives every x_k.
template <class FA, class FB, class FO>
__device__ void block_linear_scan(int64_t m, FA A, FB B, FO out) {
  __shared__ double sa[kScanThreads], sb[kScanThreads];
  const int t = threadIdx.x;
  const int64_t chunk = (m + kScanThreads - 1) / kScanThreads;
  const int64_t k0 = t * chunk, k1 = min(m, k0 + chunk);
  Affine f{1.0, 0.0};
  for (int64_t k = k0; k < k1; ++k) f = compose(f, Affine{A(k), B(k)});
  sa[t] = f.a;
  sb[t] = f.b;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {  // inclusive scan of the chunk maps
    Affine prev{1.0, 0.0};
    if (t >= o) prev = Affine{sa[t - o], sb[t - o]};
    __syncthreads();
    if (t >= o) {
      const Affine cur = compose(prev, Affine{sa[t], sb[t]});
      sa[t] = cur.a;
      sb[t] = cur.b;
    }
    __syncthreads();
  }
  double x = t > 0 ? sb[t - 1] : 0.0;  // value entering this chunk (x_{-1} = 0)
  __syncthreads();
  for (int64_t k = k0; k < k1; ++k) {
    x = A(k) * x + B(k);
    out(k, x);
  }
  __syncthreads();
}

// One block per component; pbar (adjoint of ypp) is overwritten, ybar accumulates; work: n doubles
// per component.
__global__ void __launch_bounds__(kScanThreads) k_adj_spline_solve(const double* __restrict__ knots, int64_t n,
                                                                     double* __restrict__ ybar,
                                                                     double* __restrict__ pbar,
                                                                     double* __restrict__ work) {
  const int c = blockIdx.x;
  const double* X = knots;
  const double* diag = knots + 19 * n;
  double* B = pbar + c * n;
  double* U = work + c * n;
  double* Yb = ybar + c * n;
  auto sig = [&](int64_t i) { return (X[i] - X[i - 1]) / (X[i + 1] - X[i - 1]); };
  // (1) B'_0 = B_0, B'_k = B_k + diag_{k-1} B'_{k-1}
  block_linear_scan(n, [&](int64_t k) { return k > 0 ? diag[k - 1] : 0.0; }, [&](int64_t k) { return B[k]; },
                    [&](int64_t k, double x) { U[k] = x; });
  // (2) u_{n-2} also feeds ypp_{n-1}
  if (threadIdx.x == 0) U[n - 2] += -0.5 / (0.5 * diag[n - 2] + 1.) * U[n - 1];
  __syncthreads();
  // (3) V_{n-2} = U_{n-2}, V_{j} = U_j + (-sig_{j+1} / p_{j+1}) V_{j+1}, j = n-3 .. 1 (written into B)
  const int64_t m = n - 2;  // j = n-2 .. 1 -> k = 0 .. m-1
  block_linear_scan(m,
                    [&](int64_t k) {
                      const int64_t j = n - 2 - k;
                      if (j == n - 2) return 0.0;
                      const double sg = sig(j + 1);
                      return -sg / (sg * diag[j] + 2.0);
                    },
                    [&](int64_t k) { return U[n - 2 - k]; }, [&](int64_t k, double x) { B[n - 2 - k] = x; });
  // (4) udb_i = V_i 6 / ((X_{i+1} - X_{i-1}) p_i), i = 1 .. n-2 (into U), then the three-point gather
  for (int64_t i = 1 + threadIdx.x; i <= n - 2; i += blockDim.x) {
    const double sg = sig(i);
    U[i] = B[i] * 6.0 / ((X[i + 1] - X[i - 1]) * (sg * diag[i - 1] + 2.0));
  }
  __syncthreads();
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    double acc = 0;
    if (j - 1 >= 1 && j - 1 <= n - 2) acc += U[j - 1] / (X[j] - X[j - 1]);
    if (j >= 1 && j <= n - 2) acc += -U[j] / (X[j + 1] - X[j]) - U[j] / (X[j] - X[j - 1]);
    if (j + 1 >= 1 && j + 1 <= n - 2) acc += U[j + 1] / (X[j + 1] - X[j]);
    Yb[j] += acc;
  }
}

// ---- 5. RK4 adjoint ---------------------------------------------------------------------------
struct AdjFields {
  const DevField* fs;
  int nf;
  const double* vals;
  int param_field;   // index of the field whose half-period factors are the parameters
  double qomg;
  double* pbar;      // gradient of the parameters (n_half of the parameter field)
};

// Field value at a point, and, when Bb != nullptr, the vector-Jacobian products of B with respect to
// the position (added to posb) and to the parameter field's half-period factors (added to pbar).
__device__ void field_vjp(const AdjFields& F, double x, double y, double z, double t, double* B, const double* Bb,
                          double* posb) {
  B[0] = B[1] = B[2] = 0;
  for (int i = 0; i < F.nf; ++i) {
    const DevField& f = F.fs[i];
    const double d = (x - f.center[0]) * f.period_unit[0] + (y - f.center[1]) * f.period_unit[1] +
                     (z - f.center[2]) * f.period_unit[2];
    const double tc = 1 + d * f.taper;
    const double w = f.frequency == 0 ? 1.0 : cos(2.0 * kPiD * f.frequency * (t + f.time_offset) + f.frequency_phase);
    const int nblk = f.kind == 1 ? 2 : 1;
    for (int blk = 0; blk < nblk; ++blk) {
      const double* amp = blk == 0 ? f.a : f.b;
      const double shift = f.kind == 0 ? f.phase * f.period_mag / (2.0 * kPiD)
                                       : (blk == 0 ? 1.0 : -1.0) * f.phase / 2. * f.period_mag / (2.0 * kPiD);
      const double L = f.length, lam = f.period_length;
      if (d > L / 2. + shift || d < -L / 2. + shift) continue;
      const double th = 2.0 * kPiD * (d - shift) / lam;
      const double s = sin(th), c = cos(th);
      double kf = 1.0;
      int64_t hk = -1;
      if (d < -L / 2. + shift + lam || d > L / 2. + shift - lam) {
        kf = (d < -L / 2. + shift + lam / 2. || d > L / 2. + shift - lam / 2.) ? 0.25 : 0.75;
      } else if (f.n_half > 0) {
        hk = (int64_t)((d - (-L / 2. + shift + lam)) / (lam / 2.));
        hk = hk < 0 ? 0 : (hk >= f.n_half ? f.n_half - 1 : hk);
        kf = F.vals[f.half_off + hk];
      }
      const double phi = kf * s * tc;
      B[0] += amp[0] * phi * w;
      B[1] += amp[1] * phi * w;
      B[2] += amp[2] * phi * w;
      if (Bb) {
        const double gA = (Bb[0] * amp[0] + Bb[1] * amp[1] + Bb[2] * amp[2]) * w;
        const double dphi = kf * (c * (2.0 * kPiD / lam) * tc + s * f.taper);
        posb[0] += gA * dphi * f.period_unit[0];
        posb[1] += gA * dphi * f.period_unit[1];
        posb[2] += gA * dphi * f.period_unit[2];
        if (hk >= 0 && i == F.param_field) atomicAdd(&F.pbar[hk], gA * s * tc);
      }
    }
  }
}

__device__ void f_eval(const AdjFields& F, double t, const double* y, double* dy) {
  double B[3];
  field_vjp(F, y[0], y[2], y[4], t, B, nullptr, nullptr);
  dy[0] = y[1];
  dy[1] = F.qomg * (-y[5] * B[1] + y[3] * B[2]);
  dy[2] = y[3];
  dy[3] = F.qomg * (y[5] * B[0] - y[1] * B[2]);
  dy[4] = y[5];
  dy[5] = F.qomg * (y[1] * B[1] - y[3] * B[0]);
}

// yb += (df/dy)^T fb at (t, y); parameter gradient accumulated by field_vjp.
__device__ void f_vjp(const AdjFields& F, double t, const double* y, const double* fb, double* yb) {
  const double vx = y[1], vy = y[3], vz = y[5];
  double B[3];
  const double Bb[3] = {F.qomg * (fb[3] * vz - fb[5] * vy), F.qomg * (-fb[1] * vz + fb[5] * vx),
                        F.qomg * (fb[1] * vy - fb[3] * vx)};
  double posb[3] = {0, 0, 0};
  field_vjp(F, y[0], y[2], y[4], t, B, Bb, posb);
  yb[0] += posb[0];
  yb[2] += posb[1];
  yb[4] += posb[2];
  yb[1] += fb[0] + F.qomg * (-fb[3] * B[2] + fb[5] * B[1]);
  yb[3] += fb[2] + F.qomg * (fb[1] * B[2] - fb[5] * B[0]);
  yb[5] += fb[4] + F.qomg * (-fb[1] * B[1] + fb[3] * B[0]);
}

__device__ void rk4_step(const AdjFields& F, double* y, double t, double h) {
  double k1[6], k2[6], k3[6], k4[6], yt[6];
  f_eval(F, t, y, k1);
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + h * 0.5 * k1[i];
  f_eval(F, t + h * 0.5, yt, k2);
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + h * 0.5 * k2[i];
  f_eval(F, t + h * 0.5, yt, k3);
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + h * k3[i];
  f_eval(F, t + h, yt, k4);
  for (int i = 0; i < 6; ++i) y[i] = y[i] + h / 6.0 * (k1[i] + k4[i] + 2.0 * (k2[i] + k3[i]));
}

// lam (adjoint of the step's output) -> adjoint of its input y (returned in lam).
__device__ void rk4_vjp(const AdjFields& F, const double* y, double t, double h, double* lam) {
  double k1[6], k2[6], k3[6], y2[6], y3[6], y4[6];
  f_eval(F, t, y, k1);
  for (int i = 0; i < 6; ++i) y2[i] = y[i] + h * 0.5 * k1[i];
  f_eval(F, t + h * 0.5, y2, k2);
  for (int i = 0; i < 6; ++i) y3[i] = y[i] + h * 0.5 * k2[i];
  f_eval(F, t + h * 0.5, y3, k3);
  for (int i = 0; i < 6; ++i) y4[i] = y[i] + h * k3[i];
  double yb[6], k1b[6], k2b[6], k3b[6], k4b[6], tmp[6];
  for (int i = 0; i < 6; ++i) {
    yb[i] = lam[i];
    k1b[i] = h / 6.0 * lam[i];
    k2b[i] = h / 3.0 * lam[i];
    k3b[i] = h / 3.0 * lam[i];
    k4b[i] = h / 6.0 * lam[i];
  }
  for (int i = 0; i < 6; ++i) tmp[i] = 0;
  f_vjp(F, t + h, y4, k4b, tmp);
  for (int i = 0; i < 6; ++i) { yb[i] += tmp[i]; k3b[i] += h * tmp[i]; tmp[i] = 0; }
  f_vjp(F, t + h * 0.5, y3, k3b, tmp);
  for (int i = 0; i < 6; ++i) { yb[i] += tmp[i]; k2b[i] += h * 0.5 * tmp[i]; tmp[i] = 0; }
  f_vjp(F, t + h * 0.5, y2, k2b, tmp);
  for (int i = 0; i < 6; ++i) { yb[i] += tmp[i]; k1b[i] += h * 0.5 * tmp[i]; tmp[i] = 0; }
  f_vjp(F, t, y, k1b, tmp);
  for (int i = 0; i < 6; ++i) lam[i] = yb[i] + tmp[i];
}

// The two integration chains: z_0 = initial state; the forward chain has z_i at t0 + i dt at knot
// nb + i (i = 0 .. nf-1, knot nb + i + 1 holds f(t_i, z_i), knot nb also f(t_0, z_0)); the backward
// chain has z_i at t0 - i dt at knot nb - i (i = 0 .. nb; knot nb - 1 - i holds f(t_i, z_i)).  The
// states are read from the knots only at checkpoints, every kCheckpointSteps-th step of a chain, and
// recomputed between them (k_adj_rk4_recompute).  Each chain's reverse pass is cut into segments
// (s0, s1] of kSegSteps steps.
constexpr int kSegSteps = 64;
constexpr int kCheckpointSteps = 256;

struct AdjSegs {
  double t0, dt;
  int nf, nb;
  const double* knots;  // t | y[9] | ... (n each)
  const double* zs;     // recomputed states: forward chain 0..nf-1, then backward chain 0..nb (6 each)
  const double* kb;     // knot adjoints, 9 x n
  int64_t nseg[2];      // segments of the forward and backward chains
  int64_t base[2];      // index of each chain's first segment
  double* lam_loc;      // per segment: adjoint leaving it with zero adjoint entering (6)
  double* jt;           // per segment: J^T e_r for r = 0..5 (6 x 6)
  double* pseg;         // per segment: parameter gradient of the pass with e_r entering (6 x n_params)
  int n_params;
};

__device__ __forceinline__ void chain_state(const AdjSegs& S, int dir, int64_t i, double* z) {
  const int64_t n = (int64_t)S.nf + S.nb;
  const int64_t j = dir == 0 ? S.nb + i : S.nb - i;
  const double* y = S.knots + n;
  z[0] = y[j];
  z[1] = y[3 * n + j] * kCLight;
  z[2] = y[n + j];
  z[3] = y[4 * n + j] * kCLight;
  z[4] = y[2 * n + j];
  z[5] = y[5 * n + j] * kCLight;
}

// State i of chain dir from the recomputed states.
__device__ __forceinline__ void seg_state(const AdjSegs& S, int dir, int64_t i, double* z) {
  const double* p = S.zs + 6 * ((dir == 0 ? 0 : (int64_t)S.nf) + i);
  for (int k = 0; k < 6; ++k) z[k] = p[k];
}

// Checkpoint interval c of a chain: its first state from the knots (chain_state), the next
// kCheckpointSteps - 1 recomputed by RK4 steps (rk4_step, the stages of src/OSCARSSR.cc:1247-1386)
// into zs.  One thread per interval; nck0 intervals of the forward chain, then those of the backward.
__global__ void k_adj_rk4_recompute(AdjFields F, AdjSegs S, double* __restrict__ zs, int64_t nck0, int64_t nck1) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nck0 + nck1) return;
  const int dir = g < nck0 ? 0 : 1;
  const int64_t c = dir == 0 ? g : g - nck0;
  const int64_t M = dir == 0 ? (int64_t)S.nf - 1 : (int64_t)S.nb;  // last state of the chain
  const int64_t i0 = c * kCheckpointSteps, i1 = min(M, i0 + kCheckpointSteps - 1);
  const double h = dir == 0 ? S.dt : -S.dt;
  double* out = zs + 6 * ((dir == 0 ? 0 : (int64_t)S.nf) + i0);
  double z[6];
  chain_state(S, dir, i0, z);
  for (int k = 0; k < 6; ++k) out[k] = z[k];
  for (int64_t i = i0 + 1; i <= i1; ++i) {
    rk4_step(F, z, S.t0 + h * (double)(i - 1), h);
    for (int k = 0; k < 6; ++k) out[6 * (i - i0) + k] = z[k];
  }
}

// Knot state / acceleration adjoints in the RK4 state layout.
__device__ __forceinline__ void knot_state_adj(const double* kb, int64_t n, int64_t j, double* lam) {
  lam[0] += kb[j]; lam[2] += kb[n + j]; lam[4] += kb[2 * n + j];
  lam[1] += kb[3 * n + j] / kCLight; lam[3] += kb[4 * n + j] / kCLight; lam[5] += kb[5 * n + j] / kCLight;
}
__device__ __forceinline__ void knot_accel_adj(const double* kb, int64_t n, int64_t j, double* fb) {
  fb[0] = 0; fb[2] = 0; fb[4] = 0;
  fb[1] = kb[6 * n + j] / kCLight; fb[3] = kb[7 * n + j] / kCLight; fb[5] = kb[8 * n + j] / kCLight;
}

// One block per segment; thread 0 runs the segment's reverse pass with the knot adjoints and zero
// adjoint entering (its parameter gradient goes straight to the result), threads 1..6 run it with the
// unit adjoint e_{r-1} entering and no knot adjoints (the columns of the segment's transposed
// Jacobian and parameter sensitivities, combined by k_adj_rk4_lam and k_adj_rk4_pgrad).
__global__ void __launch_bounds__(32) k_adj_rk4_segments(AdjFields F, AdjSegs S) {
  const int r = threadIdx.x;
  if (r > 6) return;
  const int64_t g = blockIdx.x;
  const int dir = g < S.base[1] ? 0 : 1;
  const int64_t m = g - S.base[dir];
  const int64_t n = (int64_t)S.nf + S.nb;
  const double h = dir == 0 ? S.dt : -S.dt;
  const int64_t M = dir == 0 ? (int64_t)S.nf - 1 : (int64_t)S.nb;
  const int64_t s0 = m * kSegSteps, s1 = min(M, s0 + kSegSteps);
  const int64_t lo = m == 0 ? 0 : s0 + 1;
  AdjFields Fr = F;
  if (r > 0) Fr.pbar = S.pseg + (g * 6 + (r - 1)) * S.n_params;
  double lam[6] = {0, 0, 0, 0, 0, 0};
  if (r > 0) lam[r - 1] = 1.0;
  double zi[6], zp[6];
  for (int64_t i = s1; i >= lo; --i) {
    seg_state(S, dir, i, zi);
    if (r == 0) {
      const int64_t sk = dir == 0 ? S.nb + i : (i >= 1 ? S.nb - i : -1);
      if (sk >= 0) knot_state_adj(S.kb, n, sk, lam);
      const int64_t ak = dir == 0 ? (i + 1 <= (int64_t)S.nf - 1 ? S.nb + i + 1 : -1)
                                  : (i <= (int64_t)S.nb - 1 ? S.nb - 1 - i : -1);
      double fb[6];
      if (ak >= 0) {
        knot_accel_adj(S.kb, n, ak, fb);
        f_vjp(Fr, S.t0 + h * (double)i, zi, fb, lam);
      }
      if (dir == 0 && i == 0) {  // knot nb also holds f(t_0, z_0)
        knot_accel_adj(S.kb, n, S.nb, fb);
        f_vjp(Fr, S.t0, zi, fb, lam);
      }
    }
    if (i > 0) {
      seg_state(S, dir, i - 1, zp);
      rk4_vjp(Fr, zp, S.t0 + h * (double)(i - 1), h, lam);
    }
  }
  if (r == 0) {
    for (int k = 0; k < 6; ++k) S.lam_loc[g * 6 + k] = lam[k];
  } else {
    for (int k = 0; k < 6; ++k) S.jt[(g * 6 + (r - 1)) * 6 + k] = lam[k];
  }
}

// The adjoint entering every segment: a sequential sweep over the segments of each chain (block 0:
// forward chain, block 1: backward chain), the adjoint entering segment m being the one leaving
// segment m + 1 (lam_loc + J^T lam).  The segments' transposed Jacobians are staged through shared
// memory a chunk at a time; one thread runs the 6 x 6 recurrence.
constexpr int kLamChunk = 128;
__global__ void __launch_bounds__(128) k_adj_rk4_lam(AdjSegs S, double* __restrict__ lam_in) {
  __shared__ double sj[kLamChunk][42];  // per segment: J^T e_r (36), lam_loc (6)
  const int d = blockIdx.x;
  double lam[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t hi = S.nseg[d]; hi > 0; hi -= kLamChunk) {
    const int64_t lo = hi > kLamChunk ? hi - kLamChunk : 0;
    for (int64_t idx = threadIdx.x; idx < (hi - lo) * 42; idx += blockDim.x) {
      const int64_t g = S.base[d] + lo + idx / 42;
      const int k = (int)(idx % 42);
      sj[idx / 42][k] = k < 36 ? S.jt[g * 36 + k] : S.lam_loc[g * 6 + (k - 36)];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int64_t m = hi - 1; m >= lo; --m) {
        const double* J = sj[m - lo];
        double* out = lam_in + 6 * (S.base[d] + m);
        double nl[6];
        for (int jj = 0; jj < 6; ++jj) {
          out[jj] = lam[jj];
          double v = J[36 + jj];
          for (int r = 0; r < 6; ++r) v = fma(J[r * 6 + jj], lam[r], v);
          nl[jj] = v;
        }
        for (int jj = 0; jj < 6; ++jj) lam[jj] = nl[jj];
      }
    }
    __syncthreads();
  }
}

// Parameter gradient of the unit-adjoint passes: pbar[k] += sum over segments g and r of
// lam_in[g][r] * pseg[g][r][k], a block per chunk of 32 segments, a thread per parameter.
__global__ void k_adj_rk4_pgrad(AdjSegs S, const double* __restrict__ lam_in, int64_t nseg, double* __restrict__ pbar) {
  const int64_t g0 = (int64_t)blockIdx.x * 32, g1 = min(nseg, g0 + 32);
  for (int k = threadIdx.x; k < S.n_params; k += blockDim.x) {
    double acc = 0;
    for (int64_t g = g0; g < g1; ++g)
      for (int r = 0; r < 6; ++r) acc = fma(lam_in[6 * g + r], S.pseg[(g * 6 + r) * S.n_params + k], acc);
    if (acc != 0) atomicAdd(&pbar[k], acc);
  }
}

}  // namespace dev

// ---------------------------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------------------------
// Geometry of the two integration chains of the current trajectory and its fields on the device.
struct RkChains {
  std::vector<DevField> df;
  std::vector<double> fvals;
  double dt;
  int64_t nf, nb;
};
static RkChains rk_chains(const Model& model, int64_t n) {
  RkChains c;
  for (const FieldSpec& f : model.fields) c.df.push_back(to_dev_field(f, c.fvals));
  if (c.fvals.empty()) c.fvals.push_back(0.0);
  const Particle& P = model.particle;
  c.dt = ((model.ctstop - model.ctstart) / kC / (model.npoints - 1));
  c.nf = (int64_t)(1 + (model.ctstop - P.t0) / kC / c.dt);
  c.nb = (int64_t)((P.t0 - model.ctstart) / kC / c.dt);
  if (c.nf + c.nb != n) throw Error{OSC_ERR_STATE, "trajectory and its knots disagree"};
  return c;
}

// The RK4 adjoint's trajectory states: read from the knots at checkpoints every kCheckpointSteps
// steps and recomputed between them (k_adj_rk4_recompute), on the side stream -- they depend on the
// trajectory only, so the recomputation overlaps the radiation part of the adjoint -- into adj_z_
// (the fields, their values, then the states), kept until the trajectory changes.
void Engine::prepare_rk4_states(cudaStream_t st) {
  if (zs_version_ == knots_version_) return;
  const int64_t n = nknots_;
  const RkChains c = rk_chains(model, n);
  const size_t field_bytes = (sizeof(DevField) * c.df.size() + 255) & ~(size_t)255;
  if (zs_pending_) check(cudaStreamSynchronize(aux_), "trajectory states");  // the buffer may be in use
  zs_pending_ = false;
  adj_z_.reserve(field_bytes + sizeof(double) * (c.fvals.size() + 6 * (n + 1)));
  char* base = adj_z_.as<char>();
  DevField* d_fields = reinterpret_cast<DevField*>(base);
  double* d_vals = reinterpret_cast<double*>(base + field_bytes);
  double* d_zs = d_vals + c.fvals.size();
  check(cudaMemcpyAsync(d_fields, c.df.data(), sizeof(DevField) * c.df.size(), cudaMemcpyHostToDevice, st), "fields");
  check(cudaMemcpyAsync(d_vals, c.fvals.data(), sizeof(double) * c.fvals.size(), cudaMemcpyHostToDevice, st), "fields");
  dev::AdjFields AF{d_fields, (int)c.df.size(), d_vals, -1, model.particle.qomg, nullptr};
  dev::AdjSegs S{};
  S.t0 = model.particle.t0 / kC;
  S.dt = c.dt;
  S.nf = (int)c.nf;
  S.nb = (int)c.nb;
  S.knots = knots_.as<double>();
  const int64_t nck0 = c.nf > 0 ? (c.nf + dev::kCheckpointSteps - 1) / dev::kCheckpointSteps : 0;
  const int64_t nck1 = (c.nb + 1 + dev::kCheckpointSteps - 1) / dev::kCheckpointSteps;
  check(cudaEventRecord(zs_fork_ev_, st), "event");
  check(cudaStreamWaitEvent(aux_, zs_fork_ev_, 0), "stream wait");
  dev::k_adj_rk4_recompute<<<(unsigned)((nck0 + nck1 + 31) / 32), 32, 0, aux_>>>(AF, S, d_zs, nck0, nck1);
  check(cudaGetLastError(), "trajectory states");
  check(cudaEventRecord(zs_ev_, aux_), "event");
  ++last_launches;
  zs_version_ = knots_version_;
  zs_pending_ = true;
}

// The stream `st` waits for the recomputed states (before their use, or before the knots change).
void Engine::join_rk4_states(cudaStream_t st) {
  if (!zs_pending_) return;
  check(cudaStreamWaitEvent(st, zs_ev_, 0), "stream wait");
  zs_pending_ = false;
}

// Knot adjoints (9 x n on the device, layout of the knot values) -> gradient of the half-period
// factors of field `param_field` (device pointer, n_params values; valid after the stream
// completes).
double* Engine::rk4_adjoint(const double* d_kb, int param_field, int64_t n_params, cudaStream_t st) {
  const Particle& P = model.particle;
  const int64_t n = nknots_;
  prepare_rk4_states(st);
  join_rk4_states(st);
  const RkChains c = rk_chains(model, n);
  const size_t field_bytes = (sizeof(DevField) * c.df.size() + 255) & ~(size_t)255;
  char* zbase = adj_z_.as<char>();
  const DevField* d_fields = reinterpret_cast<const DevField*>(zbase);
  const double* d_vals = reinterpret_cast<const double*>(zbase + field_bytes);
  const double* d_zs = d_vals + c.fvals.size();
  auto segs = [](int64_t M) -> int64_t { return M < 0 ? 0 : (M == 0 ? 1 : (M + dev::kSegSteps - 1) / dev::kSegSteps); };
  const int64_t ns0 = segs(c.nf - 1), ns1 = segs(c.nb), nseg = ns0 + ns1;
  adj_r_.reserve(sizeof(double) * (n_params + nseg * (6 + 36 + 6 * n_params + 6)));
  double* d_pgrad = adj_r_.as<double>();
  double* d_lam = d_pgrad + n_params;
  double* d_jt = d_lam + 6 * nseg;
  double* d_pseg = d_jt + 36 * nseg;
  double* d_lam_in = d_pseg + 6 * n_params * nseg;  // adjoint entering each segment
  check(cudaMemsetAsync(d_pgrad, 0, sizeof(double) * n_params, st), "memset");
  check(cudaMemsetAsync(d_pseg, 0, sizeof(double) * 6 * n_params * nseg, st), "memset");
  dev::AdjFields AF{d_fields, (int)c.df.size(), d_vals, param_field, P.qomg, d_pgrad};
  dev::AdjSegs S{};
  S.t0 = P.t0 / kC;
  S.dt = c.dt;
  S.nf = (int)c.nf;
  S.nb = (int)c.nb;
  S.knots = knots_.as<double>();
  S.zs = d_zs;
  S.kb = d_kb;
  S.nseg[0] = ns0;
  S.nseg[1] = ns1;
  S.base[0] = 0;
  S.base[1] = ns0;
  S.lam_loc = d_lam;
  S.jt = d_jt;
  S.pseg = d_pseg;
  S.n_params = (int)n_params;
  if (nseg > 0) {
    dev::k_adj_rk4_segments<<<(unsigned)nseg, 32, 0, st>>>(AF, S);
    dev::k_adj_rk4_lam<<<2, 128, 0, st>>>(S, d_lam_in);
    dev::k_adj_rk4_pgrad<<<(unsigned)((nseg + 31) / 32), 128, 0, st>>>(S, d_lam_in, nseg, d_pgrad);
  }
  check(cudaGetLastError(), "trajectory adjoint");
  last_launches += 3;
  return d_pgrad;
}

static int param_field_of(const Model& model, int64_t n_params) {
  int param_field = -1;
  for (size_t i = 0; i < model.fields.size(); ++i) {
    const FieldSpec& f = model.fields[i];
    if (f.kind == 2) throw Error{OSC_ERR_INVALID, "the adjoint supports ideal undulator and EPU fields"};
    if (!f.half_scale.empty()) {
      if (param_field >= 0) throw Error{OSC_ERR_INVALID, "more than one field has half-period factors"};
      param_field = (int)i;
    }
  }
  if (param_field < 0) throw Error{OSC_ERR_STATE, "no field has half-period factors to differentiate"};
  if ((int64_t)model.fields[param_field].half_scale.size() != n_params)
    throw Error{OSC_ERR_LENGTH, "gradient length must equal the number of half-period factors"};
  return param_field;
}

void Engine::trajectory_vjp(const double* knot_grad, double* grad_params, int64_t n_params) {
  const int param_field = param_field_of(model, n_params);
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  check(cudaSetDevice(device), "cudaSetDevice");
  use_stream(stream);
  cudaStream_t st = stream;
  model.ensure_trajectory();
  upload_trajectory();
  const int64_t n = nknots_;
  adj_.reserve(sizeof(double) * 9 * n);
  check(cudaMemcpyAsync(adj_.p, knot_grad, sizeof(double) * 9 * n, cudaMemcpyHostToDevice, st), "knot gradient");
  double* d_pgrad = rk4_adjoint(adj_.as<double>(), param_field, n_params, st);
  check(cudaMemcpyAsync(grad_params, d_pgrad, sizeof(double) * n_params, cudaMemcpyDeviceToHost, st), "download");
  check(cudaStreamSynchronize(st), "trajectory adjoint");
}

// FNV-1a over the bytes of an array (the key of the kept forward sums).
static uint64_t bytes_hash(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

void Engine::flux_vjp(const double* obs, int64_t n_obs, const std::vector<double>& omega, int level,
                      const osc_rad_opts& o, bool current_abs, const double* grad_flux, double* flux_out,
                      double* grad_params, int64_t n_params, double* grad_knots) {
  if (level < 1 || level > 20) throw Error{OSC_ERR_RANGE, "adjoint level must be in [1, 20]"};
  const int param_field = grad_flux ? param_field_of(model, n_params) : -1;
  double pol[6];
  bool project = false;
  polarization_vector(o, pol, project);
  if (project) throw Error{OSC_ERR_INVALID, "the adjoint supports polarization 'all'"};
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  check(cudaSetDevice(device), "cudaSetDevice");
  use_stream(stream);
  pending_.clear();
  last_samples = last_launches = last_not_converged = 0;
  cudaStream_t st = stream;
  const bool mixed = o.precision_mode == OSC_MIXED;
  const int64_t n_e = (int64_t)omega.size();
  const int64_t N = n_obs * n_e;
  if (N <= 0) return;

  model.ensure_trajectory();
  upload_trajectory();
  bool tuned_field = false;  // a forward pass of the tuning: the backward pass will need the states
  for (const FieldSpec& f : model.fields) tuned_field = tuned_field || !f.half_scale.empty();
  if (grad_flux || tuned_field) prepare_rk4_states(st);  // overlaps the radiation part
  set_level_grid(kMaxLevelMemory);  // fixed levels on the memory grid
  const Particle& P = model.particle;
  const double dtL = dt_inclusive(tstart_, tstop_, level);
  const double c0 = P.q / (four_pi() * kC * kEps0 * kSqrt2Pi);
  const double cur = current_abs ? std::fabs(P.current) : P.current;
  const double c2 = four_pi() * cur / (kH * std::fabs(P.q) * kMu0 * kC) * 1e-6 * 0.001;
  const int64_t s_end = (int64_t)2 << level;
  unsigned* cnt = cnt_.as<unsigned>();

  // ---- forward sums S of every entry at level L, kept for a following call on the same inputs
  // (same trajectory, observers, energies, level, arithmetic and normalisation)
  uint64_t key = bytes_hash(obs, sizeof(double) * 3 * n_obs);
  key = bytes_hash(omega.data(), sizeof(double) * n_e, key);
  const int64_t kv[6] = {(int64_t)knots_version_, n_obs, n_e, level, mixed ? 1 : 0, current_abs ? 1 : 0};
  key = bytes_hash(kv, sizeof kv, key);
  adj_sums_.reserve(sizeof(double) * 7 * N);
  double* d_S = adj_sums_.as<double>();
  double* d_flux = d_S + 6 * N;
  // inputs and level samples (shared with other requests, so always refreshed; cheap when resident)
  obs_.reserve(sizeof(double) * 3 * n_obs);
  omega_.reserve(sizeof(double) * n_e);
  check(cudaMemcpyAsync(obs_.p, obs, sizeof(double) * 3 * n_obs, cudaMemcpyHostToDevice, st), "obs");
  check(cudaMemcpyAsync(omega_.p, omega.data(), sizeof(double) * n_e, cudaMemcpyHostToDevice, st), "omega");
  if (mixed) ensure_mixed(level);
  else ensure_levels(level);
  if (!(adj_key_valid_ && adj_key_ == key)) {
    adj_key_valid_ = false;
    // the first-wave kernel at level L with one span per segment (levels 0..L-1, level L)
    unsigned long long* work = reinterpret_cast<unsigned long long*>(cnt + 4) + 2;
    check(cudaMemsetAsync(work, 0, sizeof(unsigned long long), st), "memset");
    FdWaveArgs w{};
    w.obs = obs_.as<double>(); w.omega = omega_.as<double>();
    w.n_e = n_e; w.n_items = N; w.act = nullptr; w.n_act = nullptr; w.first = 1; w.level = level;
    w.min_span = 32; w.target_units = 1; w.err = cnt + kCntErr; w.work = work; w.fused = 0;
    int te = 0;
    if (mixed) {
      const int v = variant_in_use(2);
      te = mixed_entries_per_cta(v);
      part_.reserve(sizeof(double) * 2 * kFdPartials * te * ((N + te - 1) / te));
      w.lev = reinterpret_cast<const double*>(mrec_.p); w.tile_entries = te; w.part = part_.as<double>();
      check(launch_fd_wave_mixed(w, frame_, (int)std::min<int64_t>((N + te - 1) / te, wave_grid(2, v)), v, st),
            "adjoint forward (mixed)");
    } else {
      const int v = variant_in_use(0);
      const int tev = fp64_entries_per_cta(v);  // entries per CTA of that variant
      part_.reserve(sizeof(double) * 2 * kFdPartials * N);
      w.lev = lev_.as<double>(); w.cap = lev_cap_; w.tile_entries = tev; w.part = part_.as<double>();
      check(launch_fd_wave_fp64(w, (int)std::min<int64_t>((N + tev - 1) / tev, wave_grid(0, v)), v, st),
            "adjoint forward");
    }
    check(cudaMemsetAsync(work, 0, sizeof(unsigned long long), st), "memset");  // counters start at zero
    dev::k_adj_sums<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(part_.as<double>(), N, te, c0 * dtL, c2, d_S, d_flux);
    check(cudaGetLastError(), "adjoint sums");
    last_launches += 2;
    adj_key_ = key;
    adj_key_valid_ = true;
  }
  auto finish = [&]() {  // wait, then report the forward's device errors
    unsigned err = 0;
    check(cudaMemcpyAsync(&err, cnt + kCntErr, sizeof err, cudaMemcpyDeviceToHost, st), "error word");
    check(cudaStreamSynchronize(st), "adjoint");
    if (err) {
      adj_key_valid_ = false;
      check(cudaMemset(cnt + kCntErr, 0, sizeof(unsigned)), "error word");
      if (err & dev::kErrTmaTimeout)
        throw Error{OSC_ERR_TIMEOUT, "a staged trajectory copy did not complete (device wait limit reached)"};
      if (err & dev::kErrPlan) throw Error{OSC_ERR_STATE, "a sample-sum kernel variant was planned with another tile size"};
      throw Error{OSC_ERR_INVALID, kMixedGeometryMessage};
    }
  };
  if (flux_out) check(cudaMemcpyAsync(flux_out, d_flux, sizeof(double) * N, cudaMemcpyDeviceToHost, st), "download");
  if (!grad_flux) {  // forward only
    finish();
    return;
  }

  // ---- weights and per-sample gradients
  adj_.reserve(sizeof(double) * (N /*grad*/ + 6 * N /*W*/ + 1 /*max |W|*/));
  double* d_grad = adj_.as<double>();
  double* d_W = d_grad + N;
  unsigned long long* d_wmax = reinterpret_cast<unsigned long long*>(d_W + 6 * N);
  check(cudaMemcpyAsync(d_grad, grad_flux, sizeof(double) * N, cudaMemcpyHostToDevice, st), "grad");
  check(cudaMemsetAsync(d_wmax, 0, sizeof(unsigned long long), st), "memset");
  dev::k_adj_weights<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(d_S, N, d_grad, c0 * dtL, c2, d_W, d_wmax);
  const int64_t n = nknots_;
  const int64_t gcap = mixed ? s_end : lev_cap_;  // stride of the 9 per-sample gradient arrays
  adj_s_.reserve(sizeof(double) * (9 * gcap + 2 * 9 * n + 9 * n));
  double* d_gs = adj_s_.as<double>();
  double* d_yb = d_gs + 9 * gcap;
  double* d_pb = d_yb + 9 * n;
  double* d_diag = d_pb + 9 * n;
  check(cudaMemsetAsync(d_gs, 0, sizeof(double) * (9 * gcap + 2 * 9 * n), st), "memset");
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attr");
  if (mixed) {
    const int64_t n_pairs = s_end / 2;
    const int64_t gx = (n_pairs + dev::kAdjMxThreads - 1) / dev::kAdjMxThreads;
    const int64_t want = 12 * (int64_t)sms;  // CTAs in flight
    int64_t gy = std::max<int64_t>(1, std::min<int64_t>((want + gx - 1) / gx, (N + dev::kAdjMxStage - 1) / dev::kAdjMxStage));
    const int64_t per = ((N + gy - 1) / gy + dev::kAdjMxStage - 1) / dev::kAdjMxStage * dev::kAdjMxStage;
    gy = (N + per - 1) / per;
    dev::k_adj_samples_mixed<<<dim3((unsigned)gx, (unsigned)gy), dev::kAdjMxThreads, 0, st>>>(
        reinterpret_cast<const float4*>(mrec_.p), n_pairs, frame_, obs_.as<double>(), omega_.as<double>(), n_e, d_W,
        d_wmax, N, per, d_gs, gcap);
  } else {
    const int64_t gx = (s_end - 1 + dev::kAdjThreads - 1) / dev::kAdjThreads;
    const int64_t want = 16 * (int64_t)sms;  // CTAs in flight
    int64_t gy = std::max<int64_t>(1, std::min<int64_t>((want + gx - 1) / gx, (N + dev::kAdjStage - 1) / dev::kAdjStage));
    const int64_t per = ((N + gy - 1) / gy + dev::kAdjStage - 1) / dev::kAdjStage * dev::kAdjStage;
    gy = (N + per - 1) / per;
    dev::k_adj_samples<<<dim3((unsigned)gx, (unsigned)gy), dev::kAdjThreads, 0, st>>>(
        lev_.as<double>(), lev_cap_, s_end, obs_.as<double>(), omega_.as<double>(), n_e, d_W, N, per, d_gs);
  }
  dev::k_adj_spline_eval<<<(unsigned)((s_end - 1 + 255) / 256), 256, 0, st>>>(knots_.as<double>(), n, tstart_, tstop_,
                                                                             s_end, d_gs, gcap, d_yb, d_pb);
  dev::k_adj_spline_solve<<<9, dev::kScanThreads, 0, st>>>(knots_.as<double>(), n, d_yb, d_pb, d_diag);
  check(cudaGetLastError(), "adjoint");
  last_launches += 4;
  // RK4 adjoint
  double* d_pgrad = rk4_adjoint(d_yb, param_field, n_params, st);
  if (grad_knots) check(cudaMemcpyAsync(grad_knots, d_yb, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, st), "download");
  check(cudaMemcpyAsync(grad_params, d_pgrad, sizeof(double) * n_params, cudaMemcpyDeviceToHost, st), "download");
  finish();
  last_samples = N * (s_end - 1);
}

}  // namespace osc
