// kernels_mixed.cu -- mixed-precision frequency-domain sum (FP64 trajectory and retarded-time
// offsets, FP32 amplitudes, sincos and per-chunk sums folded into FP64).
//
// Frame: every trajectory is expressed in a frame whose origin is the particle's initial position
// X0 and whose third axis e3 is its initial direction, so observers downstream sit near the axis.
// With R = O - X = (Rx, Ry, Rz) in that frame and rho^2 = Rx^2 + Ry^2,
//     D = |R| = Rz + corr,   corr = rho^2 / (Rz + D)                       (no cancellation)
//     w (t + D/c) = w (t - z/c) + w Oz/c + (w/c) corr      (the sum uses exp(-i w (t + D/c)))
// The middle term is a constant phase per (observer, energy) entry; it multiplies the whole sum by a
// unit complex number and drops out of |E|^2, of the polarization projection and of the phase
// differences of the stop rule, so it is not computed.  tau_s = t - z/c (a few 1e-16 s) is formed in
// FP64 per sample and stored as float; (w/c) corr is a few 1e3 rad, so the phase carries
// ~1e-4..1e-3 rad of rounding per sample, which averages down as 1/sqrt(samples) in the sum.
//
// Amplitude (src/OSCARSSR.cc:4219), with u = n - b, om = 1 - n.b and |n| = 1:
//     (1-b^2) u / (D^2 om^2) + n x (u x a) / (D om^2)
//   = u (1/(D om^2)) ((1-b^2)/D + n.a) - a / (D om)        [n x (u x a) = u (n.a) - a (n.u), n.u = om]
// with the small differences formed without cancellation from per-sample FP64-exact inputs:
//     1 - n_z = corr / D,  u_z = (1 - b_z) - (1 - n_z),
//     om = (1-n_z) + (1-b_z) - (1-n_z)(1-b_z) - n_x b_x - n_y b_y.
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "fd_common.cuh"
#include "kernels.h"

namespace osc {
namespace dev {

constexpr double kCl = 2.99792458e8;

// Per-sample record, 3 x float4 = 48 bytes: (x, y, z, tau_s) (bx, by, 1-bz, 1-b^2) (ax, ay, az, 0)
__global__ void k_mixed_records(const double* __restrict__ lev, int64_t cap, int64_t s_begin, int64_t s_end,
                                MixedFrame F, float4* __restrict__ rec) {
  const int64_t s = s_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= s_end) return;
  const double t = lev[s];
  const double dx = lev[cap + s] - F.x0[0], dy = lev[2 * cap + s] - F.x0[1], dz = lev[3 * cap + s] - F.x0[2];
  const double bx = lev[4 * cap + s], by = lev[5 * cap + s], bz = lev[6 * cap + s];
  const double ax = lev[7 * cap + s], ay = lev[8 * cap + s], az = lev[9 * cap + s];
  const double* R = F.rot;  // rows: e1, e2, e3
  const double x = R[0] * dx + R[1] * dy + R[2] * dz;
  const double y = R[3] * dx + R[4] * dy + R[5] * dz;
  const double z = R[6] * dx + R[7] * dy + R[8] * dz;
  const double px = R[0] * bx + R[1] * by + R[2] * bz;
  const double py = R[3] * bx + R[4] * by + R[5] * bz;
  const double pz = R[6] * bx + R[7] * by + R[8] * bz;
  const double qx = R[0] * ax + R[1] * ay + R[2] * az;
  const double qy = R[3] * ax + R[4] * ay + R[5] * az;
  const double qz = R[6] * ax + R[7] * ay + R[8] * az;
  const double g2 = 1.0 - (px * px + py * py + pz * pz);       // 1 - b^2, ~1/gamma^2
  const double ebz = (g2 + px * px + py * py) / (1.0 + pz);     // 1 - b_z without cancellation
  const double taus = (t - F.t_ref) - z / kCl;
  rec[3 * s] = make_float4((float)x, (float)y, (float)z, (float)taus);
  rec[3 * s + 1] = make_float4((float)px, (float)py, (float)ebz, (float)g2);
  rec[3 * s + 2] = make_float4((float)qx, (float)qy, (float)qz, 0.f);
}

constexpr int kMxThreads = 128;
constexpr int kMxChunk = 256;
constexpr int kMxFold = 32;  // FP32 partial sums are folded into FP64 every kMxFold samples

struct MixedStage {
  float4 v[2][kMxChunk * 3];
  uint64_t bar[2];
};

template <int EPT, int MINB>
__global__ void __launch_bounds__(kMxThreads, MINB) k_fd_wave_mixed(FdWaveArgs A, MixedFrame F) {
  if (A.tile_entries != kMxThreads * EPT) {  // the host sized the partials for another tile
    if (threadIdx.x == 0) atomicOr(A.err, kErrPlan);
    return;
  }
  __shared__ __align__(16) MixedStage st;
  __shared__ int s_last;
  const int tid = threadIdx.x;
  if (A.fused && blockIdx.x == 0 && tid == 0) {  // counters of the following wave
    if (A.zero_u32) *A.zero_u32 = 0;
    if (A.zero_u64) *A.zero_u64 = 0;
  }
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  // the plan is uniform over the CTA; keeping it in shared memory frees the registers its
  // fields would otherwise hold across the sample loop
  __shared__ WavePlan P;
  if (threadIdx.x == 0) P = wave_plan(A.first, A.level, n_act, kMxThreads * EPT, A.target_units, A.min_span);
  __syncthreads();
  const int64_t units = P.tiles * P.spans;
  const float4* rec = reinterpret_cast<const float4*>(A.lev);
  if (tid == 0) {
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  uint32_t phase_bits = 0;
  __shared__ int64_t next_unit;
  for (;;) {  // CTAs take (tile, span) units from a shared counter until the wave's units run out
    if (tid == 0) next_unit = (int64_t)atomicAdd(A.work, 1ull);
    __syncthreads();
    const int64_t u = next_unit;
    __syncthreads();
    if (u >= units) break;
    const int64_t tile = u / P.spans;
    const int span = (int)(u % P.spans);
    // entry constants
    float Ox[EPT], Oy[EPT], Oz[EPT], w[EPT], wc[EPT];
    bool live[EPT];
    int64_t slot[EPT];
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      slot[e] = tile * kMxThreads * EPT + (int64_t)e * kMxThreads + tid;
      live[e] = slot[e] < n_act;
      const int64_t item = live[e] ? (A.act ? (int64_t)A.act[slot[e]] : slot[e]) : 0;
      const int64_t io = item / A.n_e, ie = item % A.n_e;
      const double* R = F.rot;
      const double ox = A.obs[3 * io] - F.x0[0], oy = A.obs[3 * io + 1] - F.x0[1], oz = A.obs[3 * io + 2] - F.x0[2];
      const double fx = R[0] * ox + R[1] * oy + R[2] * oz;
      const double fy = R[3] * ox + R[4] * oy + R[5] * oz;
      const double fz = R[6] * ox + R[7] * oy + R[8] * oz;
      Ox[e] = (float)fx; Oy[e] = (float)fy; Oz[e] = (float)fz;
      const double om = A.omega[ie];
      w[e] = (float)om;
      wc[e] = (float)(om / kCl);
      // validity of the near-axis phase form: small angle from the frame axis and a bounded
      // correction phase (see the file comment); otherwise the caller must use the FP64 path
      if (live[e] && span == 0 && !mixed_geometry_ok(fx, fy, fz, om, F.xperp_max, F.z_max)) atomicOr(A.err, kErrBadArgs);
    }
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      double S[EPT][6];
      float first[EPT], last[EPT], dmax[EPT];
      bool have[EPT];
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
#pragma unroll
        for (int k = 0; k < 6; ++k) S[e][k] = 0.0;
        first[e] = last[e] = 0.f;
        dmax[e] = 0.f;
        have[e] = false;
      }
      const int64_t nchunks = b1 > b0 ? (b1 - b0 + kMxChunk - 1) / kMxChunk : 0;
      if (tid == 0 && nchunks > 0) {
        const int64_t hi = min(b1, b0 + kMxChunk);
        mbar_arrive_expect_tx(&st.bar[0], (uint32_t)((hi - b0) * 48));
        tma_load_1d(&st.v[0][0], rec + 3 * b0, (uint32_t)((hi - b0) * 48), &st.bar[0]);
      }
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = b0 + c * kMxChunk, hi = min(b1, lo + kMxChunk);
        if (tid == 0 && c + 1 < nchunks) {
          const int64_t lo2 = lo + kMxChunk, hi2 = min(b1, lo2 + kMxChunk);
          mbar_arrive_expect_tx(&st.bar[buf ^ 1], (uint32_t)((hi2 - lo2) * 48));
          tma_load_1d(&st.v[buf ^ 1][0], rec + 3 * lo2, (uint32_t)((hi2 - lo2) * 48), &st.bar[buf ^ 1]);
        }
        if (!mbar_wait(&st.bar[buf], (phase_bits >> buf) & 1u)) {
          if (tid == 0) atomicOr(A.err, kErrTmaTimeout);
          return;
        }
        phase_bits ^= 1u << buf;
        const float4* sv = st.v[buf];
        const int j0 = lo == 0 ? 1 : 0;  // sample 0 is the unused slot
        const int n = (int)(hi - lo);
        for (int jb = j0; jb < n; jb += kMxFold) {
          const int je = min(n, jb + kMxFold);
          float s32[EPT][6];
#pragma unroll
          for (int e = 0; e < EPT; ++e)
#pragma unroll
            for (int k = 0; k < 6; ++k) s32[e][k] = 0.f;
          for (int j = jb; j < je; ++j) {
            const float4 r0 = sv[3 * j], r1 = sv[3 * j + 1], r2 = sv[3 * j + 2];
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
              const float ph = mixed_sample(r0, r1, r2, Ox[e], Oy[e], Oz[e], w[e], wc[e], s32[e]);
              if (have[e]) {
                const float dp = fabsf(ph - last[e]);
                dmax[e] = fmaxf(dmax[e], dp);
              } else {
                first[e] = ph;
                have[e] = true;
              }
              last[e] = ph;
            }
          }
#pragma unroll
          for (int e = 0; e < EPT; ++e)
#pragma unroll
            for (int k = 0; k < 6; ++k) S[e][k] += (double)s32[e][k];
        }
        __syncthreads();
      }
#pragma unroll
      for (int e = 0; e < EPT; ++e) {
        if (!live[e]) continue;
        // entry-major for the finalize kernel; tile-major when fused
        double* p = A.fused ? A.part + fused_part_index(P, tile, g, span, 0, e * kMxThreads + tid, kMxThreads * EPT)
                            : A.part + (slot[e] * P.nseg * P.spans + g * P.spans + span) * kFdPartials;
        const int64_t cs = A.fused ? kMxThreads * EPT : 1;  // stride between components
#pragma unroll
        for (int k = 0; k < 6; ++k) p[k * cs] = S[e][k];
        p[6 * cs] = have[e] ? (double)first[e] : 0.0;
        p[7 * cs] = have[e] ? (double)last[e] : 0.0;
        p[8 * cs] = have[e] ? (double)dmax[e] : -1.0;
      }
    }
    if (A.fused) fused_unit_done<EPT, kMxThreads>(A, P, tile, n_act, &s_last);
  }
}

// Sample-split variant: the CTA's 128 threads form SUB groups of TE = 128 / SUB threads; group s
// handles, for the same TE entries, the s-th of SUB equal parts of every staged chunk.  Each part
// starts from the phase of the sample before it, so the largest phase step needs no exchange
// between groups or spans (dmax_spans_joined); the groups' sums are reduced in shared memory and
// one partial per entry and span is stored.  Smaller tiles mean fewer spans per entry.
template <int SUB, int MINB>
__global__ void __launch_bounds__(kMxThreads, MINB) k_fd_wave_mixed_split(FdWaveArgs A, MixedFrame F) {
  constexpr int TE = kMxThreads / SUB;
  if (A.tile_entries != TE) {  // the host sized the partials for another tile
    if (threadIdx.x == 0) atomicOr(A.err, kErrPlan);
    return;
  }
  constexpr int PART = kMxChunk / SUB;
  __shared__ __align__(16) MixedStage st;
  __shared__ __align__(16) float4 prev_rec[3];
  __shared__ int prev_valid;
  __shared__ double red[SUB > 1 ? SUB - 1 : 1][7][TE];
  __shared__ int s_last;
  __shared__ WavePlan P;
  __shared__ int64_t next_unit;
  const int tid = threadIdx.x;
  const int grp = tid / TE, q = tid % TE;
  if (A.fused && blockIdx.x == 0 && tid == 0) {  // counters of the following wave
    if (A.zero_u32) *A.zero_u32 = 0;
    if (A.zero_u64) *A.zero_u64 = 0;
  }
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  if (tid == 0) {
    P = wave_plan(A.first, A.level, n_act, TE, A.target_units, A.min_span);
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t units = P.tiles * P.spans;
  const float4* rec = reinterpret_cast<const float4*>(A.lev);
  uint32_t phase_bits = 0;
  for (;;) {
    if (tid == 0) next_unit = (int64_t)atomicAdd(A.work, 1ull);
    __syncthreads();
    const int64_t u = next_unit;
    __syncthreads();
    if (u >= units) break;
    const int64_t tile = u / P.spans;
    const int span = (int)(u % P.spans);
    const int64_t slot = tile * TE + q;
    const bool live = slot < n_act;
    const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
    const int64_t io = item / A.n_e, ie = item % A.n_e;
    float Ox, Oy, Oz, w, wc;
    {
      const double* R = F.rot;
      const double ox = A.obs[3 * io] - F.x0[0], oy = A.obs[3 * io + 1] - F.x0[1], oz = A.obs[3 * io + 2] - F.x0[2];
      const double fx = R[0] * ox + R[1] * oy + R[2] * oz;
      const double fy = R[3] * ox + R[4] * oy + R[5] * oz;
      const double fz = R[6] * ox + R[7] * oy + R[8] * oz;
      Ox = (float)fx; Oy = (float)fy; Oz = (float)fz;
      const double om = A.omega[ie];
      w = (float)om;
      wc = (float)(om / kCl);
      if (live && grp == 0 && span == 0 && !mixed_geometry_ok(fx, fy, fz, om, F.xperp_max, F.z_max))
        atomicOr(A.err, kErrBadArgs);
    }
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      double S[6] = {0, 0, 0, 0, 0, 0};
      float dmax = 0.f;
      bool any = false;
      const int64_t nchunks = b1 > b0 ? (b1 - b0 + kMxChunk - 1) / kMxChunk : 0;
      if (tid == 0) {
        // the sample before the span, if it belongs to the same segment (span > 0)
        prev_valid = span > 0 && b0 < b1;
        if (prev_valid) {
          prev_rec[0] = rec[3 * (b0 - 1)];
          prev_rec[1] = rec[3 * (b0 - 1) + 1];
          prev_rec[2] = rec[3 * (b0 - 1) + 2];
        }
        if (nchunks > 0) {
          const int64_t hi = min(b1, b0 + kMxChunk);
          mbar_arrive_expect_tx(&st.bar[0], (uint32_t)((hi - b0) * 48));
          tma_load_1d(&st.v[0][0], rec + 3 * b0, (uint32_t)((hi - b0) * 48), &st.bar[0]);
        }
      }
      __syncthreads();
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = b0 + c * kMxChunk, hi = min(b1, lo + kMxChunk);
        if (tid == 0 && c + 1 < nchunks) {
          const int64_t lo2 = lo + kMxChunk, hi2 = min(b1, lo2 + kMxChunk);
          mbar_arrive_expect_tx(&st.bar[buf ^ 1], (uint32_t)((hi2 - lo2) * 48));
          tma_load_1d(&st.v[buf ^ 1][0], rec + 3 * lo2, (uint32_t)((hi2 - lo2) * 48), &st.bar[buf ^ 1]);
        }
        if (!mbar_wait(&st.bar[buf], (phase_bits >> buf) & 1u)) {
          if (tid == 0) atomicOr(A.err, kErrTmaTimeout);
          return;
        }
        phase_bits ^= 1u << buf;
        const float4* sv = st.v[buf];
        const int n = (int)(hi - lo);
        int j0 = grp * PART;
        const int j1 = min(n, (grp + 1) * PART);
        if (live && j0 < j1) {
          float last = __int_as_float(0x7fc00000);  // NaN: no step into the first sample
          if (lo + j0 == 0) {
            j0 = 1;  // sample 0 is the unused slot and has no successor step
          } else if (j0 > 0) {
            last = mixed_phase(sv[3 * (j0 - 1)], Ox, Oy, Oz, w, wc);
          } else if (prev_valid) {
            last = mixed_phase(prev_rec[0], Ox, Oy, Oz, w, wc);
          }
          for (int jb = j0; jb < j1; jb += kMxFold) {
            const int je = min(j1, jb + kMxFold);
            float s32[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int j = jb; j < je; ++j) {
              const float ph = mixed_sample(sv[3 * j], sv[3 * j + 1], sv[3 * j + 2], Ox, Oy, Oz, w, wc, s32);
              dmax = fmaxf(dmax, fabsf(ph - last));
              last = ph;
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) S[k] += (double)s32[k];
          }
          any = any || j0 < j1;
        }
        __syncthreads();  // everyone is done with `buf` (and prev_rec) before they are refilled
        if (tid == 0 && c + 1 < nchunks) {
          prev_rec[0] = sv[3 * (n - 1)];
          prev_rec[1] = sv[3 * (n - 1) + 1];
          prev_rec[2] = sv[3 * (n - 1) + 2];
          prev_valid = 1;
        }
        __syncthreads();
      }
      // reduce the groups' sums in group order; group 0 stores the span's partial
      if (SUB > 1) {
        if (grp > 0) {
#pragma unroll
          for (int k = 0; k < 6; ++k) red[grp - 1][k][q] = S[k];
          red[grp - 1][6][q] = any ? (double)dmax : -1.0;
        }
        __syncthreads();
        if (grp == 0) {
          double dm = any ? (double)dmax : -1.0;
          for (int o = 0; o < SUB - 1; ++o) {
#pragma unroll
            for (int k = 0; k < 6; ++k) S[k] += red[o][k][q];
            dm = fmax(dm, red[o][6][q]);
          }
          if (live) {
            double* p = A.part + fused_part_index(P, tile, g, span, 0, q, TE);
#pragma unroll
            for (int k = 0; k < 6; ++k) p[k * TE] = S[k];
            p[6 * TE] = 0.0;
            p[7 * TE] = 0.0;
            p[8 * TE] = dm;  // -1: empty span
          }
        }
        __syncthreads();
      }
    }
    fused_unit_done<1, kMxThreads>(A, P, tile, n_act, &s_last, TE);
  }
}


// ---------------------------------------------------------------------------------------------
// Packed-FP32 (f32x2) sample sum over pair records.
//
// Pair records: samples 2p and 2p + 1 share 6 float4 (96 bytes); component c of sample 2p + b is
// float 4 (c / 2) + 2 (c % 2) + b of the pair, with the components
//   x, y, z, tau_s | -bx, -by, 1-bz, bz | 1-b^2, az, ax, ay
// so that every half of a loaded float4 is one component of both samples, the operand of one
// packed instruction (fma/mul/add.rn.f32x2, two FP32 lanes per issue on sm_100).  Sample 0, the
// unused slot of the level ladder, holds a zero-amplitude record at the position and time of
// sample 1 (no contribution, no phase step), so every span is a whole number of pairs (spans begin
// and end at even samples).  The positive phase P = w tau_s + (w/c) corr enters as exp(-i P).
// ---------------------------------------------------------------------------------------------
constexpr int kPrChunk = 256;   // samples per staged chunk (128 pairs, 12 KB)
constexpr int kPrFold = 16;     // pairs per FP32 partial sum before it is folded into FP64
constexpr float kRoundF = 12582912.f;  // 1.5 * 2^23: t + kRoundF rounds t to an integer for |t| < 2^22

struct PairStage {
  float4 v[2][kPrChunk * 3];
  uint64_t bar[2];
};

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// Per-entry constants of the pair kernel (observer in the particle frame, w, w/c), both lanes equal.
struct PairObs {
  float2 ox, oy, oz, w, wc;
};

// P of one sample with the per-lane operations of pair_sample (same value).
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

// Phase of sample b (0 or 1) of the pair record at `q` (shared or global memory).
__device__ __forceinline__ float pair_phase_at(const float* q, int b, const PairObs& o) {
  return pair_phase(q[b], q[2 + b], q[4 + b], q[6 + b], o);
}

// Both samples of one pair for one entry: adds e (cos P, sin P) per lane to acc (x re, x im, y re,
// y im, z re, z im; the imaginary parts with the sign of +sin P) and returns P of both samples.
// The amplitude is that of mixed_sample with u = n - b, om = 1 - n.b formed as
//   om = (1-bz) + (1-nz) bz - nx bx - ny by,  uz = (1-bz) - (1-nz).
__device__ __forceinline__ float2 pair_sample(const float4* __restrict__ q, const PairObs& o, float2* acc) {
  const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5];
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
  // Cody-Waite reduction to [-pi, pi]: t - kRoundF = rint(P / 2pi) = k, nk = -k exactly
  const float2 t = fma2(P, f2(kInvTwoPiF), f2(kRoundF));
  const float2 nk = fma2(t, M1, f2(kRoundF));
  const float2 rr = fma2(nk, f2(kTwoPiLoF), fma2(nk, f2(kTwoPiHiF), P));
  float2 sn, cs;
  sincos_ftz(rr.x, &sn.x, &cs.x);
  sincos_ftz(rr.y, &sn.y, &cs.y);
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

// Pair records from the FP64 level cache for samples [s_begin, s_end) (thread per sample).
__global__ void k_mixed_records_pair(const double* __restrict__ lev, int64_t cap, int64_t s_begin, int64_t s_end,
                                     MixedFrame F, float* __restrict__ rec) {
  const int64_t s = s_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= s_end) return;
  const int64_t src = s == 0 ? 1 : s;  // sample 0: position and time of sample 1, zero amplitude
  const double t = lev[src];
  const double dx = lev[cap + src] - F.x0[0], dy = lev[2 * cap + src] - F.x0[1], dz = lev[3 * cap + src] - F.x0[2];
  const double bx = lev[4 * cap + src], by = lev[5 * cap + src], bz = lev[6 * cap + src];
  const double ax = lev[7 * cap + src], ay = lev[8 * cap + src], az = lev[9 * cap + src];
  const double* R = F.rot;
  const double x = R[0] * dx + R[1] * dy + R[2] * dz;
  const double y = R[3] * dx + R[4] * dy + R[5] * dz;
  const double z = R[6] * dx + R[7] * dy + R[8] * dz;
  const double px = R[0] * bx + R[1] * by + R[2] * bz;
  const double py = R[3] * bx + R[4] * by + R[5] * bz;
  const double pz = R[6] * bx + R[7] * by + R[8] * bz;
  const double qx = R[0] * ax + R[1] * ay + R[2] * az;
  const double qy = R[3] * ax + R[4] * ay + R[5] * az;
  const double qz = R[6] * ax + R[7] * ay + R[8] * az;
  const double g2 = 1.0 - (px * px + py * py + pz * pz);
  const double ebz = (g2 + px * px + py * py) / (1.0 + pz);
  const double taus = (t - F.t_ref) - z / kCl;
  float v[12] = {(float)x, (float)y, (float)z, (float)taus, (float)-px, (float)-py,
                 (float)ebz, (float)pz, (float)g2, (float)qz, (float)qx, (float)qy};
  if (s == 0) {
    v[4] = v[5] = 0.f;
    v[6] = 1.f;
    v[7] = v[8] = v[9] = v[10] = v[11] = 0.f;
  }
  float* base = rec + 24 * (s >> 1) + (s & 1);
#pragma unroll
  for (int c = 0; c < 12; ++c) base[4 * (c >> 1) + 2 * (c & 1)] = v[c];
}

// Sample-split sum over pair records: SUB groups of TE = 128 / SUB threads (one entry per thread)
// each take 1/SUB of every staged chunk, two samples per packed step.  The largest phase step of a
// part starts from the sample before it (inside the chunk, the previous chunk's last sample carried
// by group 0, or the span's predecessor read from global memory), so the span maxima already
// include the step into each span (dmax_spans_joined).  Partials and the fused finalize are those
// of k_fd_wave_mixed_split.
template <int SUB, int MINB>
__global__ void __launch_bounds__(kMxThreads, MINB) k_fd_wave_mixed_pair(FdWaveArgs A, MixedFrame F) {
  constexpr int TE = kMxThreads / SUB;
  if (A.tile_entries != TE) {  // the host sized the partials for another tile
    if (threadIdx.x == 0) atomicOr(A.err, kErrPlan);
    return;
  }
  constexpr int CP = kPrChunk / 2;  // pairs per chunk
  constexpr int PP = CP / SUB;      // pairs per group and chunk
  __shared__ __align__(16) PairStage st;
  __shared__ double red[SUB > 1 ? SUB - 1 : 1][7][TE];
  __shared__ int s_last;
  __shared__ WavePlan P;
  __shared__ int64_t next_unit;
  const int tid = threadIdx.x;
  const int grp = tid / TE, q = tid % TE;
  if (A.fused && blockIdx.x == 0 && tid == 0) {  // counters of the following wave
    if (A.zero_u32) *A.zero_u32 = 0;
    if (A.zero_u64) *A.zero_u64 = 0;
  }
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  if (tid == 0) {
    P = wave_plan(A.first, A.level, n_act, TE, A.target_units, A.min_span);
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t units = P.tiles * P.spans;
  const float4* rec = reinterpret_cast<const float4*>(A.lev);
  const float* recf = reinterpret_cast<const float*>(A.lev);
  uint32_t phase_bits = 0;
  for (;;) {
    if (tid == 0) next_unit = (int64_t)atomicAdd(A.work, 1ull);
    __syncthreads();
    const int64_t u = next_unit;
    __syncthreads();
    if (u >= units) break;
    const int64_t tile = u / P.spans;
    const int span = (int)(u % P.spans);
    const int64_t slot = tile * TE + q;
    const bool live = slot < n_act;
    const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
    const int64_t io = item / A.n_e, ie = item % A.n_e;
    PairObs o;
    {
      const double* R = F.rot;
      const double ox = A.obs[3 * io] - F.x0[0], oy = A.obs[3 * io + 1] - F.x0[1], oz = A.obs[3 * io + 2] - F.x0[2];
      const double fx = R[0] * ox + R[1] * oy + R[2] * oz;
      const double fy = R[3] * ox + R[4] * oy + R[5] * oz;
      const double fz = R[6] * ox + R[7] * oy + R[8] * oz;
      const double om = A.omega[ie];
      o.ox = f2((float)fx);
      o.oy = f2((float)fy);
      o.oz = f2((float)fz);
      o.w = f2((float)om);
      o.wc = f2((float)(om / kCl));
      if (live && grp == 0 && span == 0 && !mixed_geometry_ok(fx, fy, fz, om, F.xperp_max, F.z_max))
        atomicOr(A.err, kErrBadArgs);
    }
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      const int64_t p0 = b0 >> 1, p1 = b1 > b0 ? b1 >> 1 : p0;  // spans are whole pairs
      double S[6] = {0, 0, 0, 0, 0, 0};
      float dmax = 0.f;
      bool any = false;
      const int64_t nchunks = (p1 - p0 + CP - 1) / CP;
      // phase of the sample before the next part of group 0: the span's predecessor (span > 0)
      float carry = __int_as_float(0x7fc00000);  // NaN: no step into the segment's first sample
      if (grp == 0 && live && span > 0 && nchunks > 0) carry = pair_phase_at(recf + 24 * (p0 - 1), 1, o);
      if (tid == 0 && nchunks > 0) {
        const int64_t hi = min(p1, p0 + CP);
        mbar_arrive_expect_tx(&st.bar[0], (uint32_t)((hi - p0) * 96));
        tma_load_1d(&st.v[0][0], rec + 6 * p0, (uint32_t)((hi - p0) * 96), &st.bar[0]);
      }
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = p0 + c * CP, hi = min(p1, lo + CP);
        if (tid == 0 && c + 1 < nchunks) {
          const int64_t lo2 = lo + CP, hi2 = min(p1, lo2 + CP);
          mbar_arrive_expect_tx(&st.bar[buf ^ 1], (uint32_t)((hi2 - lo2) * 96));
          tma_load_1d(&st.v[buf ^ 1][0], rec + 6 * lo2, (uint32_t)((hi2 - lo2) * 96), &st.bar[buf ^ 1]);
        }
        if (!mbar_wait(&st.bar[buf], (phase_bits >> buf) & 1u)) {
          if (tid == 0) atomicOr(A.err, kErrTmaTimeout);
          return;
        }
        phase_bits ^= 1u << buf;
        const float4* sv = st.v[buf];
        const int n = (int)(hi - lo);
        const int j0 = grp * PP, j1 = min(n, j0 + PP);
        if (live && j0 < j1) {
          float last = j0 > 0 ? pair_phase_at(reinterpret_cast<const float*>(sv + 6 * (j0 - 1)), 1, o) : carry;
          for (int jb = j0; jb < j1; jb += kPrFold) {
            const int je = min(j1, jb + kPrFold);
            float2 acc[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[k] = f2(0.f);
#pragma unroll 2
            for (int j = jb; j < je; ++j) {
              const float2 ph = pair_sample(sv + 6 * j, o, acc);
              dmax = fmaxf(dmax, fmaxf(fabsf(ph.x - last), fabsf(ph.y - ph.x)));
              last = ph.y;
            }
#pragma unroll
            for (int k = 0; k < 6; k += 2) {
              S[k] += (double)acc[k].x + (double)acc[k].y;
              S[k + 1] -= (double)acc[k + 1].x + (double)acc[k + 1].y;
            }
          }
          any = true;
        }
        if (grp == 0 && live && c + 1 < nchunks)  // the chunk is full: its last sample precedes the next
          carry = pair_phase_at(reinterpret_cast<const float*>(sv + 6 * (CP - 1)), 1, o);
        __syncthreads();  // everyone is done with `buf` before it is refilled
      }
      // reduce the groups' sums in group order; group 0 stores the span's partial
      if (SUB > 1 && grp > 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) red[grp - 1][k][q] = S[k];
        red[grp - 1][6][q] = any ? (double)dmax : -1.0;
      }
      if (SUB > 1) __syncthreads();
      if (grp == 0) {
        double dm = any ? (double)dmax : -1.0;
        for (int o2 = 0; o2 < SUB - 1; ++o2) {
#pragma unroll
          for (int k = 0; k < 6; ++k) S[k] += red[o2][k][q];
          dm = fmax(dm, red[o2][6][q]);
        }
        if (live) {
          double* p = A.part + fused_part_index(P, tile, g, span, 0, q, TE);
#pragma unroll
          for (int k = 0; k < 6; ++k) p[k * TE] = S[k];
          p[6 * TE] = 0.0;
          p[7 * TE] = 0.0;
          p[8 * TE] = dm;  // -1: empty span
        }
      }
      if (SUB > 1) __syncthreads();
    }
    fused_unit_done<1, kMxThreads>(A, P, tile, n_act, &s_last, TE);
  }
}

}  // namespace dev

cudaError_t launch_mixed_records(const double* lev, int64_t cap, int64_t s_begin, int64_t s_end, const MixedFrame& F,
                                 float4* rec, int layout, cudaStream_t st) {
  if (layout == 1 && s_begin == 1) s_begin = 0;  // pair records also fill the zero-amplitude sample 0
  if (s_end <= s_begin) return cudaSuccess;
  const int T = 256;
  const unsigned grid = (unsigned)((s_end - s_begin + T - 1) / T);
  if (layout == 1)
    dev::k_mixed_records_pair<<<grid, T, 0, st>>>(lev, cap, s_begin, s_end, F, reinterpret_cast<float*>(rec));
  else
    dev::k_mixed_records<<<grid, T, 0, st>>>(lev, cap, s_begin, s_end, F, rec);
  return cudaGetLastError();
}

// Compiled variants of the mixed wave kernel.  Variants 0-6: (entries per thread, minimum CTAs per
// SM) over sample records; 7-9: sample-split (groups, minimum CTAs) over sample records; 10-12:
// sample-split packed-FP32 over pair records.  Split variants need the fused finalize.
static const int kMixedEpt[kMixedVariants] = {1, 1, 2, 2, 2, 4, 4, 0, 0, 0, 0, 0, 0};
static const int kMixedSub[kMixedVariants] = {0, 0, 0, 0, 0, 0, 0, 4, 4, 2, 4, 4, 2};

int mixed_entries_per_cta(int variant) {
  return kMixedSub[variant] ? dev::kMxThreads / kMixedSub[variant] : dev::kMxThreads * kMixedEpt[variant];
}
bool mixed_variant_is_split(int variant) { return kMixedSub[variant] != 0; }
const char* mixed_variant_name(int variant) {
  static const char* const kNames[kMixedVariants] = {
      "k_fd_wave_mixed<1,1>", "k_fd_wave_mixed<1,8>", "k_fd_wave_mixed<2,1>", "k_fd_wave_mixed<2,5>",
      "k_fd_wave_mixed<2,6>", "k_fd_wave_mixed<4,1>", "k_fd_wave_mixed<4,3>", "k_fd_wave_mixed_split<4,1>",
      "k_fd_wave_mixed_split<4,6>", "k_fd_wave_mixed_split<2,4>", "k_fd_wave_mixed_pair<4,4>",
      "k_fd_wave_mixed_pair<4,1>", "k_fd_wave_mixed_pair<2,4>"};
  return variant >= 0 && variant < kMixedVariants ? kNames[variant] : "";
}
int mixed_variant_layout(int variant) { return variant >= 10 ? 1 : 0; }

template <int EPT, int MINB>
static void mixed_occ(int& n) {
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed<EPT, MINB>, dev::kMxThreads, 0);
}

int mixed_blocks_per_sm(int variant) {
  int n = 0;
  switch (variant) {
    case 0: mixed_occ<1, 1>(n); break;
    case 1: mixed_occ<1, 8>(n); break;
    case 2: mixed_occ<2, 1>(n); break;
    case 3: mixed_occ<2, 5>(n); break;
    case 4: mixed_occ<2, 6>(n); break;
    case 5: mixed_occ<4, 1>(n); break;
    case 6: mixed_occ<4, 3>(n); break;
    case 7: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_split<4, 1>, dev::kMxThreads, 0); break;
    case 8: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_split<4, 6>, dev::kMxThreads, 0); break;
    case 9: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_split<2, 4>, dev::kMxThreads, 0); break;
    case 10: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_pair<4, 4>, dev::kMxThreads, 0); break;
    case 11: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_pair<4, 1>, dev::kMxThreads, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_pair<2, 4>, dev::kMxThreads, 0); break;
  }
  return n > 0 ? n : 1;
}

cudaError_t launch_fd_wave_mixed(const FdWaveArgs& a, const MixedFrame& F, int grid, int variant, cudaStream_t st) {
  const int T = dev::kMxThreads;
  switch (variant) {
    case 0: dev::k_fd_wave_mixed<1, 1><<<grid, T, 0, st>>>(a, F); break;
    case 1: dev::k_fd_wave_mixed<1, 8><<<grid, T, 0, st>>>(a, F); break;
    case 2: dev::k_fd_wave_mixed<2, 1><<<grid, T, 0, st>>>(a, F); break;
    case 3: dev::k_fd_wave_mixed<2, 5><<<grid, T, 0, st>>>(a, F); break;
    case 4: dev::k_fd_wave_mixed<2, 6><<<grid, T, 0, st>>>(a, F); break;
    case 5: dev::k_fd_wave_mixed<4, 1><<<grid, T, 0, st>>>(a, F); break;
    case 6: dev::k_fd_wave_mixed<4, 3><<<grid, T, 0, st>>>(a, F); break;
    case 7: dev::k_fd_wave_mixed_split<4, 1><<<grid, T, 0, st>>>(a, F); break;
    case 8: dev::k_fd_wave_mixed_split<4, 6><<<grid, T, 0, st>>>(a, F); break;
    case 9: dev::k_fd_wave_mixed_split<2, 4><<<grid, T, 0, st>>>(a, F); break;
    case 10: dev::k_fd_wave_mixed_pair<4, 4><<<grid, T, 0, st>>>(a, F); break;
    case 11: dev::k_fd_wave_mixed_pair<4, 1><<<grid, T, 0, st>>>(a, F); break;
    default: dev::k_fd_wave_mixed_pair<2, 4><<<grid, T, 0, st>>>(a, F); break;
  }
  return cudaGetLastError();
}

}  // namespace osc
