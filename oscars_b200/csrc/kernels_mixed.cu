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

}  // namespace dev

cudaError_t launch_mixed_records(const double* lev, int64_t cap, int64_t s_begin, int64_t s_end, const MixedFrame& F,
                                 float4* rec, cudaStream_t st) {
  if (s_end <= s_begin) return cudaSuccess;
  const int T = 256;
  dev::k_mixed_records<<<(unsigned)((s_end - s_begin + T - 1) / T), T, 0, st>>>(lev, cap, s_begin, s_end, F, rec);
  return cudaGetLastError();
}

// Compiled variants of the mixed wave kernel: (entries per thread, minimum resident CTAs per SM).
// Variants 0-6: (entries per thread, minimum CTAs per SM); 7-9: sample-split (groups, minimum CTAs),
// which need the fused finalize.
static const int kMixedEpt[kMixedVariants] = {1, 1, 2, 2, 2, 4, 4, 0, 0, 0};
static const int kMixedSub[kMixedVariants] = {0, 0, 0, 0, 0, 0, 0, 4, 4, 2};

int mixed_entries_per_cta(int variant) {
  return kMixedSub[variant] ? dev::kMxThreads / kMixedSub[variant] : dev::kMxThreads * kMixedEpt[variant];
}
bool mixed_variant_is_split(int variant) { return kMixedSub[variant] != 0; }

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
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_split<2, 4>, dev::kMxThreads, 0); break;
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
    default: dev::k_fd_wave_mixed_split<2, 4><<<grid, T, 0, st>>>(a, F); break;
  }
  return cudaGetLastError();
}

}  // namespace osc
