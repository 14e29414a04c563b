// kernels_mixed.cu -- mixed-precision frequency-domain sum of one trajectory: FP64 trajectory,
// FP64 retarded phase and range reduction, FP32 amplitudes, sin / cos and per-fold sums folded
// into FP64.  The sample term, the pair-record layout and the error budget are described in
// fd_common.cuh ("Mixed-precision sample term over pair records").
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "fd_common.cuh"
#include "kernels.h"

namespace osc {
namespace dev {

constexpr int kMxThreads = 128;
constexpr int kPrFold = 16;     // pairs per FP32 partial sum before it is folded into FP64

template <int CP>  // CP pair records per staged chunk, two buffers
struct PairStage {
  float4 v[2][CP * kPairF4];
  uint64_t bar[2];
};

// Pair records of level samples [s_begin, s_end) straight from the trajectory spline (one thread per
// sample): the level time (levels above ext_from are extended levels, see level_time), the spline values
// (include/TOMATH.h:92-121, bit-identical to the FP64 level cache), the particle frame and the record.
// Sample 0 is the zero-amplitude record at the position and time of sample 1.  The two samples of a
// pair sit in adjacent lanes (s_begin and the block size are even) and exchange their FP64 values
// for the pair's step, so every lane of the grid's last warp takes part (past s_end on a clamped
// sample, writing nothing).
__global__ void k_mixed_records(const double* __restrict__ knots, int64_t n, double tstart, double tstop,
                                int64_t s_begin, int64_t s_end, int ext_from, MixedFrame F,
                                float* __restrict__ rec) {
  const int64_t s_raw = s_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s_raw < s_end;
  const int64_t s = active ? s_raw : s_end - 2 + (s_raw & 1);
  const double t = level_time(tstart, tstop, s == 0 ? 1 : s, ext_from);
  double v[9];
  spline_eval9(knots, n, t, v);
  const double dx = v[0] - F.x0[0], dy = v[1] - F.x0[1], dz = v[2] - F.x0[2];
  const double* R = F.rot;
  const double x = R[0] * dx + R[1] * dy + R[2] * dz;
  const double y = R[3] * dx + R[4] * dy + R[5] * dz;
  const double z = R[6] * dx + R[7] * dy + R[8] * dz;
  const double px = R[0] * v[3] + R[1] * v[4] + R[2] * v[5];
  const double py = R[3] * v[3] + R[4] * v[4] + R[5] * v[5];
  const double pz = R[6] * v[3] + R[7] * v[4] + R[8] * v[5];
  const double qx = R[0] * v[6] + R[1] * v[7] + R[2] * v[8];
  const double qy = R[3] * v[6] + R[4] * v[7] + R[5] * v[8];
  const double qz = R[6] * v[6] + R[7] * v[7] + R[8] * v[8];
  const double taus = (t - F.t_ref) - z / kCLight;
  const unsigned full = 0xffffffffu;
  const double xo = __shfl_xor_sync(full, x, 1), yo = __shfl_xor_sync(full, y, 1);
  const double zo = __shfl_xor_sync(full, z, 1), to = __shfl_xor_sync(full, taus, 1);
  if (active) write_pair_record(rec, s, s == 0, x, y, z, taus, px, py, pz, qx, qy, qz, xo, yo, zo, to);
}

// Sample sum over pair records, sample-split: the CTA's 128 threads form SUB groups of TE = 128 / SUB
// threads (one entry per thread); each group takes 1/SUB of every staged chunk, two samples per
// packed step.  The largest phase step of a part starts from the sample before it (inside the
// chunk, the previous chunk's last sample carried by group 0, or the span's predecessor read from
// global memory), so the span maxima already include the step into each span (dmax_spans_joined).
// The groups' sums are reduced in shared memory in group order and one tile-major partial per entry
// and span is stored; the CTA that finishes a tile's last span finalizes the tile (fused_unit_done).
// With A.fused == 0 the partials are only stored (the adjoint's forward sums read them).
template <int SUB, int MINB, int CP, bool SSM>
__global__ void __launch_bounds__(kMxThreads, MINB) k_fd_wave_mixed_pair(FdWaveArgs A, MixedFrame F) {
  constexpr int TE = kMxThreads / SUB;
  if (A.tile_entries != TE) {  // the host sized the partials for another tile
    if (threadIdx.x == 0) atomicOr(A.err, kErrPlan);
    return;
  }
  __shared__ __align__(16) PairStage<CP> st;
  __shared__ double ssum[SSM ? 6 : 1][SSM ? kMxThreads : 1];
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
      o = make_pair_obs(fx, fy, fz, om);
      if (live && grp == 0 && span == 0 && !mixed_geometry_ok(fx, fy, fz, om, F)) atomicOr(A.err, kErrBadArgs);
    }
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      const int64_t p0 = b0 >> 1, p1 = b1 > b0 ? b1 >> 1 : p0;  // spans are whole pairs
      double S[6] = {0, 0, 0, 0, 0, 0};
      if (SSM)
#pragma unroll
        for (int k = 0; k < 6; ++k) ssum[k][tid] = 0.0;
      float dmax = 0.f;
      bool any = false;
      const int64_t nchunks = (p1 - p0 + CP - 1) / CP;
      // phase of the sample before a part that starts a chunk: the span's predecessor (span > 0), then
      // the previous chunk's last sample (whichever group's part starts at the chunk's first pair)
      float carry = __int_as_float(0x7fc00000);  // NaN: no step into the segment's first sample
      if (live && span > 0 && nchunks > 0) carry = pair_phase_at(recf + kPairFloats * (p0 - 1), 1, o);
      if (tid == 0 && nchunks > 0) {
        const int64_t hi = min(p1, p0 + CP);
        mbar_arrive_expect_tx(&st.bar[0], (uint32_t)((hi - p0) * (kPairFloats * 4)));
        tma_load_1d(&st.v[0][0], rec + kPairF4 * p0, (uint32_t)((hi - p0) * (kPairFloats * 4)), &st.bar[0]);
      }
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = p0 + c * CP, hi = min(p1, lo + CP);
        if (tid == 0 && c + 1 < nchunks) {
          const int64_t lo2 = lo + CP, hi2 = min(p1, lo2 + CP);
          mbar_arrive_expect_tx(&st.bar[buf ^ 1], (uint32_t)((hi2 - lo2) * (kPairFloats * 4)));
          tma_load_1d(&st.v[buf ^ 1][0], rec + kPairF4 * lo2, (uint32_t)((hi2 - lo2) * (kPairFloats * 4)), &st.bar[buf ^ 1]);
        }
        if (!mbar_wait(&st.bar[buf], (phase_bits >> buf) & 1u)) {
          if (tid == 0) atomicOr(A.err, kErrTmaTimeout);
          return;
        }
        phase_bits ^= 1u << buf;
        const float4* sv = st.v[buf];
        const int n = (int)(hi - lo);
        const int j0 = (grp * n) / SUB, j1 = ((grp + 1) * n) / SUB;  // the chunk's pairs split evenly
        if (live && j0 < j1) {
          float last = j0 > 0 ? pair_phase_at(reinterpret_cast<const float*>(sv + kPairF4 * (j0 - 1)), 1, o) : carry;
          for (int jb = j0; jb < j1; jb += kPrFold) {
            const int je = min(j1, jb + kPrFold);
            float2 acc[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[k] = f2(0.f);
#pragma unroll 2
            for (int j = jb; j < je; ++j) {
              const float2 ph = pair_sample(sv + kPairF4 * j, o, acc);
              dmax = fmaxf(dmax, fmaxf(fabsf(ph.x - last), fabsf(ph.y - ph.x)));
              last = ph.y;
            }
            if (SSM) {
#pragma unroll
              for (int k = 0; k < 6; k += 2) {
                ssum[k][tid] += (double)acc[k].x + (double)acc[k].y;
                ssum[k + 1][tid] -= (double)acc[k + 1].x + (double)acc[k + 1].y;
              }
            } else {
#pragma unroll
              for (int k = 0; k < 6; k += 2) {
                S[k] += (double)acc[k].x + (double)acc[k].y;
                S[k + 1] -= (double)acc[k + 1].x + (double)acc[k + 1].y;
              }
            }
          }
          any = true;
        }
        if (live && c + 1 < nchunks)  // the chunk is full: its last sample precedes the next
          carry = pair_phase_at(reinterpret_cast<const float*>(sv + kPairF4 * (CP - 1)), 1, o);
        __syncthreads();  // everyone is done with `buf` before it is refilled
      }
      if (SSM)
#pragma unroll
        for (int k = 0; k < 6; ++k) S[k] = ssum[k][tid];
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
    if (A.fused) fused_unit_done_grouped<kMxThreads>(A, P, tile, n_act, &s_last, TE, &red[0][0][0]);
  }
}

}  // namespace dev

cudaError_t launch_mixed_records(const double* knots, int64_t n, double tstart, double tstop, int64_t s_begin,
                                 int64_t s_end, int ext_from, const MixedFrame& F, float4* rec, cudaStream_t st) {
  if (s_end <= s_begin) return cudaSuccess;
  const int T = 128;
  const unsigned grid = (unsigned)((s_end - s_begin + T - 1) / T);
  dev::k_mixed_records<<<grid, T, 0, st>>>(knots, n, tstart, tstop, s_begin, s_end, ext_from, F,
                                            reinterpret_cast<float*>(rec));
  return cudaGetLastError();
}

// Compiled variants of the mixed wave kernel: groups SUB of 128 / SUB entries, minimum CTAs per SM,
// pair records per staged chunk, FP64 span sums kept in shared memory.
#define OSC_MIXED_VARIANTS(X) \
  X(0, 4, 4, 128, false)      \
  X(1, 4, 4, 64, true)        \
  X(2, 4, 5, 64, false)       \
  X(3, 2, 5, 64, true)

#define OSC_SUB(i, sub, minb, cp, ssm) sub,
static const int kMixedSub[kMixedVariants] = {OSC_MIXED_VARIANTS(OSC_SUB)};

int mixed_entries_per_cta(int variant) { return dev::kMxThreads / kMixedSub[variant]; }
const char* mixed_variant_name(int variant) {
#define OSC_NAME(i, sub, minb, cp, ssm) "k_fd_wave_mixed_pair<" #sub "," #minb "," #cp "," #ssm ">",
  static const char* const kNames[kMixedVariants] = {OSC_MIXED_VARIANTS(OSC_NAME)};
  return variant >= 0 && variant < kMixedVariants ? kNames[variant] : "";
}

int mixed_blocks_per_sm(int variant) {
  int n = 0;
  switch (variant) {
#define OSC_OCC(i, sub, minb, cp, ssm) \
    case i: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_mixed_pair<sub, minb, cp, ssm>, dev::kMxThreads, 0); break;
    OSC_MIXED_VARIANTS(OSC_OCC)
  }
  return n > 0 ? n : 1;
}

cudaError_t launch_fd_wave_mixed(const FdWaveArgs& a, const MixedFrame& F, int grid, int variant, cudaStream_t st) {
  const int T = dev::kMxThreads;
  switch (variant) {
#define OSC_LAUNCH(i, sub, minb, cp, ssm) \
    case i: dev::k_fd_wave_mixed_pair<sub, minb, cp, ssm><<<grid, T, 0, st>>>(a, F); break;
    OSC_MIXED_VARIANTS(OSC_LAUNCH)
  }
  return cudaGetLastError();
}

}  // namespace osc
