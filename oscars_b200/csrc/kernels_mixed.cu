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
// pair sit in adjacent lanes (s_begin and the samples per warp are even) and exchange their FP64 values
// for the pair's step, so every lane of the grid's last warp takes part (past s_end on a clamped
// sample, writing nothing).  Also folds, per level, the largest |beta_i - beta_{i-1}| over its
// samples i >= 1 into bd_bits (the power-density stop rule, src/OSCARSSR.cc:2887-2891; the FP64 values
// and operations of k_level_betadiff): the predecessor's beta comes from the lane before (lanes 0
// and 1 of every warp evaluate the warp's two predecessors).
constexpr int kRecWarpSamples = 30;  // samples per warp of k_mixed_records (32 lanes, 2 of them a halo)
__global__ void k_mixed_records(const double* __restrict__ knots, int64_t n, double tstart, double tstop,
                                int64_t s_begin, int64_t s_end, int ext_from, MixedFrame F,
                                float* __restrict__ rec, unsigned long long* __restrict__ bd_bits) {
  __shared__ unsigned long long blk[32];  // per-level maxima of this block
  if (threadIdx.x < 32) blk[threadIdx.x] = 0;
  __syncthreads();
  // Each warp holds kRecWarpSamples samples in lanes 2..31 and their two predecessors in lanes 0..1
  // (a halo: evaluated, not written), so every sample finds the one before it in the lane before and
  // lane pairs stay (even, odd) samples.
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t s_raw = s_begin + gw * kRecWarpSamples + lane - 2;
  const bool active = lane >= 2 && s_raw < s_end;
  // halo lanes before sample 0 and lanes past the end evaluate a valid sample of the same parity
  const int64_t s = s_raw < 0 ? s_raw + 4 : (s_raw < s_end ? s_raw : s_end - 2 + (s_raw & 1));
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
  // beta step from the previous sample of the same level
  double pbx = __shfl_up_sync(full, v[3], 1), pby = __shfl_up_sync(full, v[4], 1), pbz = __shfl_up_sync(full, v[5], 1);
  const int L = 63 - __clzll((unsigned long long)(s == 0 ? 1 : s));
  const bool step = active && s >= 1 && s - ((int64_t)1 << L) > 0;
  if (step && bd_bits) {
    const double dx = __dsub_rn(v[3], pbx), dy = __dsub_rn(v[4], pby), dz = __dsub_rn(v[5], pbz);
    const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    atomicMax(&blk[L & 31], (unsigned long long)__double_as_longlong(d));
  }
  __syncthreads();
  if (bd_bits && threadIdx.x < 32 && blk[threadIdx.x]) atomicMax(&bd_bits[threadIdx.x], blk[threadIdx.x]);
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

// ---------------------------------------------------------------------------------------------
// Power density over the pair records, mixed precision (src/OSCARSSR.cc:2869-2922):
//   sum += |N1 x ((N1 - b) x a/c)|^2 / (1 - b.N1)^5 / |O - X|^2 * (N1 . normal)
// (the sum of the squared projections on N2 and N3, an orthonormal pair across N1, is the squared
// norm of the numerator, which is across N1).  Geometry, 1 - b.N1 without cancellation
// ((1 - b_z) + (1 - n_z) b_z - n_x b_x - n_y b_y, with 1 - n_z = (rho^2 / (D + |R_z|) + |R_z| - R_z) / D
// for any direction) and the numerator run on packed f32x2 operands in the particle frame; the fifth
// power of 1 / (1 - b.N1) (~1e40 near the axis, beyond FP32) and the sums in FP64.  Sample-split like
// the flux kernel: SUB groups of TE = 128 / SUB entries, each taking 1/SUB of every staged chunk, the
// groups' sums reduced in group order; entry-major partials for k_pd_finalize.
// ---------------------------------------------------------------------------------------------
struct PdObsMx {
  float2 ox, oy, oz;  // observer in the particle frame (both lanes)
  float2 nx, ny, nz;  // surface normal in the particle frame (both lanes)
};

// Exact float -> double of any finite normal float or zero on the integer pipe (denormals, which the
// flushed FP32 arithmetic does not produce, would come out as ~6e-39).
__device__ __forceinline__ double float_to_double_bits(float x) {
  const unsigned u = __float_as_uint(x);
  const unsigned hi = (u & 0x7FFFFFFFu) ? ((((u & 0x7FFFFFFFu) >> 3) + 0x38000000u) | (u & 0x80000000u)) : u;
  return __hiloint2double((int)hi, (int)(u << 29));
}

template <bool NORMAL, bool DIRECTIONAL>
__device__ __forceinline__ double pd_pair(const float4* __restrict__ q, const PdObsMx& o) {
  const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5];
  const float2 X = make_float2(q0.x, q0.y), Y = make_float2(q0.z, q0.w), Z = make_float2(q1.x, q1.y);
  const float2 MBX = make_float2(q2.x, q2.y), MBY = make_float2(q2.z, q2.w);
  const float2 EB = make_float2(q3.x, q3.y), BZ = make_float2(q3.z, q3.w);
  const float2 AZ = make_float2(q4.z, q4.w), AX = make_float2(q5.x, q5.y), AY = make_float2(q5.z, q5.w);
  const float2 M1 = f2(-1.f);
  const float2 rx = fma2(X, M1, o.ox), ry = fma2(Y, M1, o.oy), rz = fma2(Z, M1, o.oz);
  const float2 rho2 = fma2(rx, rx, mul2(ry, ry));
  const float2 d2 = fma2(rz, rz, rho2);
  const float2 iD = make_float2(rsqrt_ftz(d2.x), rsqrt_ftz(d2.y));
  const float2 arz = make_float2(fabsf(rz.x), fabsf(rz.y));
  const float2 den = fma2(d2, iD, arz);  // D + |R_z|
  const float2 ide = make_float2(rcp_ftz(den.x), rcp_ftz(den.y));
  const float2 en = mul2(fma2(rho2, ide, fma2(rz, M1, arz)), iD);  // 1 - n_z
  const float2 nx = mul2(rx, iD), ny = mul2(ry, iD), nz = fma2(en, M1, f2(1.f));
  const float2 om = fma2(ny, MBY, fma2(nx, MBX, fma2(en, BZ, EB)));  // 1 - n.b
  const float2 iom = make_float2(rcp_ftz(om.x), rcp_ftz(om.y));
  const float2 ux = add2(nx, MBX), uy = add2(ny, MBY), uz = fma2(en, M1, EB);  // n - b
  const float2 wx = fma2(uy, AZ, mul2(mul2(uz, AY), M1));
  const float2 wy = fma2(uz, AX, mul2(mul2(ux, AZ), M1));
  const float2 wz = fma2(ux, AY, mul2(mul2(uy, AX), M1));
  const float2 mx = fma2(ny, wz, mul2(mul2(nz, wy), M1));
  const float2 my = fma2(nz, wx, mul2(mul2(nx, wz), M1));
  const float2 mz = fma2(nx, wy, mul2(mul2(ny, wx), M1));
  float2 t = mul2(mul2(fma2(mx, mx, fma2(my, my, mul2(mz, mz))), iD), iD);
  if (NORMAL) {
    const float2 n1dn = fma2(nx, o.nx, fma2(ny, o.ny, mul2(nz, o.nz)));
    t = mul2(t, n1dn);
    if (DIRECTIONAL) t = make_float2(n1dn.x > 0.f ? t.x : 0.f, n1dn.y > 0.f ? t.y : 0.f);
  }
  const double q0d = nonneg_float_to_double(iom.x), q1d = nonneg_float_to_double(iom.y);
  const double q02 = q0d * q0d, q12 = q1d * q1d;
  return fma(float_to_double_bits(t.x), q02 * q02 * q0d, float_to_double_bits(t.y) * (q12 * q12 * q1d));
}

template <int SUB, int MINB, int CP>
__global__ void __launch_bounds__(kMxThreads, MINB) k_pd_wave_mixed(PdWaveArgs A, MixedFrame F) {
  constexpr int TE = kMxThreads / SUB;
  if (A.tile_entries != TE) {  // the host sized the partials for another tile
    if (threadIdx.x == 0) atomicOr(A.err, kErrPlan);
    return;
  }
  __shared__ __align__(16) PairStage<CP> st;
  __shared__ double red[SUB > 1 ? SUB - 1 : 1][TE];
  __shared__ WavePlan P;
  __shared__ int64_t next_unit;
  __shared__ int s_last;
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
    PdObsMx o;
    {
      const double* R = F.rot;
      const double ox = A.obs[3 * item] - F.x0[0], oy = A.obs[3 * item + 1] - F.x0[1], oz = A.obs[3 * item + 2] - F.x0[2];
      o.ox = f2((float)(R[0] * ox + R[1] * oy + R[2] * oz));
      o.oy = f2((float)(R[3] * ox + R[4] * oy + R[5] * oz));
      o.oz = f2((float)(R[6] * ox + R[7] * oy + R[8] * oz));
      double nx = 0, ny = 0, nz = 0;
      if (A.has_normal) { nx = A.normals[3 * item]; ny = A.normals[3 * item + 1]; nz = A.normals[3 * item + 2]; }
      o.nx = f2((float)(R[0] * nx + R[1] * ny + R[2] * nz));
      o.ny = f2((float)(R[3] * nx + R[4] * ny + R[5] * nz));
      o.nz = f2((float)(R[6] * nx + R[7] * ny + R[8] * nz));
    }
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      const int64_t p0 = b0 >> 1, p1 = b1 > b0 ? b1 >> 1 : p0;  // spans are whole pairs
      double S = 0;
      const int64_t nchunks = (p1 - p0 + CP - 1) / CP;
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
        if (live) {
          if (A.has_normal && A.directional)
            for (int j = j0; j < j1; ++j) S += pd_pair<true, true>(sv + kPairF4 * j, o);
          else if (A.has_normal)
            for (int j = j0; j < j1; ++j) S += pd_pair<true, false>(sv + kPairF4 * j, o);
          else
            for (int j = j0; j < j1; ++j) S += pd_pair<false, false>(sv + kPairF4 * j, o);
        }
        __syncthreads();  // everyone is done with `buf` before it is refilled
      }
      // reduce the groups' sums in group order; group 0 stores the span's partial (entry-major, or
      // tile-major for the fused finalize)
      if (SUB > 1 && grp > 0) red[grp - 1][q] = S;
      if (SUB > 1) __syncthreads();
      if (grp == 0) {
        for (int o2 = 0; o2 < SUB - 1; ++o2) S += red[o2][q];
        if (live) {
          if (A.fused) A.part[((tile * P.nseg + g) * P.spans + span) * TE + q] = S;
          else A.part[slot * P.nseg * P.spans + g * P.spans + span] = S;
        }
      }
      if (SUB > 1) __syncthreads();
    }
    if (A.fused) {  // the CTA that finishes a tile's last span finalizes the tile
      __threadfence();
      __syncthreads();
      if (tid == 0) {
        const unsigned done = atomicAdd(&A.tile_done[tile], 1u);
        s_last = done == (unsigned)(P.spans - 1);
        if (s_last) __threadfence();
      }
      __syncthreads();
      if (s_last) {
        pd_tile_finalize(A.fin, P, tile, n_act, TE);
        if (tid == 0) A.tile_done[tile] = 0;
      }
    }
  }
}

}  // namespace dev

cudaError_t launch_mixed_records(const double* knots, int64_t n, double tstart, double tstop, int64_t s_begin,
                                 int64_t s_end, int ext_from, const MixedFrame& F, float4* rec,
                                 unsigned long long* bd_bits, cudaStream_t st) {
  if (s_end <= s_begin) return cudaSuccess;
  const int T = 128;
  const int64_t warps = (s_end - s_begin + dev::kRecWarpSamples - 1) / dev::kRecWarpSamples;
  const unsigned grid = (unsigned)((warps * 32 + T - 1) / T);
  dev::k_mixed_records<<<grid, T, 0, st>>>(knots, n, tstart, tstop, s_begin, s_end, ext_from, F,
                                            reinterpret_cast<float*>(rec), bd_bits);
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

// The mixed power-density kernel: 4 groups of 32 entries, at least 4 CTAs per SM, 128 pair records
// per staged chunk.
constexpr int kPdMxSub = 4;
int pd_mixed_entries_per_cta() { return dev::kMxThreads / kPdMxSub; }
int pd_mixed_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_pd_wave_mixed<kPdMxSub, 4, 128>, dev::kMxThreads, 0);
  return n > 0 ? n : 1;
}
cudaError_t launch_pd_wave_mixed(const PdWaveArgs& a, const MixedFrame& F, int grid, cudaStream_t st) {
  dev::k_pd_wave_mixed<kPdMxSub, 4, 128><<<grid, dev::kMxThreads, 0, st>>>(a, F);
  return cudaGetLastError();
}

}  // namespace osc
