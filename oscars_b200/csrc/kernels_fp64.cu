// kernels_fp64.cu -- the reference's FP64 method on sm_100a.
//
// Level samples (trajectory spline evaluated at the level-ladder times), the frequency-domain
// (flux / spectrum) and time-domain (power density) sums over those samples, and the per-level
// convergence tests.  Every operation whose rounding can move the retarded phase or the
// 1 - n.beta denominators is written with explicit round-to-nearest intrinsics in the reference's
// association order, so those quantities are bit-identical to the reference CPU build; only the
// order of the final summation and the last-ulp behaviour of sin/cos/pow differ.
//
// Work decomposition ("waves"): every (observer, energy) entry that is still unconverged at level
// L needs the 2^L samples of that level.  A wave launches one CTA per (128 entries x span of the
// level); each thread owns one entry and walks the span's samples, which a single elected thread
// stages into shared memory with 1-D TMA bulk copies (double buffered, mbarrier completion).
// All threads read the same sample at the same time (shared-memory broadcast).  Per-span partial
// sums go to global memory and a finalize kernel reduces them in span order, applies the
// reference's stop rule and compacts the still-active entries for the next wave.
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "fd_common.cuh"
#include "kernels.h"

namespace osc {
namespace dev {

// ---------------------------------------------------------------------------------------------
// Level samples: TParticleTrajectoryInterpolated::FillTParticleTrajectoryPointsLevel
// (src/TParticleTrajectoryInterpolated.cc:124-158) + TSpline1D3::GetValue (include/TOMATH.h:92-121).
// Sample i of level L lives at index 2^L + i of each of the 10 SoA arrays (index 0 unused), so the
// union of levels 0..L is the contiguous range [1, 2^(L+1)) and every level starts 16-byte aligned.
// Levels above ext_from hold the reference's extended levels (same count 2^L, their own spacing:
// level_time), which it evaluates on the fly instead of storing.
// ---------------------------------------------------------------------------------------------
__global__ void k_level_fill(const double* __restrict__ knots, int64_t n, double tstart, double tstop,
                             int64_t s_begin, int64_t s_end, double* __restrict__ lev, int64_t cap, int ext_from) {
  const int64_t s = s_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= s_end) return;
  const double T = level_time(tstart, tstop, s, ext_from);
  double v[9];
  spline_eval9(knots, n, T, v);
  lev[s] = T;
#pragma unroll
  for (int c = 0; c < 9; ++c) lev[(1 + c) * cap + s] = v[c];
}

// Per-level max |beta_i - beta_{i-1}| over i >= 1 (the power-density stop rule, src/OSCARSSR.cc:
// 2887-2891).  Positive doubles order like their bit patterns, so atomicMax on the bits is exact.
__global__ void k_level_betadiff(const double* __restrict__ lev, int64_t cap, int64_t s_begin, int64_t s_end,
                                 unsigned long long* __restrict__ bdmax_bits) {
  __shared__ unsigned long long blk[32];  // per-level maxima of this block, merged into global at the end
  if (threadIdx.x < 32) blk[threadIdx.x] = 0;
  __syncthreads();
  const int64_t s = s_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < s_end) {
    const int L = 63 - __clzll((unsigned long long)s);
    const int64_t i = s - ((int64_t)1 << L);
    if (i > 0) {
      const double* bx = lev + 4 * cap;
      const double* by = lev + 5 * cap;
      const double* bz = lev + 6 * cap;
      const double dx = __dsub_rn(bx[s], bx[s - 1]), dy = __dsub_rn(by[s], by[s - 1]), dz = __dsub_rn(bz[s], bz[s - 1]);
      const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
      atomicMax(&blk[L & 31], (unsigned long long)__double_as_longlong(d));
    }
  }
  __syncthreads();
  if (threadIdx.x < 32 && blk[threadIdx.x]) atomicMax(&bdmax_bits[threadIdx.x], blk[threadIdx.x]);
}

// ---------------------------------------------------------------------------------------------
// Shared-memory staging of sample ranges.
// ---------------------------------------------------------------------------------------------
template <int NARR, int CH>
struct Stage {
  // CH + 2 slots so that a range whose start is rounded down to an even index still fits.
  double v[2][NARR][CH + 2];
  uint64_t bar[2];
};

// Issue the bulk copies of samples [lo_al, hi_al) of the NARR arrays into buffer `b`.
template <int NARR, int CH>
__device__ __forceinline__ void stage_issue(Stage<NARR, CH>& st, int b, const double* lev, int64_t cap,
                                            int64_t lo_al, int64_t hi_al) {
  const uint32_t bytes = (uint32_t)((hi_al - lo_al) * sizeof(double));
  mbar_arrive_expect_tx(&st.bar[b], bytes * NARR);
#pragma unroll
  for (int k = 0; k < NARR; ++k) tma_load_1d(&st.v[b][k][0], lev + k * cap + lo_al, bytes, &st.bar[b]);
}

// ---------------------------------------------------------------------------------------------
// Frequency-domain wave (flux / spectrum).  Integrand: src/OSCARSSR.cc:4202-4220 (flux) and
// :1976-1989 (spectrum), both
//   [ (1-b^2)(n-b) / (D^2 (1-n.b)^2) + n x ((n-b) x a/c) / (D (1-n.b)^2) ] exp(-i w (t + D/c)).
// ---------------------------------------------------------------------------------------------
constexpr int kFdThreads = 128;
constexpr int kFdChunk = 128;

// Phase -w (t + D/c) of one staged sample for an observer, with the operations of the sum below.
__device__ __forceinline__ double fd_phase(double T, double X, double Y, double Z, double Ox, double Oy, double Oz,
                                           double mw) {
  const double Rx = __dsub_rn(Ox, X), Ry = __dsub_rn(Oy, Y), Rz = __dsub_rn(Oz, Z);
  const double D = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(Rx, Rx), __dmul_rn(Ry, Ry)), __dmul_rn(Rz, Rz)));
  return __dmul_rn(mw, __dadd_rn(T, __ddiv_rn(D, kCLight)));
}

// Sample-split FP64 sum: the CTA's 128 threads form SUB groups of TE = 128 / SUB threads, one entry
// per thread; group g takes the g-th of SUB equal parts of every staged chunk of the 10 level arrays.
// Each part starts from the phase of the sample before it (the chunk's previous sample, the previous
// chunk's last one, or the span's predecessor read from the level cache), so the largest phase step
// of a span covers exactly the consecutive pairs of the serial order and spans need no joining
// (dmax_spans_joined); the groups' sums are combined in shared memory in group order.  Fused waves
// finalize their tiles with all threads (fused_unit_done_grouped); unfused waves store entry-major
// partials for k_fd_finalize.
template <int SUB, int MINB>
__global__ void __launch_bounds__(kFdThreads, MINB) k_fd_wave_fp64(FdWaveArgs A) {
  constexpr int TE = kFdThreads / SUB;
  if (A.tile_entries != TE) {  // the host sized the partials for another tile
    if (threadIdx.x == 0) atomicOr(A.err, kErrPlan);
    return;
  }
  __shared__ __align__(16) Stage<10, kFdChunk> st;
  __shared__ double red[SUB > 1 ? SUB - 1 : 1][7][TE];
  __shared__ int s_last;
  const int tid = threadIdx.x;
  const int grp = tid / TE, q = tid % TE;
  if (A.fused && blockIdx.x == 0 && tid == 0) {  // counters of the following wave
    if (A.zero_u32) *A.zero_u32 = 0;
    if (A.zero_u64) *A.zero_u64 = 0;
  }
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  // the plan is uniform over the CTA; keeping it in shared memory frees the registers its
  // fields would otherwise hold across the sample loop
  __shared__ WavePlan P;
  if (threadIdx.x == 0) P = wave_plan(A.first, A.level, n_act, TE, A.target_units, A.min_span);
  __syncthreads();
  const int64_t units = P.tiles * P.spans;
  if (tid == 0) {
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  uint32_t phase_bits = 0;  // parity of the next completion expected on each buffer
  __shared__ int64_t next_unit;
  for (;;) {  // CTAs take (tile, span) units from a shared counter until the wave's units run out
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
    const double Ox = A.obs[3 * io], Oy = A.obs[3 * io + 1], Oz = A.obs[3 * io + 2];
    const double mw = -A.omega[ie];
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      double sxr = 0, sxi = 0, syr = 0, syi = 0, szr = 0, szi = 0;
      double dmax = 0;
      bool any = false;
      const int64_t nchunks = b1 > b0 ? (b1 - b0 + kFdChunk - 1) / kFdChunk : 0;
      // phase of the sample before a part that starts a chunk: the span's predecessor (span > 0;
      // sample 0, the unused slot, never is one), then the previous chunk's last sample
      double carry = 0;
      bool have_carry = false;
      if (live && span > 0 && nchunks > 0 && b0 - 1 >= 1) {
        const int64_t s = b0 - 1;
        const double* L = A.lev;
        carry = fd_phase(L[s], L[A.cap + s], L[2 * A.cap + s], L[3 * A.cap + s], Ox, Oy, Oz, mw);
        have_carry = true;
      }
      if (tid == 0 && nchunks > 0) {
        const int64_t lo = b0, hi = min(b1, b0 + kFdChunk);
        stage_issue<10, kFdChunk>(st, 0, A.lev, A.cap, lo & ~(int64_t)1, (hi + 1) & ~(int64_t)1);
      }
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = b0 + c * kFdChunk, hi = min(b1, lo + kFdChunk);
        if (tid == 0 && c + 1 < nchunks) {  // prefetch the next chunk into the other buffer
          const int64_t lo2 = lo + kFdChunk, hi2 = min(b1, lo2 + kFdChunk);
          stage_issue<10, kFdChunk>(st, buf ^ 1, A.lev, A.cap, lo2 & ~(int64_t)1, (hi2 + 1) & ~(int64_t)1);
        }
        if (!mbar_wait(&st.bar[buf], (phase_bits >> buf) & 1u)) {
          if (tid == 0) atomicOr(A.err, kErrTmaTimeout);
          return;
        }
        phase_bits ^= 1u << buf;
        const int64_t lo_al = lo & ~(int64_t)1;
        const double* sT = st.v[buf][0];
        const double* sX = st.v[buf][1];
        const double* sY = st.v[buf][2];
        const double* sZ = st.v[buf][3];
        const double* sBx = st.v[buf][4];
        const double* sBy = st.v[buf][5];
        const double* sBz = st.v[buf][6];
        const double* sAx = st.v[buf][7];
        const double* sAy = st.v[buf][8];
        const double* sAz = st.v[buf][9];
        const int ja = (int)(max(lo, (int64_t)1) - lo_al);  // sample 0 is the unused slot
        const int jb = (int)(hi - lo_al);
        const int j0 = ja + ((jb - ja) * grp) / SUB, j1 = ja + ((jb - ja) * (grp + 1)) / SUB;  // this group's part
        if (live && j0 < j1) {
          double last;
          bool have;
          if (j0 > ja) {
            last = fd_phase(sT[j0 - 1], sX[j0 - 1], sY[j0 - 1], sZ[j0 - 1], Ox, Oy, Oz, mw);
            have = true;
          } else {
            last = carry;
            have = have_carry;
          }
          for (int j = j0; j < j1; ++j) {
            const double T = sT[j];
            const double Rx = __dsub_rn(Ox, sX[j]), Ry = __dsub_rn(Oy, sY[j]), Rz = __dsub_rn(Oz, sZ[j]);
            const double D = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(Rx, Rx), __dmul_rn(Ry, Ry)), __dmul_rn(Rz, Rz)));
            const double ph = __dmul_rn(mw, __dadd_rn(T, __ddiv_rn(D, kCLight)));
            if (have) {
              const double dp = fabs(__dsub_rn(ph, last));
              dmax = dp > dmax ? dp : dmax;
            }
            have = true;
            last = ph;
            const double bx = sBx[j], by = sBy[j], bz = sBz[j];
            const double nx = __ddiv_rn(Rx, D), ny = __ddiv_rn(Ry, D), nz = __ddiv_rn(Rz, D);
            const double b2 = __dadd_rn(__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)), __dmul_rn(bz, bz));
            const double ndb = __dadd_rn(__dadd_rn(__dmul_rn(nx, bx), __dmul_rn(ny, by)), __dmul_rn(nz, bz));
            const double om = __dsub_rn(1.0, ndb);
            const double p2 = __dmul_rn(om, om);
            const double den1 = __dmul_rn(__dmul_rn(D, D), p2);
            const double den2 = __dmul_rn(D, p2);
            const double ob2 = __dsub_rn(1.0, b2);
            const double ux = __dsub_rn(nx, bx), uy = __dsub_rn(ny, by), uz = __dsub_rn(nz, bz);
            const double ax = sAx[j], ay = sAy[j], az = sAz[j];
            const double wx = __dsub_rn(__dmul_rn(uy, az), __dmul_rn(ay, uz));
            const double wy = __dsub_rn(__dmul_rn(uz, ax), __dmul_rn(az, ux));
            const double wz = __dsub_rn(__dmul_rn(ux, ay), __dmul_rn(ax, uy));
            const double vx = __dsub_rn(__dmul_rn(ny, wz), __dmul_rn(wy, nz));
            const double vy = __dsub_rn(__dmul_rn(nz, wx), __dmul_rn(wz, nx));
            const double vz = __dsub_rn(__dmul_rn(nx, wy), __dmul_rn(wx, ny));
            // The two amplitude terms need only relative accuracy: one quotient per term, then
            // multiplications (the reference divides each component; the difference is ~1 ulp).
            const double f1 = ob2 / den1, f2 = 1.0 / den2;
            const double ex = fma(ux, f1, vx * f2);
            const double ey = fma(uy, f1, vy * f2);
            const double ez = fma(uz, f1, vz * f2);
            double sn, cs;
            sincos(reduce_2pi(ph), &sn, &cs);
            sxr = fma(ex, cs, sxr); sxi = fma(ex, sn, sxi);
            syr = fma(ey, cs, syr); syi = fma(ey, sn, syi);
            szr = fma(ez, cs, szr); szi = fma(ez, sn, szi);
          }
          any = true;
        }
        if (live && c + 1 < nchunks) {  // a full chunk: its last sample precedes the next chunk
          const int jl = jb - 1;
          carry = fd_phase(sT[jl], sX[jl], sY[jl], sZ[jl], Ox, Oy, Oz, mw);
          have_carry = true;
        }
        __syncthreads();  // everyone is done with `buf` before it is refilled
      }
      // combine the groups' sums in group order; group 0 stores the span's partial
      double S[6] = {sxr, sxi, syr, syi, szr, szi};
      double dm = any ? dmax : -1.0;
      if (SUB > 1) {
        if (grp > 0) {
#pragma unroll
          for (int k = 0; k < 6; ++k) red[grp - 1][k][q] = S[k];
          red[grp - 1][6][q] = dm;
        }
        __syncthreads();
        if (grp == 0)
          for (int o = 0; o < SUB - 1; ++o) {
#pragma unroll
            for (int k = 0; k < 6; ++k) S[k] += red[o][k][q];
            dm = fmax(dm, red[o][6][q]);
          }
        __syncthreads();
      }
      if (live && grp == 0) {
        // entry-major for the finalize kernel (an entry's spans contiguous); tile-major when fused
        double* p = A.fused ? A.part + fused_part_index(P, tile, g, span, 0, q, TE)
                            : A.part + (slot * P.nseg * P.spans + g * P.spans + span) * kFdPartials;
        const int64_t cs = A.fused ? TE : 1;  // stride between components
#pragma unroll
        for (int k = 0; k < 6; ++k) p[k * cs] = S[k];
        p[6 * cs] = 0.0;
        p[7 * cs] = 0.0;
        p[8 * cs] = dm;  // -1 marks an empty span
      }
    }
    if (A.fused) fused_unit_done_grouped<kFdThreads>(A, P, tile, n_act, &s_last, TE, &red[0][0][0]);
  }
}

// Reduce the span partials of the wave, apply the stop rule of src/OSCARSSR.cc:4222-4238, finish
// converged / last-level entries (:4246-4267) and append the others to the next active list
// (span partials reduced by kFinLanes-lane groups, fd_common.cuh).

__global__ void k_fd_finalize(FdFinalArgs A) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.work_reset) *A.work_reset = 0;
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  const int lane = threadIdx.x % kFinLanes;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kFinLanes;
  if ((int64_t)blockIdx.x * blockDim.x / kFinLanes >= n_act) return;  // whole block idle
  const bool live = slot < n_act;
  const WavePlan P = wave_plan(A.first, A.level, n_act, A.tile_entries, A.target_units, A.min_span);
  const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
  // sums and max phase step of segment g over this lane's spans, then over the group
  auto seg_sum = [&](int g, C3& s, double& dmax) {
    C3 t = {0, 0, 0, 0, 0, 0};
    double dm = 0;
    if (live) {
      const double* base = A.part + (slot * P.nseg * P.spans + g * P.spans) * kFdPartials;
      for (int sp = lane; sp < P.spans; sp += kFinLanes) {
        const double* p = base + sp * kFdPartials;
        t.xr += p[0]; t.xi += p[1]; t.yr += p[2]; t.yi += p[3]; t.zr += p[4]; t.zi += p[5];
        if (p[8] >= 0) {  // non-empty span (empty spans only trail the segment)
          dm = fmax(dm, p[8]);
          if (sp > 0) dm = fmax(dm, fabs(__dsub_rn(p[6], p[-kFdPartials + 7])));
        }
      }
    }
    s.xr += group_sum(t.xr); s.xi += group_sum(t.xi); s.yr += group_sum(t.yr);
    s.yi += group_sum(t.yi); s.zr += group_sum(t.zr); s.zi += group_sum(t.zi);
    dmax = fmax(dmax, group_max(dm));
  };
  const int64_t N = A.n_items;
  C3 S = {0, 0, 0, 0, 0, 0};
  double last_mag = -1;
  double dmax = 0;
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
    if (live) {
      S = {A.state[item], A.state[N + item], A.state[2 * N + item], A.state[3 * N + item], A.state[4 * N + item],
           A.state[5 * N + item]};
      last_mag = A.state[6 * N + item];
    }
    seg_sum(0, S, dmax);
  }
  bool finished = false, unconverged = false, survive = false;
  if (live && lane == 0) fd_entry_decide(A, item, S, last_mag, dmax, finished, unconverged, survive);
  finalize_bookkeeping(finished, unconverged, survive, item, A.level, A.act_next, A.n_next, A.not_converged, A.samples,
                       A.level_max);
}

// ---------------------------------------------------------------------------------------------
// Power density (src/OSCARSSR.cc:2869-2922):
//   sum += [(N1 x ((N1 - b) x a/c)) . Nk]^2 / (1 - b.N1)^5 / |O - X|^2 * (N1 . normal),  k = 2, 3
// N1 and 1 - b.N1 keep the reference's operations (the difference is ill-conditioned, so its value
// depends on them); the well-conditioned rest is summed as |N1 x W|^2 / ((1 - b.N1)^5 |O - X|^2),
// equal to the two projections to rounding.
// ---------------------------------------------------------------------------------------------
constexpr int kPdThreads = 128;
constexpr int kPdChunk = 128;

__device__ __forceinline__ void unit3(double x, double y, double z, double& ux, double& uy, double& uz) {
  const double m = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
  ux = __ddiv_rn(x, m); uy = __ddiv_rn(y, m); uz = __ddiv_rn(z, m);
}

__global__ void __launch_bounds__(kPdThreads) k_pd_wave_fp64(PdWaveArgs A) {
  __shared__ __align__(16) Stage<10, kPdChunk> st;
  const int tid = threadIdx.x;
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  // the plan is uniform over the CTA; keeping it in shared memory frees the registers its
  // fields would otherwise hold across the sample loop
  __shared__ WavePlan P;
  if (threadIdx.x == 0) P = wave_plan(A.first, A.level, n_act, kPdThreads, A.target_units, A.min_span);
  __syncthreads();
  const int64_t units = P.tiles * P.spans;
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
    const int64_t slot = tile * kPdThreads + tid;
    const bool live = slot < n_act;
    const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
    const double Ox = A.obs[3 * item], Oy = A.obs[3 * item + 1], Oz = A.obs[3 * item + 2];
    double Nx = 0, Ny = 0, Nz = 0;
    if (A.has_normal) { Nx = A.normals[3 * item]; Ny = A.normals[3 * item + 1]; Nz = A.normals[3 * item + 2]; }
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      double sum = 0;
      const int64_t nchunks = b1 > b0 ? (b1 - b0 + kPdChunk - 1) / kPdChunk : 0;
      if (tid == 0 && nchunks > 0) {
        const int64_t lo = b0, hi = min(b1, b0 + kPdChunk);
        stage_issue<10, kPdChunk>(st, 0, A.lev, A.cap, lo & ~(int64_t)1, (hi + 1) & ~(int64_t)1);
      }
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = b0 + c * kPdChunk, hi = min(b1, lo + kPdChunk);
        if (tid == 0 && c + 1 < nchunks) {
          const int64_t lo2 = lo + kPdChunk, hi2 = min(b1, lo2 + kPdChunk);
          stage_issue<10, kPdChunk>(st, buf ^ 1, A.lev, A.cap, lo2 & ~(int64_t)1, (hi2 + 1) & ~(int64_t)1);
        }
        if (!mbar_wait(&st.bar[buf], (phase_bits >> buf) & 1u)) {
          if (tid == 0) atomicOr(A.err, kErrTmaTimeout);
          return;
        }
        phase_bits ^= 1u << buf;
        const int64_t lo_al = lo & ~(int64_t)1;
        const int j0 = (int)(max(lo, (int64_t)1) - lo_al), j1 = (int)(hi - lo_al);
        if (live) {
          for (int j = j0; j < j1; ++j) {
            const double Rx = __dsub_rn(Ox, st.v[buf][1][j]), Ry = __dsub_rn(Oy, st.v[buf][2][j]), Rz = __dsub_rn(Oz, st.v[buf][3][j]);
            // N1 and 1 - B.N1 with the reference's operations: the difference 1 - B.N1 (~1e-8) carries
            // the rounding of B.N1, which its result shares
            double n1x, n1y, n1z;
            unit3(Rx, Ry, Rz, n1x, n1y, n1z);
            const double n1dn = A.has_normal
                                    ? __dadd_rn(__dadd_rn(__dmul_rn(n1x, Nx), __dmul_rn(n1y, Ny)), __dmul_rn(n1z, Nz))
                                    : 1.0;
            if (A.directional && n1dn <= 0) continue;
            const double bx = st.v[buf][4][j], by = st.v[buf][5][j], bz = st.v[buf][6][j];
            const double ax = st.v[buf][7][j], ay = st.v[buf][8][j], az = st.v[buf][9][j];
            const double ux = __dsub_rn(n1x, bx), uy = __dsub_rn(n1y, by), uz = __dsub_rn(n1z, bz);
            const double wx = __dsub_rn(__dmul_rn(uy, az), __dmul_rn(ay, uz));
            const double wy = __dsub_rn(__dmul_rn(uz, ax), __dmul_rn(az, ux));
            const double wz = __dsub_rn(__dmul_rn(ux, ay), __dmul_rn(ax, uy));
            const double mx = __dsub_rn(__dmul_rn(n1y, wz), __dmul_rn(wy, n1z));
            const double my = __dsub_rn(__dmul_rn(n1z, wx), __dmul_rn(wz, n1x));
            const double mz = __dsub_rn(__dmul_rn(n1x, wy), __dmul_rn(wx, n1y));
            const double bdn = __dadd_rn(__dadd_rn(__dmul_rn(bx, n1x), __dmul_rn(by, n1y)), __dmul_rn(bz, n1z));
            // the rest is well conditioned: the squared projections on N2 and N3 (an orthonormal pair
            // across N1) sum to |N1 x W|^2, which is across N1; (1 - B.N1)^5 by products; one division
            const double om = __dsub_rn(1.0, bdn), om2 = om * om;
            const double m2 = __dadd_rn(__dadd_rn(__dmul_rn(Rx, Rx), __dmul_rn(Ry, Ry)), __dmul_rn(Rz, Rz));
            const double num = fma(mx, mx, fma(my, my, mz * mz));
            sum = fma(num / (om2 * om2 * om * m2), n1dn, sum);
          }
        }
        __syncthreads();
      }
      if (live) A.part[slot * P.nseg * P.spans + g * P.spans + span] = sum;
    }
  }
}

// src/OSCARSSR.cc:2924-2968
__global__ void k_pd_finalize(PdFinalArgs A) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.work_reset) *A.work_reset = 0;
  const int64_t n_act = A.act ? (int64_t)*A.n_act : A.n_items;
  const int lane = threadIdx.x % kFinLanes;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kFinLanes;
  if ((int64_t)blockIdx.x * blockDim.x / kFinLanes >= n_act) return;
  const bool live = slot < n_act;
  const WavePlan P = wave_plan(A.first, A.level, n_act, A.tile_entries, A.target_units, A.min_span);
  const int64_t item = live ? (A.act ? (int64_t)A.act[slot] : slot) : 0;
  const int64_t N = A.n_items;
  auto seg_sum = [&](int g) {
    double t = 0;
    if (live)
      for (int sp = lane; sp < P.spans; sp += kFinLanes) t += A.part[slot * P.nseg * P.spans + g * P.spans + sp];
    return group_sum(t);
  };
  double sum = 0, last_sum = -1;
  if (A.first) {
    if (P.nseg == 2) {
      sum += seg_sum(0);
      last_sum = sum * A.dt_prev;
    }
    sum += seg_sum(P.nseg - 1);
  } else {
    if (live) {
      sum = A.state[item];
      last_sum = A.state[N + item];
    }
    sum += seg_sum(0);
  }
  bool finished = false, unconverged = false, survive = false;
  if (live && lane == 0) pd_entry_decide(A, item, sum, last_sum, finished, unconverged, survive);
  finalize_bookkeeping(finished, unconverged, survive, item, A.level, A.act_next, A.n_next, A.not_converged, A.samples,
                       A.level_max);
}

}  // namespace dev

// ---- launch wrappers ------------------------------------------------------------------------
cudaError_t launch_level_fill(const double* knots, int64_t n, double tstart, double tstop, int64_t s_begin,
                              int64_t s_end, double* lev, int64_t cap, int ext_from,
                              unsigned long long* bdmax_bits, cudaStream_t st) {
  if (s_end <= s_begin) return cudaSuccess;
  const int T = 256;
  const int64_t nblk = (s_end - s_begin + T - 1) / T;
  dev::k_level_fill<<<(unsigned)nblk, T, 0, st>>>(knots, n, tstart, tstop, s_begin, s_end, lev, cap, ext_from);
  dev::k_level_betadiff<<<(unsigned)nblk, T, 0, st>>>(lev, cap, s_begin, s_end, bdmax_bits);
  return cudaGetLastError();
}

// Compiled variants of the FP64 wave kernel: (groups SUB of 128 / SUB entries, minimum CTAs per SM).
// Variant 0 keeps 128 entries per CTA (the allocation-free entry point sizes its partials for it).
static const int kFp64Sub[kFp64Variants] = {1, 2, 4, 4};

int fp64_entries_per_cta(int variant) { return dev::kFdThreads / kFp64Sub[variant]; }

cudaError_t launch_fd_wave_fp64(const FdWaveArgs& a, int grid, int variant, cudaStream_t st) {
  switch (variant) {
    case 1: dev::k_fd_wave_fp64<2, 7><<<grid, dev::kFdThreads, 0, st>>>(a); break;
    case 2: dev::k_fd_wave_fp64<4, 7><<<grid, dev::kFdThreads, 0, st>>>(a); break;
    case 3: dev::k_fd_wave_fp64<4, 5><<<grid, dev::kFdThreads, 0, st>>>(a); break;
    default: dev::k_fd_wave_fp64<1, 7><<<grid, dev::kFdThreads, 0, st>>>(a); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_fd_finalize(const FdFinalArgs& a, int64_t n_act_bound, cudaStream_t st) {
  if (n_act_bound == 0) return cudaSuccess;
  const int T = 256;
  const int64_t threads = n_act_bound * dev::kFinLanes;
  dev::k_fd_finalize<<<(unsigned)((threads + T - 1) / T), T, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_pd_wave_fp64(const PdWaveArgs& a, int grid, cudaStream_t st) {
  dev::k_pd_wave_fp64<<<grid, dev::kPdThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_pd_finalize(const PdFinalArgs& a, int64_t n_act_bound, cudaStream_t st) {
  if (n_act_bound == 0) return cudaSuccess;
  const int T = 256;
  const int64_t threads = n_act_bound * dev::kFinLanes;
  dev::k_pd_finalize<<<(unsigned)((threads + T - 1) / T), T, 0, st>>>(a);
  return cudaGetLastError();
}

int fp64_blocks_per_sm(bool power_density, int variant) {
  int n = 0;
  if (power_density) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_pd_wave_fp64, dev::kPdThreads, 0);
  } else {
    switch (variant) {
      case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_fp64<2, 7>, dev::kFdThreads, 0); break;
      case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_fp64<4, 7>, dev::kFdThreads, 0); break;
      case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_fp64<4, 5>, dev::kFdThreads, 0); break;
      default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_fd_wave_fp64<1, 7>, dev::kFdThreads, 0); break;
    }
  }
  return n > 0 ? n : 1;
}

}  // namespace osc
