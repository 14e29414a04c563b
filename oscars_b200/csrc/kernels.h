// kernels.h -- argument blocks and launch wrappers of the radiation kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace osc {

constexpr int kFdPartials = 9;  // 6 complex-sum components, first phase, last phase, max |dphase|

// Work plan of one wave, computed identically by the host (buffer sizes), the wave kernel and the
// finalize kernel from the device-resident active count.  Level L's samples occupy [2^L, 2^(L+1));
// the first wave also integrates levels 0..L-1 = [1, 2^L) as a separate segment (its magnitude is
// the "last" value of the first stop test).  Segment starts are rounded down to an even index (the
// kernels skip sample 0); `spans` splits every segment so that tiles x spans reaches target_units.
struct WavePlan {
  int nseg;
  int spans;
  int64_t tiles;
  int64_t seg_b[2], seg_e[2], span_len[2];
};

// Segments of a wave with a given span count (tiles left to the caller).
__host__ __device__ inline WavePlan wave_plan_spans(int first, int L, int spans) {
  WavePlan p;
  const int64_t lo = (int64_t)1 << L, hi = (int64_t)2 << L;
  p.nseg = (first && L >= 1) ? 2 : 1;
  // segment 0: levels 0..L-1 on the first wave (level 0 alone when L == 0), else level L
  const int64_t b0 = first ? 1 : lo, e0 = first ? (L >= 1 ? lo : 2) : hi;
  const int64_t b1 = lo, e1 = hi;  // segment 1 (first wave with L >= 1): level L
  p.tiles = 0;
  p.spans = spans;
  const int64_t a0 = b0 & ~(int64_t)1, a1 = b1 & ~(int64_t)1;
  p.seg_b[0] = a0;
  p.seg_e[0] = e0;
  p.span_len[0] = ((e0 - a0 + spans - 1) / spans + 1) & ~(int64_t)1;
  p.seg_b[1] = p.nseg == 2 ? a1 : 0;
  p.seg_e[1] = p.nseg == 2 ? e1 : 0;
  p.span_len[1] = p.nseg == 2 ? (((e1 - a1 + spans - 1) / spans + 1) & ~(int64_t)1) : 0;
  return p;
}

// Smallest power-of-two span count with tiles x spans >= target_units, keeping spans of at least
// min_span samples of level L.
__host__ __device__ inline int wave_spans(int L, int64_t tiles, int64_t target_units, int min_span) {
  const int64_t lo = (int64_t)1 << L;
  int spans = 1;
  while (tiles * spans < target_units && lo / (spans * 2) >= min_span) spans *= 2;
  return spans;
}

__host__ __device__ inline WavePlan wave_plan(int first, int L, int64_t n_act, int tile_entries, int64_t target_units,
                                              int min_span) {
  const int64_t tiles = (n_act + tile_entries - 1) / tile_entries;
  WavePlan p = wave_plan_spans(first, L, wave_spans(L, tiles, target_units, min_span));
  p.tiles = tiles;
  return p;
}

// Register-friendly accessors (g is 0 or 1; selects instead of a runtime array index).
__host__ __device__ inline int64_t seg_begin(const WavePlan& p, int g) { return g ? p.seg_b[1] : p.seg_b[0]; }
__host__ __device__ inline int64_t seg_end(const WavePlan& p, int g) { return g ? p.seg_e[1] : p.seg_e[0]; }
__host__ __device__ inline int64_t seg_span(const WavePlan& p, int g) { return g ? p.span_len[1] : p.span_len[0]; }

struct FdFinalArgs {
  const double* part;
  int first, level, max_level, quantity, project, tile_entries, min_span;
  int64_t target_units;
  double dt_prev, dt_level;  // DeltaT inclusive to level-1 (first wave) and to level
  double precision, c0, c2, weight;
  double pol[6];            // polarization vector (re, im) x 3
  int64_t n_items;
  const int* act;
  const unsigned* n_act;
  double* state;            // 7 * n_items: complex sum (6) + last magnitude
  int* act_next;
  unsigned* n_next;
  double* out;
  int* level_out;
  unsigned long long* not_converged;
  unsigned long long* samples;
  unsigned long long* work_reset;  // the wave's unit counter, zeroed for the next wave
  int dmax_spans_joined;    // the span maxima include the step from the previous span's last sample
  unsigned* level_max;      // highest level at which an entry finished (may be NULL)
};

// One wave of the frequency-domain sum over level `level` for the active entries.
struct FdWaveArgs {
  const double* lev;        // FP64 level cache (10 arrays of `cap`) or mixed pair records
  int64_t cap;
  const double* obs;        // 3 * n_obs
  const double* omega;      // n_e
  int64_t n_e;
  int64_t n_items;          // n_obs * n_e (entry = obs_index * n_e + energy_index)
  const int* act;           // active entry ids (NULL: entries 0..n_items-1)
  const unsigned* n_act;    // device count of `act`
  int first, level, tile_entries, min_span;
  int64_t target_units;
  double* part;             // partials, entry-major: [slot][seg][span][kFdPartials]; fused: see below
  unsigned* err;
  unsigned long long* work;  // next unit to take (zero at launch; the finalize resets it)
  // Fused finalize: the last CTA to finish a tile's spans reduces them, applies the stop rule and
  // appends survivors (no finalize launch).  Partials are then tile-major,
  // [tile][seg][span][kFdPartials][entry in tile], so writes and the finalizer's reads coalesce.
  // zero_u32 / zero_u64 are the counters of the following wave, zeroed by block 0 at start.
  int fused;
  unsigned* tile_done;      // per tile: spans finished (the finalizer resets it to 0)
  unsigned* zero_u32;
  unsigned long long* zero_u64;
  FdFinalArgs fin;
};

struct PdFinalArgs {
  const double* part;
  int first, level, max_level, quantity, directional, tile_entries, min_span;
  int64_t target_units;
  double dt_prev, dt_level, precision, scale, weight, two_over_gamma;
  const double* bdmax_levels;  // device, per level max |beta_i - beta_{i-1}| (-1 for level 0)
  int64_t n_items;
  const int* act;
  const unsigned* n_act;
  double* state;            // 2 * n_items: running sum, last level value
  int* act_next;
  unsigned* n_next;
  double* out;
  int* level_out;
  unsigned long long* not_converged;
  unsigned long long* samples;
  unsigned long long* work_reset;
  unsigned* level_max;      // highest level at which an entry finished (may be NULL)
};

struct PdWaveArgs {
  const double* lev;
  int64_t cap;
  const double* obs;
  const double* normals;
  int has_normal, directional;
  int64_t n_items;
  const int* act;
  const unsigned* n_act;
  int first, level, tile_entries, min_span;
  int64_t target_units;
  double* part;             // partials, entry-major: [slot][seg][span]; fused: [tile][seg][span][entry in tile]
  unsigned* err;
  unsigned long long* work;
  // Fused finalize (the mixed kernel): the last CTA to finish a tile's spans applies the stop rule of
  // `fin` to the tile's entries and appends survivors; zero_u32 / zero_u64 are the counters of the
  // following wave, zeroed by block 0 at start.
  int fused;
  unsigned* tile_done;
  unsigned* zero_u32;
  unsigned long long* zero_u64;
  PdFinalArgs fin;
};

// One level of the STL power density (kernels_stl.cu): one CTA per facet not yet done.
struct StlLevelArgs {
  const double* lev;        // FP64 level cache (10 arrays of cap doubles)
  int64_t cap;
  const double* geometry;   // n x 9: vertex A, B - A, C - A of each facet
  const double* centers;    // n x 3: facet centres (the observation points)
  const double* normals;    // n x 3: stored facet normals
  int64_t n;
  int level;
  double dt_level, precision, two_over_gamma;
  double* state;            // n x 4: running sum, last level value, result precision, last level
  int* done;                // n: stopped
  int* level_out;           // n: level at which the facet stopped (-1 set by the host beforehand)
  unsigned* n_active;       // facets not stopped after this level (zeroed by the host per level)
};
cudaError_t launch_stl_level(const StlLevelArgs& a, cudaStream_t st);

// Frame of the mixed-precision path: origin x0 (particle start), rows of rot = e1, e2, e3 with e3 the
// initial direction; xperp_max / z_max bound the trajectory in that frame; t_ref = t0 / c;
// theta_max = the largest observer angle the path accepts (mixed_theta_max of the particle's gamma);
// tau_max bounds |tau_s| (the phase range check of mixed_geometry_ok).
struct MixedFrame {
  double rot[9];
  double x0[3];
  double t_ref;
  double xperp_max, z_max;
  double theta_max;
  double tau_max;  // largest |t - t_ref - z/c| over the trajectory knots
};

// Refusal of an observer outside the mixed path's validity region (mixed_geometry_ok).
constexpr const char* kMixedGeometryMessage =
    "compute='mixed' needs observers near the beam axis (angle below min(1e-2, 20/gamma), a correction "
    "phase below 3e4 rad and retarded phases below 2^20 turns); use compute='fp64' for this geometry";

// Largest observer angle from the frame axis the mixed path accepts for a particle of Lorentz
// factor gamma: min(1e-2, 20 / gamma) (see mixed_geometry_ok in fd_common.cuh).
__host__ __device__ inline double mixed_theta_max(double gamma) {
  const double t = 20.0 / gamma;
  return t < 1e-2 ? t : 1e-2;
}

// Mixed pair records (fd_common.cuh, 144 bytes per two samples) of level samples [s_begin, s_end),
// evaluated from the trajectory knots (t | y[9] | y''[9], n points); levels above ext_from are the
// reference's extended levels (their own time spacing, fd_common.cuh level_time).  bd_bits (32
// words, may be NULL): per level, the largest |beta_i - beta_{i-1}| is folded in (atomicMax on the
// bits of the positive double; the caller zeroes the words of the levels it fills).
cudaError_t launch_mixed_records(const double* knots, int64_t n, double tstart, double tstop, int64_t s_begin,
                                 int64_t s_end, int ext_from, const MixedFrame& F, float4* rec,
                                 unsigned long long* bd_bits, cudaStream_t st);
constexpr int kMixedRecordBytesPerSample = 72;
// Compiled kernel variants (see kernels_fp64.cu / kernels_mixed.cu); the engine's autotuner picks one.
constexpr int kFp64Variants = 4;
constexpr int kMixedVariants = 4;
cudaError_t launch_fd_wave_mixed(const FdWaveArgs& a, const MixedFrame& F, int grid, int variant, cudaStream_t st);
int mixed_entries_per_cta(int variant);
const char* mixed_variant_name(int variant);  // kernel and template arguments of a variant
int mixed_blocks_per_sm(int variant);
int fp64_blocks_per_sm(bool power_density, int variant);
int fp64_entries_per_cta(int variant);

// FP64 level samples [s_begin, s_end) (10 SoA arrays of stride cap) and their per-level beta-difference
// maxima; levels above ext_from are the reference's extended levels.
cudaError_t launch_level_fill(const double* knots, int64_t n, double tstart, double tstop, int64_t s_begin,
                              int64_t s_end, double* lev, int64_t cap, int ext_from,
                              unsigned long long* bdmax_bits, cudaStream_t st);
cudaError_t launch_fd_wave_fp64(const FdWaveArgs& a, int grid, int variant, cudaStream_t st);
cudaError_t launch_fd_finalize(const FdFinalArgs& a, int64_t n_act_bound, cudaStream_t st);
cudaError_t launch_pd_wave_fp64(const PdWaveArgs& a, int grid, cudaStream_t st);
// Mixed-precision power density over the pair records (kernels_mixed.cu): a.lev = the records,
// partials entry-major like the FP64 kernel's, tile_entries = pd_mixed_entries_per_cta().
cudaError_t launch_pd_wave_mixed(const PdWaveArgs& a, const MixedFrame& F, int grid, cudaStream_t st);
int pd_mixed_entries_per_cta();
int pd_mixed_blocks_per_sm();
cudaError_t launch_pd_finalize(const PdFinalArgs& a, int64_t n_act_bound, cudaStream_t st);

}  // namespace osc
