// kernels.h -- argument blocks and launch wrappers of the radiation kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace osc {

constexpr int kFdPartials = 9;  // 6 complex-sum components, first phase, last phase, max |dphase|

// One wave of the frequency-domain sum: every active entry integrates the samples
// [seg_b[g], seg_e[g]) of the level cache, split into gridDim.y spans of span_len[g] samples.
struct FdWaveArgs {
  const double* lev;        // level cache, 10 arrays of `cap` doubles
  int64_t cap;
  const double* obs;        // 3 * n_obs
  const double* omega;      // n_e
  int64_t n_e;
  int64_t n_items;          // n_obs * n_e (entry = obs_index * n_e + energy_index)
  const int* act;           // active entry ids (NULL: entries 0..n_items-1)
  const unsigned* n_act;    // device count of `act`
  int nseg;
  int64_t seg_b[2], seg_e[2], span_len[2];
  double* part;             // partials [(seg*spans + span) * kFdPartials + k][part_stride]
  int64_t part_stride;
  unsigned* err;
};

struct FdFinalArgs {
  const double* part;
  int64_t part_stride;
  int spans, nseg, first, level, max_level, quantity, project;
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
  int nseg;
  int64_t seg_b[2], seg_e[2], span_len[2];
  double* part;             // partials [(seg*spans + span)][part_stride]
  int64_t part_stride;
  unsigned* err;
};

struct PdFinalArgs {
  const double* part;
  int64_t part_stride;
  int spans, nseg, first, level, max_level, quantity, directional;
  double dt_prev, dt_level, precision, scale, weight, bdmax, two_over_gamma;
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
};

// Frame of the mixed-precision path: origin x0 (particle start), rows of rot = e1, e2, e3 with e3 the
// initial direction; xperp_max / z_max bound the trajectory in that frame; t_ref = t0 / c.
struct MixedFrame {
  double rot[9];
  double x0[3];
  double t_ref;
  double xperp_max, z_max;
};

cudaError_t launch_mixed_records(const double* lev, int64_t cap, int64_t s_begin, int64_t s_end, const MixedFrame& F,
                                 float4* rec, cudaStream_t st);
cudaError_t launch_fd_wave_mixed(const FdWaveArgs& a, const MixedFrame& F, int64_t n_act_bound, int spans, int ept,
                                 cudaStream_t st);
int mixed_entries_per_cta(int ept);

cudaError_t launch_level_fill(const double* knots, int64_t n, double tstart, double tstop, int64_t s_begin,
                              int64_t s_end, double* lev, int64_t cap, int extended_level,
                              unsigned long long* bdmax_bits, cudaStream_t st);
cudaError_t launch_fd_wave_fp64(const FdWaveArgs& a, int64_t n_act_bound, int spans, cudaStream_t st);
cudaError_t launch_fd_finalize(const FdFinalArgs& a, int64_t n_act_bound, cudaStream_t st);
cudaError_t launch_pd_wave_fp64(const PdWaveArgs& a, int64_t n_act_bound, int spans, cudaStream_t st);
cudaError_t launch_pd_finalize(const PdFinalArgs& a, int64_t n_act_bound, cudaStream_t st);

}  // namespace osc
