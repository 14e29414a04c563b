// batch.h -- device-side description of a batch of radiation jobs: many particles of one beam, or
// many unrelated undulator jobs with their own trajectory lengths, observers and energies, all
// integrated in the same kernel launches (mixed precision).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "kernels.h"

namespace osc {

// A field source on the device (FieldSpec after finish()).
struct DevField {
  int kind;                 // 0 undulator, 1 EPU, 2 grid
  int nperiods;
  double a[3], b[3], center[3], period_unit[3];
  double phase, taper, frequency, frequency_phase, time_offset;
  double period_length, period_mag, length;
  // per-field constants of the device evaluation: 2 pi / period length, 2 / period length, and the
  // pole-block shifts (undulator: shift[0]; EPU: A at shift[0], B at shift[1])
  double k_arg, inv_half_period, shift[2];
  // undulator half-period factors: n_half values at half_off of the batch's value array (0: none)
  int64_t half_off;
  int n_half;
  // grid: points, start / step / stop per axis, dimension code, values (3 per point) at grid_off,
  // sin and cos of the rotation angles (computed on the host, as the host model computes them)
  int grid_dim;
  int64_t grid_n[3];
  double grid_start[3], grid_step[3], grid_stop[3];
  int64_t grid_off;
  double rot_sin[3], rot_cos[3];
};

struct DevJob {
  MixedFrame frame;         // particle frame; xperp_max / z_max are written on the device
  double b0[3];             // initial velocity / c
  double qomg;              // q / (m gamma)
  double dt;                // RK4 step [s]
  double tstart, tstop;     // first and last knot time [s]
  double c0, c2;            // field and flux constants (src/OSCARSSR.cc:4106-4109)
  double pol[6];            // polarization vector in the job frame (re, im) x 3
  int nf, nb;               // RK4 points forward / backward of t0
  int field_begin, field_count;
  int64_t knots;            // offset of the job's knot block t | y[9] | ypp[9] (19 x n doubles)
  int64_t u_off;            // offset of the job's 9 x n spline work block
  int64_t obs_begin, omega_begin, n_obs, n_e;
  int64_t entry_begin;      // first entry of the job in its chunk (job-major; obs-major, energy fastest)
};

// Offsets of one wave, written by k_batch_plan: prefix sums over the jobs of the chunk.
struct BatchPlan {
  int64_t* unit_start;      // njobs + 1: first (tile, span) unit of each job
  int64_t* part_start;      // njobs + 1: first partial-sum double of each job
  int64_t* act_start;       // njobs + 1: first active entry of each job in the finalize order
  int* spans;               // spans per segment, common to the wave
};

struct BatchWaveArgs {
  const DevJob* jobs;
  int njobs;
  const float4* rec;        // pair records: job j from float4 5 * j * stride, sample s at local index s - s_off
  int64_t stride, s_off;
  const double* obs;
  const double* omega;
  const int* act;           // per-job active lists at entry_begin (unused on the first wave)
  const unsigned* cnt;      // per-job active counts (unused on the first wave)
  BatchPlan plan;
  int first, level;
  double* part;             // per job: [slot][seg][span][kFdPartials] from part_start[j]
  unsigned* err;
  unsigned long long* work;  // next unit to take (zero at launch; the finalize resets it)
};

struct BatchFinalArgs {
  const DevJob* jobs;
  int njobs;
  const int* act;
  const unsigned* cnt;
  BatchPlan plan;
  const double* part;
  int first, level, max_level, quantity, project;
  double precision;
  int64_t n_entries;        // entries of the chunk (state stride)
  double* state;            // 7 x n_entries: complex sum (6) + last magnitude, at entry_begin + item
  int* act_next;
  unsigned* cnt_next;
  double* out;              // value of every entry of the chunk (weight 1)
  int* level_out;
  unsigned long long* not_converged;
  unsigned long long* samples;
  unsigned long long* work_reset;
};

struct FieldSpec;
// Device form of a field; grid values and half-period factors are appended to `vals`.
DevField to_dev_field(FieldSpec f, std::vector<double>& vals);

// Compiled variants of the batched wave kernel (groups per CTA, minimum CTAs per SM).
constexpr int kBatchVariants = 4;

}  // namespace osc
