// batch.cu -- many radiation jobs integrated in the same launches (mixed precision).
//
// A job is one particle through its own field set and trajectory range, observed on its own
// observer list at its own energies.  A multi-particle beam is a batch of jobs that share fields,
// observers and energies and whose results are averaged (src/OSCARSSR.cc:4026-4062); a set of
// uneven undulator jobs is a batch of unrelated jobs.  Per chunk of jobs every stage runs once over
// all of them:
//   k_batch_rk4       FP64 RK4, one thread per (job, direction)           src/OSCARSSR.cc:910-1009
//   k_batch_extent    trajectory extent in the job frame (validity bound of the mixed phase form)
//   k_batch_spline    clamped cubic spline, one thread per (job, component) include/TOMATH.h:141-203
//   k_batch_fill      level samples written straight as mixed pair records, one thread per sample
//   k_batch_plan      per-job tiles, units, partial offsets and active offsets of a wave (one block)
//   k_batch_wave      the mixed sample sum; persistent CTAs take (job, tile, span) units from a counter
//   k_batch_finalize  span reduction and the stop rule of src/OSCARSSR.cc:4222-4238 per entry
//   k_batch_average   compensated mean over the jobs of a beam, in particle order
// The launches of a chunk up to the prefilled level are captured once into a CUDA graph and
// replayed; only waves beyond that level need the host (to size the next level's records).
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

// ---------------------------------------------------------------------------------------------
// Fields and RK4 on the device.  The host model's field formulas (TField3D_IdealUndulator /
// TField3D_IdealEPU and TParticleA::RK4) with the per-field divisions replaced by constants
// computed once on the host (DevField::k_arg, inv_half_period, shift) and CUDA's sin and cos, so a
// trajectory agrees with the host's to rounding, not bit for bit -- this path is the mixed-precision
// one.  The integrator is a serial FP64 dependency chain per (job, direction), so what bounds it is
// the latency of each step's operations, not throughput.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void pole_block_d(const DevField& f, const double* __restrict__ vals, const double* amp,
                                             double d, double shift, double tc, double* F) {
  const double L = f.length, lam = f.period_length;
  if (d > L / 2. + shift || d < -L / 2. + shift) return;
  const double s = sin(f.k_arg * (d - shift));
  if (d < -L / 2. + shift + lam || d > L / 2. + shift - lam) {  // 1/4 and 3/4 end poles
    const double k = (d < -L / 2. + shift + lam / 2. || d > L / 2. + shift - lam / 2.) ? 0.25 : 0.75;
    F[0] += amp[0] * k * s * tc;
    F[1] += amp[1] * k * s * tc;
    F[2] += amp[2] * k * s * tc;
    return;
  }
  double h = 1.0;
  if (f.n_half > 0) {  // half-period k of the full-strength region
    int64_t k = (int64_t)((d - (-L / 2. + shift + lam)) * f.inv_half_period);
    k = k < 0 ? 0 : (k >= f.n_half ? f.n_half - 1 : k);
    h = vals[f.half_off + k];
  }
  F[0] += amp[0] * s * tc * h;
  F[1] += amp[1] * s * tc * h;
  F[2] += amp[2] * s * tc * h;
}

// Grid field (src/TField3D_Grid.cc:153-283), the host model's operations.
__device__ void grid_field_d(const DevField& f, const double* __restrict__ vals, double x, double y, double z,
                             double t, double* B) {
  // TVector3D::RotateSelfXYZ with the host's sin / cos of the angles, then the translation
  double vx = x, vy = y, vz = z, tt;
  tt = vy; vy = f.rot_cos[0] * tt - f.rot_sin[0] * vz; vz = f.rot_sin[0] * tt + f.rot_cos[0] * vz;
  tt = vz; vz = f.rot_cos[1] * tt - f.rot_sin[1] * vx; vx = f.rot_sin[1] * tt + f.rot_cos[1] * vx;
  tt = vx; vx = f.rot_cos[2] * tt - f.rot_sin[2] * vy; vy = f.rot_sin[2] * tt + f.rot_cos[2] * vy;
  const double p[3] = {vx - f.center[0], vy - f.center[1], vz - f.center[2]};
  int64_t ni[3] = {0, 0, 0};
  double di[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) {
    if (f.grid_n[a] > 1) {
      if (p[a] <= f.grid_start[a] || p[a] >= f.grid_stop[a]) return;
      ni[a] = (int64_t)((p[a] - f.grid_start[a]) / f.grid_step[a]);
      di[a] = (p[a] - f.grid_start[a]) - ni[a] * f.grid_step[a];
      if (ni[a] > f.grid_n[a] - 2) ni[a] = f.grid_n[a] - 2;
    }
  }
  const double* V = vals + f.grid_off;
  const int64_t NY = f.grid_n[1], NZ = f.grid_n[2];
  auto lerp = [&](const double* a0, const double* a1, double d, double step, double* o) {
    for (int c = 0; c < 3; ++c) o[c] = a0[c] + (a1[c] - a0[c]) * d / step;
  };
  auto at = [&](int64_t ix, int64_t iy, int64_t iz) { return V + 3 * (ix * NY * NZ + iy * NZ + iz); };
  const int64_t nx = ni[0], ny = ni[1], nz = ni[2];
  double F[3];
  switch (f.grid_dim) {
    case kGridXYZ: {
      double v00[3], v10[3], v01[3], v11[3], v0[3], v1[3];
      lerp(at(nx, ny, nz), at(nx + 1, ny, nz), di[0], f.grid_step[0], v00);
      lerp(at(nx, ny + 1, nz), at(nx + 1, ny + 1, nz), di[0], f.grid_step[0], v10);
      lerp(at(nx, ny, nz + 1), at(nx + 1, ny, nz + 1), di[0], f.grid_step[0], v01);
      lerp(at(nx, ny + 1, nz + 1), at(nx + 1, ny + 1, nz + 1), di[0], f.grid_step[0], v11);
      lerp(v00, v10, di[1], f.grid_step[1], v0);
      lerp(v01, v11, di[1], f.grid_step[1], v1);
      lerp(v0, v1, di[2], f.grid_step[2], F);
      break;
    }
    case kGridX: lerp(V + 3 * nx, V + 3 * (nx + 1), di[0], f.grid_step[0], F); break;
    case kGridY: lerp(V + 3 * ny, V + 3 * (ny + 1), di[1], f.grid_step[1], F); break;
    case kGridZ: lerp(V + 3 * nz, V + 3 * (nz + 1), di[2], f.grid_step[2], F); break;
    case kGridXY: {
      double v0[3], v1[3];
      lerp(at(nx, ny, 0), at(nx + 1, ny, 0), di[0], f.grid_step[0], v0);
      lerp(at(nx, ny + 1, 0), at(nx + 1, ny + 1, 0), di[0], f.grid_step[0], v1);
      lerp(v0, v1, di[1], f.grid_step[1], F);
      break;
    }
    case kGridXZ: {
      double v0[3], v1[3];
      lerp(at(nx, 0, nz), at(nx + 1, 0, nz), di[0], f.grid_step[0], v0);
      lerp(at(nx, 0, nz + 1), at(nx + 1, 0, nz + 1), di[0], f.grid_step[0], v1);
      lerp(v0, v1, di[2], f.grid_step[2], F);
      break;
    }
    default: {
      double v0[3], v1[3];
      lerp(at(0, ny, nz), at(0, ny + 1, nz), di[1], f.grid_step[1], v0);
      lerp(at(0, ny, nz + 1), at(0, ny + 1, nz + 1), di[1], f.grid_step[1], v1);
      lerp(v0, v1, di[2], f.grid_step[2], F);
      break;
    }
  }
  const double w = cos(2.0 * kPiD * f.frequency * (t + f.time_offset) + f.frequency_phase);
  B[0] += F[0] * w;
  B[1] += F[1] * w;
  B[2] += F[2] * w;
}

__device__ void field_sum_d(const DevField* __restrict__ fs, int nf, const double* __restrict__ vals, double x,
                            double y, double z, double t, double* B) {
  B[0] = B[1] = B[2] = 0;
  for (int i = 0; i < nf; ++i) {
    const DevField& f = fs[i];
    if (f.kind == 2) {
      grid_field_d(f, vals, x, y, z, t, B);
      continue;
    }
    const double d = (x - f.center[0]) * f.period_unit[0] + (y - f.center[1]) * f.period_unit[1] +
                     (z - f.center[2]) * f.period_unit[2];
    const double tc = 1 + d * f.taper;
    double F[3] = {0, 0, 0};
    pole_block_d(f, vals, f.a, d, f.shift[0], tc, F);
    if (f.kind == 1) pole_block_d(f, vals, f.b, d, f.shift[1], tc, F);  // EPU (src/TField3D_IdealEPU.cc:127-165)
    const double w = f.frequency == 0 ? 1.0 : cos(2.0 * kPiD * f.frequency * (t + f.time_offset) + f.frequency_phase);
    B[0] += F[0] * w;
    B[1] += F[1] * w;
    B[2] += F[2] * w;
  }
}

struct Rk4Ctx {
  const DevField* fs;
  int nf;
  const double* vals;
  double qomg;
  bool superluminal;
};

__device__ __forceinline__ void derivs_d(Rk4Ctx& c, double t, const double* x, double* dxdt) {
  constexpr double kInvC2 = 1.0 / (kCLight * kCLight);
  const double one_minus = 1. - (x[1] * x[1] + x[3] * x[3] + x[5] * x[5]) * kInvC2;
  if (one_minus <= 0) {  // a state at or above c: reported to the host, dxdt left as it was
    c.superluminal = true;
    return;
  }
  double B[3];
  field_sum_d(c.fs, c.nf, c.vals, x[0], x[2], x[4], t, B);
  dxdt[0] = x[1];
  dxdt[1] = c.qomg * (-x[5] * B[1] + x[3] * B[2]);
  dxdt[2] = x[3];
  dxdt[3] = c.qomg * (x[5] * B[0] - x[1] * B[2]);
  dxdt[4] = x[5];
  dxdt[5] = c.qomg * (x[1] * B[1] - x[3] * B[0]);
}

__device__ __forceinline__ void rk4_step_d(Rk4Ctx& c, double* y, const double* dydx, double x, double h) {
  double dym[6], dyt[6], yt[6];
  const double hh = h * 0.5, h6 = h / 6.0, xh = x + hh;
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dydx[i];
  derivs_d(c, xh, yt, dyt);
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
  derivs_d(c, xh, yt, dym);
  for (int i = 0; i < 6; ++i) {
    yt[i] = y[i] + h * dym[i];
    dym[i] += dyt[i];
  }
  derivs_d(c, x + h, yt, dyt);
  for (int i = 0; i < 6; ++i) y[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
}

// One thread per (job, direction).  Forward points land at [nb, nb + nf), backward points at
// [0, nb) in time order; each point carries the acceleration of the state before it, as the
// reference's integrator stores it (src/OSCARSSR.cc:930-1004).
__global__ void k_batch_rk4(const DevJob* __restrict__ jobs, int njobs, const DevField* __restrict__ fields,
                            const double* __restrict__ field_vals, double* __restrict__ arena,
                            unsigned* __restrict__ err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * njobs) return;
  const DevJob& J = jobs[t >> 1];
  const bool fwd = (t & 1) == 0;
  const int64_t n = (int64_t)J.nf + J.nb;
  double* K = arena + J.knots;
  Rk4Ctx c{fields + J.field_begin, J.field_count, field_vals, J.qomg, false};
  const double* x0 = J.frame.x0;
  double x[6] = {x0[0], J.b0[0] * kCLight, x0[1], J.b0[1] * kCLight, x0[2], J.b0[2] * kCLight};
  double dxdt[6] = {0, 0, 0, 0, 0, 0};
  const double t0 = J.frame.t_ref;
  // beta and a/c by one product with 1/c (within an ulp of the host's division): divisions here would
  // sit in the in-order instruction stream of the serial chain
  constexpr double kInvC = 1.0 / kCLight;
  auto store = [&](int64_t i, double tt) {
    K[i] = tt;
    K[n + i] = x[0];
    K[2 * n + i] = x[2];
    K[3 * n + i] = x[4];
    K[4 * n + i] = x[1] * kInvC;
    K[5 * n + i] = x[3] * kInvC;
    K[6 * n + i] = x[5] * kInvC;
    K[7 * n + i] = dxdt[1] * kInvC;
    K[8 * n + i] = dxdt[3] * kInvC;
    K[9 * n + i] = dxdt[5] * kInvC;
  };
  if (fwd) {
    derivs_d(c, t0, x, dxdt);
    for (int i = 0; i < J.nf; ++i) {
      const double tt = t0 + J.dt * i;
      store(J.nb + i, tt);
      derivs_d(c, tt, x, dxdt);
      rk4_step_d(c, x, dxdt, tt, J.dt);
    }
  } else {
    const double dtr = -J.dt;
    for (int i = 0; i < J.nb; ++i) {
      const double t1 = t0 + dtr * i;
      derivs_d(c, t1, x, dxdt);
      rk4_step_d(c, x, dxdt, t1, dtr);
      store(J.nb - 1 - i, t0 + dtr * (i + 1));
    }
  }
  if (c.superluminal) atomicOr(err, kErrSuperluminal);
}

// The same clamped spline with each sweep split across the threads of a block (one block per job
// and component).  Every sweep is a first-order recurrence: the factor yp_i = (sig_i - 1) /
// (sig_i yp_{i-1} + 2) a Moebius map of yp_{i-1}, the right side u_i = (6 d_i - sig_i u_{i-1}) / p_i
// and the back substitution ypp_k = yp_k ypp_{k+1} + u_k affine ones.  Each thread composes the maps
// of its chunk of points, a block-wide inclusive scan of the chunk maps gives every chunk its entering
// value, and each thread then runs its chunk with the reference's operations from that value.  The
// maps contract (|d yp_i / d yp_{i-1}| < 1/4, |sig_i / p_i| < 1/2, |yp_k| < 1/2), so the entering
// values' rounding does not grow along the chunk.
constexpr int kSplThreads = 256;

struct Mob { double a, b, c, d; };  // y -> (a y + b) / (c y + d)
__device__ __forceinline__ Mob mob_then(Mob f, Mob g) {  // g(f(y)), scaled by its largest entry
  Mob h{g.a * f.a + g.b * f.c, g.a * f.b + g.b * f.d, g.c * f.a + g.d * f.c, g.c * f.b + g.d * f.d};
  const double m = fmax(fmax(fabs(h.a), fabs(h.b)), fmax(fabs(h.c), fabs(h.d)));
  const double r = m > 0 ? 1.0 / m : 1.0;
  return {h.a * r, h.b * r, h.c * r, h.d * r};
}
struct Aff { double a, b; };  // x -> a x + b
__device__ __forceinline__ Aff aff_then(Aff f, Aff g) { return {g.a * f.a, g.a * f.b + g.b}; }

// Inclusive block scan of the threads' maps (kSplThreads of them) in shared memory; returns the
// composition of the maps of threads 0 .. t-1 (identity for thread 0).
template <class M, class Then>
__device__ __forceinline__ M block_prefix(M mine, M identity, M* sh, Then then) {
  const int t = threadIdx.x;
  sh[t] = mine;
  __syncthreads();
  for (int o = 1; o < kSplThreads; o <<= 1) {
    M prev = identity;
    if (t >= o) prev = sh[t - o];
    __syncthreads();
    if (t >= o) sh[t] = then(prev, sh[t]);
    __syncthreads();
  }
  const M before = t > 0 ? sh[t - 1] : identity;
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kSplThreads) k_batch_spline_scan(const DevJob* __restrict__ jobs,
                                                                   double* __restrict__ arena,
                                                                   double* __restrict__ work) {
  __shared__ Mob shm[kSplThreads];
  __shared__ Aff sha[kSplThreads];
  const DevJob& J = jobs[blockIdx.x / 9];
  const int c = blockIdx.x % 9;
  const int t = threadIdx.x;
  const int64_t n = (int64_t)J.nf + J.nb;
  const double* X = arena + J.knots;
  const double* Y = X + (1 + c) * n;
  double* ypp = arena + J.knots + (10 + c) * n;
  double* u = work + J.u_off + c * n;
  auto sigma = [&](int64_t i) {
    return __ddiv_rn(__dsub_rn(X[i], X[i - 1]), __dsub_rn(X[i + 1], X[i - 1]));
  };
  // interior points i = 1 .. n-2 in chunks
  const int64_t m = n - 2;
  const int64_t chunk = (m + kSplThreads - 1) / kSplThreads;
  const int64_t i0 = 1 + t * chunk, i1 = min(n - 1, i0 + chunk);
  // boundary values (src: the clamped first-derivative end conditions of the reference's sweep)
  const double dydx0 = __ddiv_rn(__dsub_rn(Y[1], Y[0]), __dsub_rn(X[1], X[0]));
  const double u0 = __dmul_rn(__ddiv_rn(3., __dsub_rn(X[1], X[0])),
                              __dsub_rn(__ddiv_rn(__dsub_rn(Y[1], Y[0]), __dsub_rn(X[1], X[0])), dydx0));
  // 1. yp (stored in ypp for now): Moebius maps [[0, sig - 1], [sig, 2]]
  Mob fm{1, 0, 0, 1};
  for (int64_t i = i0; i < i1; ++i) {
    const double sg = sigma(i);
    fm = mob_then(fm, Mob{0.0, sg - 1.0, sg, 2.0});
  }
  const Mob pm = block_prefix<Mob>(fm, Mob{1, 0, 0, 1}, shm, mob_then);
  double yp_prev = (pm.a * -0.5 + pm.b) / (pm.c * -0.5 + pm.d);  // yp_{i0-1}
  if (t == 0) {
    yp_prev = -0.5;
    ypp[0] = -0.5;
    u[0] = u0;
  }
  for (int64_t i = i0; i < i1; ++i) {
    const double sg = sigma(i);
    const double p = __dadd_rn(__dmul_rn(sg, yp_prev), 2.0);
    yp_prev = __ddiv_rn(__dsub_rn(sg, 1.), p);
    ypp[i] = yp_prev;
  }
  __syncthreads();
  // 2. u: affine maps u_i = (-sig / p) u_{i-1} + (6 d_i / (x_{i+1} - x_{i-1})) / p
  auto d_i = [&](int64_t i) {
    return __dsub_rn(__ddiv_rn(__dsub_rn(Y[i + 1], Y[i]), __dsub_rn(X[i + 1], X[i])),
                     __ddiv_rn(__dsub_rn(Y[i], Y[i - 1]), __dsub_rn(X[i], X[i - 1])));
  };
  Aff fa{1, 0};
  for (int64_t i = i0; i < i1; ++i) {
    const double sg = sigma(i);
    const double p = __dadd_rn(__dmul_rn(sg, i == 1 ? -0.5 : ypp[i - 1]), 2.0);
    fa = aff_then(fa, Aff{-sg / p, __ddiv_rn(__dmul_rn(6., d_i(i)), __dsub_rn(X[i + 1], X[i - 1])) / p});
  }
  const Aff pa = block_prefix<Aff>(fa, Aff{1, 0}, sha, aff_then);
  double u_prev = t == 0 ? u0 : pa.a * u0 + pa.b;  // u_{i0-1}
  for (int64_t i = i0; i < i1; ++i) {
    const double sg = sigma(i);
    const double p = __dadd_rn(__dmul_rn(sg, i == 1 ? -0.5 : ypp[i - 1]), 2.0);
    u_prev = __ddiv_rn(__dsub_rn(__ddiv_rn(__dmul_rn(6., d_i(i)), __dsub_rn(X[i + 1], X[i - 1])), __dmul_rn(sg, u_prev)), p);
    u[i] = u_prev;
  }
  __syncthreads();
  // 3. back substitution from ypp_{n-1}: ypp_k = yp_k ypp_{k+1} + u_k, k = n-2 .. 0, in chunks of the
  // reversed index
  const double dydxn = __ddiv_rn(__dsub_rn(Y[n - 1], Y[n - 2]), __dsub_rn(X[n - 1], X[n - 2]));
  const double un = __dmul_rn(__ddiv_rn(3., __dsub_rn(X[n - 1], X[n - 2])),
                              __dsub_rn(dydxn, __ddiv_rn(__dsub_rn(Y[n - 1], Y[n - 2]), __dsub_rn(X[n - 1], X[n - 2]))));
  const double last = __ddiv_rn(__dsub_rn(un, __dmul_rn(0.5, u[n - 2])), __dadd_rn(__dmul_rn(0.5, ypp[n - 2]), 1.));
  const int64_t mb = n - 1;  // k = n-2 .. 0
  const int64_t cb = (mb + kSplThreads - 1) / kSplThreads;
  const int64_t r0 = t * cb, r1 = min(mb, r0 + cb);  // reversed positions r: k = n - 2 - r
  Aff fb{1, 0};
  for (int64_t r = r0; r < r1; ++r) {
    const int64_t k = n - 2 - r;
    fb = aff_then(fb, Aff{ypp[k], u[k]});
  }
  const Aff pb = block_prefix<Aff>(fb, Aff{1, 0}, sha, aff_then);
  double next = pb.a * last + pb.b;  // ypp_{k+1} entering the chunk
  if (t == 0) next = last;
  __syncthreads();  // every chunk has read its yp and u before any is overwritten
  if (t == 0) ypp[n - 1] = last;
  for (int64_t r = r0; r < r1; ++r) {
    const int64_t k = n - 2 - r;
    next = __dadd_rn(__dmul_rn(ypp[k], next), u[k]);
    ypp[k] = next;
  }
}

// Trajectory extent in the job frame: max transverse distance from the axis, max longitudinal
// coordinate and max |tau_s| (one block of 256 threads per job).
__global__ void k_batch_extent(DevJob* __restrict__ jobs, const double* __restrict__ arena) {
  __shared__ double sx[256], sz[256], st[256];
  DevJob& J = jobs[blockIdx.x];
  const int64_t n = (int64_t)J.nf + J.nb;
  const double* K = arena + J.knots;
  const double* R = J.frame.rot;
  const double* x0 = J.frame.x0;
  double xp = 0, zm = -1e300, tm = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double dx = K[n + i] - x0[0], dy = K[2 * n + i] - x0[1], dz = K[3 * n + i] - x0[2];
    const double a = R[0] * dx + R[1] * dy + R[2] * dz;
    const double b = R[3] * dx + R[4] * dy + R[5] * dz;
    const double c = R[6] * dx + R[7] * dy + R[8] * dz;
    xp = fmax(xp, sqrt(a * a + b * b));
    zm = fmax(zm, c);
    tm = fmax(tm, fabs((K[i] - J.frame.t_ref) - c / kCLight));
  }
  sx[threadIdx.x] = xp;
  sz[threadIdx.x] = zm;
  st[threadIdx.x] = tm;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + o]);
      sz[threadIdx.x] = fmax(sz[threadIdx.x], sz[threadIdx.x + o]);
      st[threadIdx.x] = fmax(st[threadIdx.x], st[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    J.frame.xperp_max = sx[0];
    J.frame.z_max = sz[0];
    J.frame.tau_max = st[0];
  }
}

// Clamped spline second derivatives (end slopes from the end differences, as TSpline1D3 sets
// them), one thread per (job, component); `work` holds the forward-sweep terms.
__global__ void k_batch_spline(const DevJob* __restrict__ jobs, int njobs, double* __restrict__ arena,
                               double* __restrict__ work) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 9 * njobs) return;
  const DevJob& J = jobs[t / 9];
  const int c = t % 9;
  const int64_t n = (int64_t)J.nf + J.nb;
  const double* X = arena + J.knots;
  const double* Y = X + (1 + c) * n;
  double* ypp = arena + J.knots + (10 + c) * n;
  double* u = work + J.u_off + c * n;
  // The sweeps carry the recurrence (ypp[i-1], u[i-1] forward, ypp[k+1] backward) in registers and
  // read the knots through the read-only path a few points ahead, so each step waits only on its own
  // arithmetic; the operations and their order are those of the reference's sweep.
  const double dydx0 = __ddiv_rn(__dsub_rn(__ldg(Y + 1), __ldg(Y)), __dsub_rn(__ldg(X + 1), __ldg(X)));
  double yp_prev = -0.5;
  double u_prev = __dmul_rn(__ddiv_rn(3., __dsub_rn(__ldg(X + 1), __ldg(X))),
                            __dsub_rn(__ddiv_rn(__dsub_rn(__ldg(Y + 1), __ldg(Y)), __dsub_rn(__ldg(X + 1), __ldg(X))),
                                      dydx0));
  ypp[0] = yp_prev;
  u[0] = u_prev;
  double xm = __ldg(X), x0 = __ldg(X + 1), ym = __ldg(Y), y0 = __ldg(Y + 1);
  constexpr int B = 16;  // knots read per block of points, ahead of the block's recurrence
  for (int64_t i0 = 1; i0 < n - 1; i0 += B) {
    double xv[B], yv[B];
#pragma unroll
    for (int j = 0; j < B; ++j) {
      const int64_t q = min(i0 + j + 1, n - 1);
      xv[j] = __ldg(X + q);
      yv[j] = __ldg(Y + q);
    }
#pragma unroll
    for (int j = 0; j < B; ++j) {
      const int64_t i = i0 + j;
      if (i < n - 1) {
        const double xp = xv[j], yp = yv[j];
        const double sig = __ddiv_rn(__dsub_rn(x0, xm), __dsub_rn(xp, xm));
        const double p = __dadd_rn(__dmul_rn(sig, yp_prev), 2.0);
        const double ypi = __ddiv_rn(__dsub_rn(sig, 1.), p);
        const double ui = __dsub_rn(__ddiv_rn(__dsub_rn(yp, y0), __dsub_rn(xp, x0)),
                                    __ddiv_rn(__dsub_rn(y0, ym), __dsub_rn(x0, xm)));
        const double uu = __ddiv_rn(__dsub_rn(__ddiv_rn(__dmul_rn(6., ui), __dsub_rn(xp, xm)), __dmul_rn(sig, u_prev)), p);
        ypp[i] = ypi;
        u[i] = uu;
        yp_prev = ypi;
        u_prev = uu;
        xm = x0; x0 = xp; ym = y0; y0 = yp;
      }
    }
  }
  const double dydxn = __ddiv_rn(__dsub_rn(__ldg(Y + n - 1), __ldg(Y + n - 2)), __dsub_rn(__ldg(X + n - 1), __ldg(X + n - 2)));
  const double un = __dmul_rn(__ddiv_rn(3., __dsub_rn(__ldg(X + n - 1), __ldg(X + n - 2))),
                              __dsub_rn(dydxn, __ddiv_rn(__dsub_rn(__ldg(Y + n - 1), __ldg(Y + n - 2)),
                                                         __dsub_rn(__ldg(X + n - 1), __ldg(X + n - 2)))));
  double next = __ddiv_rn(__dsub_rn(un, __dmul_rn(0.5, u_prev)), __dadd_rn(__dmul_rn(0.5, yp_prev), 1.));
  ypp[n - 1] = next;
  int64_t k = n - 2;
  for (; k >= 7; k -= 8) {  // blocks of 8: the block's forward-sweep values are read before its stores
    double yv[8], uv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      yv[j] = ypp[k - j];
      uv[j] = u[k - j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      next = __dadd_rn(__dmul_rn(yv[j], next), uv[j]);
      ypp[k - j] = next;
    }
  }
  for (; k >= 0; --k) {
    next = __dadd_rn(__dmul_rn(ypp[k], next), u[k]);
    ypp[k] = next;
  }
}

// Clamped splines of a chunk's trajectories: the serial sweeps (one thread per job and component)
// take the latency of the longest trajectory's recurrences (~1.6 us per point for both sweeps on
// B200), the block-parallel ones the chunk's total work (~1.3 ns per point, all 9 components).  mode
// 0 takes whichever the chunk's shape makes shorter, 1 the serial and 2 the block-parallel kernel.
void launch_batch_splines(const DevJob* d_jobs, int nj, int64_t n_max, int64_t n_total, double* knots, double* work,
                          int mode, cudaStream_t st) {
  const double serial_ms = 1.6e-3 * (double)n_max, parallel_ms = 1.3e-6 * (double)n_total;
  if (mode == 2 || (mode == 0 && parallel_ms < serial_ms))
    k_batch_spline_scan<<<9 * nj, kSplThreads, 0, st>>>(d_jobs, knots, work);
  else
    k_batch_spline<<<(9 * nj + 63) / 64, 64, 0, st>>>(d_jobs, nj, knots, work);
}


// Level samples [s_begin, s_end) of every job whose active count is non-zero (all jobs when `cnt` is
// NULL), evaluated from its spline and written as pair records (fd_common.cuh): job j's records
// start at float kPairFloats / 2 * j * stride of `rec`, sample s at local index s - s_off (s_off
// even); sample 0 is the zero-amplitude record; levels above ext_from are extended levels
// (level_time).  One thread per (job, sample).
__global__ void k_batch_fill(const DevJob* __restrict__ jobs, int njobs, const double* __restrict__ arena,
                             const unsigned* __restrict__ cnt, float* __restrict__ rec, int64_t stride,
                             int64_t s_off, int64_t s_begin, int64_t s_end, int ext_from) {
  // The two samples of a pair sit in adjacent lanes (per = s_end - s_begin, s_begin and the block
  // size are even) and exchange their FP64 values for the pair's step: every lane reaches the
  // shuffles, lanes past the grid's end or of a finished job on a valid sample, writing nothing.
  const int64_t per = s_end - s_begin;
  const int64_t g_raw = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t g = g_raw < per * njobs ? g_raw : per * njobs - 2 + (g_raw & 1);
  const int j = (int)(g / per);
  const bool active = g_raw < per * njobs && !(cnt && cnt[j] == 0);
  const DevJob& J = jobs[j];
  const int64_t s = s_begin + g % per;
  const int64_t n = (int64_t)J.nf + J.nb;
  const double T = level_time(J.tstart, J.tstop, s == 0 ? 1 : s, ext_from);
  double v[9];
  spline_eval9(arena + J.knots, n, T, v);
  const MixedFrame& F = J.frame;
  const double* R = F.rot;
  const double dx = v[0] - F.x0[0], dy = v[1] - F.x0[1], dz = v[2] - F.x0[2];
  const double x = R[0] * dx + R[1] * dy + R[2] * dz;
  const double y = R[3] * dx + R[4] * dy + R[5] * dz;
  const double z = R[6] * dx + R[7] * dy + R[8] * dz;
  const double px = R[0] * v[3] + R[1] * v[4] + R[2] * v[5];
  const double py = R[3] * v[3] + R[4] * v[4] + R[5] * v[5];
  const double pz = R[6] * v[3] + R[7] * v[4] + R[8] * v[5];
  const double qx = R[0] * v[6] + R[1] * v[7] + R[2] * v[8];
  const double qy = R[3] * v[6] + R[4] * v[7] + R[5] * v[8];
  const double qz = R[6] * v[6] + R[7] * v[7] + R[8] * v[8];
  const double taus = (T - F.t_ref) - z / kCLight;
  const unsigned full = 0xffffffffu;
  const double xo = __shfl_xor_sync(full, x, 1), yo = __shfl_xor_sync(full, y, 1);
  const double zo = __shfl_xor_sync(full, z, 1), to = __shfl_xor_sync(full, taus, 1);
  if (active)
    write_pair_record(rec + (kPairFloats / 2) * (int64_t)j * stride, s - s_off, s == 0, x, y, z, taus, px, py, pz, qx,
                      qy, qz, xo, yo, zo, to);
}

// Offsets of one wave over the chunk (one block of 1024 threads): per job the active count n_j (all
// entries on the first wave), units = ceil(n_j / tile) x spans, partial doubles
// n_j x nseg x spans x kFdPartials, and exclusive prefix sums of the three.  `spans` is common to
// the wave: the smallest power of two giving at least target_units units in total (wave_spans).
__global__ void __launch_bounds__(1024) k_batch_plan(const DevJob* __restrict__ jobs, int njobs,
                                                     const unsigned* __restrict__ cnt, int first, int L, int tile,
                                                     int64_t target, int min_span, BatchPlan P) {
  constexpr int T = 1024;
  __shared__ int64_t red[3][T];
  __shared__ int64_t carry[3];
  __shared__ int spans_s;
  const int tid = threadIdx.x;
  int64_t tiles = 0;
  for (int j = tid; j < njobs; j += T) {
    const int64_t na = first ? jobs[j].n_obs * jobs[j].n_e : (int64_t)cnt[j];
    tiles += (na + tile - 1) / tile;
  }
  red[0][tid] = tiles;
  __syncthreads();
  for (int o = T / 2; o > 0; o >>= 1) {
    if (tid < o) red[0][tid] += red[0][tid + o];
    __syncthreads();
  }
  if (tid == 0) {
    spans_s = wave_spans(L, red[0][0], target, min_span);
    *P.spans = spans_s;
    carry[0] = carry[1] = carry[2] = 0;
  }
  __syncthreads();
  const int spans = spans_s;
  const int nseg = (first && L >= 1) ? 2 : 1;
  for (int base = 0; base < njobs; base += T) {
    const int j = base + tid;
    int64_t v[3] = {0, 0, 0};
    if (j < njobs) {
      const int64_t na = first ? jobs[j].n_obs * jobs[j].n_e : (int64_t)cnt[j];
      v[0] = (na + tile - 1) / tile * spans;
      v[1] = na * nseg * spans * kFdPartials;
      v[2] = na;
    }
    for (int q = 0; q < 3; ++q) red[q][tid] = v[q];
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {  // inclusive scans (Hillis-Steele)
      int64_t w[3];
      for (int q = 0; q < 3; ++q) w[q] = tid >= o ? red[q][tid - o] : 0;
      __syncthreads();
      for (int q = 0; q < 3; ++q) red[q][tid] += w[q];
      __syncthreads();
    }
    if (j < njobs) {
      P.unit_start[j] = carry[0] + red[0][tid] - v[0];
      P.part_start[j] = carry[1] + red[1][tid] - v[1];
      P.act_start[j] = carry[2] + red[2][tid] - v[2];
    }
    __syncthreads();
    if (tid == T - 1)
      for (int q = 0; q < 3; ++q) carry[q] += red[q][T - 1];
    __syncthreads();
  }
  if (tid == 0) {
    P.unit_start[njobs] = carry[0];
    P.part_start[njobs] = carry[1];
    P.act_start[njobs] = carry[2];
  }
}

// Last j with starts[j] <= x (starts non-decreasing, starts[0] = 0 <= x).
__device__ __forceinline__ int find_job(const int64_t* __restrict__ starts, int njobs, int64_t x) {
  int lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (starts[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

constexpr int kBThreads = 128;
constexpr int kBChunk = 256;   // samples per staged chunk (128 pair records, 20 KB)
constexpr int kBFold = 16;     // pairs per FP32 partial sum before it is folded into FP64

struct BatchStage {
  float4 v[2][kBChunk / 2 * kPairF4];
  uint64_t bar[2];
};

// The mixed sample sum over all jobs of a chunk.  Persistent CTAs take (job, tile, span) units from a
// shared counter (the job by binary search of the unit prefix); within a unit the sum is that of
// k_fd_wave_mixed_pair: SUB groups of TE = 128 / SUB threads, one entry per thread, each group
// taking 1/SUB of every staged chunk of pair records, the largest phase step carried across parts
// and spans (the span maxima include the step into each span).  One partial per entry and span,
// entry-major per job from part_start[j]; k_batch_finalize reduces them.
template <int SUB, int MINB>
__global__ void __launch_bounds__(kBThreads, MINB) k_batch_wave(BatchWaveArgs A) {
  constexpr int TE = kBThreads / SUB;
  constexpr int CP = kBChunk / 2;  // pairs per chunk
  __shared__ __align__(16) BatchStage st;
  __shared__ double red[SUB > 1 ? SUB - 1 : 1][7][TE];
  __shared__ WavePlan P;
  __shared__ int64_t next_unit;
  const int tid = threadIdx.x;
  const int grp = tid / TE, q = tid % TE;
  if (tid == 0) {
    P = wave_plan_spans(A.first, A.level, *A.plan.spans);
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t units = A.plan.unit_start[A.njobs];
  uint32_t phase_bits = 0;
  for (;;) {  // CTAs take (job, tile, span) units from a shared counter until the wave's units run out
    if (tid == 0) next_unit = (int64_t)atomicAdd(A.work, 1ull);
    __syncthreads();
    const int64_t u = next_unit;
    __syncthreads();
    if (u >= units) break;
    const int j = find_job(A.plan.unit_start, A.njobs, u);
    const DevJob& J = A.jobs[j];
    const int64_t local = u - A.plan.unit_start[j];
    const int64_t tile = local / P.spans;
    const int span = (int)(local % P.spans);
    const int64_t n_act = A.first ? J.n_obs * J.n_e : (int64_t)A.cnt[j];
    const int64_t slot = tile * TE + q;
    const bool live = slot < n_act;
    const int64_t item = live ? (A.first ? slot : (int64_t)A.act[J.entry_begin + slot]) : 0;
    PairObs o;
    {
      const int64_t io = J.obs_begin + item / J.n_e, ie = J.omega_begin + item % J.n_e;
      const double* R = J.frame.rot;
      const double ox = A.obs[3 * io] - J.frame.x0[0], oy = A.obs[3 * io + 1] - J.frame.x0[1];
      const double oz = A.obs[3 * io + 2] - J.frame.x0[2];
      const double fx = R[0] * ox + R[1] * oy + R[2] * oz;
      const double fy = R[3] * ox + R[4] * oy + R[5] * oz;
      const double fz = R[6] * ox + R[7] * oy + R[8] * oz;
      const double om = A.omega[ie];
      o = make_pair_obs(fx, fy, fz, om);
      if (live && grp == 0 && span == 0 && !mixed_geometry_ok(fx, fy, fz, om, J.frame)) atomicOr(A.err, kErrBadArgs);
    }
    // pair records of job j: absolute pair p at rec_j[kPairF4 * (p - s_off / 2)]
    const float4* rec_j = A.rec + kPairF4 * ((int64_t)j * (A.stride >> 1)) - kPairF4 * (A.s_off >> 1);  // stride even
    for (int g = 0; g < P.nseg; ++g) {
      const int64_t b0 = seg_begin(P, g) + (int64_t)span * seg_span(P, g);
      const int64_t b1 = min(seg_end(P, g), b0 + seg_span(P, g));
      const int64_t p0 = b0 >> 1, p1 = b1 > b0 ? b1 >> 1 : p0;  // spans are whole pairs
      double S[6] = {0, 0, 0, 0, 0, 0};
      float dmax = 0.f;
      bool any = false;
      const int64_t nchunks = (p1 - p0 + CP - 1) / CP;
      float carry = __int_as_float(0x7fc00000);  // NaN: no step into the segment's first sample
      if (live && span > 0 && nchunks > 0)
        carry = pair_phase_at(reinterpret_cast<const float*>(rec_j + kPairF4 * (p0 - 1)), 1, o);
      if (tid == 0 && nchunks > 0) {
        const int64_t hi = min(p1, p0 + CP);
        mbar_arrive_expect_tx(&st.bar[0], (uint32_t)((hi - p0) * (kPairFloats * 4)));
        tma_load_1d(&st.v[0][0], rec_j + kPairF4 * p0, (uint32_t)((hi - p0) * (kPairFloats * 4)), &st.bar[0]);
      }
      for (int64_t c = 0; c < nchunks; ++c) {
        const int buf = (int)(c & 1);
        const int64_t lo = p0 + c * CP, hi = min(p1, lo + CP);
        if (tid == 0 && c + 1 < nchunks) {  // prefetch the next chunk into the other buffer
          const int64_t lo2 = lo + CP, hi2 = min(p1, lo2 + CP);
          mbar_arrive_expect_tx(&st.bar[buf ^ 1], (uint32_t)((hi2 - lo2) * (kPairFloats * 4)));
          tma_load_1d(&st.v[buf ^ 1][0], rec_j + kPairF4 * lo2, (uint32_t)((hi2 - lo2) * (kPairFloats * 4)),
                      &st.bar[buf ^ 1]);
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
          for (int jb = j0; jb < j1; jb += kBFold) {
            const int je = min(j1, jb + kBFold);
            float2 acc[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[k] = f2(0.f);
#pragma unroll 2
            for (int jj = jb; jj < je; ++jj) {
              const float2 ph = pair_sample(sv + kPairF4 * jj, o, acc);
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
        if (live && c + 1 < nchunks)  // the chunk is full: its last sample precedes the next
          carry = pair_phase_at(reinterpret_cast<const float*>(sv + kPairF4 * (CP - 1)), 1, o);
        __syncthreads();  // everyone is done with `buf` before it is refilled
      }
      // reduce the groups' sums in group order; group 0 stores the span's partial
      if (SUB > 1 && grp > 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) red[grp - 1][k][q] = S[k];
        red[grp - 1][6][q] = any ? (double)dmax : -1.0;
      }
      if (SUB > 1) __syncthreads();
      if (grp == 0 && live) {
        double dm = any ? (double)dmax : -1.0;
        for (int o2 = 0; o2 < SUB - 1; ++o2) {
#pragma unroll
          for (int k = 0; k < 6; ++k) S[k] += red[o2][k][q];
          dm = fmax(dm, red[o2][6][q]);
        }
        double* p = A.part + A.plan.part_start[j] + (slot * P.nseg * P.spans + g * P.spans + span) * kFdPartials;
#pragma unroll
        for (int k = 0; k < 6; ++k) p[k] = S[k];
        p[6] = 0.0;
        p[7] = 0.0;
        p[8] = dm;  // -1 marks an empty span
      }
      if (SUB > 1) __syncthreads();
    }
  }
}

// Groups of kFinLanes lanes take the active entries of all jobs in act_start order (grid-stride;
// the loop bound is block-uniform so every warp stays converged for its shuffles and ballots).
// Lanes of a group summing one entry's spans (LANES = 1: one thread per entry, its spans in order).
template <int LANES>
__device__ __forceinline__ double lanes_sum(double v) {
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, LANES);
  return v;
}
template <int LANES>
__device__ __forceinline__ double lanes_max(double v) {
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o, LANES));
  return v;
}

// Span reduction and stop rule of every active entry of the chunk.  LANES threads per entry; with one
// (the launch below) a warp's 32 entries read their adjacent partial records together, which the
// waves with one span per entry -- the large ones -- make contiguous.
template <int LANES>
__global__ void __launch_bounds__(256) k_batch_finalize(BatchFinalArgs A) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *A.work_reset = 0;
  const int64_t total = A.plan.act_start[A.njobs];
  const int spans = *A.plan.spans;
  const int L = A.level;
  const int nseg = (A.first && L >= 1) ? 2 : 1;
  const int lane = threadIdx.x % LANES;
  const unsigned full = 0xffffffffu;
  const int lane32 = threadIdx.x & 31;
  const int64_t per_pass = (int64_t)gridDim.x * blockDim.x / LANES;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x / LANES; base < total; base += per_pass) {
    const int64_t gidx = base + threadIdx.x / LANES;
    const bool live = gidx < total;
    const int j = live ? find_job(A.plan.act_start, A.njobs, gidx) : 0;
    const DevJob& J = A.jobs[j];
    const int64_t slot = live ? gidx - A.plan.act_start[j] : 0;
    const int64_t item = live ? (A.first ? slot : (int64_t)A.act[J.entry_begin + slot]) : 0;
    const int64_t e = J.entry_begin + item;
    const double* pbase = A.part + A.plan.part_start[j] + slot * nseg * spans * kFdPartials;
    auto seg_sum = [&](int g, C3& s, double& dmax) {
      C3 t = {0, 0, 0, 0, 0, 0};
      double dm = 0;
      if (live) {
        for (int sp = lane; sp < spans; sp += LANES) {
          const double* p = pbase + (g * spans + sp) * kFdPartials;
          t.xr += p[0]; t.xi += p[1]; t.yr += p[2]; t.yi += p[3]; t.zr += p[4]; t.zi += p[5];
          if (p[8] >= 0) dm = fmax(dm, p[8]);  // the span maxima include the step into each span
        }
      }
      s.xr += lanes_sum<LANES>(t.xr); s.xi += lanes_sum<LANES>(t.xi); s.yr += lanes_sum<LANES>(t.yr);
      s.yi += lanes_sum<LANES>(t.yi); s.zr += lanes_sum<LANES>(t.zr); s.zi += lanes_sum<LANES>(t.zi);
      dmax = fmax(dmax, lanes_max<LANES>(dm));
    };
    auto mag = [&](C3 v, double scale) {
      C3 t = c3_scale(v, scale);
      if (A.project) t = c3_project(t, J.pol);
      return c3_mag2(t);
    };
    const double T = J.tstop - J.tstart;
    C3 S = {0, 0, 0, 0, 0, 0};
    double last_mag = -1, dmax = 0;
    if (A.first) {
      double unused = 0;
      if (nseg == 2) {
        seg_sum(0, S, unused);
        last_mag = mag(S, T / (ldexp(1.0, L) - 1));  // DeltaT inclusive to level L-1
      }
      seg_sum(nseg - 1, S, dmax);
    } else {
      if (live) {
        const int64_t N = A.n_entries;
        S = {A.state[e], A.state[N + e], A.state[2 * N + e], A.state[3 * N + e], A.state[4 * N + e],
             A.state[5 * N + e]};
        last_mag = A.state[6 * N + e];
      }
      seg_sum(0, S, dmax);
    }
    bool finished = false, unconverged = false, survive = false;
    if (live && lane == 0) {
      const double dtl = T / (ldexp(1.0, L + 1) - 1);  // DeltaT inclusive to level L
      const double this_mag = mag(S, dtl);
      const double prec = fabs(this_mag - last_mag) / last_mag;
      const bool stop = (L > 8 && prec < A.precision && dmax < kPiD) || (L > 8 && dmax < kPiD && this_mag == last_mag);
      if (stop || L >= A.max_level) {
        const int result_level = stop ? L : -1;
        double v;
        if (A.quantity == 1) v = prec;
        else if (A.quantity == 2) v = (double)result_level;
        else v = J.c2 * mag(S, J.c0 * dtl);
        A.out[e] = v;
        if (A.level_out) A.level_out[e] = result_level;
        finished = true;
        unconverged = !stop;
      } else {
        const int64_t N = A.n_entries;
        A.state[e] = S.xr; A.state[N + e] = S.xi; A.state[2 * N + e] = S.yr;
        A.state[3 * N + e] = S.yi; A.state[4 * N + e] = S.zr; A.state[5 * N + e] = S.zi;
        A.state[6 * N + e] = this_mag;
        survive = true;
      }
    }
    const unsigned fin = __ballot_sync(full, finished), unc = __ballot_sync(full, unconverged);
    if (lane32 == 0) {
      if (fin) atomicAdd(A.samples, (unsigned long long)__popc(fin) * (unsigned long long)((2ll << L) - 1));
      if (unc) atomicAdd(A.not_converged, (unsigned long long)__popc(unc));
    }
    // survivors join their job's next list; one atomic per (warp, job)
    const unsigned sur_all = __ballot_sync(full, survive);
    const unsigned peers = __match_any_sync(full, survive ? j : -1) & sur_all;
    const int leader = survive ? __ffs(peers) - 1 : lane32;
    unsigned pos = 0;
    if (survive && lane32 == leader) pos = atomicAdd(&A.cnt_next[j], (unsigned)__popc(peers));
    pos = __shfl_sync(full, pos, leader);
    if (survive) A.act_next[J.entry_begin + pos + __popc(peers & ((1u << lane32) - 1u))] = (int)item;
  }
}

// acc[m] += weight x value of entry m of every job of the chunk, in job order, compensated
// (T3DScalarContainer::AddToPoint over particles).
__global__ void k_batch_average(const double* __restrict__ vals, const DevJob* __restrict__ jobs, int njobs,
                                int64_t m_count, double weight, double* __restrict__ acc, double* __restrict__ comp) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= m_count) return;
  double S = acc[m], c = comp[m];
  for (int j = 0; j < njobs; ++j) {
    const double v = __dmul_rn(vals[jobs[j].entry_begin + m], weight);
    const double y = __dsub_rn(v, c);
    const double t = __dadd_rn(S, y);
    c = __dsub_rn(__dsub_rn(t, S), y);
    S = t;
  }
  acc[m] = S;
  comp[m] = c;
}

}  // namespace dev

// ---------------------------------------------------------------------------------------------
// Variants of the batched wave kernel: (entries per thread, minimum resident CTAs per SM).
// ---------------------------------------------------------------------------------------------
static const int kBatchSub[kBatchVariants] = {4, 4, 2, 1};  // groups per CTA: tiles of 128 / SUB entries

template <int SUB, int MINB>
static int batch_occ() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::k_batch_wave<SUB, MINB>, dev::kBThreads, 0);
  return n > 0 ? n : 1;
}

static int batch_blocks_per_sm(int variant) {
  switch (variant) {
    case 0: return batch_occ<4, 4>();
    case 1: return batch_occ<4, 1>();
    case 2: return batch_occ<2, 4>();
    default: return batch_occ<1, 4>();
  }
}

static int batch_tile(int variant) { return dev::kBThreads / kBatchSub[variant]; }

static cudaError_t launch_batch_wave(const BatchWaveArgs& a, int grid, int variant, cudaStream_t st) {
  const int T = dev::kBThreads;
  switch (variant) {
    case 0: dev::k_batch_wave<4, 4><<<grid, T, 0, st>>>(a); break;
    case 1: dev::k_batch_wave<4, 1><<<grid, T, 0, st>>>(a); break;
    case 2: dev::k_batch_wave<2, 4><<<grid, T, 0, st>>>(a); break;
    default: dev::k_batch_wave<1, 4><<<grid, T, 0, st>>>(a); break;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------------------------
namespace {
constexpr int kBatchPrefill = 13;        // levels enqueued without the host (records kept resident)
constexpr int kBatchMinSpan = 128;
constexpr int kBatchMaxJobsPerChunk = 8192;
}  // namespace

DevField to_dev_field(FieldSpec f, std::vector<double>& vals) {
  f.finish();
  DevField d;
  std::memset(&d, 0, sizeof d);
  if (f.kind == 2) {
    const GridData& g = *f.grid;
    d.kind = 2;
    d.grid_dim = g.dimx;
    for (int a = 0; a < 3; ++a) {
      d.grid_n[a] = g.n[a];
      d.grid_start[a] = g.start[a];
      d.grid_step[a] = g.step[a];
      d.grid_stop[a] = g.stop[a];
    }
    d.grid_off = (int64_t)vals.size();
    vals.insert(vals.end(), g.v.begin(), g.v.end());
    const double r[3] = {f.rotations.x, f.rotations.y, f.rotations.z};
    for (int a = 0; a < 3; ++a) {
      d.rot_sin[a] = std::sin(r[a]);
      d.rot_cos[a] = std::cos(r[a]);
    }
    d.center[0] = f.center.x; d.center[1] = f.center.y; d.center[2] = f.center.z;
    d.frequency = f.frequency; d.frequency_phase = f.frequency_phase; d.time_offset = f.time_offset;
    return d;
  }
  if (!f.half_scale.empty()) {
    d.half_off = (int64_t)vals.size();
    d.n_half = (int)f.half_scale.size();
    vals.insert(vals.end(), f.half_scale.begin(), f.half_scale.end());
  }
  d.kind = f.kind;
  d.nperiods = f.nperiods;
  const Vec3 a = f.a, b = f.b, c = f.center, u = f.period_unit;
  d.a[0] = a.x; d.a[1] = a.y; d.a[2] = a.z;
  d.b[0] = b.x; d.b[1] = b.y; d.b[2] = b.z;
  d.center[0] = c.x; d.center[1] = c.y; d.center[2] = c.z;
  d.period_unit[0] = u.x; d.period_unit[1] = u.y; d.period_unit[2] = u.z;
  d.phase = f.phase; d.taper = f.taper; d.frequency = f.frequency; d.frequency_phase = f.frequency_phase;
  d.time_offset = f.time_offset; d.period_length = f.period_length; d.period_mag = mag(f.period);
  d.length = f.length;
  d.k_arg = 2.0 * kPi / f.period_length;
  d.inv_half_period = 2.0 / f.period_length;
  if (f.kind == 0) {
    d.shift[0] = f.phase * d.period_mag / (2.0 * kPi);
  } else {  // EPU: A shifted by +phase/2, B by -phase/2
    d.shift[0] = f.phase / 2. * d.period_mag / (2.0 * kPi);
    d.shift[1] = -f.phase / 2. * d.period_mag / (2.0 * kPi);
  }
  return d;
}

// Device descriptors of a batch's jobs, validated like Model::compute_trajectory: frame, RK4 step and
// point counts, flux constants, polarization vector in the job frame (pol), field and entry ranges
// (the latter only with_entries).
static std::vector<DevJob> build_dev_jobs(size_t n_fields, const std::vector<BatchJob>& jobs, int64_t n_obs_total,
                                          int64_t n_omega_total, bool average, const double* pol, bool with_entries) {
  std::vector<DevJob> dj(jobs.size());
  for (size_t k = 0; k < jobs.size(); ++k) {
    const BatchJob& S = jobs[k];
    const Particle& P = S.particle;
    if (S.field_begin < 0 || S.field_count < 0 || (size_t)S.field_begin + S.field_count > n_fields)
      throw Error{OSC_ERR_RANGE, "job field range outside the field array"};
    if (with_entries && (S.obs_begin < 0 || S.n_obs < 1 || S.obs_begin + S.n_obs > n_obs_total))
      throw Error{OSC_ERR_RANGE, "job observer range outside the observer array"};
    if (with_entries && (S.omega_begin < 0 || S.n_e < 1 || S.omega_begin + S.n_e > n_omega_total))
      throw Error{OSC_ERR_RANGE, "job energy range outside the energy array"};
    if (S.n_obs * S.n_e > 2147483647ll) throw Error{OSC_ERR_LENGTH, "more than 2^31-1 entries in one job"};
    if (average && (S.obs_begin != jobs[0].obs_begin || S.n_obs != jobs[0].n_obs ||
                    S.omega_begin != jobs[0].omega_begin || S.n_e != jobs[0].n_e))
      throw Error{OSC_ERR_INVALID, "averaged jobs must share their observers and energies"};
    if (!P.set) throw Error{OSC_ERR_RANGE, "particle not initialized.  make sure you have a particle or beam defined"};
    if (S.ctstart > P.t0 || S.ctstop < P.t0)
      throw Error{OSC_ERR_RANGE, "start time is greater than T0 or stop time is less than T0"};
    if (S.ctstart >= S.ctstop)
      throw Error{OSC_ERR_RANGE, "start time is greater than stop time.  check that set_ctstartstop is set"};
    if (S.npoints < 2) throw Error{OSC_ERR_LENGTH, "Not enough points in this trajectory"};
    const double dt = ((S.ctstop - S.ctstart) / kC / (S.npoints - 1));
    const int64_t nf = (int64_t)(1 + (S.ctstop - P.t0) / kC / dt);
    const int64_t nb = (int64_t)((P.t0 - S.ctstart) / kC / dt);
    if (nf + nb < 3)
      throw Error{OSC_ERR_LENGTH, "TSpline1D3 does not see enough points for interpolation.  Please use >= 3 points"};
    if (nf + nb > 2147483647ll) throw Error{OSC_ERR_LENGTH, "trajectory too long"};
    DevJob& d = dj[k];
    std::memset(&d, 0, sizeof d);
    const Vec3 e3 = unit(P.b0);
    const Vec3 e1 = unit(orthogonal(e3));
    const Vec3 e2 = cross(e3, e1);
    const Vec3 rows[3] = {e1, e2, e3};
    for (int r = 0; r < 3; ++r) {
      d.frame.rot[3 * r] = rows[r].x;
      d.frame.rot[3 * r + 1] = rows[r].y;
      d.frame.rot[3 * r + 2] = rows[r].z;
    }
    d.frame.x0[0] = P.x0.x; d.frame.x0[1] = P.x0.y; d.frame.x0[2] = P.x0.z;
    d.frame.t_ref = P.t0 / kC;
    d.frame.theta_max = mixed_theta_max(P.gamma);
    d.b0[0] = P.b0.x; d.b0[1] = P.b0.y; d.b0[2] = P.b0.z;
    d.qomg = P.qomg;
    d.dt = dt;
    d.tstart = P.t0 / kC + (-dt) * (double)nb;
    d.tstop = P.t0 / kC + dt * (double)(nf - 1);
    d.c0 = P.q / (four_pi() * kC * kEps0 * kSqrt2Pi);                                           // :4106
    const double cur = S.current_abs ? std::fabs(P.current) : P.current;
    d.c2 = four_pi() * cur / (kH * std::fabs(P.q) * kMu0 * kC) * 1e-6 * 0.001;                  // :4109
    for (int ri = 0; ri < 2; ++ri)  // P' = R P in the job frame (R orthogonal: E'.P' = E.P)
      for (int r = 0; r < 3; ++r)
        d.pol[2 * r + ri] = d.frame.rot[3 * r] * pol[ri] + d.frame.rot[3 * r + 1] * pol[2 + ri] +
                            d.frame.rot[3 * r + 2] * pol[4 + ri];
    d.nf = (int)nf;
    d.nb = (int)nb;
    d.field_begin = S.field_begin;
    d.field_count = S.field_count;
    d.obs_begin = S.obs_begin; d.omega_begin = S.omega_begin; d.n_obs = S.n_obs; d.n_e = S.n_e;
  }

  return dj;
}

int Engine::batch_resident(int v) {
  if (wave_grid_[3][v] == 0) {
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attr");
    wave_grid_[3][v] = sms * batch_blocks_per_sm(v);
  }
  return wave_grid_[3][v];
}

void Engine::batch(const std::vector<FieldSpec>& fields, const std::vector<BatchJob>& jobs, const double* obs,
                   int64_t n_obs_total, const double* omega, int64_t n_omega_total, const osc_rad_opts& o,
                   bool average, double* out, int32_t* level_out, double average_weight) {
  pending_.clear();
  last_samples = last_launches = last_not_converged = 0;
  if (jobs.empty()) return;
  // the chunking sizes every job's records up to the prefill level, so the levels stop at 26 here
  int ext_from = kMaxLevelMemory;  // levels above it are extended levels (level_time)
  const int lstop = request_levels(o, kMaxLevelMemory, &ext_from);
  const int Lfirst = std::min(9, lstop);
  const int Lpre = std::min(lstop, std::max(Lfirst, kBatchPrefill));
  double pol[6];
  bool project = false;
  polarization_vector(o, pol, project);

  // ---- job descriptors, validated like Model::compute_trajectory ----
  std::vector<DevJob> dj = build_dev_jobs(fields.size(), jobs, n_obs_total, n_omega_total, average, pol, true);
  const int64_t m_avg = average ? jobs[0].n_obs * jobs[0].n_e : 0;

  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  check(cudaSetDevice(device), "cudaSetDevice");
  use_stream(stream);
  cudaStream_t st = stream;
  std::vector<DevField> df;
  std::vector<double> fvals;
  for (const FieldSpec& f : fields) df.push_back(to_dev_field(f, fvals));
  if (df.empty()) df.push_back(DevField{});
  if (fvals.empty()) fvals.push_back(0.0);
  b_fields_.reserve(sizeof(DevField) * df.size());
  b_fvals_.reserve(sizeof(double) * fvals.size());
  check(cudaMemcpyAsync(b_fvals_.p, fvals.data(), sizeof(double) * fvals.size(), cudaMemcpyHostToDevice, st),
        "field values");
  b_obs_.reserve(sizeof(double) * 3 * n_obs_total);
  b_omega_.reserve(sizeof(double) * n_omega_total);
  // stream-ordered copies (pageable sources are staged before the calls return)
  check(cudaMemcpyAsync(b_fields_.p, df.data(), sizeof(DevField) * df.size(), cudaMemcpyHostToDevice, st), "fields");
  check(cudaMemcpyAsync(b_obs_.p, obs, sizeof(double) * 3 * n_obs_total, cudaMemcpyHostToDevice, st), "observers");
  check(cudaMemcpyAsync(b_omega_.p, omega, sizeof(double) * n_omega_total, cudaMemcpyHostToDevice, st), "energies");
  if (average) {
    b_acc_.reserve(sizeof(double) * 2 * m_avg);
    check(cudaMemsetAsync(b_acc_.p, 0, sizeof(double) * 2 * m_avg, st), "memset");
  }

  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attr");
  int max_resident = 0, max_tile = 0;
  for (int v = 0; v < kBatchVariants; ++v) {
    max_resident = std::max(max_resident, batch_resident(v));
    max_tile = std::max(max_tile, batch_tile(v));
  }
  const int64_t target = 4 * (int64_t)max_resident;  // >= 4 units per resident CTA when work allows

  // ---- chunks of jobs sized to the free device memory ----
  size_t free_b = 0, total_b = 0;
  check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  const size_t budget = std::min<size_t>(free_b / 2, (size_t)64 << 30);
  const int64_t rec_per_job = (int64_t)2 << Lpre;  // levels 0..Lpre, sample s at index s
  auto job_bytes = [&](const DevJob& d) {
    return sizeof(double) * 28 * ((size_t)d.nf + d.nb) + kMixedRecordBytesPerSample * (size_t)rec_per_job +
           (size_t)(d.n_obs * d.n_e) * (56 + 8 + 4 + 8 + 16 * kFdPartials);
  };
  // Chunks: the jobs that fit the budget from the start, then, when more than one chunk is needed,
  // the same number of chunks with the jobs spread evenly (each chunk runs its serial RK4 once, so
  // fewer, fuller chunks are faster).
  size_t fit = 0;
  {
    size_t bytes = 0;
    while (fit < dj.size() && fit < (size_t)kBatchMaxJobsPerChunk) {
      const size_t need = job_bytes(dj[fit]);
      if (fit > 0 && bytes + need > budget) break;
      bytes += need;
      ++fit;
    }
  }
  const size_t n_chunks = (dj.size() + fit - 1) / fit;
  const size_t per_chunk = (dj.size() + n_chunks - 1) / n_chunks;
  size_t done_entries = 0;
  size_t j0 = 0;
  while (j0 < dj.size()) {
    size_t j1 = j0, bytes = 0;
    while (j1 < dj.size() && j1 - j0 < per_chunk) {
      const size_t need = job_bytes(dj[j1]);
      if (j1 > j0 && bytes + need > budget) break;
      bytes += need;
      ++j1;
    }
    const int nj = (int)(j1 - j0);
    int64_t knots = 0, work = 0, N = 0, n_max = 0, n_total = 0;
    for (int k = 0; k < nj; ++k) {
      DevJob& d = dj[j0 + k];
      const int64_t n = (int64_t)d.nf + d.nb;
      n_max = std::max(n_max, n);
      n_total += n;
      d.knots = knots;
      knots += 19 * n;
      d.u_off = work;
      work += 9 * n;
      d.entry_begin = N;
      N += d.n_obs * d.n_e;
    }
    // partial sums: spans = 1 gives 2 segments x N entries; a wave split into more spans has fewer
    // than 2 x target units of at most max_tile entries each (wave_spans)
    const size_t part_doubles = (size_t)std::max<int64_t>(2 * N, 4 * target * max_tile) * kFdPartials;
    b_jobs_.reserve(sizeof(DevJob) * nj);
    b_knots_.reserve(sizeof(double) * knots);
    b_work_.reserve(sizeof(double) * work);
    b_rec_.reserve((size_t)kMixedRecordBytesPerSample * rec_per_job * nj);
    b_state_.reserve(sizeof(double) * 7 * N);
    b_out_.reserve(sizeof(double) * N);
    b_lvl_.reserve(sizeof(int32_t) * N);
    b_act_[0].reserve(sizeof(int) * N);
    b_act_[1].reserve(sizeof(int) * N);
    b_part_.reserve(sizeof(double) * part_doubles);
    b_plan_.reserve(sizeof(int64_t) * 3 * (nj + 1) + 64);
    b_cnt_.reserve(sizeof(unsigned) * 2 * nj + 256);
    check(cudaMemcpyAsync(b_jobs_.p, dj.data() + j0, sizeof(DevJob) * nj, cudaMemcpyHostToDevice, st), "jobs");
    DevJob* d_jobs = b_jobs_.as<DevJob>();
    unsigned* cnt0 = b_cnt_.as<unsigned>();
    unsigned* cnts[2] = {cnt0, cnt0 + nj};
    // after the two count arrays: [0] error word, [2..] 3 x u64 (not converged, samples, unit counter)
    unsigned* misc = cnt0 + ((2 * nj + 7) & ~7);
    unsigned long long* m64 = reinterpret_cast<unsigned long long*>(misc + 2);
    BatchPlan plan;
    plan.unit_start = b_plan_.as<int64_t>();
    plan.part_start = plan.unit_start + (nj + 1);
    plan.act_start = plan.part_start + (nj + 1);
    plan.spans = reinterpret_cast<int*>(plan.act_start + (nj + 1));

    int cur = 0;  // active list / count array of the next wave
    auto wave = [&](int L, int v, int64_t stride, int64_t s_off, const float4* rec) {
      const bool first = L == Lfirst;
      unsigned* cin = cnts[cur];
      unsigned* cout = cnts[cur ^ 1];
      check(cudaMemsetAsync(cout, 0, sizeof(unsigned) * nj, st), "memset");
      const int tile = batch_tile(v);
      dev::k_batch_plan<<<1, 1024, 0, st>>>(d_jobs, nj, cin, first, L, tile, target, kBatchMinSpan, plan);
      BatchWaveArgs w{};
      w.jobs = d_jobs; w.njobs = nj; w.rec = rec; w.stride = stride; w.s_off = s_off;
      w.obs = b_obs_.as<double>(); w.omega = b_omega_.as<double>(); w.act = b_act_[cur].as<int>(); w.cnt = cin;
      w.plan = plan; w.first = first; w.level = L; w.part = b_part_.as<double>(); w.err = misc; w.work = m64 + 2;
      check(launch_batch_wave(w, batch_resident(v), v, st), "batch wave");
      BatchFinalArgs f{};
      f.jobs = d_jobs; f.njobs = nj; f.act = w.act; f.cnt = cin; f.plan = plan; f.part = w.part;
      f.first = first; f.level = L; f.max_level = lstop; f.quantity = o.quantity; f.project = project;
      f.precision = o.precision; f.n_entries = N; f.state = b_state_.as<double>();
      f.act_next = b_act_[cur ^ 1].as<int>(); f.cnt_next = cout; f.out = b_out_.as<double>();
      f.level_out = b_lvl_.as<int32_t>(); f.not_converged = m64; f.samples = m64 + 1; f.work_reset = m64 + 2;
      dev::k_batch_finalize<1><<<sms * 8, 256, 0, st>>>(f);
      check(cudaGetLastError(), "batch finalize");
      last_launches += 3;
      cur ^= 1;
    };
    // trajectories, splines, the resident levels' records and the waves up to Lpre: no host sync
    auto front = [&](int v, bool tune) {
      check(cudaMemsetAsync(misc, 0, 64, st), "memset");
      dev::k_batch_rk4<<<(2 * nj + 63) / 64, 64, 0, st>>>(d_jobs, nj, b_fields_.as<DevField>(),
                                                          b_fvals_.as<double>(), b_knots_.as<double>(), misc);
      dev::k_batch_extent<<<nj, 256, 0, st>>>(d_jobs, b_knots_.as<double>());
      dev::launch_batch_splines(d_jobs, nj, n_max, n_total, b_knots_.as<double>(), b_work_.as<double>(), spline_kernel,
                                st);
      const int64_t fill_n = rec_per_job * nj;  // samples 0 .. 2^(Lpre+1) - 1 of every job
      dev::k_batch_fill<<<(unsigned)((fill_n + 255) / 256), 256, 0, st>>>(
          d_jobs, nj, b_knots_.as<double>(), nullptr, b_rec_.as<float>(), rec_per_job, 0, 0, rec_per_job, ext_from);
      check(cudaGetLastError(), "batch trajectories");
      last_launches += 4;
      if (tune) v = tune_batch(nj, Lfirst, target, d_jobs, plan, misc, m64, rec_per_job);
      for (int L = Lfirst; L <= Lpre; ++L) wave(L, v, rec_per_job, 0, b_rec_.as<float4>());
      return v;
    };
    // a new shape is tuned and run eagerly; a known shape is captured and replayed as a graph
    const auto key = std::make_tuple(nj, N, Lfirst, Lpre);
    const auto chunk_ev = timed_begin(st);  // with profiling on: device time of the whole chunk
    int v = forced_variant[3] >= 0 ? forced_variant[3] : current_variant_[3];
    const bool need_tune = forced_variant[3] < 0 && autotune && tuned_batch_.find(key) == tuned_batch_.end();
    if (forced_variant[3] < 0 && autotune && !need_tune) v = tuned_batch_[key];
    if (need_tune || !use_graphs) {
      v = front(v, need_tune);
      if (need_tune) {
        tuned_batch_[key] = v;
        current_variant_[3] = v;
      }
    } else {
      cudaGraph_t g = nullptr;
      check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
      try {
        front(v, false);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
      }
      check(cudaStreamEndCapture(st, &g), "capture");
      bool updated = false;
      if (graph_exec_) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(graph_exec_, g, &info) == cudaSuccess;
        if (!updated) {
          cudaGetLastError();
          cudaGraphExecDestroy(graph_exec_);
          graph_exec_ = nullptr;
        }
      }
      if (!updated) {
        const cudaError_t e = cudaGraphInstantiate(&graph_exec_, g, 0);
        if (e != cudaSuccess) {
          cudaGraphDestroy(g);
          graph_exec_ = nullptr;
          check(e, "graph instantiate");
        }
      }
      cudaGraphDestroy(g);
      check(cudaGraphLaunch(graph_exec_, st), "graph launch");
      ++graph_launches_;
    }
    // levels beyond the resident ones: records of one level at a time, for the jobs still active
    for (int L = Lpre + 1; L <= lstop; ++L) {
      std::vector<unsigned> c(nj);
      check(cudaMemcpyAsync(c.data(), cnts[cur], sizeof(unsigned) * nj, cudaMemcpyDeviceToHost, st), "counts");
      check(cudaStreamSynchronize(st), "counts");
      bool any = false;
      for (unsigned x : c) any = any || x > 0;
      if (!any) break;
      const int64_t len = (int64_t)1 << L;
      b_rec_ext_.reserve((size_t)kMixedRecordBytesPerSample * len * nj);
      const int64_t fill_n = len * nj;
      dev::k_batch_fill<<<(unsigned)((fill_n + 255) / 256), 256, 0, st>>>(
          d_jobs, nj, b_knots_.as<double>(), cnts[cur], b_rec_ext_.as<float>(), len, len, len, 2 * len, ext_from);
      check(cudaGetLastError(), "batch fill");
      ++last_launches;
      wave(L, v, len, len, b_rec_ext_.as<float4>());
    }
    // results of the chunk
    if (average) {
      dev::k_batch_average<<<(unsigned)((m_avg + 255) / 256), 256, 0, st>>>(
          b_out_.as<double>(), d_jobs, nj, m_avg, average_weight > 0 ? average_weight : 1.0 / (double)jobs.size(),
          b_acc_.as<double>(),
          b_acc_.as<double>() + m_avg);
      check(cudaGetLastError(), "batch average");
      ++last_launches;
      if (level_out && j1 == dj.size())  // levels of the last particle, as the reference leaves them
        check(cudaMemcpyAsync(level_out, b_lvl_.as<int32_t>() + dj[j1 - 1].entry_begin, sizeof(int32_t) * m_avg,
                              cudaMemcpyDeviceToHost, st), "levels");
    } else {
      check(cudaMemcpyAsync(out + done_entries, b_out_.p, sizeof(double) * N, cudaMemcpyDeviceToHost, st), "download");
      if (level_out)
        check(cudaMemcpyAsync(level_out + done_entries, b_lvl_.p, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, st),
              "download");
    }
    timed_end(chunk_ev, st);
    unsigned long long* h64 = reinterpret_cast<unsigned long long*>(ctl_host_ + 4);  // pinned
    check(cudaMemcpyAsync(h64, m64, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "stats");
    check(cudaMemcpyAsync(ctl_host_ + 8, misc, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "stats");
    check(cudaStreamSynchronize(st), "batch");
    const unsigned err = ctl_host_[8];
    if (err & dev::kErrTmaTimeout)
      throw Error{OSC_ERR_TIMEOUT, "a staged trajectory copy did not complete (device wait limit reached)"};
    if (err & dev::kErrSuperluminal)
      throw Error{OSC_ERR_RANGE, "a trajectory reached the speed of light (check the fields)"};
    if (err & dev::kErrBadArgs)
      throw Error{OSC_ERR_INVALID, kMixedGeometryMessage};
    last_not_converged += (long long)h64[0];
    last_samples += (long long)h64[1];
    if (profiling) {
      prof_samples += (long long)h64[1];
      collect_timings();
    }
    done_entries += (size_t)N;
    j0 = j1;
  }
  if (average) {
    check(cudaMemcpyAsync(out, b_acc_.p, sizeof(double) * m_avg, cudaMemcpyDeviceToHost, st), "download");
    check(cudaStreamSynchronize(st), "download");
  }
}

// Trajectories of the jobs as the batched path computes them (k_batch_rk4, k_batch_spline, one chunk):
// per job 19 x n knot values in job order (t | x y z bx by bz ax/c ay/c az/c | their 9 spline second
// derivatives), npoints[k] = n of job k.  For comparing the device integration with the host's.
void Engine::batch_trajectories(const std::vector<FieldSpec>& fields, const std::vector<BatchJob>& jobs, double* out,
                                int64_t capacity, int64_t* npoints) {
  const double pol[6] = {0, 0, 0, 0, 0, 0};
  std::vector<DevJob> dj = build_dev_jobs(fields.size(), jobs, 0, 0, false, pol, false);
  int64_t knots = 0, work = 0, n_max = 0, n_total = 0;
  for (DevJob& d : dj) {
    const int64_t n = (int64_t)d.nf + d.nb;
    d.knots = knots;
    knots += 19 * n;
    d.u_off = work;
    work += 9 * n;
    n_max = std::max(n_max, n);
    n_total += n;
  }
  if (knots > capacity) throw Error{OSC_ERR_LENGTH, "output capacity below 19 x points summed over the jobs"};
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  if (dj.empty()) return;
  check(cudaSetDevice(device), "cudaSetDevice");
  use_stream(stream);
  cudaStream_t st = stream;
  std::vector<DevField> df;
  std::vector<double> fvals;
  for (const FieldSpec& f : fields) df.push_back(to_dev_field(f, fvals));
  if (df.empty()) df.push_back(DevField{});
  if (fvals.empty()) fvals.push_back(0.0);
  const int nj = (int)dj.size();
  b_fields_.reserve(sizeof(DevField) * df.size());
  b_fvals_.reserve(sizeof(double) * fvals.size());
  b_jobs_.reserve(sizeof(DevJob) * nj);
  b_knots_.reserve(sizeof(double) * knots);
  b_work_.reserve(sizeof(double) * work);
  b_cnt_.reserve(64);
  check(cudaMemcpyAsync(b_fvals_.p, fvals.data(), sizeof(double) * fvals.size(), cudaMemcpyHostToDevice, st), "fields");
  check(cudaMemcpyAsync(b_fields_.p, df.data(), sizeof(DevField) * df.size(), cudaMemcpyHostToDevice, st), "fields");
  check(cudaMemcpyAsync(b_jobs_.p, dj.data(), sizeof(DevJob) * nj, cudaMemcpyHostToDevice, st), "jobs");
  unsigned* err = b_cnt_.as<unsigned>();
  check(cudaMemsetAsync(err, 0, sizeof(unsigned), st), "memset");
  dev::k_batch_rk4<<<(2 * nj + 63) / 64, 64, 0, st>>>(b_jobs_.as<DevJob>(), nj, b_fields_.as<DevField>(),
                                                      b_fvals_.as<double>(), b_knots_.as<double>(), err);
  dev::launch_batch_splines(b_jobs_.as<DevJob>(), nj, n_max, n_total, b_knots_.as<double>(), b_work_.as<double>(),
                            spline_kernel, st);
  check(cudaGetLastError(), "batch trajectories");
  check(cudaMemcpyAsync(out, b_knots_.p, sizeof(double) * knots, cudaMemcpyDeviceToHost, st), "download");
  unsigned e = 0;
  check(cudaMemcpyAsync(&e, err, sizeof e, cudaMemcpyDeviceToHost, st), "error word");
  check(cudaStreamSynchronize(st), "batch trajectories");
  if (e & dev::kErrSuperluminal) throw Error{OSC_ERR_RANGE, "a trajectory reached the speed of light (check the fields)"};
  for (int k = 0; k < nj; ++k) npoints[k] = (int64_t)dj[k].nf + dj[k].nb;
}

// Autotuner of the batched wave: times the first wave of the chunk with every compiled variant
// (each run rewrites only the partial sums, so the runs are interchangeable) and keeps the fastest.
int Engine::tune_batch(int nj, int Lfirst, int64_t target, const DevJob* d_jobs, const BatchPlan& plan,
                       unsigned* misc, unsigned long long* m64, int64_t rec_stride) {
  cudaStream_t st = stream;
  cudaEvent_t a, b;
  check(cudaEventCreate(&a), "event");
  check(cudaEventCreate(&b), "event");
  int best = current_variant_[3];
  float best_ms = 1e30f;
  for (int v = 0; v < kBatchVariants; ++v) {
    const int tile = batch_tile(v);
    dev::k_batch_plan<<<1, 1024, 0, st>>>(d_jobs, nj, nullptr, 1, Lfirst, tile, target, kBatchMinSpan, plan);
    BatchWaveArgs w{};
    w.jobs = d_jobs; w.njobs = nj; w.rec = b_rec_.as<float4>(); w.stride = rec_stride; w.s_off = 0;
    w.obs = b_obs_.as<double>(); w.omega = b_omega_.as<double>(); w.act = nullptr; w.cnt = nullptr;
    w.plan = plan; w.first = 1; w.level = Lfirst; w.part = b_part_.as<double>(); w.err = misc; w.work = m64 + 2;
    float ms_v = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      check(cudaMemsetAsync(m64 + 2, 0, sizeof(unsigned long long), st), "memset");
      check(cudaEventRecord(a, st), "event");
      check(launch_batch_wave(w, batch_resident(v), v, st), "batch wave");
      check(cudaEventRecord(b, st), "event");
      check(cudaEventSynchronize(b), "event");
      float ms = 0;
      check(cudaEventElapsedTime(&ms, a, b), "event");
      ms_v = std::min(ms_v, ms);
    }
    if (ms_v < best_ms) {
      best_ms = ms_v;
      best = v;
    }
  }
  check(cudaMemsetAsync(m64 + 2, 0, sizeof(unsigned long long), st), "memset");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

}  // namespace osc
