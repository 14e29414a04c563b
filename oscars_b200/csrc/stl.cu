// stl.cu -- host side of the power density on STL facets (src/OSCARSSR.cc:3154-3521): the particle
// loop, the per-level launches of k_stl_level (kernels_stl.cu) on the FP64 level cache, and the
// per-facet results with the reference's bookkeeping.
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.h"
#include "kernels.h"

namespace osc {

double dt_inclusive(double tstart, double tstop, int L);

void Engine::power_density_stl(const double* tri, const double* centers, int64_t n, const osc_rad_opts& o,
                               double* out, int32_t* level_out) {
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  check(cudaSetDevice(device), "cudaSetDevice");
  use_stream(stream);
  cudaStream_t st = stream;
  pending_.clear();
  last_samples = last_launches = last_not_converged = 0;
  // one CTA per facet walks a whole level, so the levels stop at 26 here
  int ext_from = kMaxLevelMemory;
  const int lstop = request_levels(o, kMaxLevelMemory, &ext_from);
  if (n <= 0) return;
  set_level_grid(ext_from);
  for (int64_t i = 0; i < n; ++i) out[i] = 0;
  // facet geometry as RayIntersectionDistance forms it: A, B - A, C - A (src/TTriangle3D.cc)
  std::vector<double> geo(9 * n), nrm(3 * n);
  for (int64_t i = 0; i < n; ++i) {
    const double* t = tri + 12 * i;
    for (int c = 0; c < 3; ++c) {
      geo[9 * i + c] = t[c];
      geo[9 * i + 3 + c] = t[3 + c] - t[c];
      geo[9 * i + 6 + c] = t[6 + c] - t[c];
      nrm[3 * i + c] = t[9 + c];
    }
  }
  stl_geo_.reserve(sizeof(double) * 9 * n);
  stl_cen_.reserve(sizeof(double) * 3 * n);
  stl_nrm_.reserve(sizeof(double) * 3 * n);
  stl_state_.reserve(sizeof(double) * 4 * n);
  stl_flags_.reserve(sizeof(int) * 2 * n);
  check(cudaMemcpyAsync(stl_geo_.p, geo.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice, st), "facets");
  check(cudaMemcpyAsync(stl_cen_.p, centers, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st), "facets");
  check(cudaMemcpyAsync(stl_nrm_.p, nrm.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st), "facets");
  unsigned* n_active = cnt_.as<unsigned>();  // word 0 of the request counters
  std::vector<double> init(4 * n), state(4 * n);
  for (int64_t i = 0; i < n; ++i) {  // sum 0, last level value -1, result precision -1, level 0
    init[4 * i] = 0;
    init[4 * i + 1] = -1;
    init[4 * i + 2] = -1;
    init[4 * i + 3] = 0;
  }
  std::vector<int32_t> flags(2 * n);
  const int np = o.nparticles;
  const double weight = np > 0 ? 1.0 / (double)np : 1.0;
  for (int ip = 0; ip < (np > 0 ? np : 1); ++ip) {
    if (np > 0) {  // src/OSCARSSR.cc:3234-3240: a new random particle and its trajectory
      model.random_particle();
      model.compute_trajectory();
    } else {
      model.ensure_trajectory();
    }
    check(cudaStreamSynchronize(st), "particle");  // the previous particle's launches read the caches
    upload_trajectory();
    const Particle& P = model.particle;
    check(cudaMemcpyAsync(stl_state_.p, init.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice, st), "state");
    check(cudaMemsetAsync(stl_flags_.p, 0, sizeof(int) * n, st), "memset");
    check(cudaMemsetAsync(stl_flags_.as<int>() + n, 0xff, sizeof(int) * n, st), "memset");  // levels -1
    StlLevelArgs a{};
    a.geometry = stl_geo_.as<double>();
    a.centers = stl_cen_.as<double>();
    a.normals = stl_nrm_.as<double>();
    a.n = n;
    a.precision = o.precision;
    a.two_over_gamma = 2. / P.gamma;
    a.state = stl_state_.as<double>();
    a.done = stl_flags_.as<int>();
    a.level_out = stl_flags_.as<int>() + n;
    a.n_active = n_active;
    int last_level = 0;
    for (int L = 0; L <= lstop; ++L) {
      ensure_levels(L);
      a.lev = lev_.as<double>();
      a.cap = lev_cap_;
      a.level = L;
      a.dt_level = dt_inclusive(tstart_, tstop_, L);
      check(cudaMemsetAsync(n_active, 0, sizeof(unsigned), st), "memset");
      check(launch_stl_level(a, st), "stl level");
      last_launches += 2;
      last_samples += ((int64_t)1 << L) * n;
      last_level = L;
      if (L > 8) {  // facets can stop from level 9 on
        check(cudaMemcpyAsync(ctl_host_ + 9, n_active, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "count");
        check(cudaStreamSynchronize(st), "count");
        if (ctl_host_[9] == 0) break;
      }
    }
    (void)last_level;
    check(cudaMemcpyAsync(state.data(), stl_state_.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st), "state");
    check(cudaMemcpyAsync(flags.data(), stl_flags_.p, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost, st), "state");
    check(cudaStreamSynchronize(st), "state");
    // src/OSCARSSR.cc:3503-3521.  Result_Level lives outside the loop over facets: a facet that does
    // not stop reports the level of the last facet that did (-1 before any).
    const double scale = std::fabs(P.q * P.current) / (16 * (kPi * kPi) * kEps0 * kC);
    int carried = -1;
    for (int64_t i = 0; i < n; ++i) {
      const int lv = flags[n + i];
      if (lv >= 0) carried = lv;
      else ++last_not_converged;
      double v;
      switch (o.quantity) {
        case 1: v = state[4 * i + 2] * weight; break;
        case 2: v = ((double)carried) * weight; break;
        default: {
          double sum = state[4 * i] * (scale * dt_inclusive(tstart_, tstop_, (int)state[4 * i + 3]));
          sum /= 1e6;
          v = sum * weight;
        }
      }
      out[i] = v + out[i];  // TTriangle3D::AddToValue
      if (level_out) level_out[i] = carried;
    }
  }
}

}  // namespace osc
