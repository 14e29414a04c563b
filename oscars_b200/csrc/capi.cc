// capi.cc -- the extern "C" boundary (include/oscars_b200.h).  Every entry point catches osc::Error
// and any other exception and turns it into a status code plus a message for osc_last_error().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <cuda_runtime.h>

#include "../../include/oscars_b200.h"
#include "engine.h"

struct osc_ctx {
  osc::Engine* eng = nullptr;
  std::string err;
};

namespace {

thread_local std::string g_create_error;

template <class F>
int guarded(osc_ctx* ctx, F&& f) {
  if (!ctx) return OSC_ERR_INVALID;
  try {
    f();
    ctx->err.clear();
    return OSC_OK;
  } catch (const osc::Error& e) {
    ctx->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->err = "host allocation failed";
    return OSC_ERR_ALLOC;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return OSC_ERR_INVALID;
  } catch (...) {
    ctx->err = "unexpected exception";
    return OSC_ERR_INVALID;
  }
}

osc::Vec3 V3(const double* p) { return p ? osc::v3(p[0], p[1], p[2]) : osc::Vec3{}; }

int particle_qm(int code, double charge, double mass, double& q, double& m) {
  using namespace osc;
  switch (code) {  // TParticleA::SetParticleType (src/TParticleA.cc:78-121)
    case OSC_PARTICLE_ELECTRON: q = -kQe; m = kMe; return 0;
    case OSC_PARTICLE_POSITRON: q = kQe; m = kMe; return 0;
    case OSC_PARTICLE_MUON: q = -kQe; m = gev_to_kg(0.1056583715); return 0;
    case OSC_PARTICLE_ANTIMUON: q = kQe; m = gev_to_kg(0.1056583715); return 0;
    case OSC_PARTICLE_PROTON: q = kQe; m = gev_to_kg(0.938272046); return 0;
    case OSC_PARTICLE_ANTIPROTON: q = -kQe; m = gev_to_kg(0.938272046); return 0;
    case OSC_PARTICLE_PIPLUS: q = kQe; m = gev_to_kg(0.13957018); return 0;
    case OSC_PARTICLE_PIMINUS: q = -kQe; m = gev_to_kg(0.13957018); return 0;
    case OSC_PARTICLE_CUSTOM: q = charge; m = mass; return 0;
    default: return -1;
  }
}

void check_opts(const osc_rad_opts* o) {
  if (!o) throw osc::Error{OSC_ERR_INVALID, "options are required"};
  if (o->nparticles < 0) throw osc::Error{OSC_ERR_INVALID, "'nparticles' must be >= 1 (sort of)"};
  if (o->quantity < 0 || o->quantity > 2)
    throw osc::Error{OSC_ERR_INVALID, "'quantity' must be: 'flux', 'precision', 'level', or blank"};
  if (o->precision_mode != OSC_FP64 && o->precision_mode != OSC_MIXED)
    throw osc::Error{OSC_ERR_INVALID, "unknown precision mode"};
  if (o->shard_count < 0 || (o->shard_count > 1 && (o->shard_rank < 0 || o->shard_rank >= o->shard_count)))
    throw osc::Error{OSC_ERR_RANGE, "shard_rank must be in [0, shard_count)"};
}

}  // namespace

extern "C" {

OSC_API const char* osc_version(void) { return "oscars_b200 0.1 (sm_100a)"; }

OSC_API int osc_get_device_count(int* count) {
  if (!count) return OSC_ERR_INVALID;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return OSC_OK;
  }
  int usable = 0;
  for (int d = 0; d < n; ++d) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10 && p.minor == 0) ++usable;
  }
  *count = usable;
  return OSC_OK;
}

OSC_API int osc_ctx_create(int device, osc_ctx** out) {
  if (!out) return OSC_ERR_INVALID;
  *out = nullptr;
  if (device == -1) {  // host-only context
    osc_ctx* c = new (std::nothrow) osc_ctx;
    if (!c) return OSC_ERR_ALLOC;
    c->eng = new osc::Engine(-1);
    *out = c;
    return OSC_OK;
  }
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    g_create_error = "no CUDA device is visible";
    return OSC_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) {
    g_create_error = "device index out of range";
    return OSC_ERR_RANGE;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess || p.major != 10 || p.minor != 0) {
    g_create_error = "device is not an sm_100 (B200) GPU";
    return OSC_ERR_NO_DEVICE;
  }
  osc_ctx* c = new (std::nothrow) osc_ctx;
  if (!c) return OSC_ERR_ALLOC;
  try {
    c->eng = new osc::Engine(device);
  } catch (const osc::Error& e) {
    g_create_error = e.msg;
    delete c;
    return e.code;
  }
  *out = c;
  return OSC_OK;
}

OSC_API void osc_ctx_destroy(osc_ctx* ctx) {
  if (!ctx) return;
  delete ctx->eng;
  delete ctx;
}

OSC_API const char* osc_last_error(const osc_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

OSC_API int osc_clear_fields(osc_ctx* ctx) {
  return guarded(ctx, [&] { ctx->eng->model.clear_fields(); });
}

osc::FieldSpec field_from_desc(const osc_field_desc* f) {
  if (!f) throw osc::Error{OSC_ERR_INVALID, "field descriptor is NULL"};
  if (f->kind == OSC_FIELD_GRID) {
    if (!f->grid_values) throw osc::Error{OSC_ERR_INVALID, "grid field without values"};
    const int64_t n[3] = {f->grid_n[0], f->grid_n[1], f->grid_n[2]};
    return osc::grid_from_values(n, f->grid_start, f->grid_step, f->grid_values, V3(f->rotations), V3(f->center),
                                 f->frequency, f->frequency_phase, f->time_offset);
  }
  if (f->kind != OSC_FIELD_UNDULATOR && f->kind != OSC_FIELD_EPU) throw osc::Error{OSC_ERR_INVALID, "unknown field kind"};
  osc::FieldSpec s;
  s.kind = f->kind;
  s.a = V3(f->bfield);
  s.b = V3(f->bfield_b);
  s.period = V3(f->period);
  s.nperiods = f->nperiods;
  s.center = V3(f->center);
  s.phase = f->phase;
  s.taper = f->taper;
  s.frequency = f->frequency;
  s.frequency_phase = f->frequency_phase;
  s.time_offset = f->time_offset;
  if (f->half_period_scale && f->n_half_periods > 0) {
    if (f->kind != OSC_FIELD_UNDULATOR) throw osc::Error{OSC_ERR_INVALID, "half-period factors apply to undulators"};
    if (f->n_half_periods != 2 * f->nperiods)
      throw osc::Error{OSC_ERR_LENGTH, "n_half_periods must be 2 * nperiods"};
    s.half_scale.assign(f->half_period_scale, f->half_period_scale + f->n_half_periods);
  }
  return s;
}

OSC_API int osc_add_field(osc_ctx* ctx, const osc_field_desc* f) {
  return guarded(ctx, [&] { ctx->eng->model.add_field(field_from_desc(f)); });
}

OSC_API int osc_add_field_file(osc_ctx* ctx, const char* path, const char* format, const double rotations[3],
                               const double translation[3], const double* scaling, int n_scaling, double frequency,
                               double frequency_phase, double time_offset) {
  return guarded(ctx, [&] {
    if (!path || !format) throw osc::Error{OSC_ERR_INVALID, "path and format are required"};
    if (n_scaling < 0 || (n_scaling > 0 && !scaling)) throw osc::Error{OSC_ERR_INVALID, "bad scaling"};
    std::vector<double> sc(scaling, scaling + n_scaling);
    ctx->eng->model.add_field(osc::grid_from_file(path, format, V3(rotations), V3(translation), sc, frequency,
                                                  frequency_phase, time_offset));
  });
}

OSC_API int osc_get_bfield(osc_ctx* ctx, const double x[3], double t, double out[3]) {
  return guarded(ctx, [&] {
    const osc::Vec3 b = osc::field_sum(ctx->eng->model.fields, V3(x), t);
    out[0] = b.x; out[1] = b.y; out[2] = b.z;
  });
}

// add_particle_beam + set_particle_beam (src/OSCARSSR_Python.cc:3561-3576, 3699-4100) for a
// single user-defined beam; the TParticleBeam 10-argument constructor (src/TParticleBeam.cc:68-101).
// TParticleBeam::SetPredefinedBeam (src/TParticleBeam.cc:135-206): the beam's fields in the order
// the reference sets them (each setter's recomputation included).
static osc::BeamSpec predefined_beam(int code) {
  using namespace osc;
  BeamSpec b;
  if (particle_qm(OSC_PARTICLE_ELECTRON, 0, 0, b.q, b.m)) throw Error{OSC_ERR_INVALID, "particle type"};
  b.current = 0.500;
  b.e0 = 3 < kg_to_gev(b.m) ? b.m : 3;  // SetE0
  b.u0 = unit(v3(0, 0, 1));
  b.t0 = 0;
  b.x0 = v3(0, 0, 0);
  b.twiss_at_x0();                      // SetX0
  b.emit[0] = 0.55e-9;
  b.emit[1] = 0.008e-9;
  b.lattice_ref = v3(0, 0, 0);
  b.twiss_at_x0();                      // SetTwissLatticeReference
  const bool straight = code != OSC_BEAM_NSLSII;
  const double beta[2] = {code == OSC_BEAM_NSLSII_LONGSTRAIGHT ? 18. : 1.5,
                          code == OSC_BEAM_NSLSII_LONGSTRAIGHT ? 3.1 : 0.8};
  for (int i = 0; i < 2; ++i) {        // SetTwissBetaAlpha(beta, (0, 0))
    b.tw_beta[i] = beta[i];
    b.tw_gamma[i] = (1. + 0. * 0.) / beta[i];
    b.tw_alpha[i] = 0;
  }
  b.twiss_at_x0();
  b.sigma_e = straight ? 3. * 0.00089 : 0;
  b.vdir = unit(v3(0, 1, 0));           // SetVerticalDirection
  b.hdir = unit(cross(b.vdir, b.u0));
  b.distribution = straight ? OSC_DIST_GAUSSIAN : OSC_DIST_FILAMENT;
  return b;
}

// One beam as add_particle_beam builds it (src/OSCARSSR_Python.cc:3796-4096), from a descriptor
// whose x0 / d0 are already rotated and translated and whose horizontal direction is the one given
// or -d0.Orthogonal() of the unrotated direction.
static osc::BeamSpec build_beam(const osc_beam_desc* d) {
  using namespace osc;
  const bool pre = d->predefined != OSC_BEAM_NONE;
  if (pre && d->predefined != OSC_BEAM_NSLSII && d->predefined != OSC_BEAM_NSLSII_LONGSTRAIGHT &&
      d->predefined != OSC_BEAM_NSLSII_SHORTSTRAIGHT)
    throw Error{OSC_ERR_INVALID, "Error in predefined beam name / definition"};
  BeamSpec b;
  if (pre) {
    b = predefined_beam(d->predefined);
    if (d->energy_GeV >= 0) b.e0 = d->energy_GeV < kg_to_gev(b.m) ? b.m : d->energy_GeV;  // SetE0
  }
  const double e = d->energy_GeV == -1 ? 0 : d->energy_GeV;
  if (e < 0) throw Error{OSC_ERR_INVALID, "We do not currently support negative energy beams.  Please change 'energy_GeV' to >= 0"};
  const double w = d->weight == 0 ? 1 : d->weight;
  if (w <= 0) throw Error{OSC_ERR_INVALID, "Particle weight cannot be negative"};
  const Vec3 dir = V3(d->d0);
  const Vec3 hd = unit(V3(d->horizontal));  // the binding normalises once ...
  if (!pre) {  // the TParticleBeam constructor (src/TParticleBeam.cc:97-125)
    if (particle_qm(d->particle, d->charge, d->mass, b.q, b.m))
      throw Error{OSC_ERR_INVALID, "invalid argument in adding particle beam.  possibly 'name' already exists"};
    if (d->particle == OSC_PARTICLE_CUSTOM && (d->mass == 0 || d->charge == 0))
      throw Error{OSC_ERR_INVALID, "'mass' or 'charge' is zero"};
    b.x0 = V3(d->x0);
    b.u0 = mag2(dir) > 0 ? unit(dir) : Vec3{};
    b.e0 = e < kg_to_gev(b.m) ? b.m : e;
    b.t0 = d->t0;
    b.current = d->current != 0 ? d->current : b.q;
  } else {
    if (d->has_d0) b.u0 = unit(dir);  // SetU0
    b.x0 = V3(d->x0);                 // SetX0
    b.twiss_at_x0();
  }
  b.weight = w;
  b.hdir = unit(hd);  // ... and SetHorizontalDirection again (src/TParticleBeam.cc:374-381)
  b.vdir = -unit(cross(hd, b.u0));
  if (d->has_emittance) {
    b.emit[0] = d->emittance[0];
    b.emit[1] = d->emittance[1];
    b.distribution = OSC_DIST_GAUSSIAN;
  } else if (!pre) {
    b.distribution = OSC_DIST_FILAMENT;
  }
  if (d->distribution != OSC_DIST_DEFAULT) b.distribution = d->distribution;
  if (d->sigma_energy_GeV < 0) throw Error{OSC_ERR_INVALID, "'sigma_energy_GeV' cannot be less than zero"};
  if (d->sigma_energy_GeV > 0) b.sigma_e = d->sigma_energy_GeV;
  const Vec3 ref = d->has_lattice_reference ? V3(d->lattice_reference) : v3(0, 0, 0);
  b.lattice_ref = ref;  // SetTwissLatticeReference
  b.twiss_at_x0();
  const int bag = (d->has_beta ? 4 : 0) | (d->has_alpha ? 2 : 0) | (d->has_gamma ? 1 : 0);
  const double* B = d->beta;
  const double* A = d->alpha;
  const double* G = d->gamma;
  const bool set_ref = d->has_lattice_reference != 0;
  auto finish = [&]() {
    if (set_ref) b.lattice_ref = ref;
    b.twiss_at_x0();
  };
  switch (bag) {  // src/TParticleBeam.cc:219-350
    case 7:
      for (int i = 0; i < 2; ++i) { b.tw_beta[i] = B[i]; b.tw_alpha[i] = A[i]; b.tw_gamma[i] = G[i]; }
      finish();
      break;
    case 6:
    case 4: {
      const double a0 = bag == 6 ? A[0] : 0, a1 = bag == 6 ? A[1] : 0;
      if (B[0] <= 0 || B[1] <= 0) throw Error{OSC_ERR_RANGE, "Beta cannot be <= 0"};
      b.tw_beta[0] = B[0]; b.tw_beta[1] = B[1];
      b.tw_gamma[0] = (1. + a0 * a0) / B[0];
      b.tw_gamma[1] = (1. + a1 * a1) / B[1];
      b.tw_alpha[0] = a0; b.tw_alpha[1] = a1;
      finish();
      break;
    }
    case 5:
      for (int i = 0; i < 2; ++i) {
        b.tw_beta[i] = B[i];
        b.tw_alpha[i] = std::sqrt(G[i] * B[i] - 1);
        b.tw_gamma[i] = G[i];
      }
      finish();
      break;
    case 3:
      if (G[0] == 0 || G[1] == 0) throw Error{OSC_ERR_RANGE, "Gamma cannot be <= 0"};
      for (int i = 0; i < 2; ++i) {
        b.tw_beta[i] = (1. + A[i] * A[i]) / G[i];
        b.tw_alpha[i] = A[i];
        b.tw_gamma[i] = G[i];
      }
      finish();
      break;
    default:
      break;
  }
  b.eta[0] = d->eta[0];
  b.eta[1] = d->eta[1];
  if (d->t0 != 0) b.t0 = d->t0;
  return b;
}

static void add_beam(osc::Model& M, const osc_beam_desc* d, const char* name) {
  using namespace osc;
  if (!d) throw Error{OSC_ERR_INVALID, "beam descriptor is NULL"};
  const bool first = M.beams.empty();
  BeamSpec b = build_beam(d);
  b.name = name && *name ? std::string(name) : "_beam" + std::to_string(M.beams.size());
  for (const BeamSpec& o : M.beams)
    if (o.name == b.name)
      throw Error{OSC_ERR_INVALID, d->predefined != OSC_BEAM_NONE
                                       ? "Error in predefined beam name / definition"
                                       : "invalid argument in adding particle beam.  possibly 'name' already exists"};
  M.add_beam(b);
  if (d->has_ctstartstop) M.set_ctstartstop(d->ctstartstop[0], d->ctstartstop[1]);
  else M.set_ctstartstop(-3, 3);
  if (first) M.new_particle("", true);  // SetNewParticle("", "ideal")
}

OSC_API int osc_set_beam(osc_ctx* ctx, const osc_beam_desc* d) {
  return guarded(ctx, [&] {
    ctx->eng->model.clear_beams();
    add_beam(ctx->eng->model, d, "");
  });
}

OSC_API int osc_add_beam(osc_ctx* ctx, const osc_beam_desc* d, const char* name) {
  return guarded(ctx, [&] { add_beam(ctx->eng->model, d, name); });
}

OSC_API int osc_clear_beams(osc_ctx* ctx) {
  return guarded(ctx, [&] { ctx->eng->model.clear_beams(); });
}

OSC_API int osc_set_new_particle_of_beam(osc_ctx* ctx, const char* beam, int ideal) {
  return guarded(ctx, [&] {
    osc::Model& M = ctx->eng->model;
    if (!M.has_beam) throw osc::Error{OSC_ERR_RANGE, "no beam defined"};
    M.new_particle(beam ? std::string(beam) : std::string(), ideal != 0);
  });
}

OSC_API int osc_set_seed(osc_ctx* ctx, int seed) {
  return guarded(ctx, [&] { ctx->eng->model.rng.seed(seed); });
}

OSC_API int osc_set_new_particle(osc_ctx* ctx, int ideal) {
  return guarded(ctx, [&] {
    osc::Model& M = ctx->eng->model;
    if (!M.has_beam) throw osc::Error{OSC_ERR_RANGE, "no beam defined"};
    if (ideal) M.ideal_particle();
    else M.random_particle();
  });
}

OSC_API int osc_beam_particles(osc_ctx* ctx, long long n, int shard_rank, int shard_count, double* out,
                               long long* n_out) {
  return guarded(ctx, [&] {
    osc::Model& M = ctx->eng->model;
    if (!M.has_beam) throw osc::Error{OSC_ERR_RANGE, "no beam defined"};
    if (n < 0 || !out) throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    const int cnt = shard_count > 1 ? shard_count : 1;
    if (shard_rank < 0 || shard_rank >= cnt) throw osc::Error{OSC_ERR_RANGE, "shard_rank must be in [0, shard_count)"};
    long long k = 0;
    for (long long ip = 0; ip < n; ++ip) {
      M.random_particle();
      if (ip % cnt != shard_rank) continue;
      const osc::Particle& p = M.particle;
      const double v[6] = {p.x0.x, p.x0.y, p.x0.z, p.b0.x, p.b0.y, p.b0.z};
      for (int i = 0; i < 6; ++i) out[6 * k + i] = v[i];
      ++k;
    }
    if (n_out) *n_out = k;
  });
}

OSC_API int osc_get_particle(osc_ctx* ctx, double x0[3], double beta0[3], double* t0, double* gamma) {
  return guarded(ctx, [&] {
    const osc::Particle& p = ctx->eng->model.particle;
    if (x0) { x0[0] = p.x0.x; x0[1] = p.x0.y; x0[2] = p.x0.z; }
    if (beta0) { beta0[0] = p.b0.x; beta0[1] = p.b0.y; beta0[2] = p.b0.z; }
    if (t0) *t0 = p.t0;
    if (gamma) *gamma = p.gamma;
  });
}

OSC_API int osc_set_ctstartstop(osc_ctx* ctx, double start, double stop) {
  return guarded(ctx, [&] { ctx->eng->model.set_ctstartstop(start, stop); });
}

OSC_API int osc_get_ctstartstop(osc_ctx* ctx, double* start, double* stop) {
  return guarded(ctx, [&] {
    if (start) *start = ctx->eng->model.ctstart;
    if (stop) *stop = ctx->eng->model.ctstop;
  });
}

OSC_API int osc_set_npoints_trajectory(osc_ctx* ctx, long long n) {
  return guarded(ctx, [&] { ctx->eng->model.npoints = n; });
}

OSC_API int osc_get_npoints_trajectory(osc_ctx* ctx, long long* n) {
  return guarded(ctx, [&] { if (n) *n = ctx->eng->model.npoints; });
}

OSC_API int osc_set_trajectory_calculation(osc_ctx* ctx, const char* method, double precision) {
  return guarded(ctx, [&] {
    if (!method) throw osc::Error{OSC_ERR_INVALID, "Method requested is invalid.  Try again"};
    ctx->eng->model.set_trajectory_calculation(method, precision);
  });
}

OSC_API int osc_get_trajectory_calculation(osc_ctx* ctx, int* method_out, double* precision_out) {
  return guarded(ctx, [&] {
    if (method_out) *method_out = ctx->eng->model.traj_method;
    if (precision_out) *precision_out = ctx->eng->model.traj_precision;
  });
}

OSC_API int osc_calculate_trajectory(osc_ctx* ctx) {
  return guarded(ctx, [&] {
    osc::Model& M = ctx->eng->model;
    if (!M.particle.set) {
      if (!M.has_beam) throw osc::Error{OSC_ERR_RANGE, "particle not initialized.  make sure you have a particle or beam defined"};
      M.random_particle();
    }
    M.compute_trajectory();
  });
}

OSC_API int osc_get_trajectory(osc_ctx* ctx, double* out, long long capacity, long long* n_out) {
  return guarded(ctx, [&] {
    const osc::Knots& k = ctx->eng->model.knots;
    if (n_out) *n_out = k.n;
    if (!out) return;
    if (capacity < 10 * k.n) throw osc::Error{OSC_ERR_LENGTH, "trajectory buffer too small"};
    std::memcpy(out, k.t.data(), sizeof(double) * k.n);
    std::memcpy(out + k.n, k.y.data(), sizeof(double) * 9 * k.n);
  });
}

OSC_API int osc_set_particle_trajectory(osc_ctx* ctx, int particle, double charge, double mass, double current,
                                        const double x0[3], const double beta0[3], double t0, const double* traj,
                                        long long n) {
  return guarded(ctx, [&] {
    using namespace osc;
    if (!x0 || !beta0 || !traj) throw Error{OSC_ERR_INVALID, "bad buffers"};
    double q = 0, m = 0;
    if (particle_qm(particle, charge, mass, q, m)) throw Error{OSC_ERR_INVALID, "unknown particle type"};
    if (particle == OSC_PARTICLE_CUSTOM && (mass == 0 || charge == 0))
      throw Error{OSC_ERR_INVALID, "'mass' or 'charge' is zero"};
    Model& M = ctx->eng->model;
    Particle P;
    P.q = q;
    P.m = m;
    P.current = current;
    P.set_conditions(V3(x0), V3(beta0), t0);
    M.particle = P;
    M.set_trajectory(traj, n);
  });
}

OSC_API int osc_get_device_properties(int device, char* out, long long capacity) {
  try {
    cudaDeviceProp p;
    const cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess) {
      cudaGetLastError();
      g_create_error = cudaGetErrorString(e);
      return OSC_ERR_CUDA;
    }
    if (out && capacity > 0)
      std::snprintf(out, (size_t)capacity,
                    "%s, compute capability %d.%d, %d multiprocessors, %.1f GB device memory, %.0f kB L2", p.name,
                    p.major, p.minor, p.multiProcessorCount, p.totalGlobalMem / 1e9, p.l2CacheSize / 1e3);
    return OSC_OK;
  } catch (...) {
    return OSC_ERR_INVALID;
  }
}

OSC_API int osc_surface_rectangle(const char* plane, int nx1, int nx2, double width1, double width2,
                                  const double rotations[3], const double translation[3], int normal, double* xyz,
                                  double* normals, double* x1x2) {
  try {
    if (!plane) return OSC_ERR_INVALID;
    if (nx1 <= 0 || nx2 <= 0) {
      g_create_error = "an entry in 'npoints' is <= 0";
      return OSC_ERR_INVALID;
    }
    osc::surface_rectangle(plane, nx1, nx2, width1, width2, V3(rotations), V3(translation), normal, xyz, normals, x1x2);
    return OSC_OK;
  } catch (const osc::Error& e) {
    g_create_error = e.msg;
    return e.code;
  }
}

OSC_API int osc_surface_x0x1x2(int nx1, int nx2, const double x0x1x2[9], const double rotations[3],
                               const double translation[3], int normal, double* xyz, double* normals, double* x1x2) {
  try {
    if (!x0x1x2) {
      g_create_error = "bad buffers";
      return OSC_ERR_INVALID;
    }
    const double zero[3] = {0, 0, 0};
    osc::surface_x0x1x2(nx1, nx2, V3(x0x1x2), V3(x0x1x2 + 3), V3(x0x1x2 + 6), V3(rotations ? rotations : zero),
                        V3(translation ? translation : zero), normal, xyz, normals, x1x2);
    return OSC_OK;
  } catch (const osc::Error& e) {
    g_create_error = e.msg;
    return e.code;
  } catch (...) {
    g_create_error = "unexpected error";
    return OSC_ERR_INVALID;
  }
}

OSC_API int osc_surface_points(long long n, const double* points, const double* normals, const double rotations[3],
                               const double translation[3], int invert_normals, double* xyz, double* normals_out) {
  if (n < 0 || (n > 0 && (!points || !normals || !xyz || !normals_out))) {
    g_create_error = "bad buffers";
    return OSC_ERR_INVALID;
  }
  const double zero[3] = {0, 0, 0};
  osc::surface_points(n, points, normals, V3(rotations ? rotations : zero), V3(translation ? translation : zero),
                      invert_normals != 0, xyz, normals_out);
  return OSC_OK;
}

OSC_API int osc_flux(osc_ctx* ctx, const double* obs_xyz, long long n_obs, double energy_eV, const osc_rad_opts* opts,
                     double* out, int32_t* level_out, long long* n_not_converged) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (n_obs < 0 || (n_obs > 0 && (!obs_xyz || !out))) throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    osc::RadRequest rq;
    rq.obs = obs_xyz;
    rq.n_obs = n_obs;
    rq.omega = {osc::ev_to_omega(energy_eV)};
    rq.opts = *opts;
    rq.out = out;
    rq.level_out = level_out;
    ctx->eng->radiation(rq);
    if (n_not_converged) *n_not_converged = ctx->eng->last_not_converged;
  });
}

OSC_API int osc_spectrum(osc_ctx* ctx, const double obs[3], const double* energies_eV, long long n_energies,
                         const osc_rad_opts* opts, double* out, int32_t* level_out, long long* n_not_converged) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (!obs || n_energies < 0 || (n_energies > 0 && (!energies_eV || !out))) throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    osc::RadRequest rq;
    rq.obs = obs;
    rq.n_obs = 1;
    rq.omega.resize(n_energies);
    for (long long i = 0; i < n_energies; ++i) rq.omega[i] = osc::ev_to_omega(energies_eV[i]);
    rq.opts = *opts;
    rq.spectrum_current_abs = true;
    rq.out = out;
    rq.level_out = level_out;
    ctx->eng->radiation(rq);
    if (n_not_converged) *n_not_converged = ctx->eng->last_not_converged;
  });
}

// A batch of independent jobs (no reference counterpart: the reference runs one particle and one
// field container per call).  Mixed precision runs all jobs in shared launches; FP64 runs them one
// after another through the single-trajectory path.
// Fields of a batch request (FieldSpec after finish()).
static std::vector<osc::FieldSpec> fields_from_descs(const osc_field_desc* fields, int n_fields) {
  using namespace osc;
  std::vector<FieldSpec> fs;
  for (int i = 0; i < n_fields; ++i) {
    FieldSpec f = field_from_desc(fields + i);
    f.finish();
    fs.push_back(f);
  }
  return fs;
}

// Jobs of a batch request: the ideal particle of a beam with each job's energy and direction
// (TParticleBeam::GetNewParticle), its trajectory range and its observer / energy ranges.
static std::vector<osc::BatchJob> jobs_from_descs(const osc_job_desc* jobs, int n_jobs) {
  using namespace osc;
  std::vector<BatchJob> bj(n_jobs);
  for (int k = 0; k < n_jobs; ++k) {
    const osc_job_desc& d = jobs[k];
    BatchJob& J = bj[k];
    double q = 0, m = 0;
    if (particle_qm(d.particle, d.charge, d.mass, q, m)) throw Error{OSC_ERR_INVALID, "unknown particle type"};
    if (d.particle == OSC_PARTICLE_CUSTOM && (d.mass == 0 || d.charge == 0))
      throw Error{OSC_ERR_INVALID, "'mass' or 'charge' is zero"};
    if (d.energy_GeV < 0) throw Error{OSC_ERR_INVALID, "job energy_GeV must be >= 0"};
    const Vec3 dir = V3(d.d0);
    const Vec3 u0 = mag2(dir) > 0 ? unit(dir) : Vec3{};
    const double e0 = d.energy_GeV < kg_to_gev(m) ? m : d.energy_GeV;
    const double g = e0 / kg_to_gev(m) < 1 ? 1 : e0 / kg_to_gev(m);
    const double b = g != 1 ? std::sqrt(1.0 - 1.0 / (g * g)) : 0;
    J.particle.q = q;
    J.particle.m = m;
    J.particle.current = d.current != 0 ? d.current : q;
    J.particle.set_conditions(V3(d.x0), u0 * b, d.t0);
    J.field_begin = d.field_begin;
    J.field_count = d.field_count;
    J.ctstart = d.ctstart;
    J.ctstop = d.ctstop;
    J.npoints = d.npoints;
    J.obs_begin = d.obs_begin;
    J.n_obs = d.n_obs;
    J.omega_begin = d.energy_begin;
    J.n_e = d.n_energies;
    J.current_abs = d.spectrum != 0;
  }
  return bj;
}

OSC_API int osc_batch_flux(osc_ctx* ctx, const osc_field_desc* fields, int n_fields, const osc_job_desc* jobs,
                           int n_jobs, const double* obs_xyz, long long n_obs, const double* energies_eV,
                           long long n_energies, const osc_rad_opts* opts, int average, double* out,
                           int32_t* level_out, long long* n_not_converged) {
  return guarded(ctx, [&] {
    using namespace osc;
    check_opts(opts);
    if (opts->nparticles != 0) throw Error{OSC_ERR_INVALID, "batch jobs are single particles: nparticles must be 0"};
    if (n_fields < 0 || n_jobs < 0 || n_obs < 0 || n_energies < 0) throw Error{OSC_ERR_INVALID, "negative count"};
    if ((n_fields > 0 && !fields) || (n_jobs > 0 && (!jobs || !out)) || (n_obs > 0 && !obs_xyz) ||
        (n_energies > 0 && !energies_eV))
      throw Error{OSC_ERR_INVALID, "bad buffers"};
    std::vector<FieldSpec> fs = fields_from_descs(fields, n_fields);
    std::vector<double> omega(n_energies);
    for (long long i = 0; i < n_energies; ++i) omega[i] = ev_to_omega(energies_eV[i]);
    std::vector<BatchJob> bj = jobs_from_descs(jobs, n_jobs);
    Engine& E = *ctx->eng;
    if (opts->precision_mode == OSC_MIXED) {
      E.batch(fs, bj, obs_xyz, n_obs, omega.data(), n_energies, *opts, average != 0, out, level_out);
    } else {
      E.batch_fp64(fs, bj, obs_xyz, n_obs, omega.data(), n_energies, *opts, average != 0, out, level_out);
    }
    if (n_not_converged) *n_not_converged = E.last_not_converged;
  });
}

OSC_API int osc_batch_trajectories(osc_ctx* ctx, const osc_field_desc* fields, int n_fields, const osc_job_desc* jobs,
                                   int n_jobs, double* out, long long capacity, long long* npoints_out) {
  return guarded(ctx, [&] {
    using namespace osc;
    if (n_fields < 0 || n_jobs < 0) throw Error{OSC_ERR_INVALID, "negative count"};
    if ((n_fields > 0 && !fields) || (n_jobs > 0 && (!jobs || !out || !npoints_out)))
      throw Error{OSC_ERR_INVALID, "bad buffers"};
    std::vector<FieldSpec> fs = fields_from_descs(fields, n_fields);
    std::vector<BatchJob> bj = jobs_from_descs(jobs, n_jobs);
    std::vector<int64_t> np(n_jobs);
    ctx->eng->batch_trajectories(fs, bj, out, capacity, np.data());
    for (int k = 0; k < n_jobs; ++k) npoints_out[k] = np[k];
  });
}

OSC_API int osc_set_half_period_scale(osc_ctx* ctx, int field_index, const double* scale, long long n) {
  return guarded(ctx, [&] {
    osc::Model& M = ctx->eng->model;
    int idx = field_index;
    if (idx < 0) {
      for (size_t i = 0; i < M.fields.size(); ++i)
        if (!M.fields[i].half_scale.empty()) idx = (int)i;
    }
    if (idx < 0 || idx >= (int)M.fields.size()) throw osc::Error{OSC_ERR_RANGE, "no such field"};
    osc::FieldSpec& f = M.fields[idx];
    if (f.kind != OSC_FIELD_UNDULATOR) throw osc::Error{OSC_ERR_INVALID, "half-period factors apply to undulators"};
    if (!scale || n != 2 * (long long)f.nperiods) throw osc::Error{OSC_ERR_LENGTH, "n must be 2 * nperiods"};
    if ((long long)f.half_scale.size() == n && std::memcmp(f.half_scale.data(), scale, sizeof(double) * n) == 0)
      return;  // the same factors: the trajectory stands
    f.half_scale.assign(scale, scale + n);
    M.knots.clear();
    ++M.knots_version;
  });
}

OSC_API int osc_trajectory_vjp(osc_ctx* ctx, const double* knot_grad, long long n_points, double* grad_half_scale,
                               long long n_half) {
  return guarded(ctx, [&] {
    if (!knot_grad || !grad_half_scale) throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    osc::Model& M = ctx->eng->model;
    M.ensure_trajectory();
    if (n_points != M.knots.n) throw osc::Error{OSC_ERR_LENGTH, "n_points differs from the trajectory's"};
    ctx->eng->trajectory_vjp(knot_grad, grad_half_scale, n_half);
  });
}

OSC_API int osc_flux_vjp(osc_ctx* ctx, const double* obs_xyz, long long n_obs, const double* energies_eV,
                         long long n_energies, int level, const osc_rad_opts* opts, int spectrum,
                         const double* grad_flux, double* flux_out, double* grad_half_scale, long long n_half,
                         double* grad_knots) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (opts->nparticles != 0) throw osc::Error{OSC_ERR_INVALID, "the adjoint is for one particle: nparticles must be 0"};
    if (n_obs < 1 || n_energies < 1 || !obs_xyz || !energies_eV || (grad_flux ? !grad_half_scale : !flux_out))
      throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    std::vector<double> omega(n_energies);
    for (long long i = 0; i < n_energies; ++i) omega[i] = osc::ev_to_omega(energies_eV[i]);
    ctx->eng->flux_vjp(obs_xyz, n_obs, omega, level, *opts, spectrum != 0, grad_flux, flux_out, grad_half_scale,
                       n_half, grad_knots);
  });
}

OSC_API int osc_flux_multi(osc_ctx* ctx, const double* obs_xyz, long long n_obs, const double* energies_eV,
                           long long n_energies, const osc_rad_opts* opts, int spectrum, double* out,
                           int32_t* level_out, long long* n_not_converged) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (n_obs < 0 || n_energies < 0 || (n_obs > 0 && n_energies > 0 && (!obs_xyz || !energies_eV || !out)))
      throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    osc::RadRequest rq;
    rq.obs = obs_xyz;
    rq.n_obs = n_obs;
    rq.omega.resize(n_energies);
    for (long long i = 0; i < n_energies; ++i) rq.omega[i] = osc::ev_to_omega(energies_eV[i]);
    rq.opts = *opts;
    rq.spectrum_current_abs = spectrum != 0;
    rq.out = out;
    rq.level_out = level_out;
    ctx->eng->radiation(rq);
    if (n_not_converged) *n_not_converged = ctx->eng->last_not_converged;
  });
}

OSC_API int osc_power_density(osc_ctx* ctx, const double* obs_xyz, const double* normals, long long n_obs,
                              int directional, const osc_rad_opts* opts, double* out, int32_t* level_out,
                              long long* n_not_converged) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (n_obs < 0 || (n_obs > 0 && (!obs_xyz || !out))) throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    osc::RadRequest rq;
    rq.power_density = true;
    rq.obs = obs_xyz;
    rq.normals = normals;
    rq.n_obs = n_obs;
    rq.directional = directional != 0;
    rq.opts = *opts;
    rq.out = out;
    rq.level_out = level_out;
    ctx->eng->radiation(rq);
    if (n_not_converged) *n_not_converged = ctx->eng->last_not_converged;
  });
}

OSC_API int osc_power_density_stl(osc_ctx* ctx, const double* facets, const double* centers, long long n,
                                  const osc_rad_opts* opts, double* out, int32_t* level_out,
                                  long long* n_not_converged) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (n < 0 || (n > 0 && (!facets || !centers || !out))) throw osc::Error{OSC_ERR_INVALID, "bad buffers"};
    ctx->eng->power_density_stl(facets, centers, n, *opts, out, level_out);
    if (n_not_converged) *n_not_converged = ctx->eng->last_not_converged;
  });
}

OSC_API int osc_flux_device(osc_ctx* ctx, const double* d_obs_xyz, long long n_obs, double energy_eV,
                            const osc_rad_opts* opts, double* d_out, int32_t* d_level, void* stream) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (opts->nparticles != 0) throw osc::Error{OSC_ERR_INVALID, "device-resident calls take one particle"};
    osc::RadRequest rq;
    rq.obs = d_obs_xyz;
    rq.obs_on_device = true;
    rq.n_obs = n_obs;
    rq.omega = {osc::ev_to_omega(energy_eV)};
    rq.opts = *opts;
    rq.out = d_out;
    rq.level_out = d_level;
    rq.out_on_device = true;
    rq.stream = static_cast<cudaStream_t>(stream);
    ctx->eng->radiation(rq);
  });
}

OSC_API int osc_power_density_device(osc_ctx* ctx, const double* d_obs_xyz, const double* d_normals, long long n_obs,
                                     int directional, const osc_rad_opts* opts, double* d_out, int32_t* d_level,
                                     void* stream) {
  return guarded(ctx, [&] {
    check_opts(opts);
    if (opts->nparticles != 0) throw osc::Error{OSC_ERR_INVALID, "device-resident calls take one particle"};
    osc::RadRequest rq;
    rq.power_density = true;
    rq.obs = d_obs_xyz;
    rq.normals = d_normals;
    rq.obs_on_device = true;
    rq.n_obs = n_obs;
    rq.directional = directional != 0;
    rq.opts = *opts;
    rq.out = d_out;
    rq.level_out = d_level;
    rq.out_on_device = true;
    rq.stream = static_cast<cudaStream_t>(stream);
    ctx->eng->radiation(rq);
  });
}

OSC_API int osc_last_stats(osc_ctx* ctx, long long* samples, long long* launches) {
  return guarded(ctx, [&] {
    ctx->eng->collect();
    if (samples) *samples = ctx->eng->last_samples;
    if (launches) *launches = ctx->eng->last_launches;
  });
}

OSC_API int osc_set_beam_batch_threshold(osc_ctx* ctx, int particles) {
  return guarded(ctx, [&] {
    if (particles < 1) throw osc::Error{OSC_ERR_RANGE, "the threshold must be at least 1 particle"};
    ctx->eng->beam_batch_min = particles;
  });
}

OSC_API int osc_set_batch_spline_kernel(osc_ctx* ctx, int kernel) {
  return guarded(ctx, [&] {
    if (kernel < 0 || kernel > 2) throw osc::Error{OSC_ERR_RANGE, "kernel must be 0, 1 or 2"};
    ctx->eng->spline_kernel = kernel;
  });
}

OSC_API int osc_set_profiling(osc_ctx* ctx, int enable) {
  return guarded(ctx, [&] { ctx->eng->profiling = enable != 0; });
}

OSC_API int osc_get_profile(osc_ctx* ctx, double* kernel_ms, long long* launches, long long* samples, int reset) {
  return guarded(ctx, [&] {
    osc::Engine& E = *ctx->eng;
    E.collect();
    if (kernel_ms) *kernel_ms = E.prof_ms;
    if (launches) *launches = E.prof_launches;
    if (samples) *samples = E.prof_samples;
    if (reset) { E.prof_ms = 0; E.prof_launches = 0; E.prof_samples = 0; }
  });
}

static int n_variants_of(int kind) {
  return kind == 3 ? osc::kBatchVariants : kind == 2 ? osc::kMixedVariants : osc::kFp64Variants;
}

OSC_API int osc_set_variant(osc_ctx* ctx, int kind, int variant) {
  return guarded(ctx, [&] {
    if (kind != 0 && kind != 2 && kind != 3)
      throw osc::Error{OSC_ERR_INVALID, "kind must be 0 (fp64), 2 (mixed) or 3 (batched mixed)"};
    if (variant < -1 || variant >= n_variants_of(kind)) throw osc::Error{OSC_ERR_RANGE, "variant out of range"};
    ctx->eng->forced_variant[kind] = variant;
  });
}

OSC_API int osc_get_variant(osc_ctx* ctx, int kind, int* variant, int* n_variants) {
  return guarded(ctx, [&] {
    if (kind != 0 && kind != 2 && kind != 3)
      throw osc::Error{OSC_ERR_INVALID, "kind must be 0 (fp64), 2 (mixed) or 3 (batched mixed)"};
    if (variant) *variant = ctx->eng->variant_in_use(kind);
    if (n_variants) *n_variants = n_variants_of(kind);
  });
}

OSC_API int osc_variant_name(int kind, int variant, char* name, long long capacity) {
  try {
    if (kind != 0 && kind != 2 && kind != 3)
      throw osc::Error{OSC_ERR_INVALID, "kind must be 0 (fp64), 2 (mixed) or 3 (batched mixed)"};
    if (variant < 0 || variant >= n_variants_of(kind)) throw osc::Error{OSC_ERR_RANGE, "variant out of range"};
    static const char* const kFp64[] = {"k_fd_wave_fp64<1,7>", "k_fd_wave_fp64<2,7>", "k_fd_wave_fp64<4,7>",
                                        "k_fd_wave_fp64<4,5>"};
    static const char* const kBatch[] = {"k_batch_wave<4,4>", "k_batch_wave<4,1>", "k_batch_wave<2,4>",
                                         "k_batch_wave<1,4>"};
    static_assert(sizeof(kFp64) / sizeof(kFp64[0]) == osc::kFp64Variants, "FP64 variant names");
    static_assert(sizeof(kBatch) / sizeof(kBatch[0]) == osc::kBatchVariants, "batch variant names");
    const char* n = kind == 0 ? kFp64[variant] : kind == 2 ? osc::mixed_variant_name(variant) : kBatch[variant];
    if (!name || capacity <= (long long)std::strlen(n)) throw osc::Error{OSC_ERR_LENGTH, "name buffer too small"};
    std::strcpy(name, n);
    return OSC_OK;
  } catch (const osc::Error& e) {
    g_create_error = e.msg;
    return e.code;
  }
}

OSC_API int osc_drop_level_cache(osc_ctx* ctx) {
  return guarded(ctx, [&] { ctx->eng->drop_level_cache(); });
}

OSC_API int osc_measure_fma_peak(osc_ctx* ctx, int kind, double* tflops) {
  return guarded(ctx, [&] {
    const double v = ctx->eng->measure_fma_peak(kind);
    if (tflops) *tflops = v;
  });
}

}  // extern "C"
