/*
 * oscars_b200.h -- C ABI of the B200 (sm_100a) implementation of the OSCARS radiation hot path.
 *
 * Plain C types, caller-owned buffers, an int status return on every call (0 = OSC_OK, never an
 * exception across the boundary), one osc_ctx per host thread.  osc_last_error() gives the message
 * for the last non-zero status, worded like the reference's ValueError texts.
 *
 * The reference GPU seam these entry points replace is include/OSCARSSR_Cuda.h:28-66
 * (OSCARSSR_Cuda_CalculateFluxGPU / _CalculateSpectrumGPU / _CalculatePowerDensityGPU /
 * _GetDeviceCount), called from OSCARSSR::Calculate*GPU (src/OSCARSSR.cc:2429, 3125, 4428).
 * Those take C++ references to OSCARSSR, TSurfacePoints and the result containers; here the same
 * information crosses as plain arrays and descriptors, and the simulation state (fields, beam,
 * trajectory) lives in the osc_ctx.
 */
#ifndef OSCARS_B200_H
#define OSCARS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OSC_API __attribute__((visibility("default")))

/* Status codes.  The reference maps std::length_error / out_of_range / invalid_argument to
 * ValueError (src/OSCARSSR_Python.cc:5892-5915); the three are kept apart here. */
enum osc_status {
  OSC_OK = 0,
  OSC_ERR_INVALID = 1,      /* std::invalid_argument in the reference */
  OSC_ERR_RANGE = 2,        /* std::out_of_range */
  OSC_ERR_LENGTH = 3,       /* std::length_error */
  OSC_ERR_STATE = 4,        /* call order (no beam, no trajectory ...) */
  OSC_ERR_CUDA = 5,         /* a CUDA runtime call failed; message has the CUDA error string */
  OSC_ERR_NO_DEVICE = 6,    /* no usable sm_100 device */
  OSC_ERR_ALLOC = 7,        /* device or host allocation failed */
  OSC_ERR_TIMEOUT = 8       /* a bounded device-side wait gave up */
};

enum osc_field_kind { OSC_FIELD_UNDULATOR = 0, OSC_FIELD_EPU = 1, OSC_FIELD_GRID = 2 };

/* Particle types of TParticleA::SetParticleType (src/TParticleA.cc:78-121). */
enum osc_particle_type {
  OSC_PARTICLE_ELECTRON = 0, OSC_PARTICLE_POSITRON = 1, OSC_PARTICLE_MUON = 2,
  OSC_PARTICLE_ANTIMUON = 3, OSC_PARTICLE_PROTON = 4, OSC_PARTICLE_ANTIPROTON = 5,
  OSC_PARTICLE_PIPLUS = 6, OSC_PARTICLE_PIMINUS = 7, OSC_PARTICLE_CUSTOM = 8
};

/* Beam distributions, TParticleBeam_BeamDistribution order (include/TParticleBeam.h). */
enum osc_distribution { OSC_DIST_DEFAULT = -1, OSC_DIST_FILAMENT = 1, OSC_DIST_GAUSSIAN = 2, OSC_DIST_KV = 3 };

/* Polarization selectors (string matching of src/OSCARSSR.cc:4129-4150 is done by the caller). */
enum osc_polarization { OSC_POL_ALL = 0, OSC_POL_LH = 1, OSC_POL_LV = 2, OSC_POL_LINEAR = 3,
                        OSC_POL_CL = 4, OSC_POL_CR = 5 };

/* Quantity returned per entry, src/OSCARSSR_Python.cc:5865-5875 ('flux', 'precision', 'level'). */
enum osc_quantity { OSC_Q_VALUE = 0, OSC_Q_PRECISION = 1, OSC_Q_LEVEL = 2 };

/* Arithmetic of the radiation integral. */
enum osc_precision_mode {
  OSC_FP64 = 0,   /* the reference's FP64 method; matches the reference CPU path to <= 1e-9 */
  OSC_MIXED = 1   /* FP64 trajectory and retarded phase, FP32 amplitudes, sincos and sums */
};

typedef struct osc_ctx osc_ctx;

typedef struct {
  int kind;                 /* osc_field_kind */
  double bfield[3];         /* peak field [T] (EPU: field A) */
  double bfield_b[3];       /* EPU field B [T]; ignored for the undulator */
  double period[3];         /* period vector [m]: magnitude = period, direction = axis */
  int nperiods;
  double center[3];         /* translation [m] */
  double phase;             /* [rad] */
  double taper;             /* [1/m] */
  double frequency;         /* [Hz], 0 = static */
  double frequency_phase;   /* [rad] */
  double time_offset;       /* [s] */
  /* OSC_FIELD_UNDULATOR, optional: amplitude factor of each of the 2 * nperiods half-periods of the
   * full-strength region between the end poles (NULL / 0 = all 1). */
  const double* half_period_scale;
  int n_half_periods;
  /* OSC_FIELD_GRID (TField3D_Grid, src/TField3D_Grid.cc:153-283): grid_n points per axis from
   * grid_start in steps grid_step; grid_values holds 3 field components per point at index
   * ix * ny * nz + iy * nz + iz; `rotations` rotate the values on load and the evaluation point
   * before `center` (the translation) is subtracted; time factor
   * cos(2 pi frequency (t + time_offset) + frequency_phase). */
  long long grid_n[3];
  double grid_start[3];
  double grid_step[3];
  const double* grid_values;
  double rotations[3];
} osc_field_desc;

typedef struct {
  int particle;             /* osc_particle_type */
  double charge, mass;      /* [C], [kg]; custom particles only */
  double energy_GeV;        /* -1 = not given (the binding default) */
  double x0[3];             /* initial position [m] (already rotated/translated) */
  double d0[3];             /* direction (already rotated) */
  double horizontal[3];     /* horizontal direction before normalisation, see add_particle_beam */
  double t0;                /* [m] */
  double current;           /* [A]; 0 = use the particle charge (TParticleA::SetCurrent) */
  double sigma_energy_GeV;
  double emittance[2];
  int has_emittance;
  double beta[2], alpha[2];
  int has_beta, has_alpha;
  double eta[2];
  int distribution;         /* osc_distribution */
  double ctstartstop[2];
  int has_ctstartstop;
  /* Twiss gamma and the lattice reference point of the Twiss values (add_particle_beam's 'gamma',
   * 'lattice_reference'); any two of beta / alpha / gamma (or all three) define the optics. */
  double gamma[2];
  int has_gamma;
  double lattice_reference[3];
  int has_lattice_reference;
  int predefined;           /* osc_predefined_beam: 0 none, else TParticleBeam::SetPredefinedBeam */
  int has_d0;               /* predefined beams: d0 given (replaces the beam's direction) */
  double weight;            /* share of the particles drawn from this beam (> 0; 0 counts as 1) */
} osc_beam_desc;

/* Predefined beams of TParticleBeam::SetPredefinedBeam (src/TParticleBeam.cc:135-206). */
typedef enum {
  OSC_BEAM_NONE = 0,
  OSC_BEAM_NSLSII = 1,
  OSC_BEAM_NSLSII_LONGSTRAIGHT = 2,
  OSC_BEAM_NSLSII_SHORTSTRAIGHT = 3
} osc_predefined_beam;

typedef struct {
  int polarization;         /* osc_polarization */
  double angle;             /* [rad], OSC_POL_LINEAR */
  double horizontal[3];     /* horizontal_direction, default (1,0,0) */
  double propagation[3];    /* propogation_direction, default (0,0,1) */
  double precision;         /* relative convergence target, default 0.01 */
  int max_level;            /* default -2 (= 26) */
  int max_level_extended;   /* default 0 */
  int nparticles;           /* 0 = the current particle; N = N random particles, weight 1/N */
  int quantity;             /* osc_quantity */
  int precision_mode;       /* osc_precision_mode */
  /* Multi-particle requests split over processes (no reference counterpart): with shard_count > 1
   * all N particles are still drawn in order, but only those with index % shard_count == shard_rank
   * are integrated, each with weight 1/N, so the shards' outputs add up to the whole request (one
   * all-reduce).  0 / 0 (or 0 / 1) = the whole request. */
  int shard_rank;
  int shard_count;
} osc_rad_opts;

/* ---- device / context ---------------------------------------------------------------------- */
/* Replaces OSCARSSR_Cuda_GetDeviceCount (include/OSCARSSR_Cuda.h:66). */
OSC_API int osc_get_device_count(int* count);
/* device -1 creates a host-only context (fields, beam, trajectory, surfaces; radiation calls
 * return OSC_ERR_NO_DEVICE).  On failure osc_last_error(NULL) has the reason. */
OSC_API int osc_ctx_create(int device, osc_ctx** out);
OSC_API void osc_ctx_destroy(osc_ctx* ctx);
OSC_API const char* osc_last_error(const osc_ctx* ctx);
OSC_API const char* osc_version(void);

/* ---- fields: OSCARSSR::AddMagneticField (src/OSCARSSR.cc:157-169) with TField3D_IdealUndulator
 *      (src/TField3D_IdealUndulator.cc:113-152) and TField3D_IdealEPU (src/TField3D_IdealEPU.cc:116-170) */
OSC_API int osc_clear_fields(osc_ctx* ctx);
OSC_API int osc_add_field(osc_ctx* ctx, const osc_field_desc* field);
OSC_API int osc_get_bfield(osc_ctx* ctx, const double x[3], double t, double out[3]);
/* add_bfield_file: OSCARSSR::AddMagneticField(FileName, Format, ...) (src/OSCARSSR.cc:70-103) with
 * the TField3D_Grid readers for the 'OSCARS' (src/TField3D_Grid.cc:365-530) and 'OSCARS1D ...'
 * (:572-870) text formats; scaling may be NULL (n_scaling 0). */
OSC_API int osc_add_field_file(osc_ctx* ctx, const char* path, const char* format, const double rotations[3],
                               const double translation[3], const double* scaling, int n_scaling,
                               double frequency, double frequency_phase, double time_offset);

/* ---- beam: set_particle_beam (src/OSCARSSR_Python.cc:3561-3576, 3699-4100) ------------------ */
OSC_API int osc_set_beam(osc_ctx* ctx, const osc_beam_desc* beam);
OSC_API int osc_set_seed(osc_ctx* ctx, int seed);                 /* TRandomA::SetSeed */
/* Several beams (OSCARSSR::AddParticleBeam, binding src/OSCARSSR_Python.cc:3699-4100): append a beam
 * named `name` ("" = "_beam<k>", k the beams held; a repeated name is refused).  Each new random
 * particle comes from a beam picked by weight; adding the first beam makes its ideal particle the
 * current one.  osc_set_beam is osc_clear_beams followed by osc_add_beam with name "". */
OSC_API int osc_add_beam(osc_ctx* ctx, const osc_beam_desc* beam, const char* name);
OSC_API int osc_clear_beams(osc_ctx* ctx);
/* OSCARSSR::SetNewParticle(beam, "ideal" or random) (src/OSCARSSR.cc:510-524): beam "" picks one by
 * weight. */
OSC_API int osc_set_new_particle_of_beam(osc_ctx* ctx, const char* beam, int ideal);
OSC_API int osc_set_new_particle(osc_ctx* ctx, int ideal);         /* OSCARSSR::SetNewParticle */
OSC_API int osc_get_particle(osc_ctx* ctx, double x0[3], double beta0[3], double* t0, double* gamma);
/* Draw n particles from the beam exactly as a request with nparticles = n does (advancing the
 * context's random sequence the same way) and return those of shard shard_rank of shard_count
 * (index % shard_count == shard_rank): 6 doubles each (x0[3] [m], beta0[3]) in out, their number in
 * *n_out (out must hold 6 * ceil(n / shard_count) doubles).  Works on host-only contexts. */
OSC_API int osc_beam_particles(osc_ctx* ctx, long long n, int shard_rank, int shard_count, double* out,
                               long long* n_out);
OSC_API int osc_set_ctstartstop(osc_ctx* ctx, double start, double stop);       /* :637-647 */
OSC_API int osc_get_ctstartstop(osc_ctx* ctx, double* start, double* stop);
OSC_API int osc_set_npoints_trajectory(osc_ctx* ctx, long long n);
OSC_API int osc_get_npoints_trajectory(osc_ctx* ctx, long long* n);
/* Trajectory method (OSCARSSR::SetTrajectoryCalculation, src/OSCARSSR.cc:784-820): "RK4" (fixed
 * step; precision must be -1) or "RKAS" (adaptive Cash-Karp, src/OSCARSSR.cc:1015-1072 and
 * 1392-1618; precision > 0, or -1 to keep the current one, default 1e-6).  Case-insensitive. */
OSC_API int osc_set_trajectory_calculation(osc_ctx* ctx, const char* method, double precision);
/* method_out: 0 RK4, 1 RKAS. */
OSC_API int osc_get_trajectory_calculation(osc_ctx* ctx, int* method_out, double* precision_out);

/* ---- trajectory: OSCARSSR::CalculateTrajectory (src/OSCARSSR.cc:853-1009) -------------------- */
OSC_API int osc_calculate_trajectory(osc_ctx* ctx);
/* out: 10 x n SoA (t, x, y, z, beta_x, beta_y, beta_z, a_x/c, a_y/c, a_z/c); n_out = points. */
OSC_API int osc_get_trajectory(osc_ctx* ctx, double* out, long long capacity, long long* n_out);

/* Use a trajectory computed elsewhere -- e.g. by the reference's own host code through any of its
 * field types -- for the radiation calls that follow: the particle (osc_particle_type, custom charge
 * [C] and mass [kg], current [A], initial position x0 [m], beta0 and t0 [m] -- what TParticleA holds)
 * and its trajectory as 10 x n SoA (t [s], x y z [m], beta, a/c [1/s]; the layout of
 * osc_get_trajectory), times strictly increasing, n >= 3.  The clamped spline is computed here as for
 * an RK4 trajectory (include/TOMATH.h:141-203).  This is what the reference's GPU seam receives
 * through OSCARSSR& (src/OSCARSSR_Cuda.cu:609-614 reads OSR's current particle and trajectory). */
OSC_API int osc_set_particle_trajectory(osc_ctx* ctx, int particle, double charge, double mass, double current,
                                        const double x0[3], const double beta0[3], double t0, const double* traj,
                                        long long n);
/* Replaces OSCARSSR_Cuda_GetDeviceProperties (include/OSCARSSR_Cuda.h:30): a one-line description of
 * device `device` (name, compute capability, multiprocessors, memory), NUL-terminated into out.
 * Errors go to osc_last_error(NULL). */
OSC_API int osc_get_device_properties(int device, char* out, long long capacity);

/* ---- observation surfaces: TSurfacePoints_Rectangle::Init/GetXYZ/GetX1/GetX2
 *      (src/TSurfacePoints_Rectangle.cc:140-315).  Any pointer may be NULL. */
OSC_API int osc_surface_rectangle(const char* plane, int nx1, int nx2, double width1,
                                  double width2, const double rotations[3],
                                  const double translation[3], int normal, double* xyz,
                                  double* normals, double* x1x2);

/* Rectangle from three points (TSurfacePoints_Rectangle::Init(NX1, NX2, X0, X1, X2, Normal),
 * src/TSurfacePoints_Rectangle.cc:76-127; GetXYZ / GetX1 / GetX2, :280-317): x0x1x2 = X0, X1, X2 (9
 * doubles), rotated (RotateSelfXYZ) and translated first as the binding does
 * (src/OSCARSSR_Python.cc:6652-6658); nx1, nx2 >= 2 (the reference divides by nx - 1).  Pointers
 * other than x0x1x2 may be NULL. */
OSC_API int osc_surface_x0x1x2(int nx1, int nx2, const double x0x1x2[9], const double rotations[3],
                               const double translation[3], int normal, double* xyz, double* normals, double* x1x2);
/* Arbitrary points with normals as the point-list calls take them (calculate_flux,
 * src/OSCARSSR_Python.cc:7730-7750; calculate_power_density, :6225-6250): each point and normal
 * rotated (RotateSelfXYZ), the normal reversed when invert_normals (calculate_power_density with
 * normal = -1), the point translated.  3 x n doubles in and out. */
OSC_API int osc_surface_points(long long n, const double* points, const double* normals, const double rotations[3],
                               const double translation[3], int invert_normals, double* xyz, double* normals_out);

/* ---- radiation: host buffers in and out; results are written (not accumulated). -------------
 * osc_flux          replaces OSCARSSR_Cuda_CalculateFluxGPU         (src/OSCARSSR_Cuda.cu:516)
 * osc_spectrum      replaces OSCARSSR_Cuda_CalculateSpectrumGPU     (src/OSCARSSR_Cuda.cu:1607)
 * osc_power_density replaces OSCARSSR_Cuda_CalculatePowerDensityGPU (src/OSCARSSR_Cuda.cu:2678)
 * out[i] is the value selected by opts->quantity; level_out (may be NULL) gets the stop level,
 * -1 for entries that did not converge; *n_not_converged (may be NULL) counts those.
 * Any host buffers are accepted; page-locked ones (cudaHostAlloc / cudaHostRegister) make the
 * upload of the inputs and the download of the results faster. */
OSC_API int osc_flux(osc_ctx* ctx, const double* obs_xyz, long long n_obs, double energy_eV,
                     const osc_rad_opts* opts, double* out, int32_t* level_out,
                     long long* n_not_converged);
OSC_API int osc_spectrum(osc_ctx* ctx, const double obs[3], const double* energies_eV,
                         long long n_energies, const osc_rad_opts* opts, double* out,
                         int32_t* level_out, long long* n_not_converged);
/* Flux of every (observer, energy) pair in one request (no reference counterpart: the reference
 * computes one energy per calculate_flux call or one observer per calculate_spectrum call).  out has
 * n_obs x n_energies values, observer-major with energies fastest; spectrum = 1 normalises like
 * osc_spectrum (|current|), 0 like osc_flux. */
OSC_API int osc_flux_multi(osc_ctx* ctx, const double* obs_xyz, long long n_obs, const double* energies_eV,
                           long long n_energies, const osc_rad_opts* opts, int spectrum, double* out,
                           int32_t* level_out, long long* n_not_converged);
OSC_API int osc_power_density(osc_ctx* ctx, const double* obs_xyz, const double* normals,
                              long long n_obs, int directional, const osc_rad_opts* opts,
                              double* out, int32_t* level_out, long long* n_not_converged);
/* Power density on the facets of STL meshes (replaces OSCARSSR::CalculatePowerDensitySTL,
 * src/OSCARSSR.cc:3154-3521, behind OSCARSSR_Python.cc:6993 calculate_power_density_stl).
 * facets: n x 12 doubles = vertices A, B, C and the normal as stored; centers: n x 3 (the facet
 * centres, each the mean of its vertices before the mesh was translated, then translated).  For
 * every facet the trajectory samples whose ray to the centre crosses another facet are skipped.
 * out / level_out: n values / stop levels; a facet that does not stop reports the level of the last
 * facet before it that did (the reference's Result_Level), counted in n_not_converged.  opts: the
 * precision, levels, nparticles and quantity fields are used. */
OSC_API int osc_power_density_stl(osc_ctx* ctx, const double* facets, const double* centers, long long n,
                                  const osc_rad_opts* opts, double* out, int32_t* level_out,
                                  long long* n_not_converged);

/* ---- batches of independent jobs (no reference counterpart: the reference integrates one
 *      particle through one field container per call).  Job k is the ideal particle of a beam of
 *      `particle` at energy_GeV, starting at x0 along d0 at t0, through fields
 *      [field_begin, field_begin + field_count) of `fields`, tracked over [ctstart, ctstop] with
 *      npoints RK4 points, and observed at observers [obs_begin, obs_begin + n_obs) of obs_xyz and
 *      energies [energy_begin, energy_begin + n_energies) of energies_eV. */
typedef struct {
  int field_begin, field_count;
  int particle;             /* osc_particle_type */
  double charge, mass;      /* [C], [kg]; custom particles only */
  double energy_GeV;
  double x0[3];             /* [m] */
  double d0[3];             /* direction */
  double t0;                /* [m] */
  double current;           /* [A]; 0 = the particle charge */
  double ctstart, ctstop;   /* [m] */
  long long npoints;
  long long obs_begin, n_obs;
  long long energy_begin, n_energies;
  int spectrum;             /* 1: normalised like osc_spectrum (|current|), 0: like osc_flux */
} osc_job_desc;

/* opts->precision_mode OSC_MIXED integrates all jobs in shared launches (trajectories, splines
 * and level samples on the device; the waves up to level 13 replayed from a CUDA graph once a
 * shape is known); OSC_FP64 runs the jobs one after another through osc_flux's FP64 path.
 * opts->nparticles must be 0.  out: with average == 0, every job's n_obs x n_energies values in
 * job order (observer-major, energy fastest); with average != 0, the jobs (which must then share
 * observers and energies) are averaged with weight 1/n_jobs in job order -- a multi-particle beam.
 * level_out (may be NULL) has the same layout (the last job's levels when averaging). */
OSC_API int osc_batch_flux(osc_ctx* ctx, const osc_field_desc* fields, int n_fields,
                           const osc_job_desc* jobs, int n_jobs, const double* obs_xyz,
                           long long n_obs, const double* energies_eV, long long n_energies,
                           const osc_rad_opts* opts, int average, double* out,
                           int32_t* level_out, long long* n_not_converged);

/* The jobs' trajectories exactly as the batched mixed path integrates them on the device (its RK4
 * and spline kernels; no reference counterpart -- it exists to compare the device integration with
 * the host's, which follows src/OSCARSSR.cc:910-1009 bit for bit).  Per job, in job order, 19 x n
 * doubles: t [s]; x, y, z [m]; beta_x, beta_y, beta_z; a_x/c, a_y/c, a_z/c [1/s]; then the 9 clamped-
 * spline second derivatives of those components (include/TOMATH.h:141-203), each a row of n values.
 * npoints_out[k] = n of job k (npoints or npoints + 1, as the reference's step count gives it); out
 * must hold 19 x the sum of those (19 x (npoints + 2) per job is always enough).  The jobs' observer
 * and energy ranges are ignored. */
OSC_API int osc_batch_trajectories(osc_ctx* ctx, const osc_field_desc* fields, int n_fields, const osc_job_desc* jobs,
                                   int n_jobs, double* out, long long capacity, long long* npoints_out);

/* ---- differentiation (no reference counterpart: the reference has no gradients) ------------
 * osc_set_half_period_scale replaces the half-period amplitude factors of field `field_index`
 * (an undulator added with them; -1 = the one field that has them) and drops the trajectory (the
 * same factors again leave it in place).
 * osc_flux_vjp computes, at the fixed level `level` (all samples of levels 0..level, no stop rule),
 * the flux F of every (observer, energy) entry -- the value osc_flux / osc_spectrum return with
 * precision 0 and max_level = level -- and grad_half_scale = (dF/ds)^T grad_flux, the gradient of any
 * loss with dLoss/dF = grad_flux with respect to those factors, by reverse mode through the
 * radiation sum, the trajectory spline and the RK4 steps.  opts->precision_mode selects the
 * arithmetic of the radiation part: OSC_FP64, or OSC_MIXED (the mixed path's sums and an FP32
 * reverse sweep with the FP64 phase of each pair of samples); the RK4 part is FP64 either way and
 * recomputes the trajectory states from checkpoints every 256 steps, its reverse pass parallel in
 * time over 64-step segments joined by their 6 x 6 Jacobians.
 * grad_flux may be NULL: the call then computes flux_out only and keeps the entry sums, which a
 * following call on the same trajectory, observers, energies, level and arithmetic reuses (a
 * forward pass followed by its backward pass computes the sums once).
 * Entries are observer-major with energies fastest; spectrum = 1 normalises like osc_spectrum.
 * grad_knots (may be NULL) receives the gradient with respect to the trajectory knots (9 x n_points,
 * the layout of osc_trajectory_vjp's knot_grad).
 * Polarization 'all' only; ideal undulator / EPU fields only; opts->nparticles must be 0. */
OSC_API int osc_set_half_period_scale(osc_ctx* ctx, int field_index, const double* scale, long long n);
/* Gradient of sum_j knot_grad . knot_j (knot_grad: 9 x n_points, the layout of osc_get_trajectory
 * without its time row) with respect to the half-period factors: the trajectory part of the adjoint
 * on its own (reverse mode through the RK4 steps). */
OSC_API int osc_trajectory_vjp(osc_ctx* ctx, const double* knot_grad, long long n_points,
                               double* grad_half_scale, long long n_half);
OSC_API int osc_flux_vjp(osc_ctx* ctx, const double* obs_xyz, long long n_obs, const double* energies_eV,
                         long long n_energies, int level, const osc_rad_opts* opts, int spectrum,
                         const double* grad_flux, double* flux_out, double* grad_half_scale,
                         long long n_half, double* grad_knots);

/* ---- device-resident variants: same arithmetic, pointers are device memory on the context's
 *      device, work is queued on `stream` (a cudaStream_t, NULL = the context's stream) and the
 *      call returns without synchronising.  Single particle (opts->nparticles must be 0).  The
 *      queued work reads the inputs in place: keep them unchanged until it has run. */
OSC_API int osc_flux_device(osc_ctx* ctx, const double* d_obs_xyz, long long n_obs,
                            double energy_eV, const osc_rad_opts* opts, double* d_out,
                            int32_t* d_level, void* stream);
OSC_API int osc_power_density_device(osc_ctx* ctx, const double* d_obs_xyz,
                                     const double* d_normals, long long n_obs, int directional,
                                     const osc_rad_opts* opts, double* d_out, int32_t* d_level,
                                     void* stream);

/* Number of trajectory samples integrated by the last radiation call (sum over entries and
 * particles of 2^(L+1)-1 for stop level L), and the number of kernel launches it made. */
OSC_API int osc_last_stats(osc_ctx* ctx, long long* samples, long long* launches);

/* Profiling: when enabled, every sample-integration kernel launch is bracketed by CUDA events on
 * its stream (for batches -- osc_batch_flux and multi-particle mixed requests -- each chunk of jobs
 * from its first kernel to its last, trajectories included); osc_get_profile returns the summed
 * device time [ms] of those intervals since the last reset, their number, and the samples they
 * integrated (reset = 1 clears the counters). */
OSC_API int osc_set_profiling(osc_ctx* ctx, int enable);
OSC_API int osc_get_profile(osc_ctx* ctx, double* kernel_ms, long long* launches, long long* samples,
                            int reset);
/* Kernel variants of the sample sums.  kind 0 = FP64 flux/spectrum, 2 = mixed flux/spectrum,
 * 3 = batched mixed (osc_batch_flux and multi-particle mixed requests; tuned on the first wave).
 * variant >= 0 forces a compiled variant; -1 (default) lets the context autotune: the first call
 * of each request shape times every variant and keeps the fastest.  osc_get_variant reports the
 * variant the last request of that kind used and the number of compiled variants. */
OSC_API int osc_set_variant(osc_ctx* ctx, int kind, int variant);
OSC_API int osc_get_variant(osc_ctx* ctx, int kind, int* variant, int* n_variants);
/* Name of compiled variant `variant` of kind 0, 2 or 3: the kernel and its template arguments
 * (e.g. "k_fd_wave_mixed_pair<4,4>"), NUL-terminated into name[capacity].  No context; errors go
 * to osc_last_error(NULL).  No counterpart in the reference (it has one kernel per quantity). */
OSC_API int osc_variant_name(int kind, int variant, char* name, long long capacity);
/* Multi-particle compute='mixed' flux / spectrum requests whose share of particles reaches
 * `particles` (default 1024) run as one batch with device RK4 trajectories (the route of
 * osc_batch_flux); smaller ones integrate each particle's trajectory on host worker threads and sum
 * it with the single-trajectory mixed kernels, as the FP64 path does.  Both routes give the same
 * results to rounding; 1 forces the batch, a large value the per-particle route.  No counterpart in
 * the reference. */
OSC_API int osc_set_beam_batch_threshold(osc_ctx* ctx, int particles);
/* Spline kernel of the batched trajectories: 0 (default) picks per chunk, 1 the serial sweeps (one
 * thread per job and component: the latency of the longest trajectory), 2 the block-parallel sweeps
 * (the chunk's total work).  Both solve the same system to rounding. */
OSC_API int osc_set_batch_spline_kernel(osc_ctx* ctx, int kernel);
/* Drop the device-side level-sample cache (it is rebuilt by the next radiation call). */
OSC_API int osc_drop_level_cache(osc_ctx* ctx);
/* Measured arithmetic peak of this GPU: an FMA-throughput loop in FP64 (kind 0) or FP32 (kind 1),
 * returned in TFLOP/s counting one FMA as two floating-point operations. */
OSC_API int osc_measure_fma_peak(osc_ctx* ctx, int kind, double* tflops);

/* ---- allocation-free entry point --------------------------------------------------------------
 * No counterpart in the reference (its GPU path allocates device and pinned memory on every call).
 * For callers that cannot allocate on the call path -- a plugin running inside a host application
 * that owns all device memory, or a real-time loop that must not enter the allocator after start-up
 * -- this computes the FP64 flux at one fixed level (every observer sums exactly the samples of
 * levels 0..level, no adaptive stop) without allocating anything: no cudaMalloc/cudaFree, no host
 * heap.  Its scratch is a 16 MiB static device array held by every GPU that loads the library until
 * the process exits; a request must fit in it (224 B per trajectory point + 80 B x 2^(level+1) +
 * 176 B per observer, alignment aside) or the call returns OSC_ERR_LENGTH with the reason in
 * `message`.  The array's device address is looked up on the first call on each device (and again
 * on the first call after that device's CUDA context was destroyed and created anew, e.g. by
 * cudaDeviceReset), so make the first call on a device before any stream capture.  Calls are
 * synchronous and restore the caller's current device before returning.  Every call uses the same
 * array, which keeps the previous call's contents (what must start at zero is cleared on each call);
 * two calls whose GPU work overlaps -- from different host threads, or alongside another thread's
 * call on the same device -- race on it and may return wrong results.  trajectory: host, 10 x n SoA
 * as osc_get_trajectory returns it; obs_xyz: host, 3 x n_obs; polarization: host, 6 doubles (re, im
 * of x, y, z) or NULL for none; charge [C] and current [A] of the particle; out: host, n_obs values
 * in the units of osc_flux; message: optional buffer for a NUL-terminated reason. */
OSC_API int osc_flux_fixed_level_noalloc(int device, const double* trajectory, long long n_points,
                                         const double* obs_xyz, long long n_obs, double energy_eV,
                                         int level, double charge, double current,
                                         const double polarization[6], double* out, char* message,
                                         long long message_capacity);

#ifdef __cplusplus
}
#endif
#endif
