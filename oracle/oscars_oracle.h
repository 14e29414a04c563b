/*
 * oscars_oracle.h -- CPU restatement of the OSCARS radiation path, used ONLY as a parity checker.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library; the oscars_b200 product never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle_pin.py compares every entry point below with the reference's
 * own CPU build (oracle/_ref, built by oracle/Makefile from the reference sources) and with the
 * golden fixtures in tests/golden/ that were generated from that build.
 *
 * Every routine restates the reference algorithm operation by operation (same association order,
 * no FMA contraction: built with -ffp-contract=off) so that trajectories, level samples and
 * radiation sums match the reference bit for bit on x86-64.
 */
#ifndef OSCARS_ORACLE_H
#define OSCARS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

enum { ORC_OK = 0, ORC_ERR_ARG = -1, ORC_ERR_STATE = -2, ORC_ERR_RANGE = -3, ORC_ERR_ALLOC = -4 };

/* Polarization selectors (the string matching itself lives in the Python wrapper). */
enum { ORC_POL_ALL = 0, ORC_POL_LH = 1, ORC_POL_LV = 2, ORC_POL_LINEAR = 3, ORC_POL_CL = 4, ORC_POL_CR = 5 };

/* Beam distributions, TParticleBeam.h enum order. */
enum { ORC_DIST_NONE = 0, ORC_DIST_FILAMENT = 1, ORC_DIST_GAUSSIAN = 2, ORC_DIST_KV = 3 };

orc_sim* orc_new(void);
void     orc_free(orc_sim*);
const char* orc_last_error(const orc_sim*);

int orc_clear_fields(orc_sim*);
int orc_add_undulator(orc_sim*, const double field[3], const double period[3], int nperiods,
                      const double center[3], double phase, double taper, double frequency,
                      double frequency_phase, double time_offset);
int orc_add_epu(orc_sim*, const double field_a[3], const double field_b[3], const double period[3],
                int nperiods, const double center[3], double phase, double taper, double frequency,
                double frequency_phase, double time_offset);
int orc_get_bfield(const orc_sim*, const double x[3], double t, double out[3]);
/* Amplitude factors of the 2 * nperiods half-periods of the last added undulator's full-strength
 * region (between its end poles). */
int orc_set_half_period_scale(orc_sim*, const double* scale, int n);
/* Regular grid field (TField3D_Grid, src/TField3D_Grid.cc:153-283): values (3 per point, already
 * rotated, index ix*ny*nz + iy*nz + iz); the file readers are restated in oracle.py. */
int orc_add_grid(orc_sim*, const long n[3], const double start[3], const double step[3], const double stop[3],
                 const double* values, const double rotations[3], const double translation[3], double frequency,
                 double frequency_phase, double time_offset);

/* set_particle_beam: charge [C], mass [kg] (0,0 selects by type code 0=electron,1=positron). */
int orc_set_beam(orc_sim*, int type_code, double charge, double mass, double energy_GeV,
                 const double x0[3], const double d0[3], double t0, double current,
                 const double horizontal[3], int has_horizontal, double sigma_energy_GeV,
                 const double emittance[2], int has_emittance, const double beta[2],
                 const double alpha[2], int has_beta, int has_alpha, const double eta[2],
                 int distribution_override, const double ctstartstop[2], int has_ctstartstop,
                 const double gamma[2], int has_gamma, const double lattice_ref[3], int has_lattice_ref,
                 int predefined, int has_d0, double weight, int append);
int orc_set_new_particle_of(orc_sim*, int beam, int ideal);
int orc_set_ctstartstop(orc_sim*, double start, double stop);
int orc_set_npoints_trajectory(orc_sim*, long n);
long orc_get_npoints_trajectory(const orc_sim*);
int orc_set_seed(orc_sim*, int seed);
double orc_uniform(orc_sim*);
double orc_normal(orc_sim*);
int orc_set_new_particle(orc_sim*, int ideal);
/* A particle of the beam's species at the given initial conditions (as a drawn particle would be). */
int orc_set_particle(orc_sim*, const double x0[3], const double b0[3], double t0);
int orc_get_particle(const orc_sim*, double x0[3], double b0[3], double* t0, double* gamma,
                     double* q, double* m, double* current);

int orc_calculate_trajectory(orc_sim*);
long orc_trajectory_npoints(const orc_sim*);
/* out: 10 x n SoA (t, x, y, z, bx, by, bz, ax, ay, az) */
int orc_get_trajectory(const orc_sim*, double* out, long cap);
/* spline second derivatives, 9 x n SoA */
int orc_get_spline_ypp(const orc_sim*, double* out, long cap);
/* level samples of the current trajectory: 10 x 2^level SoA */
int orc_get_level(orc_sim*, int level, double* out, long cap);

/* Trajectory method: 0 RK4, 1 RKAS; precision -1 keeps the current one (default 1e-6). */
int orc_set_trajectory_calculation(orc_sim*, int method, double precision);

/* Radiation entry points.  out has n entries (quantity 0=value, 1=precision, 2=level);
 * out_level (optional) receives the per-entry stop level, -1 when not converged. */
int orc_flux(orc_sim*, const double* obs, long n_obs, double energy_eV, int pol, double angle,
             const double horizontal[3], const double propagation[3], double precision,
             int max_level, int max_level_extended, int nparticles, int quantity, double* out,
             int* out_level);
int orc_spectrum(orc_sim*, const double obs[3], const double* energies_eV, long n_e, int pol,
                 double angle, const double horizontal[3], const double propagation[3],
                 double precision, int max_level, int max_level_extended, int nparticles,
                 int quantity, double* out, int* out_level);
int orc_power_density(orc_sim*, const double* obs, const double* normals, long n_obs,
                      int directional, double precision, int max_level, int max_level_extended,
                      int nparticles, int quantity, double* out, int* out_level);
/* Power density on STL facets (tri: n x 12 = vertices A, B, C and normal; centers: n x 3).  out_level
 * receives the level the reference's Result_Level holds after each facet (carried over from the
 * previous facet when one does not converge). */
int orc_power_density_stl(orc_sim*, const double* tri, const double* centers, long n, double precision,
                          int max_level, int max_level_extended, int nparticles, int quantity, double* out,
                          int* out_level);

#ifdef __cplusplus
}
#endif
#endif
