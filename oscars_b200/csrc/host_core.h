// host_core.h -- host-side model of the OSCARS radiation path: fields, beam sampling, the FP64
// RK4 trajectory and its clamped cubic spline.  Everything here reproduces the reference's double
// arithmetic operation for operation (built with -ffp-contract=off), so trajectories and spline
// coefficients are bit-identical to the reference CPU build; the GPU kernels start from them.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <random>
#include <string>
#include <vector>

namespace osc {

// Constants of include/TOSCARS.h:20-76 (older CODATA values, kept for parity).
constexpr double kPi = 3.14159265358979323846;
constexpr double kC = 2.99792458e8;
constexpr double kH = 6.62606876e-34;
constexpr double kHbar = 1.054571596e-34;
constexpr double kQe = 1.602176462e-19;
constexpr double kMe = 9.10938356e-31;
constexpr double kEps0 = 8.854187817E-12;
constexpr double kMu0 = 1.2566370614E-6;
constexpr double kSqrt2Pi = 2.5066282746310002416123552393401;
constexpr int kMaxLevelMemory = 26;  // TParticleA::kMaxTrajectoryLevel

inline double two_pi() { return 2.0 * kPi; }
inline double four_pi() { return 4.0 * kPi; }
inline double kg_to_gev(double m) { return 1e-9 * m * kC * kC / kQe; }
inline double gev_to_kg(double m) { return kQe * m / (1e-9 * kC * kC); }
inline double ev_to_omega(double e) { return e * kQe / kHbar; }

struct Vec3 {
  double x = 0, y = 0, z = 0;
};
inline Vec3 v3(double x, double y, double z) { return Vec3{x, y, z}; }
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
inline Vec3 operator*(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3 operator/(Vec3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double mag2(Vec3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double mag(Vec3 a) { return __builtin_sqrt(mag2(a)); }
inline double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(Vec3 a, Vec3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline Vec3 unit(Vec3 a) { return a / mag(a); }
Vec3 orthogonal(Vec3 a);
Vec3 rotate_about(Vec3 v, double angle, Vec3 axis);  // TVector3D::RotateSelf
Vec3 rotate_xyz(Vec3 v, Vec3 r);                       // TVector3D::RotateSelfXYZ

// Field values on a regular 1-3D grid (TField3D_Grid): n[a] points along axis a from start[a] in
// steps step[a] up to stop[a]; v holds the (already rotated) field vectors, 3 doubles per point, at
// index ix * n[1] * n[2] + iy * n[2] + iz.  dimx: which axes have more than one point.
enum GridDim { kGridX = 0, kGridY, kGridZ, kGridXY, kGridXZ, kGridYZ, kGridXYZ };
struct GridData {
  int64_t n[3] = {1, 1, 1};
  double start[3] = {0, 0, 0}, step[3] = {0, 0, 0}, stop[3] = {0, 0, 0};
  int dimx = kGridZ;
  std::vector<double> v;
};

// One magnetic field source; `kind` 0 = ideal planar undulator, 1 = ideal EPU, 2 = grid.
struct FieldSpec {
  int kind = 0;
  Vec3 a, b, period, center;   // center: the translation (grid: subtracted after the rotation)
  int nperiods = 0;
  double phase = 0, taper = 0, frequency = 0, frequency_phase = 0, time_offset = 0;
  double period_length = 0, length = 0;
  Vec3 period_unit;
  // undulator only, optional: amplitude factor of each of the 2 * nperiods half-periods of the
  // full-strength region (between the end poles); empty = all 1
  std::vector<double> half_scale;
  // grid only
  Vec3 rotations;
  std::shared_ptr<const GridData> grid;
  void finish();  // derived quantities, TField3D_IdealUndulator::Init
};

// Grid fields from the reference's text formats (TField3D_Grid::ReadFile, ReadFile_OSCARS1D) and
// from memory.  Throw osc::Error.
FieldSpec grid_from_file(const std::string& path, const std::string& format, Vec3 rotations, Vec3 translation,
                         const std::vector<double>& scaling, double frequency, double frequency_phase,
                         double time_offset, char comment = '#');
FieldSpec grid_from_values(const int64_t n[3], const double start[3], const double step[3], const double* values,
                           Vec3 rotations, Vec3 translation, double frequency, double frequency_phase,
                           double time_offset);

Vec3 field_value(const FieldSpec& f, Vec3 x, double t);
Vec3 field_sum(const std::vector<FieldSpec>& fields, Vec3 x, double t);

struct Particle {
  double q = 0, m = 0, gamma = 0, qomg = 0, current = 0;
  Vec3 x0, b0;
  double t0 = 0;
  bool set = false;
  void set_conditions(Vec3 x, Vec3 b, double t);  // TParticleA::SetInitialParticleConditions
};

struct BeamSpec {
  double q = 0, m = 0, current = 0, e0 = 0, t0 = 0;
  Vec3 x0, u0, hdir, vdir;
  double sigma_e = 0;
  double emit[2] = {0, 0}, eta[2] = {0, 0};
  double tw_beta[2] = {0, 0}, tw_alpha[2] = {0, 0}, tw_gamma[2] = {0, 0};
  double beta_x0[2] = {0, 0}, alpha_x0[2] = {0, 0}, gamma_x0[2] = {0, 0};
  Vec3 lattice_ref;
  int distribution = 1;  // 1 filament, 2 gaussian, 3 KV
  double weight = 1;     // share of the particles drawn from this beam among all beams
  std::string name;
  void twiss_at_x0();
};

// libstdc++ engine and distributions, exactly as src/TRandomA.cc uses them.
struct Rng {
  std::mt19937 mt{5489u};
  std::normal_distribution<double> normal{0.0, 1.0};
  std::uniform_real_distribution<double> uniform{0.0, 1.0};
  void seed(int s) {
    mt = std::mt19937(s);
    normal = std::normal_distribution<double>(0.0, 1.0);
    uniform = std::uniform_real_distribution<double>(0.0, 1.0);
  }
};

// RK4 knots and their spline second derivatives, SoA: t[n]; y[9][n] = x y z bx by bz ax ay az
// (a = acceleration / c); ypp[9][n].
struct Knots {
  int64_t n = 0;
  std::vector<double> t, y, ypp;
  std::vector<double> diag;  // factored diagonal of the spline system (depends on t only)
  std::vector<double> work;  // spline scratch (sigma, p, 9 right-hand sides), kept between calls
  double tstart = 0, tstop = 0;
  void clear() { n = 0; t.clear(); y.clear(); ypp.clear(); diag.clear(); }
};

struct Error {
  int code;
  std::string msg;
};

class Model {
 public:
  std::vector<FieldSpec> fields;
  // Particle beams (TParticleBeamContainer, src/TParticleBeamContainer.cc): particles are drawn from
  // a beam picked at random by weight (one uniform draw when there are several beams).
  std::vector<BeamSpec> beams;
  std::vector<double> beam_weight_sums;
  bool has_beam = false;
  Particle particle;
  double ctstart = 0, ctstop = 0;
  int64_t npoints = 0, npoints_per_meter = 10000;
  Rng rng;
  Knots knots;
  uint64_t knots_version = 0;  // bumps whenever `knots` changes
  std::vector<double> sweep[2];  // forward / backward integration points, kept between calls
  // Trajectory method (OSCARSSR::SetTrajectoryCalculation, src/OSCARSSR.cc:784-820): fixed-step RK4
  // or the adaptive Cash-Karp RKAS with its precision (default 1e-6).
  enum TrajectoryMethod { kRK4 = 0, kRKAS = 1 };
  int traj_method = kRK4;
  double traj_precision = 1e-6;

  void add_field(const FieldSpec& f);
  void clear_fields();
  void set_ctstartstop(double a, double b);
  void add_beam(const BeamSpec& b);  // name must be unique (set by the caller)
  void clear_beams();
  size_t pick_beam();                 // GetRandomBeamIndexByWeight
  size_t find_beam(const std::string& name) const;
  // OSCARSSR::SetNewParticle(beam, "ideal" or random): `name` empty picks a beam by weight.
  void new_particle(const std::string& name, bool ideal);
  void ideal_particle();   // SetNewParticle("", "ideal")
  void random_particle();  // SetNewParticle(): a beam by weight, then its random particle
  void ideal_of(const BeamSpec& b);
  void sample_of(const BeamSpec& b);
  // Throws osc::Error on failure.
  void compute_trajectory();
  void ensure_trajectory();
  // The trajectory of particle P with this model's fields, times and method into `out` (knots and
  // spline); `sweep` (2 vectors) holds the forward / backward points.  Reads the model only, so
  // several threads may integrate different particles at once (threads = false: no use of the host
  // task pool inside).
  void integrate(const Particle& P, Knots& out, std::vector<double>* sweep, bool threads) const;
  // Select the method: "RK4" (precision must be -1, the binding's "not given") or "RKAS".
  void set_trajectory_calculation(const std::string& method, double precision);
  // Use a trajectory computed elsewhere (10 x n SoA: t, x y z, beta, a/c) with its spline.
  void set_trajectory(const double* traj, int64_t n);
};

// Spline second derivatives of the 9 components (TSpline1D3::Derivatives, include/TOMATH.h:141-203).
// `threads`: the 9 components on the host task pool (callers that are themselves worker threads pass
// false).
void spline_second_derivatives(Knots& k, bool threads = true);

// Runs fn(0) .. fn(n - 1) on a process-wide set of persistent host threads (the caller works too)
// and returns when all have finished; the first exception a task throws is rethrown here.  Calls
// from several threads are served one after another.
void parallel_tasks(int n, const std::function<void(int)>& fn);

// Rectangle surface (TSurfacePoints_Rectangle).  Throws osc::Error.
void surface_rectangle(const std::string& plane, int nx1, int nx2, double w1, double w2, Vec3 rot,
                       Vec3 trans, int normal, double* xyz, double* normals, double* x1x2);
// Rectangle from three points (TSurfacePoints_Rectangle x0x1x2 form).  Throws osc::Error.
void surface_x0x1x2(int nx1, int nx2, Vec3 x0, Vec3 x1, Vec3 x2, Vec3 rot, Vec3 trans, int normal, double* xyz,
                    double* normals, double* x1x2);
// Arbitrary points with normals, rotated / translated as the point-list bindings do.
void surface_points(int64_t n, const double* pts, const double* nrm, Vec3 rot, Vec3 trans, bool invert_normals,
                    double* xyz, double* normals);

}  // namespace osc
