// host_core.cc -- host model of the radiation path (see host_core.h).  Every expression keeps the
// association order of the reference expression it reproduces (file:line of the OSCARS sources).
#include "host_core.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cctype>
#include <cmath>
#include <condition_variable>
#include <exception>
#include <fstream>
#include <mutex>
#include <sstream>
#include <thread>

#include "../../include/oscars_b200.h"

namespace osc {

// ---------------------------------------------------------------------------------------------
// Persistent host threads for the independent parts of a trajectory (the two integration sweeps,
// the 9 spline components): created once, woken per call, so a trajectory costs no thread starts.
// ---------------------------------------------------------------------------------------------
namespace {

class TaskPool {
 public:
  ~TaskPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }

  void run(int n, const std::function<void(int)>& fn) {
    std::lock_guard<std::mutex> call(call_m_);
    if (threads_.empty()) {
      const unsigned hw = std::thread::hardware_concurrency();
      const int w = (int)std::min(8u, hw > 1 ? hw - 1 : 1u);
      for (int i = 0; i < w; ++i) threads_.emplace_back([this] { worker(); });
    }
    {
      std::lock_guard<std::mutex> lk(m_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      error_ = nullptr;
      ++gen_;
    }
    cv_.notify_all();
    drain();
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return active_ == 0; });
    fn_ = nullptr;
    if (error_) std::rethrow_exception(error_);
  }

 private:
  void drain() {
    for (int i; (i = next_.fetch_add(1)) < n_;) {
      try {
        (*fn_)(i);
      } catch (...) {
        std::lock_guard<std::mutex> lk(m_);
        if (!error_) error_ = std::current_exception();
      }
    }
  }
  void worker() {
    uint64_t seen = 0;
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
      cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
      if (!fn_) continue;  // woke after that call had finished
      ++active_;
      lk.unlock();
      drain();
      lk.lock();
      if (--active_ == 0) done_.notify_all();
    }
  }

  std::mutex call_m_, m_;
  std::condition_variable cv_, done_;
  std::vector<std::thread> threads_;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0, active_ = 0;
  std::atomic<int> next_{0};
  uint64_t gen_ = 0;
  bool stop_ = false;
  std::exception_ptr error_;
};

TaskPool& task_pool() {
  static TaskPool pool;
  return pool;
}

}  // namespace

void parallel_tasks(int n, const std::function<void(int)>& fn) {
  if (n <= 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  task_pool().run(n, fn);
}

Vec3 orthogonal(Vec3 a) {  // include/TVector3D.h:132-142
  double xx = a.x < 0.0 ? -a.x : a.x;
  double yy = a.y < 0.0 ? -a.y : a.y;
  double zz = a.z < 0.0 ? -a.z : a.z;
  if (xx < yy) return xx < zz ? v3(0, a.z, -a.y) : v3(a.y, -a.x, 0);
  return yy < zz ? v3(-a.z, 0, a.x) : v3(a.y, -a.x, 0);
}

Vec3 rotate_about(Vec3 o, double A, Vec3 axis) {  // TVector3D::RotateSelf (Rodrigues matrix)
  Vec3 v = unit(axis);
  double c = std::cos(A), s = std::sin(A);
  double m00 = c + v.x * v.x * (1 - c), m01 = v.x * v.y * (1 - c) - v.z * s;
  double m02 = v.x * v.z * (1 - c) + v.y * s, m10 = v.y * v.x * (1 - c) + v.z * s;
  double m11 = c + v.y * v.y * (1 - c), m12 = v.y * v.z * (1 - c) - v.x * s;
  double m20 = v.z * v.x * (1 - c) - v.y * s, m21 = v.z * v.y * (1 - c) + v.x * s;
  double m22 = c + v.z * v.z * (1 - c);
  return {m00 * o.x + m01 * o.y + m02 * o.z, m10 * o.x + m11 * o.y + m12 * o.z,
          m20 * o.x + m21 * o.y + m22 * o.z};
}

Vec3 rotate_xyz(Vec3 v, Vec3 r) {  // TVector3D::RotateSelfX, Y, Z in that order
  double s = std::sin(r.x), c = std::cos(r.x), t = v.y;
  v.y = c * t - s * v.z;
  v.z = s * t + c * v.z;
  s = std::sin(r.y); c = std::cos(r.y); t = v.z;
  v.z = c * t - s * v.x;
  v.x = s * t + c * v.x;
  s = std::sin(r.z); c = std::cos(r.z); t = v.x;
  v.x = c * t - s * v.y;
  v.y = s * t + c * v.y;
  return v;
}

// ---------------------------------------------------------------------------------------------
// Fields
// ---------------------------------------------------------------------------------------------
void FieldSpec::finish() {  // TField3D_IdealUndulator::Init :94-98
  if (kind == 2) return;
  period_length = mag(period);
  period_unit = unit(period);
  length = mag(period) * (nperiods + 2);
}

// One sinusoidal block with 1/4 and 3/4 end poles (src/TField3D_IdealUndulator.cc:125-142).  With
// half-period factors, the full-strength region [-L/2 + shift + lam, L/2 + shift - lam] (2 N
// half-periods between zeros of the sine) is scaled per half-period.
static Vec3 pole_block(const FieldSpec& f, Vec3 amp, double d, double shift, double taper_corr) {
  const double L = f.length, lam = f.period_length;
  if (d > L / 2. + shift || d < -L / 2. + shift) return Vec3{};
  const double s = std::sin(two_pi() * (d - shift) / lam);
  if (d < -L / 2. + shift + lam || d > L / 2. + shift - lam) {
    if (d < -L / 2. + shift + lam / 2. || d > L / 2. + shift - lam / 2.)
      return amp * 0.25 * s * taper_corr;
    return amp * 0.75 * s * taper_corr;
  }
  if (f.half_scale.empty()) return amp * s * taper_corr;
  const int64_t nh = (int64_t)f.half_scale.size();
  int64_t k = (int64_t)((d - (-L / 2. + shift + lam)) / (lam / 2.));
  k = k < 0 ? 0 : (k >= nh ? nh - 1 : k);
  return amp * s * taper_corr * f.half_scale[k];
}

// Grid interpolation (src/TField3D_Grid.cc:153-283): rotate, translate, zero outside the grid,
// multilinear interpolation v0 + d (v1 - v0) / step per axis, times the time factor.
static inline Vec3 grid_at(const GridData& g, int64_t i) { return v3(g.v[3 * i], g.v[3 * i + 1], g.v[3 * i + 2]); }
static inline Vec3 lerp_step(Vec3 v0, Vec3 v1, double d, double step) { return v0 + (v1 - v0) * d / step; }

static Vec3 grid_value(const FieldSpec& f, Vec3 xin, double t) {
  const GridData& g = *f.grid;
  Vec3 X = rotate_xyz(xin, f.rotations);
  X = X - f.center;
  const double p[3] = {X.x, X.y, X.z};
  int64_t ni[3] = {0, 0, 0};
  double di[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) {
    if (g.n[a] > 1) {
      if (p[a] <= g.start[a] || p[a] >= g.stop[a]) return Vec3{};
      ni[a] = (int64_t)((p[a] - g.start[a]) / g.step[a]);
      di[a] = (p[a] - g.start[a]) - ni[a] * g.step[a];
      // the reference would read one past its data if rounding put a point just below the stop
      // into the last cell; clamp to the last cell instead
      if (ni[a] > g.n[a] - 2) ni[a] = g.n[a] - 2;
    }
  }
  const int64_t NY = g.n[1], NZ = g.n[2];
  auto idx = [&](int64_t ix, int64_t iy, int64_t iz) { return ix * NY * NZ + iy * NZ + iz; };
  const int64_t nx = ni[0], ny = ni[1], nz = ni[2];
  const double dx = di[0], dy = di[1], dz = di[2];
  Vec3 F;
  switch (g.dimx) {
    case kGridXYZ: {
      const Vec3 v00 = lerp_step(grid_at(g, idx(nx, ny, nz)), grid_at(g, idx(nx + 1, ny, nz)), dx, g.step[0]);
      const Vec3 v10 = lerp_step(grid_at(g, idx(nx, ny + 1, nz)), grid_at(g, idx(nx + 1, ny + 1, nz)), dx, g.step[0]);
      const Vec3 v01 = lerp_step(grid_at(g, idx(nx, ny, nz + 1)), grid_at(g, idx(nx + 1, ny, nz + 1)), dx, g.step[0]);
      const Vec3 v11 = lerp_step(grid_at(g, idx(nx, ny + 1, nz + 1)), grid_at(g, idx(nx + 1, ny + 1, nz + 1)), dx,
                                 g.step[0]);
      const Vec3 v0 = lerp_step(v00, v10, dy, g.step[1]);
      const Vec3 v1 = lerp_step(v01, v11, dy, g.step[1]);
      F = lerp_step(v0, v1, dz, g.step[2]);
      break;
    }
    case kGridX: F = lerp_step(grid_at(g, nx), grid_at(g, nx + 1), dx, g.step[0]); break;
    case kGridY: F = lerp_step(grid_at(g, ny), grid_at(g, ny + 1), dy, g.step[1]); break;
    case kGridZ: F = lerp_step(grid_at(g, nz), grid_at(g, nz + 1), dz, g.step[2]); break;
    case kGridXY: {
      const Vec3 v0 = lerp_step(grid_at(g, idx(nx, ny, 0)), grid_at(g, idx(nx + 1, ny, 0)), dx, g.step[0]);
      const Vec3 v1 = lerp_step(grid_at(g, idx(nx, ny + 1, 0)), grid_at(g, idx(nx + 1, ny + 1, 0)), dx, g.step[0]);
      F = lerp_step(v0, v1, dy, g.step[1]);
      break;
    }
    case kGridXZ: {
      const Vec3 v0 = lerp_step(grid_at(g, idx(nx, 0, nz)), grid_at(g, idx(nx + 1, 0, nz)), dx, g.step[0]);
      const Vec3 v1 = lerp_step(grid_at(g, idx(nx, 0, nz + 1)), grid_at(g, idx(nx + 1, 0, nz + 1)), dx, g.step[0]);
      F = lerp_step(v0, v1, dz, g.step[2]);
      break;
    }
    default: {  // kGridYZ
      const Vec3 v0 = lerp_step(grid_at(g, idx(0, ny, nz)), grid_at(g, idx(0, ny + 1, nz)), dy, g.step[1]);
      const Vec3 v1 = lerp_step(grid_at(g, idx(0, ny, nz + 1)), grid_at(g, idx(0, ny + 1, nz + 1)), dy, g.step[1]);
      F = lerp_step(v0, v1, dz, g.step[2]);
      break;
    }
  }
  return F * std::cos(two_pi() * f.frequency * (t + f.time_offset) + f.frequency_phase);
}

Vec3 field_value(const FieldSpec& f, Vec3 x, double t) {
  if (f.kind == 2) return grid_value(f, x, t);
  const double d = dot(x - f.center, f.period_unit);
  const double taper_corr = 1 + d * f.taper;
  Vec3 F;
  if (f.kind == 0) {
    F = pole_block(f, f.a, d, f.phase * f.period_length / two_pi(), taper_corr);
  } else {  // src/TField3D_IdealEPU.cc:127-165: A shifted by +phase/2, B by -phase/2
    F = pole_block(f, f.a, d, f.phase / 2. * f.period_length / two_pi(), taper_corr);
    F = F + pole_block(f, f.b, d, -f.phase / 2. * f.period_length / two_pi(), taper_corr);
  }
  if (f.frequency == 0) return F;
  return F * std::cos(two_pi() * f.frequency * (t + f.time_offset) + f.frequency_phase);
}

// ---------------------------------------------------------------------------------------------
// Grid fields from files (src/TField3D_Grid.cc:365-530 OSCARS, :572-870 OSCARS1D)
// ---------------------------------------------------------------------------------------------
static int grid_dimx(const GridData& g) {
  const bool hx = g.n[0] > 1, hy = g.n[1] > 1, hz = g.n[2] > 1;
  if (hx && hy && hz) return kGridXYZ;
  if (hx && hy) return kGridXY;
  if (hx && hz) return kGridXZ;
  if (hy && hz) return kGridYZ;
  if (hx) return kGridX;
  if (hy) return kGridY;
  if (hz) return kGridZ;
  throw Error{OSC_ERR_RANGE, "invalid dimensions"};
}

static FieldSpec grid_spec(std::shared_ptr<GridData> g, Vec3 rotations, Vec3 translation, double frequency,
                           double frequency_phase, double time_offset) {
  FieldSpec f;
  f.kind = 2;
  f.rotations = rotations;
  f.center = translation;
  f.frequency = frequency;
  f.frequency_phase = frequency_phase;
  f.time_offset = time_offset;
  f.grid = std::move(g);
  return f;
}

static double header_value(const std::string& line) {  // GetHeaderValue: first number on the line
  std::istringstream S(line);
  double v = 0;
  S >> v;
  if (S.bad()) throw Error{OSC_ERR_INVALID, "cannot read header value"};
  return v;
}

static FieldSpec read_oscars_grid(const std::string& path, Vec3 rot, Vec3 trans, const std::vector<double>& sc,
                                  double fr, double fp, double to) {
  std::ifstream fi(path);
  if (!fi) throw Error{OSC_ERR_INVALID, "cannot open file for reading"};
  std::string L;
  std::getline(fi, L);  // comment
  double hv[9];
  for (int i = 0; i < 9; ++i) {
    std::getline(fi, L);
    hv[i] = header_value(L);
  }
  const double xs_in = hv[0], xst_in = hv[1], ys_in = hv[3], yst_in = hv[4], zs_in = hv[6], zst_in = hv[7];
  const int NX = (int)hv[2], NY = (int)hv[5], NZ = (int)hv[8];
  const double XStep = sc.size() > 0 ? xst_in * sc[0] : xst_in;
  const double YStep = sc.size() > 1 ? yst_in * sc[1] : yst_in;
  const double ZStep = sc.size() > 2 ? zst_in * sc[2] : zst_in;
  const double FxS = sc.size() > 3 ? sc[3] : 1, FyS = sc.size() > 4 ? sc[4] : 1, FzS = sc.size() > 5 ? sc[5] : 1;
  const double MiddleX = xs_in + xst_in * (NX - 1) / 2., XStart = MiddleX - XStep * (NX - 1) / 2.;
  const double MiddleY = ys_in + yst_in * (NY - 1) / 2., YStart = MiddleY - YStep * (NY - 1) / 2.;
  const double MiddleZ = zs_in + zst_in * (NZ - 1) / 2., ZStart = MiddleZ - ZStep * (NZ - 1) / 2.;
  if (NX < 1 || NY < 1 || NZ < 1) throw Error{OSC_ERR_RANGE, "invalid number of points in at least one dimension"};
  auto g = std::make_shared<GridData>();
  g->n[0] = NX; g->n[1] = NY; g->n[2] = NZ;
  g->start[0] = XStart; g->start[1] = YStart; g->start[2] = ZStart;
  g->step[0] = XStep; g->step[1] = YStep; g->step[2] = ZStep;
  for (int a = 0; a < 3; ++a) g->stop[a] = g->start[a] + (g->n[a] - 1) * g->step[a];
  g->dimx = grid_dimx(*g);
  g->v.reserve(3 * (size_t)NX * NY * NZ);
  std::istringstream S;
  for (int ix = 0; ix != NX; ++ix)
    for (int iy = 0; iy != NY; ++iy)
      for (int iz = 0; iz != NZ; ++iz) {
        std::getline(fi, L);
        if (fi.eof()) throw Error{OSC_ERR_INVALID, "error reading file.  Check format"};
        double fx, fy, fz;
        S.clear();
        S.str(L);
        S >> fx >> fy >> fz;
        if (FxS != 1) fx *= FxS;
        if (FyS != 1) fy *= FyS;
        if (FzS != 1) fz *= FzS;
        if (S.fail()) throw Error{OSC_ERR_INVALID, "error reading file.  Check format"};
        const Vec3 F = rotate_xyz(v3(fx, fy, fz), rot);
        g->v.push_back(F.x);
        g->v.push_back(F.y);
        g->v.push_back(F.z);
      }
  return grid_spec(g, rot, trans, fr, fp, to);
}

static FieldSpec read_oscars1d_grid(const std::string& path, const std::string& format, Vec3 rot, Vec3 trans,
                                    const std::vector<double>& sc, double fr, double fp, double to, char comment) {
  std::ifstream fi(path);
  if (!fi) throw Error{OSC_ERR_INVALID, "cannot open file for reading"};
  int order[4] = {-1, -1, -1, -1};
  std::istringstream fs(std::string(format.begin() + 8, format.end()));
  std::string c, axis;
  int index = 0, xdim = 0, fdim = 0;
  bool has[4] = {false, false, false, false};
  while (fs >> c) {
    if (index > 3) throw Error{OSC_ERR_RANGE, "spatial or B-field dimensions are too large(index>3)"};
    if (c == "X" || c == "Y" || c == "Z") {
      axis = c;
      ++xdim;
      order[index++] = 0;
    } else if (c == "Bx" || c == "Ex" || c == "Fx") {
      has[1] = true; ++fdim; order[index++] = 1;
    } else if (c == "By" || c == "Ey" || c == "Fy") {
      has[2] = true; ++fdim; order[index++] = 2;
    } else if (c == "Bz" || c == "Ez" || c == "Fz") {
      has[3] = true; ++fdim; order[index++] = 3;
    } else {
      throw Error{OSC_ERR_INVALID, "only excepts X Y Z Bx By Bz"};
    }
  }
  const int count = xdim + fdim;
  if (xdim != 1) throw Error{OSC_ERR_RANGE, "spatial or B-field dimensions are too large"};
  std::string L;
  std::getline(fi, L);  // comment line
  std::vector<std::array<double, 4>> in;
  std::istringstream S;
  while (std::getline(fi, L)) {
    const size_t first = L.find_first_not_of(" \t");
    if (first == std::string::npos || L[first] == comment) continue;
    std::replace(L.begin(), L.end(), ',', ' ');
    S.clear();
    S.str(L);
    double val[4] = {0, 0, 0, 0};
    for (int i = 0; i < count; ++i) {
      S >> val[order[i]];
      if (S.fail()) throw Error{OSC_ERR_LENGTH, "something is incorrect with data format or iformat string"};
    }
    for (size_t i = 0; i != sc.size() && i < 4; ++i) {
      if (order[i] < 0) continue;
      val[order[i]] *= sc[i];
    }
    in.push_back({val[0], val[1], val[2], val[3]});
  }
  std::sort(in.begin(), in.end(), [](const std::array<double, 4>& A, const std::array<double, 4>& B) { return A[0] < B[0]; });
  if (in.size() < 2) throw Error{OSC_ERR_LENGTH, "not enough data points"};
  const double First = in.front()[0], Last = in.back()[0];
  const size_t kPointsPerMeter = 10000;
  const size_t NPoints = (size_t)((Last - First) * kPointsPerMeter);
  const double Step = (Last - First) / (double)(NPoints - 1);
  auto g = std::make_shared<GridData>();
  const int ax = axis == "X" ? 0 : axis == "Y" ? 1 : 2;
  g->n[ax] = (int64_t)NPoints;
  g->start[ax] = First;
  g->stop[ax] = Last;
  g->step[ax] = Step;
  g->dimx = grid_dimx(*g);
  g->v.reserve(3 * NPoints);
  size_t min_bin = 0, after = 0, before = 0;
  for (size_t i = 0; i != NPoints; ++i) {
    const double z = i * Step + First;
    for (size_t j = min_bin + 1; j != in.size(); ++j) {
      if (in[j][0] > z) {
        after = j;
        before = j - 1;
        min_bin = j - 1;
        break;
      }
    }
    double nb[3];
    for (int k = 0; k < 3; ++k) {
      const double slope = !has[k + 1] ? 0 : (in[after][k + 1] - in[before][k + 1]) / (in[after][0] - in[before][0]);
      nb[k] = !has[k + 1] ? 0 : in[before][k + 1] + (z - in[before][0]) * slope;
    }
    const Vec3 F = rotate_xyz(v3(nb[0], nb[1], nb[2]), rot);
    g->v.push_back(F.x);
    g->v.push_back(F.y);
    g->v.push_back(F.z);
  }
  return grid_spec(g, rot, trans, fr, fp, to);
}

FieldSpec grid_from_file(const std::string& path, const std::string& format, Vec3 rotations, Vec3 translation,
                         const std::vector<double>& scaling, double frequency, double frequency_phase,
                         double time_offset, char comment) {
  std::string F = format;
  std::transform(F.begin(), F.end(), F.begin(), ::toupper);
  // OSCARSSR::AddMagneticField (src/OSCARSSR.cc:70-103) accepts these format names
  const bool is1d = F.size() > 8 && F.compare(0, 8, "OSCARS1D") == 0;
  if (!(F == "OSCARS" || F == "SRW" || F == "SPECTRA" || F == "BINARY" || is1d))
    throw Error{OSC_ERR_INVALID, "Incorrect format in format string"};
  if (F == "OSCARS") return read_oscars_grid(path, rotations, translation, scaling, frequency, frequency_phase, time_offset);
  if (is1d)
    return read_oscars1d_grid(path, format, rotations, translation, scaling, frequency, frequency_phase, time_offset,
                              comment);
  throw Error{OSC_ERR_INVALID, "grid file format " + F + " is not supported by this build (OSCARS and OSCARS1D are)"};
}

FieldSpec grid_from_values(const int64_t n[3], const double start[3], const double step[3], const double* values,
                           Vec3 rotations, Vec3 translation, double frequency, double frequency_phase,
                           double time_offset) {
  auto g = std::make_shared<GridData>();
  for (int a = 0; a < 3; ++a) {
    if (n[a] < 1) throw Error{OSC_ERR_RANGE, "invalid number of points in at least one dimension"};
    if (n[a] > 1 && !(step[a] > 0)) throw Error{OSC_ERR_RANGE, "grid steps must be positive"};
    g->n[a] = n[a];
    g->start[a] = start[a];
    g->step[a] = n[a] > 1 ? step[a] : 0;
    g->stop[a] = g->start[a] + (g->n[a] - 1) * g->step[a];
  }
  g->dimx = grid_dimx(*g);
  const int64_t N = n[0] * n[1] * n[2];
  g->v.resize(3 * N);
  for (int64_t i = 0; i < N; ++i) {
    const Vec3 F = rotate_xyz(v3(values[3 * i], values[3 * i + 1], values[3 * i + 2]), rotations);
    g->v[3 * i] = F.x;
    g->v[3 * i + 1] = F.y;
    g->v[3 * i + 2] = F.z;
  }
  return grid_spec(g, rotations, translation, frequency, frequency_phase, time_offset);
}

Vec3 field_sum(const std::vector<FieldSpec>& fields, Vec3 x, double t) {  // TFieldContainer::GetF
  Vec3 s{0, 0, 0};
  for (const FieldSpec& f : fields) s = s + field_value(f, x, t);
  return s;
}

// ---------------------------------------------------------------------------------------------
// Particle / beam
// ---------------------------------------------------------------------------------------------
void Particle::set_conditions(Vec3 x, Vec3 b, double t) {  // TParticleA.cc SetGamma/SetQoverMGamma
  x0 = x; b0 = b; t0 = t;
  const double beta2 = mag2(b) > 0 ? mag2(b) : 0;
  if (beta2 != 1) {
    gamma = beta2 != 0 ? 1.0 / std::sqrt(1.0 - beta2) : 1;
    if (!(m == 0 || gamma == 0)) qomg = q / m / gamma;
  }
  set = true;
}

void BeamSpec::twiss_at_x0() {  // TParticleBeam::SetTwissParametersAtX0
  const Vec3 dx = x0 - lattice_ref;
  const double D = mag(dx);
  const double L = dot(dx, u0) >= 0 ? D : -1. * D;
  for (int i = 0; i < 2; ++i) {
    beta_x0[i] = tw_beta[i] - 2 * L * tw_alpha[i] + L * L * tw_gamma[i];
    alpha_x0[i] = tw_alpha[i] - L * tw_gamma[i];
    gamma_x0[i] = tw_gamma[i];
  }
}

void Model::add_field(const FieldSpec& f) {
  fields.push_back(f);
  fields.back().finish();
  knots.clear();  // OSCARSSR::AddMagneticField clears the particle's trajectory
  ++knots_version;
}

void Model::clear_fields() {
  fields.clear();
  knots.clear();
  ++knots_version;
}

void Model::set_ctstartstop(double a, double b) {  // OSCARSSR::SetCTStartStop (:637-647)
  npoints = (int64_t)(npoints_per_meter * (b - a));
  ctstart = a;
  ctstop = b;
}

void Model::add_beam(const BeamSpec& b) {  // TParticleBeamContainer::AddNewParticleBeam
  beam_weight_sums.push_back(beam_weight_sums.empty() ? b.weight : beam_weight_sums.back() + b.weight);
  beams.push_back(b);
  has_beam = true;
}

void Model::clear_beams() {
  beams.clear();
  beam_weight_sums.clear();
  has_beam = false;
}

size_t Model::pick_beam() {  // TParticleBeamContainer::GetRandomBeamIndexByWeight (:135-166)
  const size_t N = beam_weight_sums.size();
  if (N == 0) throw Error{OSC_ERR_RANGE, "no beam defined"};
  if (N == 1) return 0;
  const double r = rng.uniform(rng.mt) * beam_weight_sums[N - 1];
  for (size_t i = 0; i != N; ++i)
    if (r < beam_weight_sums[i]) return i;
  throw Error{OSC_ERR_RANGE, "random weight out of range.  SERIOUS ERROR"};
}

size_t Model::find_beam(const std::string& name) const {
  for (size_t i = 0; i < beams.size(); ++i)
    if (beams[i].name == name) return i;
  throw Error{OSC_ERR_RANGE, "beam name not in map"};
}

void Model::new_particle(const std::string& name, bool ideal) {  // OSCARSSR::SetNewParticle (:510-524)
  const BeamSpec& b = beams[name.empty() ? pick_beam() : find_beam(name)];
  if (ideal) ideal_of(b);
  else sample_of(b);
}

void Model::ideal_particle() { ideal_of(beams[pick_beam()]); }

void Model::random_particle() { sample_of(beams[pick_beam()]); }

void Model::ideal_of(const BeamSpec& beam) {  // TParticleBeam::GetNewParticle("ideal") (:667-688)
  const double g = beam.e0 / kg_to_gev(beam.m) < 1 ? 1 : beam.e0 / kg_to_gev(beam.m);
  const double b = g != 1 ? std::sqrt(1.0 - 1.0 / (g * g)) : 0;
  particle = Particle{};
  particle.q = beam.q;
  particle.m = beam.m;
  particle.current = beam.current;
  particle.set_conditions(beam.x0, beam.u0 * b, beam.t0);
  knots.clear();
  ++knots_version;
}

void Model::sample_of(const BeamSpec& beam) {  // TParticleBeam::GetNewParticle() (:692-850)
  if (beam.distribution != 2 && beam.distribution != 3) {
    ideal_of(beam);
    return;
  }
  const double PI = kPi;
  const double mg = kg_to_gev(beam.m);
  double enew = beam.e0 + beam.sigma_e * rng.normal(rng.mt);
  if (enew < mg) enew = mg;
  const double ge = enew / mg < 1 ? 1 : enew / mg;
  const double beta = ge != 1 ? std::sqrt(1.0 - 1.0 / (ge * ge)) : 0;
  const double de = (enew - beam.e0) / beam.e0;
  Vec3 xn = beam.x0;
  Vec3 bn = cross(beam.hdir, beam.vdir) * beta;
  auto U = [&]() { return rng.uniform(rng.mt); };
  if (beam.distribution == 2) {
    if (beam.emit[0] * beam.emit[0] + beam.emit[1] * beam.emit[1] > 1e-99) {
      const int hc = beam.alpha_x0[0] > 0 ? -1 : 1, vc = beam.alpha_x0[1] > 0 ? -1 : 1;
      const double hsx = std::sqrt(beam.emit[0] * beam.beta_x0[0]);
      const double hsxp = std::sqrt(beam.emit[0] * beam.gamma_x0[0]);
      const double hr = beam.emit[0] / (hsx * hsxp);
      const double hrho = std::sqrt(1 - hr * hr);
      const double vsx = std::sqrt(beam.emit[1] * beam.beta_x0[1]);
      const double vsxp = std::sqrt(beam.emit[1] * beam.gamma_x0[1]);
      const double vr = beam.emit[1] / (vsx * vsxp);
      const double vrho = std::sqrt(1 - vr * vr);
      const double hu = U(), hv = U();
      const double hX = hsx * std::sqrt(-2 * std::log(hu)) *
                        (std::sqrt(1 - hrho * hrho) * std::cos(2 * PI * hv) + hrho * std::sin(2 * PI * hv));
      const double hXP = hc * hsxp * std::sqrt(-2 * std::log(hu)) * std::sin(2 * PI * hv);
      const double vu = U(), vv = U();
      const double vX = vsx * std::sqrt(-2 * std::log(vu)) *
                        (std::sqrt(1 - vrho * vrho) * std::cos(2 * PI * vv) + vrho * std::sin(2 * PI * vv));
      const double vXP = vc * vsxp * std::sqrt(-2 * std::log(vu)) * std::sin(2 * PI * vv);
      // `X += H * hX + eta * dE/E` adds the scalar term to each component
      const double eh = beam.eta[0] * de, ev = beam.eta[1] * de;
      const Vec3 th = beam.hdir * hX, tv = beam.vdir * vX;
      xn = xn + v3(th.x + eh, th.y + eh, th.z + eh);
      xn = xn + v3(tv.x + ev, tv.y + ev, tv.z + ev);
      bn = rotate_about(bn, hXP, beam.vdir);
      bn = rotate_about(bn, vXP, -beam.hdir);
    }
  } else {  // KV
    const int hc = beam.alpha_x0[0] > 0 ? -1 : 1, vc = beam.alpha_x0[1] > 0 ? -1 : 1;
    const double hT = U() * 2 * PI;
    const double vT = U() * 2 * PI;
    const double hAX = std::sqrt(beam.emit[0] * beam.beta_x0[0]) * std::cos(hT);
    const double vAX = std::sqrt(beam.emit[1] * beam.beta_x0[1]) * std::cos(vT);
    const double hAXP = -std::sqrt(beam.emit[0] / beam.beta_x0[0]) * (beam.alpha_x0[0] * std::cos(hT) + std::sin(hT));
    const double vAXP = -std::sqrt(beam.emit[1] / beam.beta_x0[1]) * (beam.alpha_x0[1] * std::cos(vT) + std::sin(vT));
    const double hR = std::sqrt(hAX * hAX + hAXP * hAXP), vR = std::sqrt(vAX * vAX + vAXP * vAXP);
    double hRT = std::atan(hAXP / hAX), vRT = std::atan(vAXP / vAX);
    if (hAX < 0 && hAXP > 0) hRT += PI; else if (hAX < 0 && hAXP < 0) hRT -= PI;
    if (vAX < 0 && vAXP > 0) vRT += PI; else if (vAX < 0 && vAXP < 0) vRT -= PI;
    const double hNR = std::sqrt(U()) * hR;
    const double vNR = std::sqrt(U()) * vR;
    xn = xn + beam.hdir * (hNR * std::cos(hRT));
    xn = xn + beam.vdir * (vNR * std::cos(vRT));
    bn = rotate_about(bn, hNR * std::sin(hRT) * hc, beam.vdir);
    bn = rotate_about(bn, vNR * std::sin(vRT) * vc, -beam.hdir);
  }
  particle = Particle{};
  particle.q = beam.q;
  particle.m = beam.m;
  particle.current = beam.current;
  particle.set_conditions(xn, bn, beam.t0);
  knots.clear();
  ++knots_version;
}

// ---------------------------------------------------------------------------------------------
// RK4 (src/OSCARSSR.cc:910-1009 driver, :1247-1279 DerivativesB, :1321-1386 RK4 step)
// ---------------------------------------------------------------------------------------------
namespace {

struct Integrator {
  const std::vector<FieldSpec>& fields;
  double qomg;
  bool error_gamma = false;

  void derivs(double t, const double* x, double* dxdt) {
    const double one_minus = (1. - (x[1] * x[1] + x[3] * x[3] + x[5] * x[5]) / (kC * kC));
    if (one_minus <= 0) {  // leaves dxdt untouched, as the reference does
      error_gamma = true;
      return;
    }
    const Vec3 B = field_sum(fields, v3(x[0], x[2], x[4]), t);
    dxdt[0] = x[1];
    dxdt[1] = qomg * (-x[5] * B.y + x[3] * B.z);
    dxdt[2] = x[3];
    dxdt[3] = qomg * (x[5] * B.x - x[1] * B.z);
    dxdt[4] = x[5];
    dxdt[5] = qomg * (x[1] * B.y - x[3] * B.x);
  }

  // y and yout may alias; dydx is overwritten by the step-halving branch like the reference's.
  void step(const double* y, double* dydx, double x, double h, double* yout) {
    double dym[6], dyt[6], yt[6], yo[6];
    const double hh = h * 0.5, h6 = h / 6.0, xh = x + hh;
    for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dydx[i];
    derivs(xh, yt, dyt);
    for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
    derivs(xh, yt, dym);
    for (int i = 0; i < 6; ++i) {
      yt[i] = y[i] + h * dym[i];
      dym[i] += dyt[i];
    }
    derivs(x + h, yt, dyt);
    for (int i = 0; i < 6; ++i) yo[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
    const bool this_err = 1. - (yo[1] * yo[1] + yo[3] * yo[3] + yo[5] * yo[5]) / (kC * kC) <= 0;
    if (error_gamma || this_err) {
      error_gamma = false;
      double yhalf[6], ysave[6];
      for (int i = 0; i < 6; ++i) ysave[i] = y[i];
      derivs(x, ysave, dydx);
      step(ysave, dydx, x, h / 2., yhalf);
      derivs(x + h / 2., yhalf, dydx);
      step(yhalf, dydx, x + h / 2., h / 2., yo);
    }
    for (int i = 0; i < 6; ++i) yout[i] = yo[i];
  }
};

// Adaptive Cash-Karp RK5(4) (src/OSCARSSR.cc:1392-1618, the driver / step / stage functions of the
// reference): stage and error coefficients as the reference declares them, the step controller with
// its safety factors, and output steps capped at the fixed-step interval DeltaT.
struct Rkas {
  Integrator& I;
  double delta_t, precision;

  void rkck(const double* x, const double* dxdt, double t, double h, double* xout, double* xerr) {
    static constexpr double a2 = 0.2, a3 = 0.3, a4 = 0.6, a5 = 1.0, a6 = 0.875;
    static constexpr double b21 = 0.2, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0, b41 = 0.3, b42 = -0.9, b43 = 1.2;
    static constexpr double b51 = -11.0 / 54.0, b52 = 2.5, b53 = -70.0 / 27.0, b54 = 35.0 / 27.0;
    static constexpr double b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0, b63 = 575.0 / 13824.0;
    static constexpr double b64 = 44275.0 / 110592.0, b65 = 253.0 / 4096.0;
    static constexpr double c1 = 37.0 / 378.0, c3 = 250.0 / 621.0, c4 = 125.0 / 594.0, c6 = 512.0 / 1771.0;
    static constexpr double dc5 = -277.00 / 14336.0, dc1 = c1 - 2825.0 / 27648.0, dc3 = c3 - 18575.0 / 48384.0;
    static constexpr double dc4 = c4 - 13525.0 / 55296.0, dc6 = c6 - 0.25;
    double dx2[6], dx3[6], dx4[6], dx5[6], dx6[6], xt[6];
    for (int i = 0; i != 6; ++i) xt[i] = x[i] + b21 * h * dxdt[i];
    I.derivs(t + a2 * h, xt, dx2);
    for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b31 * dxdt[i] + b32 * dx2[i]);
    I.derivs(t + a3 * h, xt, dx3);
    for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b41 * dxdt[i] + b42 * dx2[i] + b43 * dx3[i]);
    I.derivs(t + a4 * h, xt, dx4);
    for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b51 * dxdt[i] + b52 * dx2[i] + b53 * dx3[i] + b54 * dx4[i]);
    I.derivs(t + a5 * h, xt, dx5);
    for (int i = 0; i != 6; ++i)
      xt[i] = x[i] + h * (b61 * dxdt[i] + b62 * dx2[i] + b63 * dx3[i] + b64 * dx4[i] + b65 * dx5[i]);
    I.derivs(t + a6 * h, xt, dx6);
    for (int i = 0; i != 6; ++i) xout[i] = x[i] + h * (c1 * dxdt[i] + c3 * dx3[i] + c4 * dx4[i] + c6 * dx6[i]);
    for (int i = 0; i != 6; ++i)
      xerr[i] = h * (dc1 * dxdt[i] + dc3 * dx3[i] + dc4 * dx4[i] + dc5 * dx5[i] + dc6 * dx6[i]);
  }

  // One accepted step from t with trial step htry; returns the step size for the next one.
  double rkqs(double* x, double* dxdt, double* t, double htry, const double* xscale) {
    double h = htry, max_error = 0, xt[6], xe[6];
    for (;;) {
      I.error_gamma = false;
      rkck(x, dxdt, *t, h, xt, xe);
      max_error = 0.0;
      for (int i = 0; i != 6; ++i) max_error = std::fmax(max_error, std::fabs(xe[i] / xscale[i]));
      max_error /= precision;
      if (max_error <= 1.0 && !I.error_gamma) break;
      const double htemp = I.error_gamma ? 0.25 * h : 0.9 * h * std::pow(max_error, -0.25);
      h = (h >= 0.0 ? std::fmax(htemp, 0.1 * h) : std::fmin(htemp, 0.1 * h));
      if ((*t) + h == *t)
        throw Error{OSC_ERR_RANGE, "stepsize underflow in rkqs.  Possible you have a discontinuous field"};
    }
    double hnext = max_error > 1.89e-4 ? 0.9 * h * std::pow(max_error, -0.2) : 5.0 * h;
    if (std::fabs(hnext) > delta_t) hnext = delta_t * (hnext >= 0 ? 1 : -1);  // output step cap
    *t += h;
    for (int i = 0; i != 6; ++i) x[i] = xt[i];
    return hnext;
  }

  // From T1 to T2: every accepted step's start point with its derivative, then the end point (with
  // the derivative of the last step's start, as the reference stores it).
  void propagate(double* xstart, double T1, double T2, std::vector<double>& buf);
};

inline void push_point(std::vector<double>& buf, const double* x, const double* dxdt, double t) {
  buf.push_back(t);
  buf.push_back(x[0]); buf.push_back(x[2]); buf.push_back(x[4]);
  buf.push_back(x[1] / kC); buf.push_back(x[3] / kC); buf.push_back(x[5] / kC);
  buf.push_back(dxdt[1] / kC); buf.push_back(dxdt[3] / kC); buf.push_back(dxdt[5] / kC);
}

void Rkas::propagate(double* xstart, double T1, double T2, std::vector<double>& buf) {
  double x[6], dxdt[6] = {0, 0, 0, 0, 0, 0}, xscale[6];
  double t = T1;
  double h = (T2 >= T1 ? delta_t : -delta_t);
  for (int i = 0; i != 6; ++i) x[i] = xstart[i];
  for (int nstp = 0; nstp != 10000000; ++nstp) {
    I.derivs(t, x, dxdt);
    for (int i = 0; i != 6; ++i) xscale[i] = std::fabs(x[i]) + std::fabs(dxdt[i] * h) + 1.0e-30;
    push_point(buf, x, dxdt, t);
    if ((t + h - T2) * (t + h - T1) > 0.0) h = T2 - t;
    const double hnext = rkqs(x, dxdt, &t, h, xscale);
    if ((t - T2) * (T2 - T1) >= 0.0) {
      for (int i = 0; i != 6; ++i) xstart[i] = x[i];
      push_point(buf, x, dxdt, t);
      return;
    }
    if (std::fabs(hnext) <= 1e-30)
      throw Error{OSC_ERR_RANGE, "Reached minimum stepsize in PropogateRKAS without convergence"};
    h = hnext;
  }
  throw Error{OSC_ERR_RANGE, "Too many steps taken in routine PropogateRKAS"};
}

}  // namespace

void Model::set_trajectory_calculation(const std::string& method, double precision) {
  std::string m = method;
  for (char& c : m) c = (char)std::toupper((unsigned char)c);
  const char* kRk4Precision = "RK4 Trajectory does not use the precision parameter and you are attempting to set it";
  int which;
  if (m == "RK4") {
    if (precision != -1) throw Error{OSC_ERR_INVALID, kRk4Precision};
    which = kRK4;
  } else if (m == "RKAS") {
    which = kRKAS;
  } else {
    throw Error{OSC_ERR_INVALID, "Method requested is invalid.  Try again"};
  }
  traj_method = which;  // src/OSCARSSR.cc:805-818: the method is set before the precision is checked
  if (precision != -1) {
    if (which == kRK4) throw Error{OSC_ERR_INVALID, kRk4Precision};
    if (precision <= 0) throw Error{OSC_ERR_INVALID, "Trajectory precision cannot be >= 0"};
    traj_precision = precision;
  }
}

void Model::compute_trajectory() {
  knots.clear();
  ++knots_version;
  integrate(particle, knots, sweep, true);
}

void Model::integrate(const Particle& P, Knots& knots, std::vector<double>* sweep, bool threads) const {
  if (!P.set) throw Error{OSC_ERR_RANGE, "particle not initialized.  make sure you have a particle or beam defined"};
  if (ctstart > P.t0 || ctstop < P.t0)
    throw Error{OSC_ERR_RANGE, "start time is greater than T0 or stop time is less than T0"};
  if (ctstart >= ctstop)
    throw Error{OSC_ERR_RANGE, "start time is greater than stop time.  check that set_ctstartstop is set"};
  knots.clear();
  const double dt = ((ctstop - ctstart) / kC / (npoints - 1));
  if (traj_method == kRKAS) {  // src/OSCARSSR.cc:1015-1072
    std::vector<double>& fwd = sweep[0];
    std::vector<double>& bwd = sweep[1];
    fwd.clear();
    bwd.clear();
    auto run = [&](int dir) {
      Integrator I{fields, P.qomg};
      Rkas R{I, dt, traj_precision};
      double x[6] = {P.x0.x, P.b0.x * kC, P.x0.y, P.b0.y * kC, P.x0.z, P.b0.z * kC};
      double dxdt[6] = {0, 0, 0, 0, 0, 0};
      I.derivs(P.t0 / kC, x, dxdt);  // the reference evaluates it first (its value is not used)
      R.propagate(x, P.t0 / kC, (dir == 0 ? ctstop : ctstart) / kC, dir == 0 ? fwd : bwd);
    };
    if (threads) {
      parallel_tasks(2, run);
    } else {
      run(0);
      run(1);
    }
    // forward reversed, backward appended, all reversed: the backward points earliest first, then the
    // forward ones; both start at t0, so t0 appears twice (as in the reference)
    const int64_t nf = (int64_t)fwd.size() / 10, nb = (int64_t)bwd.size() / 10, n = nf + nb;
    if (n < 3)
      throw Error{OSC_ERR_LENGTH, "TSpline1D3 does not see enough points for interpolation.  Please use >= 3 points"};
    knots.n = n;
    knots.t.resize(n);
    knots.y.resize(9 * n);
    for (int64_t j = 0; j < nb; ++j) {
      const double* r = &bwd[10 * (nb - 1 - j)];
      knots.t[j] = r[0];
      for (int c = 0; c < 9; ++c) knots.y[c * n + j] = r[1 + c];
    }
    for (int64_t j = 0; j < nf; ++j) {
      const double* r = &fwd[10 * j];
      knots.t[nb + j] = r[0];
      for (int c = 0; c < 9; ++c) knots.y[c * n + nb + j] = r[1 + c];
    }
    knots.tstart = knots.t.front();
    knots.tstop = knots.t.back();
    spline_second_derivatives(knots, threads);
    return;
  }
  const size_t nf = (size_t)(1 + (ctstop - P.t0) / kC / dt);
  const size_t nb = (size_t)((P.t0 - ctstart) / kC / dt);

  // The forward and backward sweeps are independent integrations from the same initial state; they
  // run on two host threads and are stitched together afterwards (backward reversed, then forward).
  std::vector<double>& fwd = sweep[0];
  std::vector<double>& bwd = sweep[1];
  fwd.clear();
  bwd.clear();
  fwd.reserve(10 * nf);
  bwd.reserve(10 * nb);
  auto forward = [&]() {
    Integrator I{fields, P.qomg};
    double x[6] = {P.x0.x, P.b0.x * kC, P.x0.y, P.b0.y * kC, P.x0.z, P.b0.z * kC};
    double dxdt[6] = {0, 0, 0, 0, 0, 0};
    I.derivs(P.t0 / kC, x, dxdt);
    for (size_t i = 0; i != nf; ++i) {
      const double t = P.t0 / kC + dt * i;
      if (i == 0) I.derivs(t, x, dxdt);
      push_point(fwd, x, dxdt, t);
      I.derivs(t, x, dxdt);
      I.step(x, dxdt, t, dt, x);
    }
  };
  auto backward = [&]() {
    Integrator I{fields, P.qomg};
    double x[6] = {P.x0.x, P.b0.x * kC, P.x0.y, P.b0.y * kC, P.x0.z, P.b0.z * kC};
    double dxdt[6] = {0, 0, 0, 0, 0, 0};
    const double dtr = -dt;
    for (size_t i = 0; i != nb; ++i) {
      const double t1 = P.t0 / kC + dtr * (i);
      const double t2 = P.t0 / kC + dtr * (i + 1);
      I.derivs(t1, x, dxdt);
      I.step(x, dxdt, t1, dtr, x);
      push_point(bwd, x, dxdt, t2);
    }
  };
  if (threads && nf + nb > 4096) {
    parallel_tasks(2, [&](int i) {
      if (i == 0) forward();
      else backward();
    });
  } else {
    forward();
    backward();
  }
  const int64_t n = (int64_t)(nf + nb);
  if (n < 2) throw Error{OSC_ERR_LENGTH, "Not enough points in this trajectory"};
  if (n < 3) throw Error{OSC_ERR_LENGTH, "TSpline1D3 does not see enough points for interpolation.  Please use >= 3 points"};
  knots.n = n;
  knots.t.resize(n);
  knots.y.resize(9 * n);
  for (int64_t j = 0; j < (int64_t)nb; ++j) {  // backward points, earliest first
    const double* r = &bwd[10 * (nb - 1 - j)];
    knots.t[j] = r[0];
    for (int c = 0; c < 9; ++c) knots.y[c * n + j] = r[1 + c];
  }
  for (int64_t j = 0; j < (int64_t)nf; ++j) {
    const double* r = &fwd[10 * j];
    knots.t[nb + j] = r[0];
    for (int c = 0; c < 9; ++c) knots.y[c * n + nb + j] = r[1 + c];
  }
  knots.tstart = knots.t.front();
  knots.tstop = knots.t.back();
  spline_second_derivatives(knots, threads);
}

void Model::set_trajectory(const double* traj, int64_t n) {
  if (n < 3) throw Error{OSC_ERR_LENGTH, "TSpline1D3 does not see enough points for interpolation.  Please use >= 3 points"};
  // times may repeat (an RKAS trajectory stores its start time twice; the spline is then NaN there, as
  // in the reference) but not decrease
  for (int64_t i = 1; i < n; ++i)
    if (!(traj[i] >= traj[i - 1])) throw Error{OSC_ERR_INVALID, "trajectory times must not decrease"};
  knots.clear();
  ++knots_version;
  knots.n = n;
  knots.t.assign(traj, traj + n);
  knots.y.assign(traj + n, traj + 10 * n);
  knots.tstart = knots.t.front();
  knots.tstop = knots.t.back();
  spline_second_derivatives(knots);
}

void Model::ensure_trajectory() {
  if (!particle.set) {
    if (!has_beam) throw Error{OSC_ERR_RANGE, "no beam defined"};
    random_particle();
  }
  if (knots.n == 0) compute_trajectory();
}

// ---------------------------------------------------------------------------------------------
// Spline (include/TOMATH.h:141-203): the diagonal recurrence depends only on the knot times, so it
// is shared by the 9 components; each component's right-hand side sweep runs on its own.
// ---------------------------------------------------------------------------------------------
void spline_second_derivatives(Knots& k, bool threads) {
  const int64_t N = k.n;
  const double* X = k.t.data();
  k.ypp.assign(9 * N, 0.0);
  std::vector<double>& diag = k.diag;
  diag.assign(N, 0.0);
  if (k.work.size() < (size_t)(11 * N)) k.work.resize(11 * N);
  double* sigv = k.work.data();
  double* pv = sigv + N;
  diag[0] = -0.5;
  for (int64_t i = 1; i < N - 1; ++i) {
    const double sig = (X[i] - X[i - 1]) / (X[i + 1] - X[i - 1]);
    const double p = sig * diag[i - 1] + 2;
    diag[i] = (sig - 1.) / p;
    sigv[i] = sig;
    pv[i] = p;
  }
  auto component = [&](int c) {
    const double* Y = k.y.data() + c * N;
    double* ypp = k.ypp.data() + c * N;
    double* u = k.work.data() + (2 + c) * N;
    const double dydx0 = (Y[1] - Y[0]) / (X[1] - X[0]);
    u[0] = (3. / (X[1] - X[0])) * ((Y[1] - Y[0]) / (X[1] - X[0]) - dydx0);
    for (int64_t i = 1; i < N - 1; ++i) {
      double ui = (Y[i + 1] - Y[i]) / (X[i + 1] - X[i]) - (Y[i] - Y[i - 1]) / (X[i] - X[i - 1]);
      u[i] = (6. * ui / (X[i + 1] - X[i - 1]) - sigv[i] * u[i - 1]) / pv[i];
    }
    const double qn = 0.5;
    const double dydxN = (Y[N - 1] - Y[N - 2]) / (X[N - 1] - X[N - 2]);
    const double un = (3. / (X[N - 1] - X[N - 2])) * (dydxN - (Y[N - 1] - Y[N - 2]) / (X[N - 1] - X[N - 2]));
    for (int64_t i = 0; i < N - 1; ++i) ypp[i] = diag[i];
    ypp[N - 1] = (un - qn * u[N - 2]) / (qn * diag[N - 2] + 1.);
    for (int64_t j = N - 2; j >= 0; --j) ypp[j] = ypp[j] * ypp[j + 1] + u[j];
  };
  if (threads && N > 4096) {
    parallel_tasks(9, component);
  } else {
    for (int c = 0; c < 9; ++c) component(c);
  }
}

// ---------------------------------------------------------------------------------------------
// Rectangle surface (src/TSurfacePoints_Rectangle.cc:140-315)
// ---------------------------------------------------------------------------------------------
void surface_rectangle(const std::string& plane_in, int nx1, int nx2, double w1, double w2, Vec3 rot,
                       Vec3 trans, int normal, double* xyz, double* normals, double* x1x2) {
  std::string P = plane_in;
  std::transform(P.begin(), P.end(), P.begin(), ::toupper);
  const double s1 = nx1 > 1 ? w1 / (nx1 - 1) : 0;
  const double s2 = nx2 > 1 ? w2 / (nx2 - 1) : 0;
  // start for (both>1, both<=1, nx1<=1, nx2<=1), step vectors and normal per plane
  struct Layout { Vec3 both, none, only2, only1, v1, v2, n; };
  Layout L;
  if (P == "XY") L = {v3(-w1 / 2., -w2 / 2., 0), v3(0, 0, 0), v3(0., -w2 / 2., 0), v3(-w1 / 2., 0, 0), v3(s1, 0, 0), v3(0, s2, 0), v3(0, 0, 1)};
  else if (P == "YX") L = {v3(-w2 / 2., -w1 / 2., 0), v3(0, 0, 0), v3(-w2 / 2., 0, 0), v3(0, -w1 / 2., 0), v3(0, s1, 0), v3(s2, 0, 0), v3(0, 0, -1)};
  else if (P == "XZ") L = {v3(-w1 / 2., 0, -w2 / 2.), v3(0, 0, 0), v3(0, 0, -w2 / 2.), v3(-w1 / 2., 0, 0), v3(s1, 0, 0), v3(0, 0, s2), v3(0, -1, 0)};
  else if (P == "ZX") L = {v3(-w2 / 2., 0, -w1 / 2.), v3(0, 0, 0), v3(-w2 / 2., 0, 0), v3(0., 0, -w1 / 2.), v3(0, 0, s1), v3(s2, 0, 0), v3(0, 1, 0)};
  else if (P == "YZ") L = {v3(0, -w1 / 2., -w2 / 2.), v3(0, 0, 0), v3(0, 0, -w2 / 2.), v3(0, -w1 / 2., 0), v3(0, s1, 0), v3(0, 0, s2), v3(1, 0, 0)};
  else if (P == "ZY") L = {v3(0, -w2 / 2., -w1 / 2.), v3(0, 0, 0), v3(0, -w2 / 2., 0), v3(0, 0, -w1 / 2.), v3(0, 0, s1), v3(0, s2, 0), v3(-1, 0, 0)};
  else throw Error{OSC_ERR_INVALID, "not a valid surface string: XY YX XZ ZX YZ ZY"};
  Vec3 st = (nx1 > 1 && nx2 > 1) ? L.both : (nx1 <= 1 && nx2 <= 1) ? L.none : (nx1 <= 1) ? L.only2 : L.only1;
  st = rotate_xyz(st, rot);
  const Vec3 v1 = rotate_xyz(L.v1, rot), v2 = rotate_xyz(L.v2, rot);
  st = st + trans;
  Vec3 nv = rotate_xyz(L.n, rot);
  if (normal == -1) nv = nv * -1;
  else if (normal != 0 && normal != 1) throw Error{OSC_ERR_INVALID, "normal must be -1, 0, or 1"};
  const double m1 = mag(v1), m2 = mag(v2);
  const int64_t n = (int64_t)nx1 * nx2;
  for (int64_t i = 0; i < n; ++i) {
    const int ix1 = (int)(i / nx2), ix2 = (int)(i % nx2);
    if (xyz) {
      const Vec3 p = (st + v1 * (double)ix1) + v2 * (double)ix2;
      xyz[3 * i] = p.x; xyz[3 * i + 1] = p.y; xyz[3 * i + 2] = p.z;
    }
    if (normals) { normals[3 * i] = nv.x; normals[3 * i + 1] = nv.y; normals[3 * i + 2] = nv.z; }
    if (x1x2) {
      x1x2[3 * i] = s1 * ix1 - m1 * (nx1 - 1) / 2.;
      x1x2[3 * i + 1] = s2 * ix2 - m2 * (nx2 - 1) / 2.;
      x1x2[3 * i + 2] = 0;
    }
  }
}

// Rectangle from three points (TSurfacePoints_Rectangle::Init(NX1, NX2, X0, X1, X2, Normal) and
// GetXYZ / GetX1 / GetX2, src/TSurfacePoints_Rectangle.cc:76-127, 280-317): the three points are
// rotated and translated first, as the binding does (src/OSCARSSR_Python.cc:6652-6658).
void surface_x0x1x2(int nx1, int nx2, Vec3 x0, Vec3 x1, Vec3 x2, Vec3 rot, Vec3 trans, int normal, double* xyz,
                    double* normals, double* x1x2) {
  if (nx1 < 2 || nx2 < 2) throw Error{OSC_ERR_INVALID, "'npoints' must be >= 2 in each direction with 'x0x1x2'"};
  if (normal != -1 && normal != 0 && normal != 1)
    throw Error{OSC_ERR_INVALID, "fNormal is of the incorrect form.  Must be -1, 0, 1"};
  x0 = rotate_xyz(x0, rot) + trans;
  x1 = rotate_xyz(x1, rot) + trans;
  x2 = rotate_xyz(x2, rot) + trans;
  const double w1 = mag(x1 - x0), w2 = mag(x2 - x0);
  const double s1 = w1 / (nx1 - 1), s2 = w2 / (nx2 - 1);
  const Vec3 v1 = (x1 - x0) / (double)(nx1 - 1), v2 = (x2 - x0) / (double)(nx2 - 1);
  Vec3 nv = unit(cross(v1, v2));
  if (normal == -1) nv = nv * -1;
  const double m1 = mag(v1), m2 = mag(v2);
  const int64_t n = (int64_t)nx1 * nx2;
  for (int64_t i = 0; i < n; ++i) {
    const int ix1 = (int)(i / nx2), ix2 = (int)(i % nx2);
    if (xyz) {
      const Vec3 p = (x0 + v1 * (double)ix1) + v2 * (double)ix2;
      xyz[3 * i] = p.x; xyz[3 * i + 1] = p.y; xyz[3 * i + 2] = p.z;
    }
    if (normals) { normals[3 * i] = nv.x; normals[3 * i + 1] = nv.y; normals[3 * i + 2] = nv.z; }
    if (x1x2) {
      x1x2[3 * i] = s1 * ix1 - m1 * (nx1 - 1) / 2.;
      x1x2[3 * i + 1] = s2 * ix2 - m2 * (nx2 - 1) / 2.;
      x1x2[3 * i + 2] = 0;
    }
  }
}

// Arbitrary surface points with normals as the calculate_flux / calculate_power_density bindings
// take them (src/OSCARSSR_Python.cc:7730-7750, 6225-6250): point and normal rotated, the normal
// reversed when invert_normals, the point translated.
void surface_points(int64_t n, const double* pts, const double* nrm, Vec3 rot, Vec3 trans, bool invert_normals,
                    double* xyz, double* normals) {
  for (int64_t i = 0; i < n; ++i) {
    Vec3 X = rotate_xyz(v3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), rot);
    Vec3 N = rotate_xyz(v3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]), rot);
    if (invert_normals) N = N * -1;
    X = X + trans;
    xyz[3 * i] = X.x; xyz[3 * i + 1] = X.y; xyz[3 * i + 2] = X.z;
    normals[3 * i] = N.x; normals[3 * i + 1] = N.y; normals[3 * i + 2] = N.z;
  }
}

}  // namespace osc
