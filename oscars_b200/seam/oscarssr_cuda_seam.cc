// oscarssr_cuda_seam.cc -- the reference's GPU seam implemented on liboscars_b200.
//
// OSCARS compiled with -DCUDA sends every gpu=1 request of oscars.sr through four extern "C"
// functions (include/OSCARSSR_Cuda.h:28-66), called from OSCARSSR::Calculate*GPU
// (src/OSCARSSR.cc:2429, 3125, 4428) and OSCARSSR::CheckGPU / GetGPUInfo (:721, :734).  This file
// is a drop-in object for that seam: linked into the reference's own `sr` extension in place of its
// CUDA object, it makes stock `oscars.sr.sr(gpu=1)` compute on this library's sm_100a kernels.
//
// Division of work, as in the reference's own GPU code: the reference's host code draws each
// particle and integrates its trajectory (OSR.SetNewParticle / OSR.CalculateTrajectory, so every
// field type it supports works here too); the trajectory goes to the library
// (osc_set_particle_trajectory), the library's FP64 radiation path integrates it
// (osc_flux / osc_spectrum / osc_power_density: the reference's method, <= 1e-9 of its CPU path),
// and the per-point results are added into the caller's container with weight 1/N in particle
// order, exactly as OSCARSSR::CalculateFlux and friends add them (AddToPoint / AddToFlux,
// compensated).  Library errors become std::invalid_argument with the library's message, which the
// binding turns into ValueError.  One library context per host thread, on the first device of the
// request's GPU list.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "OSCARSSR_Cuda.h"
#include "TParticleA.h"
#include "TParticleTrajectoryPoints.h"
#include "TSpectrumContainer.h"
#include "TSurfacePoints.h"
#include "T3DScalarContainer.h"
#include "oscars_b200.h"

namespace {

struct SeamContext {
  osc_ctx* ctx = nullptr;
  int device = -1;
  ~SeamContext() {
    if (ctx) osc_ctx_destroy(ctx);
  }
};
thread_local SeamContext tl_ctx;

osc_ctx* context(std::vector<int> const& gpus) {
  const int device = gpus.empty() ? 0 : gpus.front();
  if (!tl_ctx.ctx || tl_ctx.device != device) {
    if (tl_ctx.ctx) osc_ctx_destroy(tl_ctx.ctx);
    tl_ctx.ctx = nullptr;
    osc_ctx* c = nullptr;
    if (osc_ctx_create(device, &c) != OSC_OK) throw std::invalid_argument(osc_last_error(nullptr));
    tl_ctx.ctx = c;
    tl_ctx.device = device;
  }
  return tl_ctx.ctx;
}

void check(osc_ctx* c, int rc) {
  if (rc != OSC_OK) throw std::invalid_argument(osc_last_error(c));
}

// Polarization selector from the request's string, matched as src/OSCARSSR.cc:4129-4150 matches it.
int polarization_code(std::string p) {
  std::transform(p.begin(), p.end(), p.begin(), ::tolower);
  std::replace(p.begin(), p.end(), ' ', '-');
  if (p.find("all") != std::string::npos) return OSC_POL_ALL;
  if (p.find("linear-horizontal") != std::string::npos || p.find("lh") != std::string::npos) return OSC_POL_LH;
  if (p.find("linear-vertical") != std::string::npos || p.find("lv") != std::string::npos) return OSC_POL_LV;
  if (p == "linear") return OSC_POL_LINEAR;
  if (p.find("circular-left") != std::string::npos || p.find("cl") != std::string::npos) return OSC_POL_CL;
  if (p.find("circular-right") != std::string::npos || p.find("cr") != std::string::npos) return OSC_POL_CR;
  throw std::invalid_argument("Polarization requested not recognized");
}

osc_rad_opts options(double precision, int max_level, int quantity) {
  osc_rad_opts o{};
  o.polarization = OSC_POL_ALL;
  o.horizontal[0] = 1;
  o.propagation[2] = 1;
  o.precision = precision;
  o.max_level = max_level;
  o.max_level_extended = 0;
  o.nparticles = 0;
  o.quantity = quantity;
  o.precision_mode = OSC_FP64;
  return o;
}

void set_polarization(osc_rad_opts& o, std::string const& pol, double angle, TVector3D const& h, TVector3D const& p) {
  o.polarization = polarization_code(pol);
  o.angle = angle;
  o.horizontal[0] = h.GetX(); o.horizontal[1] = h.GetY(); o.horizontal[2] = h.GetZ();
  o.propagation[0] = p.GetX(); o.propagation[1] = p.GetY(); o.propagation[2] = p.GetZ();
}

// The reference's current particle and its trajectory, handed to the library.
void install_trajectory(osc_ctx* c, OSCARSSR& OSR) {
  TParticleA const& P = OSR.GetCurrentParticle();
  TParticleTrajectoryPoints const& T = OSR.GetTrajectory();
  const size_t n = T.GetNPoints();
  std::vector<double> soa(10 * n);
  for (size_t i = 0; i < n; ++i) {
    const TVector3D& X = T.GetX(i);
    const TVector3D& B = T.GetB(i);
    const TVector3D& A = T.GetAoverC(i);
    soa[i] = T.GetT(i);
    soa[n + i] = X.GetX(); soa[2 * n + i] = X.GetY(); soa[3 * n + i] = X.GetZ();
    soa[4 * n + i] = B.GetX(); soa[5 * n + i] = B.GetY(); soa[6 * n + i] = B.GetZ();
    soa[7 * n + i] = A.GetX(); soa[8 * n + i] = A.GetY(); soa[9 * n + i] = A.GetZ();
  }
  const double x0[3] = {P.GetX0().GetX(), P.GetX0().GetY(), P.GetX0().GetZ()};
  const double b0[3] = {P.GetB0().GetX(), P.GetB0().GetY(), P.GetB0().GetZ()};
  check(c, osc_set_particle_trajectory(c, OSC_PARTICLE_CUSTOM, P.GetQ(), P.GetM(), P.GetCurrent(), x0, b0, P.GetT0(),
                                       soa.data(), (long long)n));
}

// Runs `one` for the current particle (NParticles == 0) or for NParticles new random particles, each
// with its trajectory, passing the weight its values are added with.
template <class F>
void for_each_particle(OSCARSSR& OSR, osc_ctx* c, int NParticles, F one) {
  if (NParticles == 0) {
    if (OSR.GetTrajectory().GetNPoints() == 0) OSR.CalculateTrajectory();
    install_trajectory(c, OSR);
    one(1.0);
    return;
  }
  const double weight = 1.0 / (double)NParticles;
  for (int i = 0; i != NParticles; ++i) {
    OSR.SetNewParticle();
    OSR.CalculateTrajectory();
    install_trajectory(c, OSR);
    one(weight);
  }
}

}  // namespace

extern "C" int OSCARSSR_Cuda_GetDeviceCount() {
  int n = 0;
  return osc_get_device_count(&n) == OSC_OK ? n : 0;
}

std::string OSCARSSR_Cuda_GetDeviceProperties(int const i) {
  char text[512];
  if (osc_get_device_properties(i, text, sizeof text) != OSC_OK) return std::string(osc_last_error(nullptr));
  return std::string(text);
}

extern "C" void OSCARSSR_Cuda_CalculateFluxGPU(OSCARSSR& OSR, TSurfacePoints const& Surface, double const Energy_eV,
                                               T3DScalarContainer& FluxContainer, std::string const& PolarizationIn,
                                               double const Angle, TVector3D const& HorizontalDirection,
                                               TVector3D const& PropogationDirection, int const NParticles,
                                               std::vector<int> const& GPUVector, double const Precision,
                                               int const MaxLevel, int const ReturnQuantity) {
  osc_ctx* c = context(GPUVector);
  osc_rad_opts o = options(Precision, MaxLevel, ReturnQuantity);
  set_polarization(o, PolarizationIn, Angle, HorizontalDirection, PropogationDirection);
  const size_t n = Surface.GetNPoints();
  std::vector<double> xyz(3 * n), out(n);
  std::vector<int32_t> level(n);
  for (size_t i = 0; i < n; ++i) {
    const TVector3D& X = Surface.GetPoint(i).GetPoint();
    xyz[3 * i] = X.GetX(); xyz[3 * i + 1] = X.GetY(); xyz[3 * i + 2] = X.GetZ();
  }
  for_each_particle(OSR, c, NParticles, [&](double weight) {
    check(c, osc_flux(c, xyz.data(), (long long)n, Energy_eV, &o, out.data(), level.data(), nullptr));
    for (size_t i = 0; i < n; ++i) {
      if (level[i] == -1) FluxContainer.SetNotConverged(i);
      FluxContainer.AddToPoint(i, out[i] * weight);
    }
  });
}

extern "C" void OSCARSSR_Cuda_CalculateSpectrumGPU(OSCARSSR& OSR, TVector3D const& ObservationPoint,
                                                   TSpectrumContainer& Spectrum, std::string const& PolarizationIn,
                                                   double const Angle, TVector3D const& HorizontalDirection,
                                                   TVector3D const& PropogationDirection, int const NParticles,
                                                   std::vector<int> const& GPUVector, double const Precision,
                                                   int const MaxLevel, int const ReturnQuantity) {
  osc_ctx* c = context(GPUVector);
  osc_rad_opts o = options(Precision, MaxLevel, ReturnQuantity);
  set_polarization(o, PolarizationIn, Angle, HorizontalDirection, PropogationDirection);
  const size_t n = Spectrum.GetNPoints();
  std::vector<double> energies(n), out(n);
  std::vector<int32_t> level(n);
  for (size_t i = 0; i < n; ++i) energies[i] = Spectrum.GetEnergy(i);
  const double obs[3] = {ObservationPoint.GetX(), ObservationPoint.GetY(), ObservationPoint.GetZ()};
  for_each_particle(OSR, c, NParticles, [&](double weight) {
    check(c, osc_spectrum(c, obs, energies.data(), (long long)n, &o, out.data(), level.data(), nullptr));
    for (size_t i = 0; i < n; ++i) {
      if (level[i] == -1) Spectrum.SetNotConverged(i);
      Spectrum.AddToFlux(i, out[i] * weight);
    }
  });
}

// The seam carries no `Directional` argument (the reference's GPU power density has none): the power
// density is the non-directional one, as the reference's GPU path computes it.
extern "C" void OSCARSSR_Cuda_CalculatePowerDensityGPU(OSCARSSR& OSR, TSurfacePoints const& Surface,
                                                       T3DScalarContainer& PowerDensityContainer, int const NParticles,
                                                       std::vector<int> const& GPUVector, double const Precision,
                                                       int const MaxLevel, int const ReturnQuantity) {
  osc_ctx* c = context(GPUVector);
  osc_rad_opts o = options(Precision, MaxLevel, ReturnQuantity);
  const size_t n = Surface.GetNPoints();
  std::vector<double> xyz(3 * n), nrm(3 * n), out(n);
  std::vector<int32_t> level(n);
  for (size_t i = 0; i < n; ++i) {
    const TSurfacePoint P = Surface.GetPoint(i);
    xyz[3 * i] = P.GetPoint().GetX(); xyz[3 * i + 1] = P.GetPoint().GetY(); xyz[3 * i + 2] = P.GetPoint().GetZ();
    nrm[3 * i] = P.GetNormal().GetX(); nrm[3 * i + 1] = P.GetNormal().GetY(); nrm[3 * i + 2] = P.GetNormal().GetZ();
  }
  for_each_particle(OSR, c, NParticles, [&](double weight) {
    check(c, osc_power_density(c, xyz.data(), nrm.data(), (long long)n, 0, &o, out.data(), level.data(), nullptr));
    for (size_t i = 0; i < n; ++i) {
      if (level[i] == -1) PowerDensityContainer.SetNotConverged(i);
      PowerDensityContainer.AddToPoint(i, out[i] * weight);
    }
  });
}
