// The reference's GPU seam (include/OSCARSSR_Cuda.h:25-28) implemented on srs_b200.
//
// Compiled INSIDE the reference's build, in place of its src/OSCARSSR_Cuda.cu: with -DCUDA the
// reference's OSCARSSR.cc calls these four functions (OSCARSSR.cc:502, 900, 1882, 2588) after it has
// computed the particle's trajectory on the host; they gather the trajectory and the surface into
// plain arrays, call the library's host-buffer sums (plain FP64, the reference's CPU operation
// order) and add value * Weight into the caller's containers exactly where the reference's CUDA
// file does (AddToFlux / AddToPoint per output).  Needs the reference's headers on the include path
// and links against libsrs_b200.so; see oracle/Makefile (target dropin) for the recipe.
#include <stdexcept>
#include <string>
#include <vector>

#include "OSCARSSR_Cuda.h"
#include "srs_b200.h"

namespace {

struct Traj {
  std::vector<double> x, b, a;
  int64_t n = 0;
  double dt = 0;
};

Traj gather(TParticleA &P, bool with_aoc) {
  TParticleTrajectoryPoints &T = P.GetTrajectory();
  Traj t;
  t.n = (int64_t)T.GetNPoints();
  t.dt = T.GetDeltaT();
  t.x.resize(3 * t.n);
  t.b.resize(3 * t.n);
  if (with_aoc) t.a.resize(3 * t.n);
  for (int64_t i = 0; i < t.n; ++i) {
    const TVector3D &X = T.GetX(i), &B = T.GetB(i);
    t.x[i] = X.GetX(); t.x[t.n + i] = X.GetY(); t.x[2 * t.n + i] = X.GetZ();
    t.b[i] = B.GetX(); t.b[t.n + i] = B.GetY(); t.b[2 * t.n + i] = B.GetZ();
    if (with_aoc) {
      const TVector3D &A = T.GetAoverC(i);
      t.a[i] = A.GetX(); t.a[t.n + i] = A.GetY(); t.a[2 * t.n + i] = A.GetZ();
    }
  }
  return t;
}

void ok(srs_status s) {
  if (s != SRS_OK) throw std::invalid_argument(std::string("srs_b200: ") + srs_last_error());
}

}  // namespace

extern "C" int OSCARSSR_Cuda_GetDeviceCount() { return srs_device_count(); }

extern "C" void OSCARSSR_Cuda_CalculateSpectrumGPU(TParticleA &Particle, TVector3D const &ObservationPoint,
                                                   TSpectrumContainer &Spectrum, double const Weight) {
  const Traj t = gather(Particle, false);
  const int64_t ne = (int64_t)Spectrum.GetNPoints();
  std::vector<double> e(ne), out(ne);
  for (int64_t i = 0; i < ne; ++i) e[i] = Spectrum.GetEnergy(i);
  const double obs[3] = {ObservationPoint.GetX(), ObservationPoint.GetY(), ObservationPoint.GetZ()};
  ok(srs_spectrum_host(t.x.data(), t.b.data(), t.n, t.dt, srs_beam_consts{Particle.GetQ(), Particle.GetCurrent()},
                       obs, e.data(), ne, SRS_PRECISION_FP64, out.data()));
  for (int64_t i = 0; i < ne; ++i) Spectrum.AddToFlux(i, out[i] * Weight);
}

extern "C" void OSCARSSR_Cuda_CalculateFluxGPU(TParticleA &Particle, TSurfacePoints const &Surface,
                                               double const Energy_eV, T3DScalarContainer &FluxContainer,
                                               int const Dimension, double const Weight,
                                               std::string const &OutFileName) {
  (void)Dimension;
  (void)OutFileName;  // the reference's CUDA path writes no file either
  const Traj t = gather(Particle, false);
  const int64_t np = (int64_t)Surface.GetNPoints();
  std::vector<double> pts(3 * np), out(np);
  for (int64_t i = 0; i < np; ++i) {
    pts[3 * i] = Surface.GetPoint(i).GetX();
    pts[3 * i + 1] = Surface.GetPoint(i).GetY();
    pts[3 * i + 2] = Surface.GetPoint(i).GetZ();
  }
  ok(srs_flux_host(t.x.data(), t.b.data(), t.n, t.dt, srs_beam_consts{Particle.GetQ(), Particle.GetCurrent()},
                   pts.data(), np, Energy_eV, out.data()));
  for (int64_t i = 0; i < np; ++i) FluxContainer.AddToPoint(i, out[i] * Weight);
}

extern "C" void OSCARSSR_Cuda_CalculatePowerDensityGPU(TParticleA &Particle, TSurfacePoints const &Surface,
                                                       T3DScalarContainer &PowerDensityContainer, int const Dimension,
                                                       bool const Directional, double const Weight,
                                                       std::string const &OutFileName) {
  (void)Dimension;
  (void)OutFileName;
  const Traj t = gather(Particle, true);
  const int64_t np = (int64_t)Surface.GetNPoints();
  std::vector<double> pts(3 * np), nrm(3 * np), out(np);
  for (int64_t i = 0; i < np; ++i) {
    const TSurfacePoint &S = Surface.GetPoint(i);
    pts[3 * i] = S.GetX(); pts[3 * i + 1] = S.GetY(); pts[3 * i + 2] = S.GetZ();
    nrm[3 * i] = S.GetNormalX(); nrm[3 * i + 1] = S.GetNormalY(); nrm[3 * i + 2] = S.GetNormalZ();
  }
  ok(srs_power_density_host(t.x.data(), t.b.data(), t.a.data(), t.n, t.dt,
                            srs_beam_consts{Particle.GetQ(), Particle.GetCurrent()}, pts.data(), nrm.data(), np,
                            Directional ? 1 : 0, out.data()));
  for (int64_t i = 0; i < np; ++i) PowerDensityContainer.AddToPoint(i, out[i] * Weight);
}
