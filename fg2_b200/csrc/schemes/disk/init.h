// schemes/disk/init.h -- initial conditions of the torus scheme (host).
//
// The reference's setup (src/disk/init.h:25-68): the hydrostatic Hawley (2000) torus with
// angular momentum l ~ R^(2 - q0), q0 = 2, pressure maximum at r0 = 16, density 1 and
// specific energy 0.01 there, inside a static background of density 1e-4 (which co-rotates
// with sin^2 theta times the torus law); the radiation energy is the background's
// equilibrium value everywhere.  Evaluated at cell centres (ln(r / r_in), theta) in the
// state's precision.
//   Hawley  (the reference's only setup; any other name selects it, as src/disk/init.h:60-68
//           does for every name)
// Added for benchmarks and tests:
//   smooth  a density bump on the equator, ln rho = -3 + 3 exp(-((ln r - l1/2)^2 +
//           (theta - pi/2)^2) / 0.3) + N(0, sigma^2), Keplerian-like Omega = (R + 1)^-1.5,
//           long-wavelength poloidal velocities of amplitude 1e-3, e = 0.01 (1 + 0.2 cos theta
//           sin(pi ln r / l1)) and radiation off its local equilibrium by a smooth factor,
//           e_rad = a_r T^4 / rho exp(0.3 cos 2 theta) (sigma=1e-4); smooth enough for
//           explicit steps of about 0.28 Delta^2
#pragma once

#include <cmath>
#include <memory>

#include "setup_common.h"

namespace scheme {

namespace detail {

// The torus in the state's precision R (float for FP32 and 16-bit states), with the
// reference's roundings: every quantity src/disk/init.h:25-58 keeps in an R variable is rounded
// to R and the mixed-precision calls (pow of an R and a double) stay in double, so FP32 states
// agree with the reference's bit for bit (tested against its own header).
struct Hawley : fg2::Setup {
  fg2::SetupCtx c;
  explicit Hawley(const fg2::SetupCtx &ctx) : c(ctx) {}
  template <class R>
  void fill(int i, double *out)
  {
    const R M = (R)c.para[MASS], rin = (R)c.para[RIN], Gamma = (R)c.para[GAMMA], ar = (R)c.para[AR];
    const R l1 = (R)c.l1, l2 = (R)c.l2;
    const R lnr = l1 * (i + 0.5) / c.n1;
    const R q0 = 2.0, r0 = 16.0, d0 = 1.0, e0 = 0.01, bg = 0.0001;
    const R g1 = Gamma - 1.0, q1 = 2.0 * q0 - 2.0;
    const R lK = std::sqrt(M * std::pow(r0, q1 - 1.0));  // specific angular momentum
    const R K = (g1 * e0) / std::pow(d0, g1);             // polytropic constant
    const R r = rin * std::exp(lnr);
    for (int j = 0; j < c.n2; ++j) {
      const R theta = l2 * (j + 0.5) / c.n2;
      const R cyl = r * std::sin(theta);
      // Bernoulli constant minus the local potential and centrifugal terms: the enthalpy
      R den = Gamma * e0 - M / r0 + lK * lK / (std::pow(r0, q1) * q1) + M / r - lK * lK / (std::pow(cyl, q1) * q1);
      if (den > 0.0) den = std::pow(den * g1 / (Gamma * K), 1.0 / g1);
      else den = -std::pow(-den * g1 / (Gamma * K), 1.0 / g1);
      R Omg = lK * std::pow(cyl, -q0);
      if (den < bg) {
        den = bg;
        Omg *= std::sin(theta) * std::sin(theta);
      }
      const R eng = K * std::pow(den, g1) / g1;
      const R tbg = K * std::pow(bg, g1);
      const R rad = ar * tbg * tbg * tbg * tbg / bg;
      double *q = out + (size_t)j * NVAR;
      q[LND] = std::log(den);
      q[UR] = 0.0;
      q[UZ] = 0.0;
      q[OMG] = Omg;
      q[LNE] = std::log(eng);
      q[LNER] = std::log(rad);
    }
  }
  void row(int i, double *out) override
  {
    if (c.single) fill<float>(i, out);
    else fill<double>(i, out);
  }
};

struct Smooth : fg2::Setup {
  fg2::SetupCtx c;
  fg2::Rng rng;
  double sigma;
  Smooth(const fg2::SetupCtx &ctx, const fg2::SetupName &nm) : c(ctx), rng(ctx.seed), sigma(nm.opt("sigma", 1e-4)) {}
  void row(int i, double *out) override
  {
    const double pi = 3.14159265358979323846;
    const double rin = c.para[RIN], gamma = c.para[GAMMA], ar = c.para[AR];
    const double lnr = c.l1 * (i + 0.5) / c.n1;
    const double r = rin * std::exp(lnr);
    for (int j = 0; j < c.n2; ++j) {
      const double th = c.l2 * (j + 0.5) / c.n2;
      const double a = lnr - 0.5 * c.l1, b = th - 0.5 * pi;
      double *q = out + (size_t)j * NVAR;
      q[LND] = -3.0 + 3.0 * std::exp(-(a * a + b * b) / 0.3) + sigma * rng.normal();
      q[UR] = 1e-3 * std::sin(2.0 * pi * lnr / c.l1) * std::sin(th);
      q[UZ] = 1e-3 * std::cos(2.0 * pi * lnr / c.l1) * std::sin(2.0 * th);
      q[OMG] = std::pow(r * std::sin(th) + 1.0, -1.5);
      const double eng = 0.01 * (1.0 + 0.2 * std::cos(th) * std::sin(pi * lnr / c.l1));
      const double temp = (gamma - 1.0) * eng;
      q[LNE] = std::log(eng);
      q[LNER] = std::log(ar * temp * temp * temp * temp / std::exp(q[LND])) + 0.3 * std::cos(2.0 * th);
    }
  }
};

}  // namespace detail

inline std::unique_ptr<fg2::Setup> pick(const char *name, const fg2::SetupCtx &ctx)
{
  const fg2::SetupName nm(name);
  if (nm.base == "smooth") return std::unique_ptr<fg2::Setup>(new detail::Smooth(ctx, nm));
  return std::unique_ptr<fg2::Setup>(new detail::Hawley(ctx));
}

}  // namespace scheme
