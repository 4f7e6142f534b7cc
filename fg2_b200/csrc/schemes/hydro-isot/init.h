// schemes/hydro-isot/init.h -- initial conditions of the isothermal scheme (host).
//
// The reference's setups (src/hydro-isot/init.h:21-49): Kf (a Kolmogorov flow plus tiny
// Gaussian noise) and the default zeros.  Added for the benchmark workloads:
//   noise  lnd = 0, u1, u2 ~ N(0, sigma^2) i.i.d. per cell  (sigma=0.01)
//   turb   lnd = 0, solenoidal random-phase velocity with E(k) ~ k^-2 on kmin <= |k| <= kmax,
//          rms |u| = mach * sqrt(cs2)  (mach=0.3, kmin=2, kmax=16)
#pragma once

#include <memory>

#include "setup_common.h"

namespace scheme {

namespace detail {

struct Kf : fg2::Setup {  // src/hydro-isot/init.h:21-33
  fg2::SetupCtx c;
  fg2::Rng rng;
  Kf(const fg2::SetupCtx &ctx) : c(ctx), rng(ctx.seed) {}
  void row(int i, double *out) override
  {
    const double x = c.l1 * (i + 0.5) / c.n1;
    const double nus = c.para[NUS], f = c.para[FAMP], k = c.para[FK];
    const double a = f / (nus * k * k);
    for (int j = 0; j < c.n2; ++j) {
      double *q = out + (size_t)j * NVAR;
      q[LND] = 0.0;
      q[U1] = 1.0e-9 * rng.normal();
      q[U2] = 1.0e-9 * rng.normal() + a * std::cos(k * x);
    }
  }
};

struct Noise : fg2::Setup {
  fg2::SetupCtx c;
  fg2::Rng rng;
  double sigma;
  Noise(const fg2::SetupCtx &ctx, const fg2::SetupName &nm) : c(ctx), rng(ctx.seed), sigma(nm.opt("sigma", 0.01)) {}
  void row(int i, double *out) override
  {
    (void)i;
    for (int j = 0; j < c.n2; ++j) {
      double *q = out + (size_t)j * NVAR;
      q[LND] = 0.0;
      q[U1] = sigma * rng.normal();
      q[U2] = sigma * rng.normal();
    }
  }
};

struct Turb : fg2::Setup {
  fg2::SetupCtx c;
  fg2::Rng rng;
  fg2::RandomVelocity vel;
  Turb(const fg2::SetupCtx &ctx, const fg2::SetupName &nm)
      : c(ctx), rng(ctx.seed),
        vel(ctx.n1, ctx.n2, nm.opt("kmin", 2), nm.opt("kmax", 16), nm.opt("slope", 2),
            nm.opt("mach", 0.3) * std::sqrt(ctx.para[CS2]), rng)
  {
  }
  void row(int i, double *out) override
  {
    vel.row(i, out, NVAR, U1, U2);
    for (int j = 0; j < c.n2; ++j) out[j * NVAR + LND] = 0.0;
  }
};

}  // namespace detail

inline std::unique_ptr<fg2::Setup> pick(const char *name, const fg2::SetupCtx &ctx)
{
  using namespace detail;
  const fg2::SetupName nm(name);
  if (nm.base == "Kf") return std::unique_ptr<fg2::Setup>(new Kf(ctx));
  if (nm.base == "noise") return std::unique_ptr<fg2::Setup>(new Noise(ctx, nm));
  if (nm.base == "turb") return std::unique_ptr<fg2::Setup>(new Turb(ctx, nm));
  return nullptr;
}

}  // namespace scheme
