// schemes/hydro/init.h -- initial conditions of the ideal-gas scheme (host).
//
// The reference's setups (src/hydro/init.h:26-112): blast, bow, implos, KH, Sod and the
// default zeros, evaluated at cell centres; rand() noise is replaced by the seeded
// generator.  Added for the benchmark workloads:
//   noise  rho = 1, p = 1/gamma, u1, u2 ~ N(0, sigma^2) i.i.d. per cell  (sigma=0.01)
//   kh     tanh shear layer: u1 = 0.5 tanh((|y - L2/2| - L2/4) / w), rho from 1 (inner
//          layer) to 2 (outer), p = 2.5, u2 = 0.01 sin(4 pi x / L1) + N(0, 1e-4^2)  (w=0.01)
//   turb   rho = 1, p = 1/gamma, solenoidal random-phase velocity with E(k) ~ k^-2 on
//          kmin <= |k| <= kmax, rms |u| = mach * c_s  (mach=0.5, kmin=2, kmax=16)
#pragma once

#include <memory>

#include "setup_common.h"

namespace scheme {

namespace detail {

// The reference's named setups (blast, bow, implos, KH, Sod) compute in the state's precision
// R, as src/hydro/init.h:19-99 does with the cell centres of src/init.cpp:30-36: every quantity
// the reference keeps in an R variable is rounded to R, and the others stay in double, so FP32
// states agree with the reference's bit for bit (tested against its own header).  eval<R> is
// instantiated for float (FP32 and 16-bit storage) and double (FP64).
template <class R>
R fermi_dirac(R x, R d)
{
  return 1.0 / (std::exp(x / d) + 1.0);
}

struct RefSetup : fg2::Setup {
  fg2::SetupCtx c;
  fg2::SetupName nm;
  fg2::Rng rng;
  double gamma;
  RefSetup(const fg2::SetupCtx &ctx, const char *name)
      : c(ctx), nm(name), rng(ctx.seed), gamma(ctx.para[GAMMA]) {}
  virtual void eval_f(float x, float y, float *q) = 0;
  virtual void eval_d(double x, double y, double *q) = 0;
  template <class R>
  void fill(int i, double *out)
  {
    const R l1 = (R)c.l1, l2 = (R)c.l2;
    const R x = l1 * (i + 0.5) / c.n1;
    R q[NVAR];
    for (int j = 0; j < c.n2; ++j) {
      const R y = l2 * (j + 0.5) / c.n2;
      if constexpr (sizeof(R) == 4) eval_f(x, y, q);
      else eval_d(x, y, q);
      for (int f = 0; f < NVAR; ++f) out[(size_t)j * NVAR + f] = q[f];
    }
  }
  void row(int i, double *out) override
  {
    if (c.single) fill<float>(i, out);
    else fill<double>(i, out);
  }
};

struct Blast : RefSetup {  // src/hydro/init.h:26-34
  using RefSetup::RefSetup;
  template <class R>
  void eval(R x, R y, R *q)
  {
    const R g = (R)gamma;
    x -= 0.5 * (R)c.l1;
    y -= 0.5 * (R)c.l2;
    const R e = ((x * x + y * y < 0.01) ? 1.0 : 0.01) / (g - 1.0);
    q[LND] = 0; q[U1] = 0; q[U2] = 0; q[LNE] = std::log(e);
  }
  void eval_f(float x, float y, float *q) override { eval<float>(x, y, q); }
  void eval_d(double x, double y, double *q) override { eval<double>(x, y, q); }
};

struct Bow : RefSetup {  // src/hydro/init.h:36-47
  using RefSetup::RefSetup;
  template <class R>
  void eval(R x, R y, R *q)
  {
    const R g = (R)gamma;
    x -= 0.5 * (R)c.l1;
    y -= 0.5 * (R)c.l2;
    const R r = std::sqrt(x * x + y * y);
    const R d = 9.9 * fermi_dirac<R>(r - 0.01, 0.001) + 0.1;
    const R u = (10.0 / d - 1.0) / 99.0;
    const R e = 0.01 / d / (g - 1.0);
    q[LND] = std::log(d); q[U1] = u; q[U2] = 0; q[LNE] = std::log(e);
  }
  void eval_f(float x, float y, float *q) override { eval<float>(x, y, q); }
  void eval_d(double x, double y, double *q) override { eval<double>(x, y, q); }
};

struct Implos : RefSetup {  // src/hydro/init.h:49-58
  using RefSetup::RefSetup;
  template <class R>
  void eval(R x, R y, R *q)
  {
    const R g = (R)gamma;
    x -= 0.5 * (R)c.l1;
    y -= 0.5 * (R)c.l2;
    const double a = 0.15 - std::fabs((double)x) - std::fabs((double)y);
    const R d = 0.125 + 0.875 * fermi_dirac<R>(a, 0.001);
    const R p = 0.14 + 0.86 * fermi_dirac<R>(a, 0.001);
    // the ratio p / d is formed in R, the rest of the quotient and its log in double
    q[LND] = std::log(d); q[U1] = 0; q[U2] = 0; q[LNE] = (R)std::log(p / d / (g - 1.0));
  }
  void eval_f(float x, float y, float *q) override { eval<float>(x, y, q); }
  void eval_d(double x, double y, double *q) override { eval<double>(x, y, q); }
};

struct KHStep : RefSetup {  // src/hydro/init.h:60-76 (step profile, +-0.005 noise)
  using RefSetup::RefSetup;
  template <class R>
  void eval(R x, R y, R *q)
  {
    (void)x;
    const R g = (R)gamma;
    y -= 0.5 * (R)c.l2;
    const bool in = std::fabs((double)y) < 0.25;
    const R d = in ? 2.0 : 1.0;
    const R u = (in ? 0.5 : -0.5) + 0.01 * rng.uniform() - 0.005;
    const R e = 2.5 / d / (g - 1.0);
    q[LND] = std::log(d); q[U1] = u; q[U2] = 0; q[LNE] = std::log(e);
  }
  void eval_f(float x, float y, float *q) override { eval<float>(x, y, q); }
  void eval_d(double x, double y, double *q) override { eval<double>(x, y, q); }
};

struct Sod : RefSetup {  // src/hydro/init.h:78-94
  using RefSetup::RefSetup;
  template <class R>
  void eval(R x, R y, R *q)
  {
    const R g = (R)gamma;
    x -= 0.5 * (R)c.l1;
    y -= 0.5 * (R)c.l2;
    // the stripe test in R (x - 2 y + 1.5 mod 1), as the reference writes its literals in R
    const R t = x - 2 * y + (R)1.5;
    const bool left = std::fmod((double)t, (double)(R)1.0) < 0.5;
    const R d = left ? 1.0 : 0.125, P = left ? 1.0 : 0.1;
    const R e = P / d / (g - 1.0);
    q[LND] = std::log(d); q[U1] = 0; q[U2] = 0; q[LNE] = std::log(e);
  }
  void eval_f(float x, float y, float *q) override { eval<float>(x, y, q); }
  void eval_d(double x, double y, double *q) override { eval<double>(x, y, q); }
};

struct PointSetup : fg2::Setup {
  fg2::SetupCtx c;
  fg2::SetupName nm;
  fg2::Rng rng;
  double gamma;
  PointSetup(const fg2::SetupCtx &ctx, const char *name)
      : c(ctx), nm(name), rng(ctx.seed), gamma(ctx.para[GAMMA]) {}
  virtual void cell(double x, double y, double *q) = 0;
  void row(int i, double *out) override
  {
    const double x = c.l1 * (i + 0.5) / c.n1;
    for (int j = 0; j < c.n2; ++j) cell(x, c.l2 * (j + 0.5) / c.n2, out + (size_t)j * NVAR);
  }
};

struct Noise : PointSetup {
  double sigma;
  Noise(const fg2::SetupCtx &ctx, const char *name) : PointSetup(ctx, name), sigma(nm.opt("sigma", 0.01)) {}
  void cell(double x, double y, double *q) override
  {
    (void)x; (void)y;
    q[LND] = 0.0;
    q[U1] = sigma * rng.normal();
    q[U2] = sigma * rng.normal();
    q[LNE] = std::log(1.0 / (gamma * (gamma - 1.0)));  // p = 1/gamma at rho = 1
  }
};

struct KHTanh : PointSetup {
  double w;
  KHTanh(const fg2::SetupCtx &ctx, const char *name) : PointSetup(ctx, name), w(nm.opt("w", 0.01)) {}
  void cell(double x, double y, double *q) override
  {
    const double s = std::tanh((std::fabs(y / c.l2 - 0.5) - 0.25) / w);
    const double rho = 1.5 + 0.5 * s;  // 1 in the inner layer, 2 outside
    q[LND] = std::log(rho);
    q[U1] = 0.5 * s;
    q[U2] = 0.01 * std::sin(4.0 * 3.14159265358979323846 * x / c.l1) + 1e-4 * rng.normal();
    q[LNE] = std::log(2.5 / (rho * (gamma - 1.0)));
  }
};

struct Turb : fg2::Setup {
  fg2::SetupCtx c;
  fg2::Rng rng;
  fg2::RandomVelocity vel;
  double lne;
  Turb(const fg2::SetupCtx &ctx, const fg2::SetupName &nm)
      : c(ctx), rng(ctx.seed),
        vel(ctx.n1, ctx.n2, nm.opt("kmin", 2), nm.opt("kmax", 16), nm.opt("slope", 2),
            nm.opt("mach", 0.5) * 1.0 /* c_s = 1 at rho = 1, p = 1/gamma */, rng),
        lne(std::log(1.0 / (ctx.para[GAMMA] * (ctx.para[GAMMA] - 1.0))))
  {
  }
  void row(int i, double *out) override
  {
    vel.row(i, out, NVAR, U1, U2);
    for (int j = 0; j < c.n2; ++j) { out[j * NVAR + LND] = 0.0; out[j * NVAR + LNE] = lne; }
  }
};

}  // namespace detail

// The setup for `name`, or nullptr (the caller then starts from zeros, as the reference's
// pick() falls back to zeros for an unknown name, src/hydro/init.h:111).
inline std::unique_ptr<fg2::Setup> pick(const char *name, const fg2::SetupCtx &ctx)
{
  using namespace detail;
  const fg2::SetupName nm(name);
  const std::string &b = nm.base;
  if (b == "blast") return std::unique_ptr<fg2::Setup>(new Blast(ctx, name));
  if (b == "bow") return std::unique_ptr<fg2::Setup>(new Bow(ctx, name));
  if (b == "implos") return std::unique_ptr<fg2::Setup>(new Implos(ctx, name));
  if (b == "KH") return std::unique_ptr<fg2::Setup>(new KHStep(ctx, name));
  if (b == "Sod") return std::unique_ptr<fg2::Setup>(new Sod(ctx, name));
  if (b == "noise") return std::unique_ptr<fg2::Setup>(new Noise(ctx, name));
  if (b == "kh") return std::unique_ptr<fg2::Setup>(new KHTanh(ctx, name));
  if (b == "turb") return std::unique_ptr<fg2::Setup>(new Turb(ctx, nm));
  return nullptr;
}

}  // namespace scheme
