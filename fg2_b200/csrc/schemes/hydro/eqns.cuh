// schemes/hydro/eqns.cuh -- right-hand side of the ideal-gas equations in log-primitive
// form, with shear/bulk viscosity, viscous heating, thermal conduction and optional
// density diffusion.  Physics and runtime keys follow src/hydro/eqns.cuh:19-92; the
// derivatives arrive precomputed in a Cell (the kernel evaluates only the ones listed
// by d2_fields()), and the arithmetic is arranged for the GPU: reciprocals instead of
// divisions, 1/e instead of (gamma-1)/temp.
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

// Parameter slots and the reference defaults (src/hydro/eqns.cuh:19-24).
enum Slot { GAMMA = 0, NUS = 1, NUB = 2, KAPPA = 3, DD = 4, NSLOT = 5 };
constexpr fg2::ParaKey PARA_KEYS[NSLOT] = {
    {"gamma", GAMMA, 5.0 / 3.0}, {"nus", NUS, 2.0e-4}, {"nub", NUB, 0.0},
    {"kappa", KAPPA, 5.0e-4},    {"dd", DD, 0.0}};

// Fields whose second derivatives (D11, D22) the kernel must evaluate for these
// parameters; D12 is needed for u1 and u2 only.
template <class C>
FG2_HD unsigned d2_fields(const fg2::Para<C> &p)
{
  unsigned m = (1u << U1) | (1u << U2);
  if (p.v[DD] != C(0)) m |= 1u << LND;
  if (p.v[KAPPA] != C(0)) m |= 1u << LNE;
  return m;
}
constexpr unsigned D12_FIELDS = (1u << U1) | (1u << U2);

template <class C>
FG2_HD C fexp(C x);
template <>
FG2_HD float fexp<float>(float x) { return expf(x); }
template <>
FG2_HD double fexp<double>(double x) { return exp(x); }

// dq/dt at one cell.  i, j are the global cell indices and delta1 the axis-1 spacing
// (all unused by this scheme).
template <class C>
FG2_HD void eqns(const fg2::Cell<C, NVAR> &c, const fg2::Para<C> &p, int i, int j, C r[NVAR], C delta1)
{
  (void)i; (void)j; (void)delta1;
  const C u1 = c.q[U1], u2 = c.q[U2];
  const C gamma = p.v[GAMMA], nus = p.v[NUS], nub = p.v[NUB];
  const C gm1 = gamma - C(1);
  const C ee = fexp(c.q[LNE]);        // specific thermal energy
  const C temp = gm1 * ee;            // p / rho
  const C iee = C(1) / ee;            // (gamma-1) / temp
  const C div = c.d1[U1] + c.d2[U2];
  const C third = C(1.0 / 3.0);

  // advection
  C rl = -(u1 * c.d1[LND] + u2 * c.d2[LND]);
  C r1 = -(u1 * c.d1[U1] + u2 * c.d2[U1]);
  C r2 = -(u1 * c.d1[U2] + u2 * c.d2[U2]);
  C re = -(u1 * c.d1[LNE] + u2 * c.d2[LNE]);

  // compression and pressure gradient
  rl -= div;
  r1 -= temp * (c.d1[LND] + c.d1[LNE]);
  r2 -= temp * (c.d2[LND] + c.d2[LNE]);
  re -= div * gm1;

  // viscous force from the density gradient, viscous heating
  const C s11 = c.d1[U1] - div * third;
  const C s12 = (c.d1[U2] + c.d2[U1]) * C(0.5);
  const C s22 = c.d2[U2] - div * third;
  const C nus2 = C(2) * nus;
  r1 += nus2 * (s11 * c.d1[LND] + s12 * c.d2[LND]);
  r2 += nus2 * (s12 * c.d1[LND] + s22 * c.d2[LND]);
  re += iee * (nus2 * (s11 * s11 + C(2) * s12 * s12 + s22 * s22) + nub * div * div);

  // viscous stress divergence
  const C mixed = nus * third + nub;
  r1 += nus * (c.d11[U1] + c.d22[U1]) + mixed * (c.d11[U1] + c.d12[U2]);
  r2 += nus * (c.d11[U2] + c.d22[U2]) + mixed * (c.d12[U1] + c.d22[U2]);

  // density diffusion and thermal conduction (Laplacian of the log plus |grad|^2)
  const C ed = gm1 * p.v[KAPPA];
  rl += p.v[DD] * (c.d11[LND] + c.d22[LND] + (c.d1[LND] * c.d1[LND] + c.d2[LND] * c.d2[LND]));
  re += ed * (c.d11[LNE] + c.d22[LNE] + (c.d1[LNE] * c.d1[LNE] + c.d2[LNE] * c.d2[LNE]));

  r[LND] = rl;
  r[U1] = r1;
  r[U2] = r2;
  r[LNE] = re;
}

// Adiabatic sound speed sqrt(gamma (gamma-1) e) for the CFL condition.
template <class C>
FG2_HD C sound_speed(const C q[NVAR], const fg2::Para<C> &p)
{
  const C gamma = p.v[GAMMA];
  return sqrt(gamma * (gamma - C(1)) * fexp(q[LNE]));
}

// Largest diffusion coefficient in the equations, for the explicit diffusive limit:
// longitudinal momentum (4/3 nus + nub), conduction ((gamma-1) kappa), density (dd).
inline double max_diffusivity(const double *v)
{
  double d = 4.0 / 3.0 * v[NUS] + v[NUB];
  const double k = (v[GAMMA] - 1.0) * v[KAPPA];
  if (k > d) d = k;
  if (v[DD] > d) d = v[DD];
  return d;
}

// Conserved densities of one cell for the FP64 sums: rho, rho u1, rho u2, total energy
// rho (e + |u|^2 / 2).
FG2_HD void conserved(const double *q, double out[4])
{
  const double rho = exp(q[LND]);
  out[0] = rho;
  out[1] = rho * q[U1];
  out[2] = rho * q[U2];
  out[3] = rho * (exp(q[LNE]) + 0.5 * (q[U1] * q[U1] + q[U2] * q[U2]));
}

}  // namespace scheme
