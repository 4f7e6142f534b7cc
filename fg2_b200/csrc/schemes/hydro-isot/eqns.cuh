// schemes/hydro-isot/eqns.cuh -- right-hand side of the isothermal equations in
// log-density form with shear/bulk viscosity, optional density diffusion and optional
// Kolmogorov forcing.  Physics and runtime keys follow src/hydro-isot/eqns.cuh:19-87;
// the derivatives arrive precomputed in a Cell.
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

// Parameter slots and the reference defaults (src/hydro-isot/eqns.cuh:19-25).
enum Slot { DD = 0, NUS = 1, NUB = 2, CS2 = 3, FAMP = 4, FK = 5, NSLOT = 6 };
constexpr fg2::ParaKey PARA_KEYS[NSLOT] = {{"dd", DD, 0.0},   {"nus", NUS, 2.0e-4}, {"nub", NUB, 0.0},
                                           {"cs2", CS2, 1.0}, {"f", FAMP, 0.0},     {"k", FK, -8.0}};

template <class C>
FG2_HD unsigned d2_fields(const fg2::Para<C> &p)
{
  unsigned m = (1u << U1) | (1u << U2);
  if (p.v[DD] != C(0)) m |= 1u << LND;
  return m;
}
constexpr unsigned D12_FIELDS = (1u << U1) | (1u << U2);

template <class C>
FG2_HD C fcos(C x);
template <>
FG2_HD float fcos<float>(float x) { return cosf(x); }
template <>
FG2_HD double fcos<double>(double x) { return cos(x); }

// dq/dt at one cell; i is the global axis-1 index (Kolmogorov forcing varies along it).
template <class C>
FG2_HD void eqns(const fg2::Cell<C, NVAR> &c, const fg2::Para<C> &p, int i, int j, C r[NVAR], C delta1)
{
  (void)j;
  const C u1 = c.q[U1], u2 = c.q[U2];
  const C nus = p.v[NUS], nub = p.v[NUB], cs2 = p.v[CS2];
  const C div = c.d1[U1] + c.d2[U2];
  const C third = C(1.0 / 3.0);

  C rl = -(u1 * c.d1[LND] + u2 * c.d2[LND]);
  C r1 = -(u1 * c.d1[U1] + u2 * c.d2[U1]);
  C r2 = -(u1 * c.d1[U2] + u2 * c.d2[U2]);

  rl -= div;
  r1 -= cs2 * c.d1[LND];
  r2 -= cs2 * c.d2[LND];

  const C s11 = c.d1[U1] - div * third;
  const C s12 = (c.d1[U2] + c.d2[U1]) * C(0.5);
  const C s22 = c.d2[U2] - div * third;
  const C nus2 = C(2) * nus;
  r1 += nus2 * (s11 * c.d1[LND] + s12 * c.d2[LND]);
  r2 += nus2 * (s12 * c.d1[LND] + s22 * c.d2[LND]);

  const C mixed = nus * third + nub;
  r1 += nus * (c.d11[U1] + c.d22[U1]) + mixed * (c.d11[U1] + c.d12[U2]);
  r2 += nus * (c.d11[U2] + c.d22[U2]) + mixed * (c.d12[U1] + c.d22[U2]);

  rl += p.v[DD] * (c.d11[LND] + c.d1[LND] * c.d1[LND] + c.d22[LND] + c.d2[LND] * c.d2[LND]);

  // Kolmogorov forcing f cos(k x1) on u2 when f k < 0 (src/hydro-isot/eqns.cuh:81-84)
  if (p.v[FAMP] * p.v[FK] < C(0)) r2 += p.v[FAMP] * fcos(p.v[FK] * C(i) * delta1);

  r[LND] = rl;
  r[U1] = r1;
  r[U2] = r2;
}

template <class C>
FG2_HD C sound_speed(const C q[NVAR], const fg2::Para<C> &p)
{
  (void)q;
  return sqrt(p.v[CS2]);
}

inline double max_diffusivity(const double *v)
{
  double d = 4.0 / 3.0 * v[NUS] + v[NUB];
  if (v[DD] > d) d = v[DD];
  return d;
}

// Conserved densities for the FP64 sums: rho, rho u1, rho u2, kinetic energy.
FG2_HD void conserved(const double *q, double out[4])
{
  const double rho = exp(q[LND]);
  out[0] = rho;
  out[1] = rho * q[U1];
  out[2] = rho * q[U2];
  out[3] = 0.5 * rho * (q[U1] * q[U1] + q[U2] * q[U2]);
}

}  // namespace scheme
