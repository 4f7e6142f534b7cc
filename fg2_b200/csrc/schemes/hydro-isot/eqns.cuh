// schemes/hydro-isot/eqns.cuh -- right-hand side of the isothermal equations in
// log-density form with shear/bulk viscosity, optional density diffusion and optional
// Kolmogorov forcing.  Physics and runtime keys follow src/hydro-isot/eqns.cuh:19-87; the
// derivatives arrive precomputed in a Cell; C is the compute type (float or double).
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

// Parameter slots and the reference defaults (src/hydro-isot/eqns.cuh:19-25), then derived
// constants.
enum Slot { DD = 0, NUS = 1, NUB = 2, CS2 = 3, FAMP = 4, FK = 5, NSLOT = 6,
            NUS2 = 6, MIXED = 7, CS = 8 };
constexpr fg2::ParaKey PARA_KEYS[NSLOT] = {{"dd", DD, 0.0},   {"nus", NUS, 2.0e-4}, {"nub", NUB, 0.0},
                                           {"cs2", CS2, 1.0}, {"f", FAMP, 0.0},     {"k", FK, -8.0}};

inline void derive(double *v)
{
  v[NUS2] = 2.0 * v[NUS];
  v[MIXED] = v[NUS] / 3.0 + v[NUB];
  v[CS] = std::sqrt(v[CS2]);
}

constexpr unsigned D2_DEFAULT = (1u << U1) | (1u << U2);
constexpr unsigned D2_ALL = (1u << U1) | (1u << U2) | (1u << LND);
constexpr unsigned D12_FIELDS = (1u << U1) | (1u << U2);
inline unsigned d2_fields(const double *v)
{
  unsigned m = (1u << U1) | (1u << U2);
  if (v[DD] != 0.0) m |= 1u << LND;
  return m;
}

// Per-column geometry of a cell (none on the Cartesian grid).
template <class C>
struct Geom {};
template <class C>
FG2_HD Geom<C> column_geom(int j, C delta2)
{
  (void)j; (void)delta2;
  return Geom<C>{};
}

// dq/dt at one cell (Kolmogorov forcing varies with its row i).
template <unsigned M2, class C>
FG2_HD void eqns(const fg2::Cell<C, NVAR> &c, const fg2::Para<C> &p, int i, int j, C r[NVAR], C delta1, C delta2,
                 const Geom<C> &)
{
  using fg2::fmac;
  using fg2::lit;
  (void)j; (void)delta2;
  const C u1 = c.q[U1], u2 = c.q[U2];
  const C div = c.d1[U1] + c.d2[U2];
  const C m1 = lit<C>(-1.0);

  const C nl = fmac(u1, c.d1[LND], fmac(u2, c.d2[LND], div));
  const C n1 = fmac(u1, c.d1[U1], fmac(u2, c.d2[U1], p.v[CS2] * c.d1[LND]));
  const C n2 = fmac(u1, c.d1[U2], fmac(u2, c.d2[U2], p.v[CS2] * c.d2[LND]));

  const C s11 = fmac(div, lit<C>(-1.0 / 3.0), c.d1[U1]);
  const C s12 = (c.d1[U2] + c.d2[U1]) * lit<C>(0.5);
  const C s22 = fmac(div, lit<C>(-1.0 / 3.0), c.d2[U2]);
  C p1 = p.v[NUS2] * fmac(s11, c.d1[LND], s12 * c.d2[LND]);
  C p2 = p.v[NUS2] * fmac(s12, c.d1[LND], s22 * c.d2[LND]);
  p1 = fmac(p.v[NUS], c.d11[U1] + c.d22[U1], fmac(p.v[MIXED], c.d11[U1] + c.d12[U2], p1));
  p2 = fmac(p.v[NUS], c.d11[U2] + c.d22[U2], fmac(p.v[MIXED], c.d12[U1] + c.d22[U2], p2));

  // Kolmogorov forcing f cos(k x1) on u2 when f k < 0 (src/hydro-isot/eqns.cuh:81-84)
  if (fg2::first(p.v[FAMP]) * fg2::first(p.v[FK]) < 0)
    p2 = fmac(p.v[FAMP], fg2::vcos(p.v[FK] * lit<C>((double)i) * delta1), p2);

  r[U1] = fmac(n1, m1, p1);
  r[U2] = fmac(n2, m1, p2);
  if (M2 & (1u << LND))
    r[LND] = fmac(nl, m1, p.v[DD] * (c.d11[LND] + c.d22[LND] + fmac(c.d1[LND], c.d1[LND], c.d2[LND] * c.d2[LND])));
  else
    r[LND] = nl * m1;
}

template <class C>
FG2_HD C sound_speed(const C q[NVAR], const fg2::Para<C> &p)
{
  (void)q;
  return p.v[CS];
}

// CFL signal rate of a cell on the Cartesian grid: (|u1| + c_s) / Delta1 + (|u2| + c_s) / Delta2.
template <class C>
FG2_HD C signal_rate(const C q[NVAR], const fg2::Para<C> &p, C inv1, C inv2, int i, int j, C delta1, C delta2,
                     const Geom<C> &)
{
  (void)i; (void)j; (void)delta1; (void)delta2;
  const C cs = sound_speed<C>(q, p);
  return fg2::fmac(fg2::vabs(q[U1]) + cs, inv1, (fg2::vabs(q[U2]) + cs) * inv2);
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
