// schemes/hydro/eqns.cuh -- right-hand side of the ideal-gas equations in log-primitive
// form, with shear/bulk viscosity, viscous heating, thermal conduction and optional
// density diffusion.  Physics and runtime keys follow src/hydro/eqns.cuh:19-92.  The
// derivatives arrive precomputed in a Cell; C is the compute type (float or double), and
// every product-sum is written as an explicit fmac.
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

// Parameter slots: the runtime keys with the reference defaults (src/hydro/eqns.cuh:19-24),
// then constants derived from them once per launch on the host.
enum Slot { GAMMA = 0, NUS = 1, NUB = 2, KAPPA = 3, DD = 4, NSLOT = 5,
            GM1 = 5, NUS2 = 6, MIXED = 7, ED = 8, CSG = 9 };
constexpr fg2::ParaKey PARA_KEYS[NSLOT] = {
    {"gamma", GAMMA, 5.0 / 3.0}, {"nus", NUS, 2.0e-4}, {"nub", NUB, 0.0},
    {"kappa", KAPPA, 5.0e-4},    {"dd", DD, 0.0}};

// gamma - 1, 2 nus, nus / 3 + nub, (gamma - 1) kappa, sqrt(gamma (gamma - 1))
inline void derive(double *v)
{
  v[GM1] = v[GAMMA] - 1.0;
  v[NUS2] = 2.0 * v[NUS];
  v[MIXED] = v[NUS] / 3.0 + v[NUB];
  v[ED] = (v[GAMMA] - 1.0) * v[KAPPA];
  v[CSG] = std::sqrt(v[GAMMA] * (v[GAMMA] - 1.0));
}

// Fields whose D11 and D22 the equations use for these parameters (u1 and u2 always, lne
// when kappa != 0, lnd when dd != 0), and the two masks the kernels are compiled for.
constexpr unsigned D2_DEFAULT = (1u << U1) | (1u << U2) | (1u << LNE);
constexpr unsigned D2_ALL = (1u << U1) | (1u << U2) | (1u << LNE) | (1u << LND);
constexpr unsigned D12_FIELDS = (1u << U1) | (1u << U2);
inline unsigned d2_fields(const double *v)
{
  unsigned m = (1u << U1) | (1u << U2);
  if (v[DD] != 0.0) m |= 1u << LND;
  if (v[KAPPA] != 0.0) m |= 1u << LNE;
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

// dq/dt at one cell.  M2 is the set of fields whose D11/D22 the caller
// evaluated; the others read as zero.  i, j and the spacings are unused by this scheme.
template <unsigned M2, class C>
FG2_HD void eqns(const fg2::Cell<C, NVAR> &c, const fg2::Para<C> &p, int i, int j, C r[NVAR], C delta1, C delta2,
                 const Geom<C> &)
{
  using fg2::fmac;
  using fg2::lit;
  (void)i; (void)j; (void)delta1; (void)delta2;
  const C u1 = c.q[U1], u2 = c.q[U2];
  const C ee = fg2::vexp(c.q[LNE]);    // specific thermal energy e
  const C iee = fg2::vexp(-c.q[LNE]);  // (gamma - 1) / temp = 1 / e
  const C temp = p.v[GM1] * ee;        // p / rho
  const C div = c.d1[U1] + c.d2[U2];
  const C m1 = lit<C>(-1.0);

  // terms of the form -(...): advection, compression, pressure gradient
  const C nl = fmac(u1, c.d1[LND], fmac(u2, c.d2[LND], div));
  const C n1 = fmac(u1, c.d1[U1], fmac(u2, c.d2[U1], temp * (c.d1[LND] + c.d1[LNE])));
  const C n2 = fmac(u1, c.d1[U2], fmac(u2, c.d2[U2], temp * (c.d2[LND] + c.d2[LNE])));
  const C ne = fmac(u1, c.d1[LNE], fmac(u2, c.d2[LNE], div * p.v[GM1]));

  // viscous stress and its divergence, viscous heating
  const C s11 = fmac(div, lit<C>(-1.0 / 3.0), c.d1[U1]);
  const C s12 = (c.d1[U2] + c.d2[U1]) * lit<C>(0.5);
  const C s22 = fmac(div, lit<C>(-1.0 / 3.0), c.d2[U2]);
  C p1 = p.v[NUS2] * fmac(s11, c.d1[LND], s12 * c.d2[LND]);
  C p2 = p.v[NUS2] * fmac(s12, c.d1[LND], s22 * c.d2[LND]);
  p1 = fmac(p.v[NUS], c.d11[U1] + c.d22[U1], fmac(p.v[MIXED], c.d11[U1] + c.d12[U2], p1));
  p2 = fmac(p.v[NUS], c.d11[U2] + c.d22[U2], fmac(p.v[MIXED], c.d12[U1] + c.d22[U2], p2));
  const C heat = fmac(p.v[NUS2], fmac(s11, s11, fmac(s12 + s12, s12, s22 * s22)), p.v[NUB] * div * div);

  // conduction (and density diffusion): Laplacian of the log plus |grad|^2
  C pe = iee * heat;
  if (M2 & (1u << LNE))
    pe = fmac(p.v[ED], c.d11[LNE] + c.d22[LNE] + fmac(c.d1[LNE], c.d1[LNE], c.d2[LNE] * c.d2[LNE]), pe);
  r[U1] = fmac(n1, m1, p1);
  r[U2] = fmac(n2, m1, p2);
  r[LNE] = fmac(ne, m1, pe);
  if (M2 & (1u << LND))
    r[LND] = fmac(nl, m1, p.v[DD] * (c.d11[LND] + c.d22[LND] + fmac(c.d1[LND], c.d1[LND], c.d2[LND] * c.d2[LND])));
  else
    r[LND] = nl * m1;
}

// Adiabatic sound speed sqrt(gamma (gamma - 1) e) = CSG exp(lne / 2), for the CFL condition.
template <class C>
FG2_HD C sound_speed(const C q[NVAR], const fg2::Para<C> &p)
{
  return p.v[CSG] * fg2::vexp(q[LNE] * fg2::lit<C>(0.5));
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
