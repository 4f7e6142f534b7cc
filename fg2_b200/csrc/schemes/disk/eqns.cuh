// schemes/disk/eqns.cuh -- right-hand side of the radiative accretion-torus equations on a
// log-r / theta grid (axis 1: ln(r / r_in), axis 2: theta), with shear/bulk and
// Shakura-Sunyaev viscosity, conduction, simple diffusions, radiation force, heating/cooling
// and flux-limited radiation diffusion, and the point-mass gravity of a pseudo-Newtonian
// potential.  Physics and runtime keys follow src/disk/eqns.cuh:19-247.
//
// The derivatives arrive precomputed in a Cell (d1/d2 along ln r and theta, already divided
// by Delta); the position of the cell comes from its indices (i, j) and the grid spacings.
// The gradient in cylindrical (R, z) components is the rotation of the coordinate gradient by
// theta divided by r, the second derivatives follow from the same rotation plus its
// curvature terms.  Evaluated in the state precision C (float or double), one cell at a time;
// exp, sin/cos, sqrt and pow are the accurate library functions, reciprocals the hardware's
// (about one ulp in FP32).  sin and cos of the column's angle come from a per-column Geom that
// the kernel computes once per tile.
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

// Parameter slots with the reference defaults (src/disk/eqns.cuh:19-36), then constants
// derived from them on the host.
enum Slot { MASS = 0, RS = 1, RIN = 2, GAMMA = 3, NUS = 4, NUB = 5, KAPPA = 6, ALPHA = 7, AR = 8,
            ES = 9, FF = 10, DD = 11, NU = 12, ED = 13, RD = 14, NSLOT = 15,
            GM1 = 15, CSG = 16, IMASS = 17 };
constexpr fg2::ParaKey PARA_KEYS[NSLOT] = {
    {"M", MASS, 1.0},        {"rS", RS, 2.0},        {"rin", RIN, 3.0},     {"gamma", GAMMA, 5.0 / 3.0},
    {"nus", NUS, 0.0},       {"nub", NUB, 0.0},      {"kappa", KAPPA, 0.0}, {"alpha", ALPHA, 0.01},
    {"ar", AR, 1.0e+8},      {"es", ES, 1.0},        {"ff", FF, 0.0},       {"dd", DD, 1.0e-4},
    {"nu", NU, 2.0e-4},      {"ed", ED, 5.0e-4},     {"rd", RD, 5.0e-4}};

// gamma - 1, sqrt(gamma (gamma - 1)) (adiabatic sound speed factor), 1 / M
inline void derive(double *v)
{
  v[GM1] = v[GAMMA] - 1.0;
  v[CSG] = std::sqrt(v[GAMMA] * (v[GAMMA] - 1.0));
  v[IMASS] = 1.0 / v[MASS];
}

// Every field carries D11 and D22 (the Laplacians of all six enter), and the mixed
// derivative of ln rho, u_R, u_z and ln e_rad (the second derivatives in R and z).
constexpr unsigned D2_DEFAULT = 0x3fu;
constexpr unsigned D2_ALL = 0x3fu;
constexpr unsigned D12_FIELDS = (1u << LND) | (1u << UR) | (1u << UZ) | (1u << LNER);
inline unsigned d2_fields(const double *) { return D2_ALL; }

// Accurate math in the state precision.
namespace m {
FG2_HD float ex(float x) { return expf(x); }
FG2_HD double ex(double x) { return exp(x); }
FG2_HD float lg(float x) { return logf(x); }
FG2_HD double lg(double x) { return log(x); }
FG2_HD float sq(float x) { return sqrtf(x); }
FG2_HD double sq(double x) { return sqrt(x); }
FG2_HD float pw(float x, float y) { return powf(x, y); }
FG2_HD double pw(double x, double y) { return pow(x, y); }
FG2_HD void sc(float x, float *s, float *c) { sincosf(x, s, c); }
FG2_HD void sc(double x, double *s, double *c) { sincos(x, s, c); }
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
#else
inline float rcp(float x) { return 1.0f / x; }
#endif
FG2_HD double rcp(double x) { return 1.0 / x; }
}  // namespace m

// The column's angle theta = (j + 1/2) Delta2: its sine, cosine and 1 / sine.
template <class C>
struct Geom {
  C sint, cost, isint;
};
template <class C>
FG2_HD Geom<C> column_geom(int j, C delta2)
{
  Geom<C> g;
  m::sc(((C)j + C(0.5)) * delta2, &g.sint, &g.cost);
  g.isint = C(1) / g.sint;
  return g;
}

// Spherical radius of row i: r_in exp((i + 1/2) Delta1) (src/disk/eqns.cuh:51).
template <class C>
FG2_HD C sphr_of(int i, C rin, C delta1) { return rin * m::ex(((C)i + C(0.5)) * delta1); }

// dq/dt at cell (i, j).  M2 is unused: every field's D11/D22 is evaluated.
template <unsigned M2, class C>
FG2_HD void eqns(const fg2::Cell<C, NVAR> &c, const fg2::Para<C> &p, int i, int j, C r[NVAR], C delta1, C delta2,
                 const Geom<C> &g)
{
  using fg2::fmac;
  (void)j; (void)delta2;
  const C sint = g.sint, cost = g.cost;
  const C sphr = sphr_of<C>(i, p.v[RIN], delta1);
  const C isp = m::rcp(sphr);
  const C rc = sphr * sint;  // cylindrical radius
  const C irc = isp * g.isint;
  const C sp2 = sphr * sphr;
  const C isp2 = isp * isp;

  const C den = m::ex(c.q[LND]), eng = m::ex(c.q[LNE]), rad = m::ex(c.q[LNER]);
  const C g1 = p.v[GM1];
  const C temp = g1 * eng;
  const C nuss = p.v[ALPHA] * p.v[GAMMA] * temp * rc * m::sq(rc * p.v[IMASS]);  // Shakura-Sunyaev

  // gradient in (R, z): the (ln r, theta) gradient rotated by theta, over r
  const C sr = sint * isp, cr = cost * isp;
  C dr[NVAR], dz[NVAR], lap[NVAR];
#pragma unroll
  for (int f = 0; f < NVAR; ++f) {
    dr[f] = fmac(sr, c.d1[f], cr * c.d2[f]);
    dz[f] = fmac(cr, c.d1[f], -(sr * c.d2[f]));
    lap[f] = (c.d11[f] + c.d22[f]) * isp2;
  }
  // second derivatives in (R, z) of the fields that need them
  const C cc = cr * cr, cs = cr * sr, ss = sr * sr, c2 = cc - ss, s2 = cs + cs;
  auto drr = [&](int f) { return fmac(ss, c.d11[f], fmac(cc, c.d22[f], fmac(s2, c.d12[f], fmac(cr, dz[f], -(sr * dr[f]))))); };
  auto drz = [&](int f) { return fmac(cs, c.d11[f] - c.d22[f], fmac(c2, c.d12[f], -fmac(cr, dr[f], sr * dz[f]))); };
  auto dzz = [&](int f) { return fmac(cc, c.d11[f], fmac(ss, c.d22[f], fmac(-s2, c.d12[f], fmac(-cr, dz[f], sr * dr[f])))); };
  const C drr_lnd = drr(LND), drr_ur = drr(UR), drr_lner = drr(LNER);
  const C drz_lnd = drz(LND), drz_ur = drz(UR), drz_uz = drz(UZ), drz_lner = drz(LNER);
  const C dzz_lnd = dzz(LND), dzz_uz = dzz(UZ), dzz_lner = dzz(LNER);

  const C ur = c.q[UR], uz = c.q[UZ], om = c.q[OMG];
  C t[NVAR];
  // advection and the centrifugal / Coriolis pseudo-forces
#pragma unroll
  for (int f = 0; f < NVAR; ++f) t[f] = -fmac(ur, dr[f], uz * dz[f]);
  t[UR] = fmac(om * om, rc, t[UR]);
  t[OMG] = fmac(C(-2) * ur * om, irc, t[OMG]);

  // compression and pressure
  const C ur_r = ur * irc;
  const C div = dr[UR] + dz[UZ] + ur_r;
  t[LND] -= div;
  t[UR] = fmac(-temp, dr[LND] + dr[LNE], t[UR]);
  t[UZ] = fmac(-temp, dz[LND] + dz[LNE], t[UZ]);
  t[LNE] = fmac(-div, g1, t[LNE]);

  // viscous stress (density-gradient terms) and viscous heating
  const C third = C(1) / C(3);
  const C srr = fmac(-div, third, dr[UR]);
  const C szz = fmac(-div, third, dz[UZ]);
  const C spp = fmac(-div, third, ur_r);
  const C srz = (dz[UR] + dr[UZ]) * C(0.5);
  const C szp = rc * dz[OMG] * C(0.5);
  const C spr = rc * dr[OMG] * C(0.5);
  const C nut = p.v[NUS] + nuss;
  const C two_nus = nut + nut;
  t[UR] = fmac(two_nus, fmac(srr, dr[LND], srz * dz[LND]), t[UR]);
  t[UZ] = fmac(two_nus, fmac(srz, dr[LND], szz * dz[LND]), t[UZ]);
  t[OMG] = fmac(two_nus * fmac(spr, dr[LND], szp * dz[LND]), irc, t[OMG]);
  const C shear2 = fmac(srr, srr, fmac(szz, szz, spp * spp)) + C(2) * fmac(srz, srz, fmac(szp, szp, spr * spr));
  const C ieng = m::rcp(eng);
  t[LNE] = fmac(fmac(two_nus, shear2, p.v[NUB] * div * div), ieng, t[LNE]);

  // viscous stress divergence (velocity-only terms)
  const C tmp1 = fmac(p.v[NU], sp2, nut);
  const C tmp2 = nut * irc;
  const C dur = dr[UR] - ur_r;
  t[UR] = fmac(tmp1, lap[UR], fmac(tmp2, dur, t[UR]));
  t[UZ] = fmac(tmp1, lap[UZ], fmac(tmp2, dr[UZ], t[UZ]));
  t[OMG] = fmac(tmp1, lap[OMG], fmac(tmp2, C(3) * dr[OMG], t[OMG]));
  const C mixed = fmac(nut, third, p.v[NUB]);
  t[UR] = fmac(mixed, drr_ur + drz_uz + dur * irc, t[UR]);
  t[UZ] = fmac(mixed, drz_ur + dzz_uz + dz[UR] * irc, t[UZ]);

  // density diffusion and thermal conduction
  const C lap_d_d = lap[LND] + fmac(dr[LND], dr[LND], dz[LND] * dz[LND]);
  const C lap_e_e = lap[LNE] + fmac(dr[LNE], dr[LNE], dz[LNE] * dz[LNE]);
  t[LND] = fmac(lap_d_d, p.v[DD] * sp2, t[LND]);
  t[LNE] = fmac(lap_e_e, fmac(p.v[ED], sp2, fmac(p.v[KAPPA], g1, p.v[GAMMA] * nuss)), t[LNE]);

  // radiation force (flux-limited: Levermore-Pomraning limiter of R = |grad ln e_rad| / chi);
  // free-free opacity only when ff != 0, since 0 * pow(...) is 0 for every physical state
  const C kap = p.v[FF] != C(0) ? p.v[FF] * den * den * m::pw(temp, C(-3.5)) : C(0);
  const C chi = fmac(p.v[ES], den, kap);
  const C ichi = m::rcp(chi);
  const C d_lner_2 = fmac(dr[LNER], dr[LNER], dz[LNER] * dz[LNER]);
  const C bigR = m::sq(d_lner_2) * ichi;
  const C denom = fmac(C(3) + bigR, bigR, C(6));
  const C idenom = m::rcp(denom);
  const C Lambda = (C(2) + bigR) * idenom;
  t[UR] = fmac(-Lambda * rad, dr[LND] + dr[LNE], t[UR]);
  t[UZ] = fmac(-Lambda * rad, dz[LND] + dz[LNE], t[UZ]);

  // radiative heating / cooling
  const C temp2 = temp * temp;
  const C cooling = kap * fmac(p.v[AR] * temp2 * temp2, m::rcp(den), -rad);
  t[LNE] = fmac(-cooling, ieng, t[LNE]);
  t[LNER] = fmac(cooling, m::rcp(rad), t[LNER]);

  // radiation diffusion
  const C d_lnd_d_lner = fmac(dr[LND], dr[LNER], dz[LND] * dz[LNER]);
  const C lap_er_er = lap[LNER] + d_lner_2;
  const C nu_rad = Lambda * ichi;
  const C Lambdap = -bigR * (C(4) + bigR) * idenom * idenom;
  const C dr_e = dr[LND] + dr[LNER], dz_e = dz[LND] + dz[LNER];
  const C drr_e = drr_lnd + drr_lner, drz_e = drz_lnd + drz_lner, dzz_e = dzz_lnd + dzz_lner;
  const C dr_chi = fmac(chi, dr[LND], C(-3.5) * kap * dr[LNE]);
  const C dz_chi = fmac(chi, dz[LND], C(-3.5) * kap * dz[LNE]);
  const C iR = m::rcp(C(1e-16) + bigR);
  const C dr_bigR = (fmac(dr_e, drr_e, dz_e * drz_e) * iR * ichi - bigR * dr_chi) * ichi;
  const C dz_bigR = (fmac(dr_e, drz_e, dz_e * dzz_e) * iR * ichi - bigR * dz_chi) * ichi;
  C er = lap_er_er * p.v[RD] * sp2;
  er = fmac(nu_rad, lap_d_d + C(2) * d_lnd_d_lner + lap_er_er, er);
  er = fmac(dr_e * ichi, fmac(Lambdap, dr_bigR, -nu_rad * dr_chi), er);
  er = fmac(dz_e * ichi, fmac(Lambdap, dz_bigR, -nu_rad * dz_chi), er);
  t[LNER] += er;

  // gravity of the central mass, pseudo-Newtonian M / (r - r_S)^2
  const C gd = sphr - p.v[RS];
  const C gr = p.v[MASS] * m::rcp(gd * gd);
  t[UR] = fmac(-sint, gr, t[UR]);
  t[UZ] = fmac(-cost, gr, t[UZ]);

#pragma unroll
  for (int f = 0; f < NVAR; ++f) r[f] = t[f];
}

// Adiabatic sound speed sqrt(gamma (gamma - 1) e).
template <class C>
FG2_HD C sound_speed(const C q[NVAR], const fg2::Para<C> &p)
{
  return p.v[CSG] * m::ex(q[LNE] * C(0.5));
}

// Signal rate of a cell for the CFL limit: the velocity components along the grid axes
// (spherical r and theta, from the cylindrical u_R, u_z) plus the adiabatic sound speed,
// over the physical cell sizes r Delta1 and r Delta2.
template <class C>
FG2_HD C signal_rate(const C q[NVAR], const fg2::Para<C> &p, C inv1, C inv2, int i, int j, C delta1, C delta2,
                     const Geom<C> &g)
{
  (void)j; (void)delta2;
  const C sint = g.sint, cost = g.cost;
  const C sphr = sphr_of<C>(i, p.v[RIN], delta1);
  const C cs = sound_speed<C>(q, p);
  using fg2::fmac;
  const C u_r = fmac(sint, q[UR], cost * q[UZ]);
  const C u_t = fmac(cost, q[UR], -(sint * q[UZ]));
  return fmac(fg2::vabs(u_r) + cs, inv1, (fg2::vabs(u_t) + cs) * inv2) / sphr;
}

// Coefficient of the coordinate-space Laplacian of the simple diffusions (nu r^2 Lap,
// dd r^2 Lap, ... make the (ln r, theta) diffusivity constant): the explicit diffusive limit
// uses their largest.  The Shakura-Sunyaev viscosity and the flux-limited radiation
// diffusion vary with the state and are not in this bound.
inline double max_diffusivity(const double *v)
{
  double d = v[NU];
  if (v[DD] > d) d = v[DD];
  if (v[ED] > d) d = v[ED];
  if (v[RD] > d) d = v[RD];
  return d;
}

// Densities for the FP64 sums, per coordinate cell: rho, rho u_R, rho u_z and the thermal
// plus radiative energy density rho (e + e_rad).
FG2_HD void conserved(const double *q, double out[4])
{
  const double rho = exp(q[LND]);
  out[0] = rho;
  out[1] = rho * q[UR];
  out[2] = rho * q[UZ];
  out[3] = rho * (exp(q[LNE]) + exp(q[LNER]));
}

}  // namespace scheme
