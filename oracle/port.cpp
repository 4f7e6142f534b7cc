/*
 * oracle/port.cpp -- TEST INFRASTRUCTURE ONLY.  This is the oracle, the CPU checker of
 * the CUDA path; nothing in the product links it or calls it.
 *
 * A CPU restatement of fg2's 2D hydro time step: the 6th-order stencils of
 * src/deriv.h:39-63, the right-hand sides of src/hydro/eqns.cuh:26-92,
 * src/hydro-isot/eqns.cuh:27-87 and src/disk/eqns.cuh:38-247, the Euler hooks of
 * src/hydro/Euler.cuh:19-22, src/hydro-isot/Euler.cuh:24-37 and src/disk/Euler.cuh:19-69,
 * the reflective sign maps of src/hydro/bcond.cuh:19-28, src/hydro-isot/bcond.cuh:19-28 and
 * src/disk/bcond.cuh:19-29, and (through oracle/loops.h) the kick / drift / bcond / step loops.
 *
 * Every expression keeps the reference's evaluation order, so that with
 * -ffp-contract=off this file and oracle/ref_harness.cpp (the reference's own headers
 * compiled for the host) give bit-identical results; tests/test_oracle.py checks that
 * against the committed golden vectors.
 *
 * Build variants (oracle/Makefile): ORC_SCHEME=1 hydro (NVAR 4), ORC_SCHEME=2 hydro-isot
 * (NVAR 3), ORC_SCHEME=3 disk (NVAR 6); ORC_DOUBLE selects R=double / E=long double as
 * -DDOUBLE does in src/fg2.h:36-45.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_DOUBLE
typedef double R;
typedef long double E;
#define K(x) (x)
#else
typedef float R;
typedef double E;
#define K(x) (x##f)
#endif

#if ORC_SCHEME == 1
#define NV 4
struct S { R lnd, u1, u2, lne; };
#elif ORC_SCHEME == 2
#define NV 3
struct S { R lnd, u1, u2; };
#elif ORC_SCHEME == 3
#define NV 6
struct S { R lnd, ur, uz, Omg, lne, lner; };
#else
#error "ORC_SCHEME must be 1 (hydro), 2 (hydro-isot) or 3 (disk)"
#endif

namespace {

// Grid spacings (src/deriv.h:22-23, set by src/config.cpp:39-41).
R Delta1 = 0, Delta2 = 0;

// ---- stencils: src/deriv.h:33-63 (ORDER 6) -------------------------------------------
// `c` is the centre cell, `s` the row stride in cells; field f of cell (c + di*s + dj).
inline R at(const S *c, int s, int f, int di, int dj) { return ((const R *)(c + di * s + dj))[f]; }
inline R dif(const S *c, int s, int f, int di, int dj) { return at(c, s, f, di, dj) - at(c, s, f, -di, -dj); }
inline R sum(const S *c, int s, int f, int di, int dj) { return at(c, s, f, di, dj) + at(c, s, f, -di, -dj); }
inline R mix(const S *c, int s, int f, int di, int dj)
{
  return at(c, s, f, di, dj) - at(c, s, f, -di, dj) + at(c, s, f, -di, -dj) - at(c, s, f, di, -dj);
}
inline R d1(const S *c, int s, int f)
{
  return ((R)(45. / 60.) * dif(c, s, f, 1, 0) + (R)(-9. / 60.) * dif(c, s, f, 2, 0) +
          (R)(1. / 60.) * dif(c, s, f, 3, 0)) / Delta1;
}
inline R d2(const S *c, int s, int f)
{
  return ((R)(45. / 60.) * dif(c, s, f, 0, 1) + (R)(-9. / 60.) * dif(c, s, f, 0, 2) +
          (R)(1. / 60.) * dif(c, s, f, 0, 3)) / Delta2;
}
inline R d11(const S *c, int s, int f)
{
  return ((R)(-490. / 180.) * at(c, s, f, 0, 0) + (R)(270. / 180.) * sum(c, s, f, 1, 0) +
          (R)(-27. / 180.) * sum(c, s, f, 2, 0) + (R)(2. / 180.) * sum(c, s, f, 3, 0)) /
         (Delta1 * Delta1);
}
inline R d22(const S *c, int s, int f)
{
  return ((R)(-490. / 180.) * at(c, s, f, 0, 0) + (R)(270. / 180.) * sum(c, s, f, 0, 1) +
          (R)(-27. / 180.) * sum(c, s, f, 0, 2) + (R)(2. / 180.) * sum(c, s, f, 0, 3)) /
         (Delta2 * Delta2);
}
inline R d12(const S *c, int s, int f)
{
  return ((R)(270. / 720.) * mix(c, s, f, 1, 1) + (R)(-27. / 720.) * mix(c, s, f, 2, 2) +
          (R)(2. / 720.) * mix(c, s, f, 3, 3)) / (Delta1 * Delta2);
}

enum { LND = 0, U1 = 1, U2 = 2, LNE = 3 };

#if ORC_SCHEME == 1
// ---- hydro: src/hydro/eqns.cuh:19-24 (keys) and :26-92 (RHS) -------------------------
R p_gamma = 5.0 / 3.0, p_nus = 2.0e-4, p_nub = 0.0, p_kappa = 5.0e-4, p_dd = 0.0;
struct Key { const char *name; R *val; } keys[] = {
    {"gamma", &p_gamma}, {"nus", &p_nus}, {"nub", &p_nub}, {"kappa", &p_kappa}, {"dd", &p_dd}};

S rhs(const S *c, int i, int j, int s)
{
  (void)i; (void)j;
  const S g1 = {d1(c, s, LND), d1(c, s, U1), d1(c, s, U2), d1(c, s, LNE)};
  const S g2 = {d2(c, s, LND), d2(c, s, U1), d2(c, s, U2), d2(c, s, LNE)};
  S r = {0.0, 0.0, 0.0, 0.0};
  {  // advection
    const R a1 = c->u1, a2 = c->u2;
    r.lnd -= a1 * g1.lnd + a2 * g2.lnd;
    r.u1 -= a1 * g1.u1 + a2 * g2.u1;
    r.u2 -= a1 * g1.u2 + a2 * g2.u2;
    r.lne -= a1 * g1.lne + a2 * g2.lne;
  }
  {  // pressure, compression, viscous heating
    const R gm1 = p_gamma - K(1.0);
    const R temp = gm1 * std::exp(c->lne);
    const R div = g1.u1 + g2.u2;
    r.lnd -= div;
    r.u1 -= temp * (g1.lnd + g1.lne);
    r.u2 -= temp * (g2.lnd + g2.lne);
    r.lne -= div * gm1;
    const R s11 = g1.u1 - div / K(3.0);
    const R s12 = (g1.u2 + g2.u1) / K(2.0);
    const R s22 = g2.u2 - div / K(3.0);
    const R nus2 = K(2.0) * p_nus;
    r.u1 += nus2 * (s11 * g1.lnd + s12 * g2.lnd);
    r.u2 += nus2 * (s12 * g1.lnd + s22 * g2.lnd);
    r.lne += (gm1 / temp) * (nus2 * (s11 * s11 + K(2.0) * s12 * s12 + s22 * s22) + p_nub * div * div);
  }
  {  // viscous stress divergence
    const R xx1 = d11(c, s, U1), xx2 = d11(c, s, U2);
    const R xy1 = d12(c, s, U1), xy2 = d12(c, s, U2);
    const R yy1 = d22(c, s, U1), yy2 = d22(c, s, U2);
    const R mixed = p_nus / K(3.0) + p_nub;
    r.u1 += p_nus * (xx1 + yy1) + mixed * (xx1 + xy2);
    r.u2 += p_nus * (xx2 + yy2) + mixed * (xy1 + yy2);
  }
  {  // density diffusion and conduction
    const R gl = g1.lnd * g1.lnd + g2.lnd * g2.lnd;
    const R ge = g1.lne * g1.lne + g2.lne * g2.lne;
    const R ed = (p_gamma - K(1.0)) * p_kappa;
    r.lnd += p_dd * (d11(c, s, LND) + d22(c, s, LND) + gl);
    r.lne += ed * (d11(c, s, LNE) + d22(c, s, LNE) + ge);
  }
  return r;
}

// src/hydro/Euler.cuh:19-22: no operator-split term.
void first_order(S *, R, int, int) {}

// src/hydro/bcond.cuh:19-28: u2 flips sign at a reflective wall.
R transform(int var, R x) { return var == U2 ? -x : x; }

#elif ORC_SCHEME == 2
// ---- hydro-isot: src/hydro-isot/eqns.cuh:19-25 (keys) and :27-87 (RHS) ---------------
R p_dd = 0.0, p_nus = 2.0e-4, p_nub = 0.0, p_cs2 = 1.0, p_f = 0.0, p_k = -8.0;
struct Key { const char *name; R *val; } keys[] = {{"dd", &p_dd},   {"nus", &p_nus}, {"nub", &p_nub},
                                                   {"cs2", &p_cs2}, {"f", &p_f},     {"k", &p_k}};
R rand1 = 0.0, rand2 = 0.0;  // src/hydro-isot/Euler.cuh:21-22

S rhs(const S *c, int i, int j, int s)
{
  (void)j;
  const S g1 = {d1(c, s, LND), d1(c, s, U1), d1(c, s, U2)};
  const S g2 = {d2(c, s, LND), d2(c, s, U1), d2(c, s, U2)};
  S r = {0.0, 0.0, 0.0};
  {
    const R a1 = c->u1, a2 = c->u2;
    r.lnd -= a1 * g1.lnd + a2 * g2.lnd;
    r.u1 -= a1 * g1.u1 + a2 * g2.u1;
    r.u2 -= a1 * g1.u2 + a2 * g2.u2;
  }
  {
    const R div = g1.u1 + g2.u2;
    r.lnd -= div;
    r.u1 -= p_cs2 * g1.lnd;
    r.u2 -= p_cs2 * g2.lnd;
    const R s11 = g1.u1 - div / K(3.0);
    const R s12 = (g1.u2 + g2.u1) / K(2.0);
    const R s22 = g2.u2 - div / K(3.0);
    const R nus2 = K(2.0) * p_nus;
    r.u1 += nus2 * (s11 * g1.lnd + s12 * g2.lnd);
    r.u2 += nus2 * (s12 * g1.lnd + s22 * g2.lnd);
  }
  {
    const R xx1 = d11(c, s, U1), xx2 = d11(c, s, U2);
    const R xy1 = d12(c, s, U1), xy2 = d12(c, s, U2);
    const R yy1 = d22(c, s, U1), yy2 = d22(c, s, U2);
    const R mixed = p_nus / K(3.0) + p_nub;
    r.u1 += p_nus * (xx1 + yy1) + mixed * (xx1 + xy2);
    r.u2 += p_nus * (xx2 + yy2) + mixed * (xy1 + yy2);
  }
  r.lnd += p_dd * (d11(c, s, LND) + g1.lnd * g1.lnd + d22(c, s, LND) + g2.lnd * g2.lnd);
  if (p_f * p_k < K(0.0)) r.u2 += p_f * std::cos(p_k * i * Delta1);  // Kolmogorov forcing
  return r;
}

// src/hydro-isot/Euler.cuh:24-37: stochastic plane-wave forcing when f * k > 0.
void first_order(S *u, R dt, int i, int j)
{
  if (p_f * p_k > K(0.0)) {
    const R k1 = p_k * std::cos(rand1);
    const R k2 = p_k * std::sin(rand1);
    const R phi = K(6.2831853071795865) * ((int)(k1 + K(0.5)) * i * Delta1 + (int)(k2 + K(0.5)) * j * Delta2);
    const R amp = std::sqrt(dt) * (p_f * std::cos(phi + rand2)) / (p_k * std::exp(u->lnd));
    u->u1 += amp * k1;
    u->u2 += amp * k2;
  }
}

R transform(int var, R x) { return var == U2 ? -x : x; }

#else
// ---- disk: src/disk/eqns.cuh:19-36 (keys) and :38-247 (RHS) --------------------------
// Log-r / theta grid: axis 1 is ln(r / r_in), axis 2 is theta.  The expressions keep the
// reference's order; sincos, exp, pow, sqrt and log are the precision-R library functions.
R p_M = 1.0, p_rS = 2.0, p_rin = 3.0, p_gamma = 5.0 / 3.0, p_nus = 0.0, p_nub = 0.0, p_kappa = 0.0,
  p_alpha = 0.01, p_ar = 1.0e+8, p_es = 1.0, p_ff = 0.0, p_dd = 1.0e-4, p_nu = 2.0e-4, p_ed = 5.0e-4,
  p_rd = 5.0e-4;
struct Key { const char *name; R *val; } keys[] = {
    {"M", &p_M},     {"rS", &p_rS}, {"rin", &p_rin}, {"gamma", &p_gamma}, {"nus", &p_nus},
    {"nub", &p_nub}, {"kappa", &p_kappa}, {"alpha", &p_alpha}, {"ar", &p_ar}, {"es", &p_es},
    {"ff", &p_ff},   {"dd", &p_dd}, {"nu", &p_nu}, {"ed", &p_ed}, {"rd", &p_rd}};
enum { UR = 1, UZ = 2, OMG = 3, LNE6 = 4, LNER = 5 };

inline void sin_cos(float x, float *s, float *c) { sincosf(x, s, c); }
inline void sin_cos(double x, double *s, double *c) { sincos(x, s, c); }

S rhs(const S *c, int i, int j, int s)
{
  R sint, cost;
  sin_cos((j + K(0.5)) * Delta2, &sint, &cost);
  const R sphr = p_rin * std::exp((i + K(0.5)) * Delta1);
  const R r = sphr * sint;  // cylindrical radius
  const R sphr_2 = sphr * sphr;

  const R den = std::exp(c->lnd), eng = std::exp(c->lne), rad = std::exp(c->lner);
  const R gamma1 = p_gamma - K(1.0);
  const R temp = gamma1 * eng;
  const R nuSS = p_alpha * p_gamma * temp * r * std::sqrt(r / p_M);

  // gradient in (R, z) from the (ln r, theta) derivatives
  R dr[NV], dz[NV], d11v[NV], d22v[NV], lap[NV];
  for (int f = 0; f < NV; ++f) {
    const R g1 = d1(c, s, f), g2 = d2(c, s, f);
    dr[f] = (sint * g1 + cost * g2) / sphr;
    dz[f] = (cost * g1 - sint * g2) / sphr;
  }
  for (int f = 0; f < NV; ++f) { d11v[f] = d11(c, s, f); d22v[f] = d22(c, s, f); }
  const R x_lnd = d12(c, s, LND), x_ur = d12(c, s, UR), x_uz = d12(c, s, UZ), x_lner = d12(c, s, LNER);
  const R cr = cost / sphr, sr = sint / sphr;
  const R cc = cr * cr, cs = cr * sr, ss = sr * sr;
  const R c2 = cc - ss, s2 = K(2.0) * cs;
  for (int f = 0; f < NV; ++f) lap[f] = (d11v[f] + d22v[f]) / sphr_2;
  auto rr = [&](int f, R x) { return ss * d11v[f] + cc * d22v[f] + s2 * x + cr * dz[f] - sr * dr[f]; };
  auto rz = [&](int f, R x) { return cs * (d11v[f] - d22v[f]) + c2 * x - cr * dr[f] - sr * dz[f]; };
  auto zz = [&](int f, R x) { return cc * d11v[f] + ss * d22v[f] - s2 * x - cr * dz[f] + sr * dr[f]; };
  const R drr_lnd = rr(LND, x_lnd), drr_ur = rr(UR, x_ur), drr_lner = rr(LNER, x_lner);
  const R drz_lnd = rz(LND, x_lnd), drz_ur = rz(UR, x_ur), drz_uz = rz(UZ, x_uz), drz_lner = rz(LNER, x_lner);
  const R dzz_lnd = zz(LND, x_lnd), dzz_uz = zz(UZ, x_uz), dzz_lner = zz(LNER, x_lner);

  R t[NV] = {0, 0, 0, 0, 0, 0};
  const R ur = c->ur, uz = c->uz, Omg = c->Omg;
  // advection and pseudo-forces
  t[LND] -= ur * dr[LND] + uz * dz[LND];
  t[UR] -= ur * dr[UR] + uz * dz[UR] - Omg * Omg * r;
  t[UZ] -= ur * dr[UZ] + uz * dz[UZ];
  t[OMG] -= ur * dr[OMG] + uz * dz[OMG] + K(2.0) * ur * Omg / r;
  t[LNE6] -= ur * dr[LNE6] + uz * dz[LNE6];
  t[LNER] -= ur * dr[LNER] + uz * dz[LNER];
  // compression and pressure
  const R ur_r = c->ur / r;
  const R div_u = dr[UR] + dz[UZ] + ur_r;
  t[LND] -= div_u;
  t[UR] -= temp * (dr[LND] + dr[LNE6]);
  t[UZ] -= temp * (dz[LND] + dz[LNE6]);
  t[LNE6] -= div_u * gamma1;
  // density- and temperature-dependent viscous terms, viscous heating
  const R Srr = dr[UR] - div_u / K(3.0);
  const R Szz = dz[UZ] - div_u / K(3.0);
  const R Spp = ur_r - div_u / K(3.0);
  const R Srz = (dz[UR] + dr[UZ]) / K(2.0);
  const R Szp = r * dz[OMG] / K(2.0);
  const R Spr = r * dr[OMG] / K(2.0);
  const R two_nus = K(2.0) * (p_nus + nuSS);
  t[UR] += two_nus * (Srr * dr[LND] + Srz * dz[LND]);
  t[UZ] += two_nus * (Srz * dr[LND] + Szz * dz[LND]);
  t[OMG] += two_nus * (Spr * dr[LND] + Szp * dz[LND]) / r;
  t[LNE6] += (two_nus * (Srr * Srr + Szz * Szz + Spp * Spp + K(2.0) * (Srz * Srz + Szp * Szp + Spr * Spr)) +
              p_nub * div_u * div_u) / eng;
  // velocity-only viscous terms
  const R tmp1 = (p_nus + nuSS) + p_nu * sphr_2;
  const R tmp2 = (p_nus + nuSS) / r;
  t[UR] += tmp1 * lap[UR] + tmp2 * (dr[UR] - c->ur / r);
  t[UZ] += tmp1 * lap[UZ] + tmp2 * (dr[UZ]);
  t[OMG] += tmp1 * lap[OMG] + tmp2 * (dr[OMG] * K(3.0));
  const R mixed = (p_nus + nuSS) / K(3.0) + p_nub;
  t[UR] += mixed * (drr_ur + drz_uz + (dr[UR] - c->ur / r) / r);
  t[UZ] += mixed * (drz_ur + dzz_uz + dz[UR] / r);
  // density diffusion and conduction
  const R lap_d_d = lap[LND] + dr[LND] * dr[LND] + dz[LND] * dz[LND];
  const R lap_e_e = lap[LNE6] + dr[LNE6] * dr[LNE6] + dz[LNE6] * dz[LNE6];
  t[LND] += lap_d_d * p_dd * sphr_2;
  t[LNE6] += lap_e_e * (p_ed * sphr_2 + p_kappa * gamma1 + p_gamma * nuSS);
  // radiation force
  const R kappa = p_ff * den * den * std::pow(temp, K(-3.5));
  const R chi = p_es * den + kappa;
  const R d_lner_2 = dr[LNER] * dr[LNER] + dz[LNER] * dz[LNER];
  const R bigR = std::sqrt(d_lner_2) / chi;
  const R denom = K(6.0) + (K(3.0) + bigR) * bigR;
  const R Lambda = (K(2.0) + bigR) / denom;
  t[UR] -= Lambda * rad * (dr[LND] + dr[LNE6]);
  t[UZ] -= Lambda * rad * (dz[LND] + dz[LNE6]);
  // heating / cooling
  const R temp2 = temp * temp;
  const R cooling = kappa * (p_ar * temp2 * temp2 / den - rad);
  t[LNE6] -= cooling / eng;
  t[LNER] += cooling / rad;
  // radiation diffusion
  const R d_lnd_d_lner = dr[LND] * dr[LNER] + dz[LND] * dz[LNER];
  const R lap_er_er = lap[LNER] + d_lner_2;
  const R nu_rad = Lambda / chi;
  const R Lambdap = -bigR * (K(4.0) + bigR) / (denom * denom);
  const R dr_e = dr[LND] + dr[LNER], dz_e = dz[LND] + dz[LNER];
  const R drr_e = drr_lnd + drr_lner, drz_e = drz_lnd + drz_lner, dzz_e = dzz_lnd + dzz_lner;
  const R dr_chi = chi * dr[LND] - K(3.5) * kappa * dr[LNE6];
  const R dz_chi = chi * dz[LND] - K(3.5) * kappa * dz[LNE6];
  const R dr_bigR = ((dr_e * drr_e + dz_e * drz_e) / (K(1e-16) + bigR) / chi - bigR * dr_chi) / chi;
  const R dz_bigR = ((dr_e * drz_e + dz_e * dzz_e) / (K(1e-16) + bigR) / chi - bigR * dz_chi) / chi;
  t[LNER] += lap_er_er * p_rd * sphr_2 + nu_rad * (lap_d_d + K(2.0) * d_lnd_d_lner + lap_er_er) +
             dr_e * (Lambdap * dr_bigR - nu_rad * dr_chi) / chi + dz_e * (Lambdap * dz_bigR - nu_rad * dz_chi) / chi;
  // gravity
  const R tmp = sphr - p_rS;
  const R gr = p_M / (tmp * tmp);
  t[UR] -= sint * gr;
  t[UZ] -= cost * gr;
  S out;
  std::memcpy(&out, t, sizeof(out));
  return out;
}

// src/disk/Euler.cuh:19-69: radiation-matter equilibrium where free-free cooling would
// overshoot it within dt (positive root of x^4 + x - x0 = 0 in closed form).
void first_order(S *u, R dt, int i, int j)
{
  (void)i; (void)j;
  const R den = std::exp(u->lnd), eng = std::exp(u->lne), rad = std::exp(u->lner);
  const R gamma1 = p_gamma - K(1.0);
  const R gamma1_2 = gamma1 * gamma1;
  const R scale = std::pow(p_ar * gamma1_2 * gamma1_2 / den, K(1.0) / K(3.0));
  const R x0 = (eng + rad) * scale;
  const R a = std::pow(std::sqrt(K(0.00390625) + x0 * x0 * x0 / K(27.0)) + K(0.0625), K(1.0) / K(3.0));
  const R b = a - x0 / (K(3.0) * a);
  const R cq = std::sqrt(K(2.0) * b);
  const R eq_eng = (std::sqrt(K(0.5) / cq - K(0.5) * b) - K(0.5) * cq) / scale;
  const R dt_eng = (eq_eng - eng) / dt;
  const R temp = gamma1 * eng;
  const R temp2 = temp * temp;
  const R kappa = p_ff * den * den * std::pow(temp, K(-3.5));
  const R cooling = kappa * (p_ar * temp2 * temp2 / den - rad);
  if (cooling * cooling > dt_eng * dt_eng) {
    u->lne = std::log(eq_eng);
    u->lner = std::log(eng + rad - eq_eng);
  }
}

// src/disk/bcond.cuh:19-29: u_R flips sign at the poles.
R transform(int var, R x) { return var == UR ? -x : x; }
#endif

}  // namespace

#define orc_eqns(c, i, j, s) rhs((c), (i), (j), (s))
#define orc_first_order(c, dt, i, j) first_order((c), (dt), (i), (j))
#define orc_transform(var, x) transform((var), (x))
#include "loops.h"

extern "C" {

int orc_nvar(void) { return NV; }
int orc_real_size(void) { return (int)sizeof(R); }
int orc_is_reference(void) { return 0; }

int orc_set_para(const char *key, double val)
{
  for (auto &k : keys)
    if (!std::strcmp(k.name, key)) { *k.val = (R)val; return 0; }
  return -1;
}
double orc_get_para(const char *key)
{
  for (auto &k : keys)
    if (!std::strcmp(k.name, key)) return (double)*k.val;
  return NAN;
}
void orc_set_delta(double a, double b) { Delta1 = (R)a; Delta2 = (R)b; }
void orc_set_rand(double r1, double r2)
{
#if ORC_SCHEME == 2
  rand1 = (R)r1; rand2 = (R)r2;
#else
  (void)r1; (void)r2;
#endif
}

int orc_threads(int n)
{
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void orc_kick(R *v, const R *u, int n1, int n2, double t, double beta) { orc::kick(v, u, n1, n2, (R)t, (R)beta); }
int orc_drift(R *u, const R *v, int n1, int n2, double dt) { return orc::drift(u, v, n1, n2, (R)dt); }
void orc_bcond(R *u, int n1, int n2, int p1, int p2) { orc::bcond(u, n1, n2, p1, p2); }
void orc_euler(R *u, int n1, int n2, double dt) { orc::euler(u, n1, n2, (R)dt); }
int orc_step(R *u, R *v, int n1, int n2, double t, double dt, int p1, int p2)
{
  return orc::step(u, v, n1, n2, (E)t, (E)dt, p1, p2);
}
// nsteps steps of fixed dt (the reference's solve loop without frames).
int orc_run(R *u, R *v, int n1, int n2, double t, double dt, int nsteps, int p1, int p2)
{
  int nan = 0;
  E tt = t;
  for (int n = 0; n < nsteps; ++n) {
    nan |= orc::step(u, v, n1, n2, tt, (E)dt, p1, p2);
    tt += dt;
  }
  return nan;
}

// One derivative of one field at every interior cell, for the stencil known-answer
// tests.  which: 0 D1, 1 D2, 2 D11, 3 D22, 4 D12.  out is n1*n2, row-major.
void orc_deriv(const R *u, int n1, int n2, int which, int field, R *out)
{
  const int s = orc::pitch(n2);
  const S *o = (const S *)(u + orc::H * (s + NV));
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < n2; ++j) {
      const S *c = o + (long)i * (s / NV) + j;
      R r = 0;
      switch (which) {
        case 0: r = d1(c, s / NV, field); break;
        case 1: r = d2(c, s / NV, field); break;
        case 2: r = d11(c, s / NV, field); break;
        case 3: r = d22(c, s / NV, field); break;
        case 4: r = d12(c, s / NV, field); break;
      }
      out[(long)i * n2 + j] = r;
    }
}

}  // extern "C"
