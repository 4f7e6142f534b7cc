/*
 * oracle/port.cpp -- TEST INFRASTRUCTURE ONLY.  This is the oracle, the CPU checker of
 * the CUDA path; nothing in the product links it or calls it.
 *
 * A CPU restatement of fg2's 2D hydro time step: the 6th-order stencils of
 * src/deriv.h:39-63, the right-hand sides of src/hydro/eqns.cuh:26-92 and
 * src/hydro-isot/eqns.cuh:27-87, the Euler hooks of src/hydro/Euler.cuh:19-22 and
 * src/hydro-isot/Euler.cuh:24-37, the reflective sign maps of src/hydro/bcond.cuh:19-28 and src/hydro-isot/bcond.cuh:19-28,
 * and (through oracle/loops.h) the kick / drift / bcond / step loops.
 *
 * Every expression keeps the reference's evaluation order, so that with
 * -ffp-contract=off this file and oracle/ref_harness.cpp (the reference's own headers
 * compiled for the host) give bit-identical results; tests/test_oracle.py checks that
 * against the committed golden vectors.
 *
 * Build variants (oracle/Makefile): ORC_SCHEME=1 hydro (NVAR 4), ORC_SCHEME=2 hydro-isot
 * (NVAR 3); ORC_DOUBLE selects R=double / E=long double as -DDOUBLE does in src/fg2.h:36-45.
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
#else
#error "ORC_SCHEME must be 1 (hydro) or 2 (hydro-isot)"
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

#else
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
