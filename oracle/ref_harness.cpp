/*
 * oracle/ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * Compiles the reference's OWN per-cell arithmetic for the host: src/fg2.h (types),
 * src/deriv.h (the 6th-order stencil macros), <scheme>/state.h, <scheme>/eqns.cuh
 * (right-hand side), <scheme>/Euler.cuh, <scheme>/bcond.cuh and, for hydro and disk, <scheme>/init.h
 * (the named initial conditions, evaluated at cell centres by orc_ref_setup), included in place from
 * the reference tree by oracle/Makefile (-I$(REF)/src -I$(REF)/src/<scheme>).  Nothing
 * of the reference is copied here: this file only provides the host stand-ins for the
 * CUDA qualifiers and the loops (oracle/loops.h), and exports the same C API as
 * oracle/port.cpp so that the two can be compared call for call.
 *
 * The output goes to oracle/_ref/ and is used to pin the port (golden vectors in
 * tests/golden/) and as the reference CPU baseline of bench.py.
 */
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#ifdef _OPENMP
#include <omp.h>
#endif

// Host stand-ins for the CUDA qualifiers used by the included headers.
#define __device__
#define __constant__
#define __global__
// The reference calls unqualified exp/cos/sin/sqrt on R; on the device R=float picks
// the float functions, so the host build must see the float overloads too.
using std::cos;
using std::exp;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
// src/disk/eqns.cuh:47 calls sincos on R; the device library has the float overload.
static inline void sincos(float x, float *s, float *c) { sincosf(x, s, c); }

// src/hydro/bcond.cuh and src/hydro-isot/bcond.cuh select the variable by threadIdx.x.
static struct { int x, y, z; } threadIdx;

#include "fg2.h"   // src/fg2.h: R, E, K(), S, NVAR, HALF; pulls <state.h>
#include "deriv.h" // src/deriv.h: Delta1, Delta2, D1 D2 D11 D22 D12
#include <eqns.cuh>
#include <Euler.cuh>
#include <bcond.cuh>

#define NV ((int)NVAR)

#define orc_eqns(c, i, j, s) eqns((c), (i), (j), (s))
#define orc_first_order(c, dt, i, j) first_order((c), (dt), (i), (j))
static inline R ref_transform(int var, R x)
{
  threadIdx.x = var;
  return transform(x);
}
#define orc_transform(var, x) ref_transform((var), (x))
#include "loops.h"

namespace {
struct Key { const char *name; R *val; };
#if defined(FG2_SCHEME_HYDRO)
Key keys[] = {{"gamma", &para_gamma}, {"nus", &para_nus}, {"nub", &para_nub},
              {"kappa", &para_kappa}, {"dd", &para_dd}};
#elif defined(FG2_SCHEME_ISOT)
Key keys[] = {{"dd", &para_dd}, {"nus", &para_nus}, {"nub", &para_nub},
              {"cs2", &para_cs2}, {"f", &para_f}, {"k", &para_k}};
#elif defined(FG2_SCHEME_DISK)
Key keys[] = {{"M", &para_M},         {"rS", &para_rS},   {"rin", &para_rin}, {"gamma", &para_gamma},
              {"nus", &para_nus},     {"nub", &para_nub}, {"kappa", &para_kappa}, {"alpha", &para_alpha},
              {"ar", &para_ar},       {"es", &para_es},   {"ff", &para_ff},   {"dd", &para_dd},
              {"nu", &para_nu},       {"ed", &para_ed},   {"rd", &para_rd}};
#else
#error "define FG2_SCHEME_HYDRO, FG2_SCHEME_ISOT or FG2_SCHEME_DISK"
#endif
}  // namespace

extern "C" {

int orc_nvar(void) { return NV; }
int orc_real_size(void) { return (int)sizeof(R); }
int orc_is_reference(void) { return 1; }

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
#if defined(FG2_SCHEME_ISOT)
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

// The reference's derivative macros evaluated at every interior cell (field by index).
void orc_deriv(const R *u, int n1, int n2, int which, int field, R *out)
{
  const int s = orc::pitch(n2);
  const S *o = (const S *)(u + orc::H * (s + NV));
  const int sc = s / NV;
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < n2; ++j) {
      const S *u = o + (long)i * sc + j;  // THIS = u, STRIDE = s (src/deriv.h:25-31)
      const int s = sc;
      R r = 0, fld[5][NVAR];
#define ORC_FIELD(k, name) \
  fld[0][k] = D1(name); fld[1][k] = D2(name); fld[2][k] = D11(name); fld[3][k] = D22(name); fld[4][k] = D12(name);
#if defined(FG2_SCHEME_DISK)
      ORC_FIELD(0, lnd) ORC_FIELD(1, ur) ORC_FIELD(2, uz) ORC_FIELD(3, Omg) ORC_FIELD(4, lne) ORC_FIELD(5, lner)
#else
      ORC_FIELD(0, lnd) ORC_FIELD(1, u1) ORC_FIELD(2, u2)
#if defined(FG2_SCHEME_HYDRO)
      ORC_FIELD(3, lne)
#endif
#endif
#undef ORC_FIELD
      r = fld[which][field];
      out[(long)i * n2 + j] = r;
    }
}

}  // extern "C"

#if defined(FG2_SCHEME_HYDRO) || defined(FG2_SCHEME_DISK)
// The reference's named initial conditions (src/hydro/init.h, included in place), evaluated at
// cell centres the way src/init.cpp:26-42 does.  Host stand-ins for the two globals the
// setups read and for the by-name symbol copy pick() makes of para_gamma.
namespace global {
R l1 = 1, l2 = 1;
}
static int cudaMemcpyFromSymbol(void *dst, const char *symbol, size_t n)
{
  for (const Key &k : keys)
    if (!std::strncmp(symbol, "para_", 5) && !std::strcmp(symbol + 5, k.name)) {
      std::memcpy(dst, k.val, n);
      return 0;
    }
  return 1;
}
#include <init.h>

extern "C" int orc_ref_setup(const char *name, int n1, int n2, double l1, double l2, R *out)
{
  global::l1 = (R)l1;
  global::l2 = (R)l2;
  S (*func)(R, R) = pick(name);
  for (Z i = 0; i < (Z)n1; ++i) {
    const R x = global::l1 * (i + 0.5) / (Z)n1;
    for (Z j = 0; j < (Z)n2; ++j) {
      const R y = global::l2 * (j + 0.5) / (Z)n2;
      ((S *)out)[i * n2 + j] = func(x, y);
    }
  }
  return 0;
}
#endif
