// schemes/hydro-isot/Euler.cuh -- stochastic plane-wave forcing applied per cell before
// each step when f k > 0 (src/hydro-isot/Euler.cuh:24-37).  The two random phases are
// drawn on the host once per step (the reference's RANDOMIZE, src/hydro-isot/Euler.cuh:
// 39-44, uses rand(); this library uses its seeded generator, or phases the caller sets).
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

struct EulerArgs {
  float r1, r2;  // forcing direction angle and phase, in [0, 2 pi)
};

template <class C>
FG2_HD bool euler_active(const fg2::Para<C> &p) { return p.v[FAMP] * p.v[FK] > C(0); }

template <class C>
FG2_HD C fcos(C x);
template <>
FG2_HD float fcos<float>(float x) { return cosf(x); }
template <>
FG2_HD double fcos<double>(double x) { return cos(x); }

template <class C>
FG2_HD C fsin(C x);
template <>
FG2_HD float fsin<float>(float x) { return sinf(x); }
template <>
FG2_HD double fsin<double>(double x) { return sin(x); }

template <class C>
FG2_HD C fexp_(C x);
template <>
FG2_HD float fexp_<float>(float x) { return expf(x); }
template <>
FG2_HD double fexp_<double>(double x) { return exp(x); }

template <class C>
FG2_HD void first_order(C *q, C dt, int i, int j, const fg2::Para<C> &p, const EulerArgs &e, C delta1,
                        C delta2)
{
  if (!euler_active(p)) return;
  const C k = p.v[FK], f = p.v[FAMP];
  const C r1 = C(e.r1), r2 = C(e.r2);
  const C k1 = k * fcos(r1);
  const C k2 = k * fsin(r1);
  // integer wave numbers along each axis, as the reference truncates them
  const C phi = C(6.2831853071795865) * (C((int)(k1 + C(0.5)) * i) * delta1 + C((int)(k2 + C(0.5)) * j) * delta2);
  const C amp = sqrt(dt) * (f * fcos(phi + r2)) / (k * fexp_(q[LND]));
  q[U1] += amp * k1;
  q[U2] += amp * k2;
}

}  // namespace scheme
