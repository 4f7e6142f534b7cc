// schemes/disk/Euler.cuh -- operator-split radiation-matter exchange before each step
// (src/disk/Euler.cuh:19-69): where free-free cooling would move the thermal energy past
// radiative equilibrium within one step, the cell is set to the equilibrium split of its
// total energy e + e_rad.  Equilibrium solves e_rad = a_r T^4 / rho with T = (gamma - 1) e,
// i.e. the quartic A e^4 + e - e_tot = 0, A = a_r (gamma - 1)^4 / rho, rescaled by A^(1/3)
// to x^4 + x - x0 = 0 and solved in closed form (resolvent cubic, Ferrari).
//
// Without free-free opacity (ff = 0, the default) the cooling rate is zero and the hook
// never changes a cell, so it is only launched when ff != 0.
#pragma once

#include <cmath>

#include "fg2b.h"

namespace scheme {

struct EulerArgs {
  float r1, r2;  // unused by this scheme
};

template <class C>
FG2_HD bool euler_active(const fg2::Para<C> &p) { return p.v[FF] != C(0); }

template <class C>
FG2_HD void first_order(C *q, C dt, int i, int j, const fg2::Para<C> &p, const EulerArgs &e, C delta1,
                        C delta2)
{
  (void)i; (void)j; (void)e; (void)delta1; (void)delta2;
  const C den = m::ex(q[LND]), eng = m::ex(q[LNE]), rad = m::ex(q[LNER]);
  const C g1 = p.v[GAMMA] - C(1);
  const C g1_2 = g1 * g1;
  const C third = C(1) / C(3);
  // equilibrium thermal energy: positive root of x^4 + x - x0 = 0, x = A^(1/3) e
  const C scale = m::pw(p.v[AR] * g1_2 * g1_2 / den, third);
  const C x0 = (eng + rad) * scale;
  const C a = m::pw(m::sq(C(0.00390625) + x0 * x0 * x0 / C(27)) + C(0.0625), third);
  const C b = a - x0 / (C(3) * a);
  const C cq = m::sq(C(2) * b);
  const C eq_eng = (m::sq(C(0.5) / cq - C(0.5) * b) - C(0.5) * cq) / scale;
  const C dt_eng = (eq_eng - eng) / dt;
  // free-free cooling rate at the current state
  const C temp = g1 * eng;
  const C temp2 = temp * temp;
  const C kap = p.v[FF] * den * den * m::pw(temp, C(-3.5));
  const C cooling = kap * (p.v[AR] * temp2 * temp2 / den - rad);
  if (cooling * cooling > dt_eng * dt_eng) {
    q[LNE] = m::lg(eq_eng);
    q[LNER] = m::lg(eng + rad - eq_eng);
  }
}

}  // namespace scheme
