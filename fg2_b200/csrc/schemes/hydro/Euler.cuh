// schemes/hydro/Euler.cuh -- operator-split per-cell update before each step.  The
// ideal-gas scheme has none (src/hydro/Euler.cuh:19-22).
#pragma once

#include "fg2b.h"

namespace scheme {

struct EulerArgs {
  float r1, r2;  // random phases (unused here)
};

template <class C>
FG2_HD bool euler_active(const fg2::Para<C> &) { return false; }

template <class C>
FG2_HD void first_order(C *q, C dt, int i, int j, const fg2::Para<C> &p, const EulerArgs &e, C delta1,
                        C delta2)
{
  (void)q; (void)dt; (void)i; (void)j; (void)p; (void)e; (void)delta1; (void)delta2;
}

}  // namespace scheme
