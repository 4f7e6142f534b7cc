// schemes/hydro/config.h -- flop model and box settings (src/hydro/config.h:19-24).
#pragma once

namespace scheme {

// Floating-point operations of one right-hand-side evaluation, the reference's count.
constexpr int EQNS_FLOP = 289;

// Scheme-specific overrides of the box and boundaries after the command line: none.
template <class R>
inline void settings(int n1, int n2, double &l1, double &l2, int &p1, int &p2)
{
  (void)n1; (void)n2; (void)l1; (void)l2; (void)p1; (void)p2;
}

}  // namespace scheme
