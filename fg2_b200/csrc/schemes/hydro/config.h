// schemes/hydro/config.h -- flop model and box settings (src/hydro/config.h:19-24).
#pragma once

namespace scheme {

// Floating-point operations of one right-hand-side evaluation, the reference's count.
constexpr int EQNS_FLOP = 289;

// Scheme-specific overrides of the box after the command line: none.
inline void settings(double &l1, double &l2) { (void)l1; (void)l2; }

}  // namespace scheme
