// schemes/disk/config.h -- flop model and box settings (src/disk/config.h:19-34): the full
// pi wedge in theta, a log-r extent that makes the cells about square, and walls on both
// axes (zero-gradient in r, reflective at the poles).
#pragma once

#include <cmath>

namespace scheme {

constexpr int EQNS_FLOP = 733;

// R is the state precision: the reference evaluates these in R (float unless DOUBLE).
template <class R>
inline void settings(int n1, int n2, double &l1, double &l2, int &p1, int &p2)
{
  l2 = (double)(R)3.14159265358979323846;
  const R hd2 = (R)(0.5 * l2 / n2);
  const R hd1 = (R)std::log(hd2 + std::sqrt(hd2 * hd2 + 1.0));
  l1 = (double)(R)(2.0 * hd1 * n1);
  p1 = 0;
  p2 = 0;
}

}  // namespace scheme
