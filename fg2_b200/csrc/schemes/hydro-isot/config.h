// schemes/hydro-isot/config.h -- flop model and box settings (src/hydro-isot/config.h:19-26).
#pragma once

namespace scheme {

constexpr int EQNS_FLOP = 214;

// The isothermal scheme works on a 2 pi periodic box whatever the command line says.
template <class R>
inline void settings(int n1, int n2, double &l1, double &l2, int &p1, int &p2)
{
  (void)n1; (void)n2; (void)p1; (void)p2;
  l1 = l2 = 2.0 * 3.14159265358979323846;
}

}  // namespace scheme
