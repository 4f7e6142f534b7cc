// schemes/hydro-isot/config.h -- flop model and box settings (src/hydro-isot/config.h:19-26).
#pragma once

namespace scheme {

constexpr int EQNS_FLOP = 214;

// The isothermal scheme works on a 2 pi periodic box whatever the command line says.
inline void settings(double &l1, double &l2) { l1 = l2 = 2.0 * 3.14159265358979323846; }

}  // namespace scheme
