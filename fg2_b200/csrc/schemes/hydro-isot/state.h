// schemes/hydro-isot/state.h -- the isothermal scheme's state {ln rho, u1, u2}, the
// field order of src/hydro-isot/state.h:19-22.
#pragma once

namespace scheme {

constexpr const char *NAME = "hydro-isot";
constexpr int NVAR = 3;
enum Field { LND = 0, U1 = 1, U2 = 2 };
// Cartesian grid: the CFL rate needs no cell position.
constexpr bool CURVILINEAR = false;
constexpr const char *FIELD_NAMES[NVAR] = {"lnd", "u1", "u2"};

}  // namespace scheme
