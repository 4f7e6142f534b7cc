// schemes/hydro/state.h -- the ideal-gas scheme's state: log-primitive variables
// {ln rho, u1, u2, ln e_th}, the field order of src/hydro/state.h:19-23.
#pragma once

namespace scheme {

constexpr const char *NAME = "hydro";
constexpr int NVAR = 4;
enum Field { LND = 0, U1 = 1, U2 = 2, LNE = 3 };
// Cartesian grid: the CFL rate needs no cell position.
constexpr bool CURVILINEAR = false;
constexpr const char *FIELD_NAMES[NVAR] = {"lnd", "u1", "u2", "lne"};

}  // namespace scheme
