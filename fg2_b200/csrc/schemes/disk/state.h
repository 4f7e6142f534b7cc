// schemes/disk/state.h -- the radiative torus scheme's state in log-r / theta coordinates:
// {ln rho, u_R, u_z, Omega, ln e_th, ln e_rad} (cylindrical radial and vertical velocity,
// angular velocity, specific thermal and radiative energy), the field order of
// src/disk/state.h:19-23.
#pragma once

namespace scheme {

constexpr const char *NAME = "disk";
constexpr int NVAR = 6;
enum Field { LND = 0, UR = 1, UZ = 2, OMG = 3, LNE = 4, LNER = 5 };
// the velocity components the framework's generic code (CFL, ghost signs) asks for
constexpr int U1 = UR, U2 = UZ;
// log-r / theta grid: the CFL rate depends on the cell position (scheme::signal_rate).
constexpr bool CURVILINEAR = true;
constexpr const char *FIELD_NAMES[NVAR] = {"lnd", "ur", "uz", "Omg", "lne", "lner"};

}  // namespace scheme
