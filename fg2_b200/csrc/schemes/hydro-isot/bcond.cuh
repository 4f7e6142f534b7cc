// schemes/hydro-isot/bcond.cuh -- sign of each field in a reflective ghost column: u2
// flips (src/hydro-isot/bcond.cuh:19-28).
#pragma once

#include "fg2b.h"

namespace scheme {

FG2_HD constexpr int reflect_sign(int f) { return f == U2 ? -1 : +1; }

}  // namespace scheme
