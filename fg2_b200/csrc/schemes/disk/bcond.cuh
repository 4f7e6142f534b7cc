// schemes/disk/bcond.cuh -- sign of each field in a reflective ghost column (the poles,
// theta = 0 and pi): u_R flips, everything else is mirrored unchanged
// (src/disk/bcond.cuh:19-29).
#pragma once

#include "fg2b.h"

namespace scheme {

FG2_HD constexpr int reflect_sign(int f) { return f == UR ? -1 : +1; }

}  // namespace scheme
