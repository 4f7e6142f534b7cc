// fg2_b200/csrc/fg2b.h -- shared host/device definitions of the B200 time-step library.
//
// Device layout of one simulation (structure of arrays, one plane per field):
//   element (f, i, j), i in [-3, n1+3), j in [-4, n2+4), lives at
//       base[f * PS + (i + GT) * P + (j + GL)]
//   GT = 3 ghost rows above/below (HALF of the 6th-order stencil, src/fg2.h:26-34);
//   GL = 4 columns left of the interior: 3 ghosts plus one so that the interior and every
//   tile's halo start on a 16-byte boundary (a TMA box must start on one);
//   P  = row pitch, >= n2 + 8, rounded up so rows start on 128 bytes;
//   PS = (n1 + 6) * P, the plane stride.
// Axis 1 (i, n1, Delta1) is the slow, strided axis and axis 2 (j, n2, Delta2) the
// contiguous one, as in the reference (src/deriv.h:33, src/init.cpp:31-35).
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define FG2_HD __host__ __device__ __forceinline__
#else
#define FG2_HD inline
#endif

namespace fg2 {

constexpr int HALF = 3;  // ghost width, ORDER / 2
constexpr int GT = 3;    // ghost rows above the interior
constexpr int GL = 4;    // padded columns left of the interior

enum Storage : int { ST_F32 = 0, ST_F64 = 1, ST_F16 = 2, ST_BF16 = 3 };

// Boundary kind per axis: periodic (the reference's p = 1), or the reference's
// non-periodic choice for that axis: zero-gradient rows along axis 1 (src/bcond.cu:45-57)
// and reflective columns along axis 2 (src/bcond.cu:59-75).
enum Bc : int { BC_WALL = 0, BC_PERIODIC = 1 };

struct Layout {
  int n1, n2;
  long long P;   // row pitch, elements
  long long PS;  // plane stride, elements
  FG2_HD long long at(int f, int i, int j) const { return f * PS + (long long)(i + GT) * P + (j + GL); }
};

inline Layout make_layout(int n1, int n2, size_t elem)
{
  Layout L;
  L.n1 = n1;
  L.n2 = n2;
  const long long align = 128 / (long long)elem;
  L.P = ((long long)n2 + 2 * GL + align - 1) / align * align;
  L.PS = (long long)(n1 + 2 * GT) * L.P;
  return L;
}

// Stencil coefficients with the grid spacing folded in (src/deriv.h:42-63 divide by
// Delta after the weighted sum; here the weights are pre-divided, computed in double on
// the host and rounded once to the compute type).
template <class C>
struct Coef {
  C a1[3], a2[3];      // first derivative weights, axis 1 / axis 2, k = 1..3
  C b1[4], b2[4];      // second derivative weights (centre, k = 1..3)
  C m[3];              // mixed derivative weights
  C delta1, delta2;    // grid spacings (the reference's Delta1/Delta2, rounded to C)
  C inv1, inv2;        // 1 / Delta
};

// Everything the right-hand side of a scheme needs at one cell.  NV fields.
template <class C, int NV>
struct Cell {
  C q[NV];    // cell value
  C d1[NV];   // first derivative along axis 1
  C d2[NV];   // first derivative along axis 2
  C d11[NV];  // second derivative along axis 1
  C d22[NV];  // second derivative along axis 2
  C d12[NV];  // mixed second derivative
};

// A runtime physics key (`key=val`, src/para.cpp:25-40): name, slot in the scheme's
// parameter array, reference default.
struct ParaKey {
  const char *name;
  int slot;
  double def;
};

// Per-launch scalar parameters of a scheme, by slot (at most 8 keys per scheme).
template <class C>
struct Para {
  C v[8];
};

// Status block shared by the kernels and the host (device memory, one per simulation).
struct Status {
  unsigned nan;                 // set when a stage produced a NaN (src/drift.cu:21,30)
  unsigned error;               // ErrorBits: a bounded wait gave up
  unsigned long long smax;      // running max of the CFL signal rate, bits of a double >= 0
  double dt;                    // time step of the current step (device-resident runs)
  double t;                     // simulation time (device-resident runs)
  double dt_next;               // time step the last dt update chose
  unsigned long long steps;     // steps taken by device-resident runs
};
enum ErrorBits : unsigned { ERR_TMA_TIMEOUT = 1u, ERR_QUEUE_TIMEOUT = 2u };

}  // namespace fg2
