// fg2_b200/csrc/fg2b.h -- shared host/device definitions of the B200 time-step library.
//
// Device layout of one simulation: cells of NVAR interleaved fields (the reference's own
// cell layout, src/setup.cpp:60-72) in rows with ghost rows and columns.  Element (f, i, j),
// i in [-3, n1+3), j in [-4, n2+4), lives at
//       base[(i + GT) * RS + (j + GL) * CS + f]            CS = NVAR
//   GT = 3 ghost rows above/below (HALF of the 6th-order stencil, src/fg2.h:26-34);
//   GL = 4 columns left of the interior: 3 ghosts plus one so that the interior and every
//   tile's halo start on a 16-byte boundary (a TMA box must start on one);
//   RS = row stride = PC * NVAR, PC >= n2 + 8 cells rounded up to a multiple of 32, so every
//   row starts on 128 bytes and holds whole 16-byte groups of cells.
// A 128-cell tile row of one array is one contiguous 2 KB (FP32 hydro) segment.  Axis 1
// (i, n1, Delta1) is the slow, strided axis and axis 2 (j, n2, Delta2) the contiguous one,
// as in the reference (src/deriv.h:33, src/init.cpp:31-35).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector_types.h>
#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

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
  long long RS;  // row stride, elements
  int CS;        // cell stride, elements (NVAR)
  FG2_HD long long at(int f, int i, int j) const { return (long long)(i + GT) * RS + (long long)(j + GL) * CS + f; }
  FG2_HD long long elems() const { return (long long)(n1 + 2 * GT) * RS; }
};

inline Layout make_layout(int n1, int n2, int nvar)
{
  Layout L;
  L.n1 = n1;
  L.n2 = n2;
  L.CS = nvar;
  L.RS = ((long long)n2 + 2 * GL + 31) / 32 * 32 * nvar;
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
  C mn[3];             // their negatives
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

// Per-launch parameters of a scheme, by slot: the runtime keys first, then constants the
// scheme derives from them on the host (scheme::derive), at most NPARA in all.
constexpr int NPARA = 24;
template <class C>
struct Para {
  C v[NPARA];
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

// Deviation storage (FP16 / BF16 state arrays).  A stored 16-bit number h of field f stands
// for bg[f] + s h, with s the scale of field f on the SCALE_TILE x SCALE_TILE tile of the
// interior cell that holds the value (a ghost cell uses the tile of the interior cell it
// images).  Fields whose sign flips at a reflecting wall have bg = 0, so a ghost image is the
// negated 16-bit number.  v (the RK3 register) is stored as plain 16-bit numbers.
constexpr int SCALE_TILE = 64;
//
// The state is kept exactly as S - e, S the stored number's value and e the rounding error of
// the encode that produced it (the residual, the low part of a two-sum).  e is stored in a
// residual array (layout of u, ghost images included; one per ping-pong parity of u) as the
// 16-bit number e / s * RESID_SCALE: |e| <= s 2^-12 for FP16 numbers |h| <= 1, so the stored
// residual is at most about 1.
constexpr int DEV_MAX_FIELDS = 4;  // the codes hold one background and scale per field
constexpr double RESID_SCALE = 4096.0;
struct DevCode {
  float bg[4];           // per-field background (field mean at upload)
  const float4 *scale;   // per tile, row-major over (n1 / 64, n2 / 64) tiles: s of each field
  const float4 *inv;     // per tile: 1 / s
  int tiles2;            // tiles along axis 2
  void *r;               // rounding residual of the state read (16-bit numbers, layout of u)
  void *r_out;           // rounding residual of the state a substage writes
};

// ---- arithmetic on a scalar or on a pair ----------------------------------------------------
// The fused kernel's stencil works on pairs of fields of a cell: for FP32 the pair is a float2
// and every operation is one packed sm_100 instruction (add/mul/fma .f32x2), for FP64 a
// double2 evaluated component-wise.  Scheme code (eqns, the CFL rate) is written against the
// same helpers and evaluated per cell on scalars.
template <class C>
struct Scalar {
  using type = C;
};
template <>
struct Scalar<float2> {
  using type = float;
};
template <>
struct Scalar<double2> {
  using type = double;
};

template <class C>
FG2_HD C lit(double x) { return (C)x; }
template <class C>
FG2_HD typename Scalar<C>::type first(C x) { return x; }
FG2_HD float fmac(float a, float b, float c) { return fmaf(a, b, c); }
FG2_HD double fmac(double a, double b, double c) { return fma(a, b, c); }

template <>
FG2_HD float2 lit<float2>(double x) { return make_float2((float)x, (float)x); }
template <>
FG2_HD double2 lit<double2>(double x) { return make_double2(x, x); }
template <>
FG2_HD float first<float2>(float2 x) { return x.x; }
template <>
FG2_HD double first<double2>(double2 x) { return x.x; }

}  // namespace fg2

// Pair arithmetic, in the global namespace like float2 and double2 themselves so that
// argument-dependent lookup finds it from scheme code.
#if defined(__CUDACC__)
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 &operator+=(float2 &a, float2 b) { return a = a + b; }
__device__ __forceinline__ float2 &operator-=(float2 &a, float2 b) { return a = a - b; }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator*(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 operator-(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 &operator+=(double2 &a, double2 b) { return a = a + b; }
__device__ __forceinline__ double2 &operator-=(double2 &a, double2 b) { return a = a - b; }
#endif

namespace fg2 {

#if defined(__CUDACC__)
__device__ __forceinline__ float2 fmac(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vabs(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float2 vexp(float2 a) { return make_float2(__expf(a.x), __expf(a.y)); }
__device__ __forceinline__ float2 vsqrt(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ float2 vmax(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ float2 vcos(float2 a) { return make_float2(cosf(a.x), cosf(a.y)); }
__device__ __forceinline__ double2 fmac(double2 a, double2 b, double2 c)
{
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 vabs(double2 a) { return make_double2(fabs(a.x), fabs(a.y)); }
__device__ __forceinline__ double2 vexp(double2 a) { return make_double2(exp(a.x), exp(a.y)); }
__device__ __forceinline__ double2 vsqrt(double2 a) { return make_double2(sqrt(a.x), sqrt(a.y)); }
__device__ __forceinline__ double2 vmax(double2 a, double2 b) { return make_double2(fmax(a.x, b.x), fmax(a.y, b.y)); }
__device__ __forceinline__ double2 vcos(double2 a) { return make_double2(cos(a.x), cos(a.y)); }
#endif

FG2_HD float vabs(float a) { return fabsf(a); }
FG2_HD double vabs(double a) { return fabs(a); }
FG2_HD float vsqrt(float a) { return sqrtf(a); }
FG2_HD double vsqrt(double a) { return sqrt(a); }
FG2_HD float vmax(float a, float b) { return fmaxf(a, b); }
FG2_HD double vmax(double a, double b) { return fmax(a, b); }
FG2_HD double vexp(double a) { return exp(a); }
FG2_HD float vcos(float a) { return cosf(a); }
FG2_HD double vcos(double a) { return cos(a); }
#if defined(__CUDACC__)
__device__ __forceinline__ float vexp(float a) { return __expf(a); }
#else
inline float vexp(float a) { return expf(a); }
#endif

}  // namespace fg2
