/*
 * oracle/loops.h -- TEST INFRASTRUCTURE ONLY (the oracle; never the product).
 *
 * Host loop structure of fg2's time step, shared by the two CPU checkers:
 *   - oracle/port.cpp        : this project's restatement of the stencils and RHS;
 *   - oracle/ref_harness.cpp : the reference's own deriv.h / eqns.cuh compiled for the host.
 * Only the loops live here; the per-cell arithmetic is supplied by the includer.
 *
 * The includer defines, before including this file:
 *   R, E            real type of the state and of time (float/double, double/long double)
 *   S               struct of NV fields of type R (one cell)
 *   NV              number of fields per cell (int constant)
 *   orc_eqns(const S *c, int i, int j, int s_cells) -> S     right-hand side at cell c
 *   orc_first_order(S *c, R dt, int i, int j)                per-cell Euler hook
 *   orc_transform(int var, R x) -> R                         reflective-boundary sign map
 *
 * Host array layout (the reference's host/device layout, src/setup.cpp:60-72):
 *   cell-interleaved (AoS) NV values per cell, HALF = 3 ghost cells on every side,
 *   row pitch s = (n2 + 6) * NV values (dense rows), `x` points at the padded origin
 *   (ghost corner), the interior origin is x + 3*(s + NV).
 */
#ifndef ORACLE_LOOPS_H
#define ORACLE_LOOPS_H

#include <cstring>

namespace orc {

constexpr int H = 3;  // HALF = ORDER / 2 (src/fg2.h:26-34)

inline int pitch(int n2) { return (n2 + 2 * H) * NV; }

// kick: v <- beta * v + F(u) on the interior (src/kick.cu:59-106; the update order
// dst = beta * dst + src is src/kick.cu:53).  u must hold valid ghosts.
inline void kick(R *v, const R *u, int n1, int n2, R t, R beta)
{
  (void)t;  // passed but unused by the equations (src/kick.cu:98)
  const int s = pitch(n2);
  const R *ui = u + H * (s + NV);
  R *vi = v + H * (s + NV);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < n2; ++j) {
      const S f = orc_eqns((const S *)(ui + (long)i * s + j * NV), i, j, s / NV);
      const R *fr = (const R *)&f;
      R *d = vi + (long)i * s + j * NV;
      for (int k = 0; k < NV; ++k) d[k] = beta * d[k] + fr[k];
    }
}

// drift: u <- u + dt * v on the interior, NaN flag (src/drift.cu:23-32).
inline int drift(R *u, const R *v, int n1, int n2, R dt)
{
  const int s = pitch(n2);
  R *ui = u + H * (s + NV);
  const R *vi = v + H * (s + NV);
  int nan = 0;
#pragma omp parallel for schedule(static) reduction(| : nan)
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < NV * n2; ++j) {
      R &x = ui[(long)i * s + j];
      x += dt * vi[(long)i * s + j];
      if (x != x) nan = 1;
    }
  return nan;
}

// Periodic fill along axis 1 (rows), full padded width (src/bcond.cu:31-36).
inline void periodic1(R *x, int n1, int n2)
{
  const int s = pitch(n2);
  const size_t w = sizeof(R) * (size_t)s;
  for (int r = 0; r < H; ++r) {
    std::memcpy(x + (long)r * s, x + (long)(n1 + r) * s, w);          // ghost rows -3..-1
    std::memcpy(x + (long)(n1 + H + r) * s, x + (long)(H + r) * s, w);  // ghost rows n1..n1+2
  }
}

// Periodic fill along axis 2 (columns) over all n1 + 6 rows (src/bcond.cu:38-43).
inline void periodic2(R *x, int n1, int n2)
{
  const int s = pitch(n2);
  const size_t w = sizeof(R) * (size_t)(H * NV);
  for (int r = 0; r < n1 + 2 * H; ++r) {
    R *row = x + (long)r * s;
    std::memcpy(row, row + n2 * NV, w);
    std::memcpy(row + (n2 + H) * NV, row + H * NV, w);
  }
}

// Zero-gradient (mirror) rows along axis 1 (src/bcond.cu:45-57).
inline void neumann1(R *x, int n1, int n2)
{
  const int s = pitch(n2);
  const size_t w = sizeof(R) * (size_t)s;
  R *o = x + (long)H * s;  // row 0, column -3
  for (int r = 0; r < H; ++r) std::memcpy(o - (long)(r + 1) * s, o + (long)r * s, w);
  o += (long)n1 * s;
  for (int r = 0; r < H; ++r) std::memcpy(o + (long)r * s, o - (long)(r + 1) * s, w);
}

// Reflective columns along axis 2 with per-variable sign map (src/bcond.cu:59-75).
inline void reflect2(R *x, int n1, int n2)
{
  const int s = pitch(n2);
  for (int r = 0; r < n1 + 2 * H; ++r) {
    R *row = x + (long)r * s + H * NV;  // column 0 of this row
    for (int side = 0; side < 2; ++side)
      for (int k = 0; k < H; ++k) {
        const int d = side ? n2 - (1 + k) : k;
        const int g = side ? n2 + k : -(1 + k);
        for (int var = 0; var < NV; ++var)
          row[g * NV + var] = orc_transform(var, row[d * NV + var]);
      }
  }
}

// bcond: axis 1 first, then axis 2 (src/bcond.cu:77-86).
inline void bcond(R *x, int n1, int n2, int p1, int p2)
{
  if (p1) periodic1(x, n1, n2);
  else    neumann1(x, n1, n2);
  if (p2) periodic2(x, n1, n2);
  else    reflect2(x, n1, n2);
}

// Euler: per-cell operator-split pre-step (src/kick.cu:121-138).
inline void euler(R *u, int n1, int n2, R dt)
{
  const int s = pitch(n2);
  R *ui = u + H * (s + NV);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < n2; ++j) orc_first_order((S *)(ui + (long)i * s + j * NV), dt, i, j);
}

// step: Williamson low-storage RK3 (src/step.cpp:22-43).  The coefficient tables are
// written with double literals and stored in E, exactly as the reference does.
inline int step(R *u, R *v, int n1, int n2, E t, E dt, int p1, int p2)
{
  const E alpha[] = {0.0, 1.0 / 3.0, 3.0 / 4.0};
  const E beta[]  = {0.0, -5.0 / 9.0, -153.0 / 128.0};
  const E gamma[] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
  euler(u, n1, n2, (R)dt);
  int nan = 0;
  for (int i = 0; i < 3; ++i) {
    bcond(u, n1, n2, p1, p2);
    kick(v, u, n1, n2, (R)(t + dt * alpha[i]), (R)beta[i]);
    nan |= drift(u, v, n1, n2, (R)(dt * gamma[i]));
  }
  return nan;
}

}  // namespace orc

#endif  // ORACLE_LOOPS_H
