// fg2_b200/csrc/substage.cuh -- the fused RK3 substage kernel (included inside namespace fg2
// by kernels.cu, once per scheme).
//
// Work decomposition.  A launch advances a list of grids (one simulation, or a batch of
// independent simulations of any sizes).  A tile is a strip of W interior columns (128, or
// 64 in batch launches) by 7 nb rows of one grid (nb blocks of 7 output rows, a launch
// parameter, 4 by default; the launch's `tail` parameter makes the last rows of each grid
// one-block tiles, and a band cut by the grid's edge has fewer blocks); the launch's tiles
// are numbered grid by grid, strip fastest, and a persistent grid of CTAs drains them from a
// queue (an atomic counter that the last CTA to finish resets, so a launch needs no host-side
// reset and replays from a CUDA graph).  Launches alternate direction: a reverse launch takes
// the grids last first and lays each grid's bands out from its last row up.  A CTA
// has W / 32 warps; a thread owns one column of the strip.  Each grid is described by a GridDesc in
// device memory: its TMA tensor maps, output pointers, layout, boundaries, time step and
// status block.
//
// Data movement.  u and v stream through a ring of NSLOT shared-memory slots by TMA
// (cp.async.bulk.tensor.3d, no multicast): chunk 0 of a tile is the 7-row warm-up box
// u[i0-4 .. i0+3) x [j0-4, j0+W+4), chunk b+1 the 7 leading rows u[i0+3+7b ..] of output
// block b together with v of the block's 7 output rows.  A box lands as [row][cell][field],
// the cells' fields interleaved as in HBM, so a thread reads a whole hydro cell with one
// 16-byte shared load.  The results u' and v are written by the threads straight from
// registers (one 16-byte store per cell and array; a warp writes 512 contiguous bytes per row).
// One CTA barrier per chunk hands the slot back to the producer thread; every wait on a TMA
// completion is bounded (%globaltimer) and the CTA agrees on a timeout before leaving, which
// raises an error bit in the launch's status block.
//
// Stencil.  Each thread walks its column down the tile.  At every leading row L it loads the
// 7 cells u(L, j-3..j+3) from shared memory and computes the axis-2 (contiguous) derivatives
// D2 and D22 of row L, pushes u(L, j) into a 7-row register window (the axis-1 stencil of row
// L-3 then needs no further loads), and feeds the mixed derivative by streaming accumulators:
// with delta_k(r) = u(r, j+k) - u(r, j-k), D12(r) = sum_k m_k (delta_k(r+k) - delta_k(r-k)),
// so delta_k(L) is added to row L-k and subtracted from row L+k (src/deriv.h:60-62
// regrouped).  Fields are handled in pairs ((lnd, u1), (u2, lne) for hydro; up to three pairs)
// so the stencil arithmetic of two fields is one packed FP32x2 instruction (add/mul/fma .f32x2
// on sm_100); the mixed derivative is accumulated for the scheme's D12 fields only.  The output row
// L-3 then has all its derivatives in registers; the scheme's eqns() gives F (with the cell's
// indices, the spacings and the scheme's per-column geometry, computed once per tile), and the
// epilogue applies v <- F + beta v, u' <- u + gamma dt v (src/kick.cu:53, src/drift.cu:29),
// stores u' with its ghost images and v, flags NaNs and, on the last stage, folds the CFL rate
// into a max.  Register slots are indexed by row mod 7 and the row loop is unrolled by 7, so
// the window never moves.
//
// Deviation storage.  With FP16 / BF16 state arrays (S = __half / __nv_bfloat16) the stencil
// still runs in FP32.  The state is the 16-bit number less its rounding residual e, which a
// second 16-bit array (one per ping-pong parity of u) holds as e / s * RESID_SCALE: each u box
// lands with the residual box of the same cells (residual numbers r), and the CTA decodes
// both into the state T = bg + s h - s r / RESID_SCALE (s of the cell's 64 x 64 tile) in an
// FP32 copy in shared memory that the stencil reads.  v is converted on load; u' = T + gamma dt v is encoded with
// its tile's 1/s, its residual e' = encode(u') - u' stored beside it, and v stored as 16-bit
// numbers, so every rounding of the state is compensated (src/step.cpp:24-35 unchanged
// otherwise).
//
// Stencil weights.  A single-grid launch folds 1/Delta into the weights (constant-bank
// operands).  A batch launch (SC) uses the reference's plain weights and multiplies each
// derivative by its grid's 1/Delta factors, which it keeps in registers, as the reference
// divides by Delta after the weighted sum (src/deriv.h:42-62).
#pragma once

namespace sub {

#ifndef FG2_NSLOT
#define FG2_NSLOT 2
#endif
constexpr int CH = 7;              // rows per chunk = register window period

// The form of a block's row loop.  Unrolled by 7, every row with its own copy of the
// right-hand side, so the compiler overlaps one row's arithmetic with the next row's loads:
// the faster form while the body fits the instruction cache (hydro: 31.7 against 29.1
// Gcell-steps/s rolled at 4096^2 FP32, 23.3 against 18.7 FP16).  Rolled, the register-window
// work of each row in a 7-way switch and one copy of the right-hand side and epilogue, for
// the six-field disk scheme, whose unrolled body stalls on instruction fetch (10.15 against
// 9.36 Gcell-steps/s at 2048^2).
__host__ __device__ constexpr bool rolled_rows() { return NV > 4; }
constexpr int NB_DEFAULT = TILE_BLOCKS_DEFAULT;  // output blocks per tile unless a launch sets nb
constexpr int NP = (NV + 1) / 2;   // field pairs

// Strip geometry of a launch: W interior columns per tile, one thread per column (W / 32
// warps per CTA), and the TMA box of u W + 8 columns wide (halo 4 + 4; the stencil uses 3).
template <int W>
struct Strip {
  static constexpr int SW = W;
  static constexpr int BW = W + 2 * GL;
  static constexpr int NT = W;
  static_assert(W % 32 == 0 && W >= 32 && W <= 256, "whole warps, at most 8 per CTA");
};

// Fields with a mixed derivative D12 (the scheme's D12_FIELDS), in field order: the k-th of
// them has streaming accumulator k.
__host__ __device__ constexpr int d12_count(unsigned m) { return m ? (int)(m & 1u) + d12_count(m >> 1) : 0; }
__host__ __device__ constexpr int d12_field(unsigned m, int k, int f = 0)
{
  return (m & 1u) ? (k == 0 ? f : d12_field(m >> 1, k - 1, f + 1)) : d12_field(m >> 1, k, f + 1);
}
constexpr int ND12 = d12_count(scheme::D12_FIELDS);
static_assert(ND12 >= 1 && d12_field(scheme::D12_FIELDS, ND12 - 1) < NV, "mixed-derivative fields");

// Cells per TMA group of a storage type: the innermost box dimension is one group of
// interleaved cells and must be a multiple of 16 bytes.
__host__ __device__ constexpr int group_of(int elem)
{
  return ((elem >= 8 ? 2 : 4) * NV * elem) % 16 == 0 ? (elem >= 8 ? 2 : 4) : 2 * (elem >= 8 ? 2 : 4);
}

// Shared memory of one CTA: NSLOT slots of [u box | v box | r box] (the v box only when the
// stage reads v, the r box -- the rounding residual of a 16-bit u box, the same cells -- only
// with 16-bit storage), two
// FP32 copies of a landed u box (deviation storage: chunk n is stenciled from one while chunk
// n + 1 is decoded into the other), then the mbarriers and the producer's bookkeeping.  The
// v and r boxes start VOFF cells left of the strip when a cell group is wider than the 4
// ghost columns.
template <class S, bool RV, bool RR, int W>
struct Geo {
  static constexpr int SW = Strip<W>::SW, BW = Strip<W>::BW;
  static constexpr bool DEV = Store<S>::DEV;
  static constexpr int NSLOT = FG2_NSLOT;
  static constexpr int CB = NV * (int)sizeof(S);  // bytes per cell
  static constexpr int G = group_of((int)sizeof(S));
  static constexpr int VOFF = GL % G;
  static constexpr int VBW = (SW + VOFF + G - 1) / G * G;
  static constexpr uint32_t U_BYTES = (uint32_t)(BW * CH * CB);
  static constexpr uint32_t V_OFF = (U_BYTES + 127) / 128 * 128;  // TMA destinations on 128 B
  static constexpr uint32_t V_BYTES = (uint32_t)(VBW * CH * CB);
  static constexpr uint32_t V_AL = (V_BYTES + 127) / 128 * 128;
  static constexpr uint32_t U_AL = (U_BYTES + 127) / 128 * 128;
  static constexpr uint32_t R_OFF = V_OFF + (RV ? V_AL : 0);
  static constexpr uint32_t SLOT = R_OFF + (RR ? U_AL : 0);
  static constexpr size_t DEC_OFF = (size_t)NSLOT * SLOT;
  static constexpr size_t DEC_ONE = DEV ? ((size_t)BW * CH * NV * sizeof(float) + 127) / 128 * 128 : 0;
  static constexpr size_t DEC_BYTES = 2 * DEC_ONE;
  static constexpr size_t BAR_OFF = DEC_OFF + DEC_BYTES;
  // tail: full[NSLOT] (mbarriers), the slots' tiles (TileSlot, 6 ints each), producer state
  // (Producer, 12 ints)
  static constexpr size_t SMEM = BAR_OFF + NSLOT * sizeof(uint64_t) + NSLOT * 6 * sizeof(int) + 12 * sizeof(int) + 64;
  static_assert(SLOT % 128 == 0, "TMA shared-memory boxes must be 128-byte aligned");
  static_assert(BW % G == 0 && VBW % G == 0 && (GL - VOFF) % G == 0, "boxes and tile origins are whole cell groups");
  static_assert(BW / G <= 256 && VBW / G <= 256 && CH <= 256 && G * NV <= 256, "TMA box dimensions");
};

// One cell's NV values as field pairs ((lnd, u1), (u2, lne)): one or two 16-byte accesses for
// a hydro cell, scalar ones for a 3-field cell.
template <class T>
__device__ __forceinline__ void ld_cell(const T *p, typename PairOf<T>::type out[NP])
{
  using PO = PairOf<T>;
  if constexpr (NV == 4 && sizeof(T) == 4) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    out[0] = make_float2(x.x, x.y);
    out[1] = make_float2(x.z, x.w);
  } else if constexpr (NV == 4 && sizeof(T) == 8) {
    out[0] = *reinterpret_cast<const double2 *>(p);
    out[1] = *reinterpret_cast<const double2 *>(p + 2);
  } else if constexpr (NV == 6) {  // 24- or 48-byte cells: three 8- or 16-byte accesses
#pragma unroll
    for (int q = 0; q < 3; ++q) out[q] = *reinterpret_cast<const typename PO::type *>(p + 2 * q);
  } else {
#pragma unroll
    for (int q = 0; q < NP; ++q) out[q] = PO::make(p[2 * q], 2 * q + 1 < NV ? p[2 * q + 1] : T(0));
  }
}

template <class T>
__device__ __forceinline__ void st_cell(T *p, const typename PairOf<T>::type in[NP])
{
  if constexpr (NV == 4 && sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(in[0].x, in[0].y, in[1].x, in[1].y);
  } else if constexpr (NV == 4 && sizeof(T) == 8) {
    *reinterpret_cast<double2 *>(p) = in[0];
    *reinterpret_cast<double2 *>(p + 2) = in[1];
  } else if constexpr (NV == 6) {
#pragma unroll
    for (int q = 0; q < 3; ++q) *reinterpret_cast<typename PairOf<T>::type *>(p + 2 * q) = in[q];
  } else {
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      p[2 * q] = in[q].x;
      if (2 * q + 1 < NV) p[2 * q + 1] = in[q].y;
    }
  }
}

// One cell of a storage array as compute-type field pairs, and back (16-bit storage converts).
template <class S>
__device__ __forceinline__ void load_cell(const S *p, typename PairOf<typename Store<S>::C>::type out[NP])
{
  using St = Store<S>;
  if constexpr (!St::DEV) {
    ld_cell<S>(p, out);
  } else if constexpr (NV == 4) {
    const uint2 w = *reinterpret_cast<const uint2 *>(p);
    out[0] = St::to2(*reinterpret_cast<const typename St::S2 *>(&w.x));
    out[1] = St::to2(*reinterpret_cast<const typename St::S2 *>(&w.y));
  } else {
#pragma unroll
    for (int q = 0; q < NP; ++q)
      out[q] = make_float2(St::to(p[2 * q]), 2 * q + 1 < NV ? St::to(p[2 * q + 1]) : 0.f);
  }
}

template <class S>
__device__ __forceinline__ void store_cell(S *p, const typename PairOf<typename Store<S>::C>::type in[NP])
{
  using St = Store<S>;
  if constexpr (!St::DEV) {
    st_cell<S>(p, in);
  } else if constexpr (NV == 4) {
    const typename St::S2 a = St::from2(in[0]), b = St::from2(in[1]);
    uint2 w;
    w.x = *reinterpret_cast<const unsigned *>(&a);
    w.y = *reinterpret_cast<const unsigned *>(&b);
    *reinterpret_cast<uint2 *>(p) = w;
  } else {
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      p[2 * q] = St::from(in[q].x);
      if (2 * q + 1 < NV) p[2 * q + 1] = St::from(in[q].y);
    }
  }
}

// Deviation storage: stores the 16-bit numbers of h (field pairs) at p and returns them as
// stored (raw) and converted back (hs).
template <class S>
__device__ __forceinline__ void encode_cell(S *p, const float2 h[NP], float2 hs[NP], S raw[NV])
{
  using St = Store<S>;
  if constexpr (NV == 4) {
    const typename St::S2 a = St::from2(h[0]), b = St::from2(h[1]);
    uint2 w;
    w.x = *reinterpret_cast<const unsigned *>(&a);
    w.y = *reinterpret_cast<const unsigned *>(&b);
    *reinterpret_cast<uint2 *>(p) = w;
    hs[0] = St::to2(a);
    hs[1] = St::to2(b);
    raw[0] = a.x;
    raw[1] = a.y;
    raw[2] = b.x;
    raw[3] = b.y;
  } else {
#pragma unroll
    for (int f = 0; f < NV; ++f) {
      raw[f] = St::from((f & 1) ? h[f >> 1].y : h[f >> 1].x);
      p[f] = raw[f];
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) hs[q] = make_float2(St::to(raw[2 * q]), 2 * q + 1 < NV ? St::to(raw[2 * q + 1]) : 0.f);
  }
}

// Interior cell whose value a padded index i (ghost or padding) holds, clamped into the grid.
__device__ __forceinline__ int source_index(int i, int n, int periodic)
{
  if (i < 0) i = periodic ? i + n : -1 - i;
  else if (i >= n) i = periodic ? i - n : 2 * n - 1 - i;
  return min(max(i, 0), n - 1);
}

// Tiles of one grid: strip fastest, so horizontally adjacent tiles run together and share
// their halo columns through L2.  The rows are cut into `bands` bands of nb blocks of 7 rows
// and then `small` tail bands of one block: with tail > 0 at least `tail` one-block bands end
// the grid, so the last tiles a launch hands out are short and the CTAs finish together
// (the persistent grid's last wave would otherwise be whole tiles on a few CTAs).  tail = 0:
// nb-block bands only, the last one cut at the grid's edge.
struct TileGrid {
  int strips, bands, small, ntiles;
};

__host__ __device__ inline TileGrid tile_grid(const Layout &L, int nb, int sw, int tail = 0)
{
  TileGrid g;
  const int th = nb * CH;
  g.strips = (L.n2 + sw - 1) / sw;
  if (tail > 0) {
    const int b = (L.n1 - CH * tail) / th;
    g.bands = b > 0 ? b : 0;
  } else {
    g.bands = (L.n1 + th - 1) / th;
  }
  const int rest = L.n1 - g.bands * th;
  g.small = rest > 0 ? (rest + CH - 1) / CH : 0;
  g.ntiles = g.strips * (g.bands + g.small);
  return g;
}

// Rows of the band at processing position q of a grid: the nb-block bands first, then the
// one-block tail bands.  A reverse launch lays the bands out from the last row up, so it too
// takes the tail bands last; the band that meets the grid's far edge is cut there.  A tile
// computes rows [i0, iend) in nbt blocks (its last block may reach past iend: those rows
// belong to the next band or lie past the grid, and are not written).
struct Band {
  int i0, iend, nbt;
};
__host__ __device__ inline Band band_rows(int n1, int nb, int bands, int q, bool reverse)
{
  const int th = nb * CH;
  const int len = q < bands ? th : CH;
  const int off = q < bands ? q * th : bands * th + (q - bands) * CH;
  Band b;
  if (!reverse) {
    b.i0 = off;
    b.iend = off + len < n1 ? off + len : n1;
  } else {
    b.iend = n1 - off;
    b.i0 = b.iend - len > 0 ? b.iend - len : 0;
  }
  b.nbt = (b.iend - b.i0 + CH - 1) / CH;
  return b;
}

// The tile a chunk slot holds, written by the issuing thread with the slot's first chunk:
// launch tile (< 0: the end of the queue), grid, rows [i0, iend) in nbt blocks, first column.
struct TileSlot {
  int tile, g, i0, iend, j0, nbt;
};

// Does field f carry second derivatives (D11, D22) under mask M2?
template <unsigned M2>
__host__ __device__ constexpr bool need(int f)
{
  return f < NV && (M2 & (1u << f));
}

// Per-thread rolling state.  Slot index = leading-row index mod 7.
template <class T>
struct Roll {
  using P = typename PairOf<T>::type;
  P w[NP][CH];    // u(row, j) per field pair, rows L-6 .. L
  P h2[NP][CH];   // D2 of each row
  P h22[NP][CH];  // D22 of each row (only the lanes under the mask are written)
  T x[ND12][CH];  // D12 accumulators of the D12 fields
};

// Everything a thread needs of the grid its current tile belongs to (registers).
template <class S>
struct GridRegs {
  using T = typename Store<S>::C;
  using P = typename PairOf<T>::type;
  Layout L;
  S *u_out, *v;
  Status *status;
  int p1, p2;
  P gdt;                       // gamma dt of this grid's step, both lanes
  P s1, s2, s11, s22;          // 1/Delta factors (batch launches)
  T s12, inv1, inv2, delta1, delta2;  // 1/(Delta1 Delta2), CFL factors, Delta1, Delta2
  // deviation storage
  P bg[NP];                    // per-field background
  const float4 *scale, *inv;   // per-tile s and 1/s
  S *r;                        // rounding residual of the state the stage writes
  int tiles2;
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Leading-row work of field pair PI for register slot R, from the pair's values at
// columns j-3 .. j+3 of the leading row.
// D2: the row is an output row of the tile, so its axis-2 derivatives are needed (the warm-up
// rows above the tile only feed the window and the mixed-derivative accumulators).
template <class T, unsigned M2, int R, int PI, bool D2>
__device__ __forceinline__ void lead_pair(const typename PairOf<T>::type (&x)[7][NP], const KParams<T> &a, Roll<T> &s,
                                          typename PairOf<T>::type dk[3])
{
  using P = typename PairOf<T>::type;
  const P l3 = x[0][PI], l2 = x[1][PI], l1 = x[2][PI], c = x[3][PI], r1 = x[4][PI], r2 = x[5][PI], r3 = x[6][PI];
  s.w[PI][R] = c;
  dk[0] = r1 - l1;
  dk[1] = r2 - l2;
  dk[2] = r3 - l3;
  if constexpr (!D2) return;
  s.h2[PI][R] = fmac(a.k.a2[0], dk[0], fmac(a.k.a2[1], dk[1], a.k.a2[2] * dk[2]));
  constexpr bool nx = need<M2>(2 * PI), ny = need<M2>(2 * PI + 1);
  if constexpr (nx && ny) {
    s.h22[PI][R] = fmac(a.k.b2[0], c, fmac(a.k.b2[1], r1 + l1, fmac(a.k.b2[2], r2 + l2, a.k.b2[3] * (r3 + l3))));
  } else if constexpr (nx) {
    s.h22[PI][R].x = fmac(a.ks.b2[0], c.x, fmac(a.ks.b2[1], r1.x + l1.x,
                                                fmac(a.ks.b2[2], r2.x + l2.x, a.ks.b2[3] * (r3.x + l3.x))));
  } else if constexpr (ny) {
    s.h22[PI][R].y = fmac(a.ks.b2[0], c.y, fmac(a.ks.b2[1], r1.y + l1.y,
                                                fmac(a.ks.b2[2], r2.y + l2.y, a.ks.b2[3] * (r3.y + l3.y))));
  }
}

// D12 of D12 field number G (field f is lane f & 1 of pair f / 2) from the leading row's
// differences: rows L+k get -m_k delta_k(L) (mn = -m), rows L-k get +m_k delta_k(L); row L-3
// is then complete.  The first contribution to row L+3 initialises its accumulator.  One
// instantiation per field, so every index is a compile-time constant.
template <class T, int R, int G>
__device__ __forceinline__ void d12_lead(const typename PairOf<T>::type (&dk)[NP][3], const KParams<T> &a, Roll<T> &s)
{
  if constexpr (G < ND12) {
    constexpr int f = d12_field(scheme::D12_FIELDS, G), pf = f >> 1;
    const T d1 = (f & 1) ? dk[pf][0].y : dk[pf][0].x;
    const T d2 = (f & 1) ? dk[pf][1].y : dk[pf][1].x;
    const T d3 = (f & 1) ? dk[pf][2].y : dk[pf][2].x;
    s.x[G][(R + 3) % CH] = a.ks.mn[2] * d3;
    s.x[G][(R + 2) % CH] = fmac(a.ks.mn[1], d2, s.x[G][(R + 2) % CH]);
    s.x[G][(R + 1) % CH] = fmac(a.ks.mn[0], d1, s.x[G][(R + 1) % CH]);
    s.x[G][(R + 6) % CH] = fmac(a.ks.m[0], d1, s.x[G][(R + 6) % CH]);
    s.x[G][(R + 5) % CH] = fmac(a.ks.m[1], d2, s.x[G][(R + 5) % CH]);
    s.x[G][(R + 4) % CH] = fmac(a.ks.m[2], d3, s.x[G][(R + 4) % CH]);
    d12_lead<T, R, G + 1>(dk, a, s);
  }
}

// The finished D12 of every D12 field at output slot S0 into the cell (other fields: 0).
template <class T, bool SC, int S0, int G, class GR>
__device__ __forceinline__ void d12_emit(const GR &gr, const Roll<T> &s, Cell<T, NV> &cell)
{
  if constexpr (G < ND12) {
    constexpr int f = d12_field(scheme::D12_FIELDS, G);
    cell.d12[f] = SC ? s.x[G][S0] * gr.s12 : s.x[G][S0];
    d12_emit<T, SC, S0, G + 1>(gr, s, cell);
  }
}

// Leading-row work for register slot R: loads the 7 cells of row R of the chunk around the
// thread's column; base points at column j-3 of row 0, rows are RSTRIDE elements apart.
template <class T, unsigned M2, int R, int RSTRIDE, bool D2 = true>
__device__ __forceinline__ void lead_row(const T *base, const KParams<T> &a, Roll<T> &s)
{
  using P = typename PairOf<T>::type;
  const T *row = base + R * RSTRIDE;
  P x[7][NP];
#pragma unroll
  for (int k = 0; k < 7; ++k) ld_cell<T>(row + k * NV, x[k]);
  P dk[NP][3];
  lead_pair<T, M2, R, 0, D2>(x, a, s, dk[0]);
  if constexpr (NP > 1) lead_pair<T, M2, R, 1, D2>(x, a, s, dk[1]);
  if constexpr (NP > 2) lead_pair<T, M2, R, 2, D2>(x, a, s, dk[2]);
  d12_lead<T, R, 0>(dk, a, s);
}

// Derivatives of field pair PI at the output row held in register slot S0, into a Cell.
template <class T, unsigned M2, bool SC, int S0, int PI, class GR>
__device__ __forceinline__ void emit_pair(const KParams<T> &a, const GR &gr, const Roll<T> &s, Cell<T, NV> &cell)
{
  using P = typename PairOf<T>::type;
  const P c = s.w[PI][S0];
  const P p1 = s.w[PI][(S0 + 1) % CH], n1 = s.w[PI][(S0 + 6) % CH];
  const P p2 = s.w[PI][(S0 + 2) % CH], n2 = s.w[PI][(S0 + 5) % CH];
  const P p3 = s.w[PI][(S0 + 3) % CH], n3 = s.w[PI][(S0 + 4) % CH];
  P d1 = fmac(a.k.a1[0], p1 - n1, fmac(a.k.a1[1], p2 - n2, a.k.a1[2] * (p3 - n3)));
  P d2 = s.h2[PI][S0];
  constexpr bool nx = need<M2>(2 * PI), ny = need<M2>(2 * PI + 1);
  P d11 = lit<P>(0.0), d22 = lit<P>(0.0);
  if constexpr (nx && ny) {
    d11 = fmac(a.k.b1[0], c, fmac(a.k.b1[1], p1 + n1, fmac(a.k.b1[2], p2 + n2, a.k.b1[3] * (p3 + n3))));
    d22 = s.h22[PI][S0];
  } else if constexpr (nx) {
    d11.x = fmac(a.ks.b1[0], c.x, fmac(a.ks.b1[1], p1.x + n1.x, fmac(a.ks.b1[2], p2.x + n2.x, a.ks.b1[3] * (p3.x + n3.x))));
    d22.x = s.h22[PI][S0].x;
  } else if constexpr (ny) {
    d11.y = fmac(a.ks.b1[0], c.y, fmac(a.ks.b1[1], p1.y + n1.y, fmac(a.ks.b1[2], p2.y + n2.y, a.ks.b1[3] * (p3.y + n3.y))));
    d22.y = s.h22[PI][S0].y;
  }
  if constexpr (SC) {
    d1 = d1 * gr.s1;
    d2 = d2 * gr.s2;
    if constexpr (nx || ny) {
      d11 = d11 * gr.s11;
      d22 = d22 * gr.s22;
    }
  }
  cell.q[2 * PI] = c.x;
  cell.d1[2 * PI] = d1.x;
  cell.d2[2 * PI] = d2.x;
  cell.d11[2 * PI] = d11.x;
  cell.d22[2 * PI] = d22.x;
  if constexpr (2 * PI + 1 < NV) {
    cell.q[2 * PI + 1] = c.y;
    cell.d1[2 * PI + 1] = d1.y;
    cell.d2[2 * PI + 1] = d2.y;
    cell.d11[2 * PI + 1] = d11.y;
    cell.d22[2 * PI + 1] = d22.y;
  }
}

// Ghost images of interior cell (i, j) for the next stage (the reference's bcond result,
// src/bcond.cu:22-86): at most one row image and one column image, and their corner, each
// stored whole; column images across a wall negate the fields the scheme reflects.  Grids
// narrower than two ghost widths take the general path.  Out of line: only cells of tiles
// near an edge call it, and one copy keeps the unrolled row loop small.
template <class S>
__device__ __forceinline__ void rim_body(S *u, const Layout L, int i, int j,
                                         const typename PairOf<typename Store<S>::C>::type (&qp)[NP], int p1, int p2)
{
  using T = typename Store<S>::C;
  using P = typename PairOf<T>::type;
  const int n1 = L.n1, n2 = L.n2;
  if (n1 < 2 * HALF || n2 < 2 * HALF) {
    T qn[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) qn[f] = (f & 1) ? qp[f >> 1].y : qp[f >> 1].x;
    store_ghosts<S, T>(u, L, i, j, qn, p1, p2);
    return;
  }
  int ia = -(1 << 30), ja = -(1 << 30);
  if (i < HALF) ia = p1 ? i + n1 : -1 - i;
  else if (i >= n1 - HALF) ia = p1 ? i - n1 : 2 * n1 - 1 - i;
  if (j < HALF) ja = p2 ? j + n2 : -1 - j;
  else if (j >= n2 - HALF) ja = p2 ? j - n2 : 2 * n2 - 1 - j;
  P f[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) f[p] = qp[p];
#pragma unroll
  for (int k = 0; k < NV; ++k)
    if (!p2 && scheme::reflect_sign(k) < 0) {
      if (k & 1) f[k >> 1].y = -f[k >> 1].y;
      else f[k >> 1].x = -f[k >> 1].x;
    }
  if (ia > -(1 << 30)) store_cell<S>(u + L.at(0, ia, j), qp);
  if (ja > -(1 << 30)) {
    store_cell<S>(u + L.at(0, i, ja), f);
    if (ia > -(1 << 30)) store_cell<S>(u + L.at(0, ia, ja), f);
  }
}

// Cells of up to two field pairs (q1 is the last pair) ...
template <class S>
__device__ __noinline__ void rim_images(S *u, const Layout L, int i, int j, typename PairOf<typename Store<S>::C>::type q0,
                                        typename PairOf<typename Store<S>::C>::type q1, int p1, int p2)
{
  using P = typename PairOf<typename Store<S>::C>::type;
  const P qp[2] = {q0, q1};
  if constexpr (NP <= 2) rim_body<S>(u, L, i, j, qp, p1, p2);
}

// ... and of three (six-field schemes).
template <class S>
__device__ __noinline__ void rim_images3(S *u, const Layout L, int i, int j, typename PairOf<typename Store<S>::C>::type q0,
                                         typename PairOf<typename Store<S>::C>::type q1,
                                         typename PairOf<typename Store<S>::C>::type q2, int p1, int p2)
{
  using P = typename PairOf<typename Store<S>::C>::type;
  const P qp[3] = {q0, q1, q2};
  if constexpr (NP == 3) rim_body<S>(u, L, i, j, qp, p1, p2);
}

// The same for 16-bit storage, with the stored numbers (reflected fields have bg = 0, so their
// images are the negated numbers).
// The stored numbers of one cell, passed by value (an array argument would put every cell's
// numbers through local memory, rim or not).
template <class S>
struct RawCell {
  S v[NV];
};

template <class S>
__device__ __noinline__ void rim_images_raw(S *u, const Layout L, int i, int j, const RawCell<S> rc, int p1, int p2)
{
  const int n1 = L.n1, n2 = L.n2;
  const S *raw = rc.v;
  if (n1 < 2 * HALF || n2 < 2 * HALF) {
    store_ghosts<S, S>(u, L, i, j, raw, p1, p2);
    return;
  }
  int ia = -(1 << 30), ja = -(1 << 30);
  if (i < HALF) ia = p1 ? i + n1 : -1 - i;
  else if (i >= n1 - HALF) ia = p1 ? i - n1 : 2 * n1 - 1 - i;
  if (j < HALF) ja = p2 ? j + n2 : -1 - j;
  else if (j >= n2 - HALF) ja = p2 ? j - n2 : 2 * n2 - 1 - j;
  auto put = [&](long long off, bool flip) {
#pragma unroll
    for (int f = 0; f < NV; ++f) u[off + f] = (flip && scheme::reflect_sign(f) < 0) ? -raw[f] : raw[f];
  };
  if (ia > -(1 << 30)) put(L.at(0, ia, j), false);
  if (ja > -(1 << 30)) {
    put(L.at(0, i, ja), !p2);
    if (ia > -(1 << 30)) put(L.at(0, ia, ja), !p2);
  }
}

// Derivatives of the output row in register slot S0 (the row 3 behind the leading row) into a
// Cell, and the row's own values as field pairs (qc).
template <class T, unsigned M2, bool SC, int S0, class GR>
__device__ __forceinline__ void gather_row(const KParams<T> &a, const GR &gr, const Roll<T> &s, Cell<T, NV> &cell,
                                           typename PairOf<T>::type qc[NP])
{
  emit_pair<T, M2, SC, S0, 0>(a, gr, s, cell);
  if constexpr (NP > 1) emit_pair<T, M2, SC, S0, 1>(a, gr, s, cell);
  if constexpr (NP > 2) emit_pair<T, M2, SC, S0, 2>(a, gr, s, cell);
#pragma unroll
  for (int f = 0; f < NV; ++f) cell.d12[f] = T(0);
  d12_emit<T, SC, S0, 0>(gr, s, cell);
#pragma unroll
  for (int p = 0; p < NP; ++p) qc[p] = s.w[p][S0];
}

// The output row of a block from its gathered derivatives: F by the scheme's eqns(), then
// the epilogue.  vr is v of the cell (read stages), rr its rounding residual (16-bit stages 0
// and 1), scv / ivv the scales of the cell's tile, cg the scheme's geometry of the column.
// u' and v go straight to HBM; edge cells also write their ghost images.
//
// Deviation storage keeps the state exactly as the 16-bit number S plus a residual: the value
// is T = S - e with e the rounding error of the last encode.  Stages 0 and 1 read e (scaled by
// 1 / s and RESID_SCALE, stored as a 16-bit number in r) and update T instead of S, so every
// rounding is compensated (the two-sum u' = T + gamma dt v = S' - e').  Stage 0's and stage 2's
// e' go to r; stage 1's e' is folded into v (stored as v - e' / (beta2 gamma2 dt)), which stage
// 2 reads once, with no carry beyond it.  The stencil itself reads S.
template <class S, unsigned M2, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL, bool SC>
__device__ __forceinline__ void finish_row(const Cell<typename Store<S>::C, NV> &cell,
                                           const typename PairOf<typename Store<S>::C>::type qc[NP],
                                           const typename PairOf<typename Store<S>::C>::type vr[NP], int i, int j,
                                           int iend, const float4 &scv, const float4 &ivv,
                                           const KParams<typename Store<S>::C> &a, const GridRegs<S> &gr, bool full,
                                           bool rim, bool &nan, typename Store<S>::C &rate,
                                           const scheme::Geom<typename Store<S>::C> &cg)
{
  using T = typename Store<S>::C;
  using P = typename PairOf<T>::type;
  using St = Store<S>;
  constexpr bool DEV = St::DEV;
  T r[NV];
  const T dl1 = SC ? gr.delta1 : a.ks.delta1, dl2 = SC ? gr.delta2 : a.ks.delta2;
  scheme::eqns<M2>(cell, a.p, i, j, r, dl1, dl2, cg);
  if (!full && (i >= iend || j >= gr.L.n2)) return;  // cells past the tile's rows or the grid
  P sc[NP], iv[NP];  // deviation storage: the scales of the cell's tile
  if constexpr (DEV && WRITE_U) {
    sc[0] = make_float2(scv.x, scv.y);
    iv[0] = make_float2(ivv.x, ivv.y);
    if constexpr (NP > 1) {
      sc[NP - 1] = make_float2(scv.z, scv.w);
      iv[NP - 1] = make_float2(ivv.z, ivv.w);
    }
  }
  P vn[NP], qp[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    vn[p] = PairOf<T>::make(r[2 * p], 2 * p + 1 < NV ? r[2 * p + 1] : T(0));
    if (READ_V) vn[p] = fmac(a.beta2, vr[p], vn[p]);
    qp[p] = fmac(gr.gdt, vn[p], qc[p]);
  }
  const long long o = gr.L.at(0, i, j);
  if constexpr (!DEV) {
    if (WRITE_U) store_cell<S>(gr.u_out + o, qp);
    if (WRITE_V) store_cell<S>(gr.v + o, vn);
  }
  using RS = typename Resid<S>::type;
  RawCell<S> raw;
  RawCell<RS> rraw;
  if constexpr (DEV) {
    if (WRITE_U) {
      // encode u' with its tile's 1/s; e' = S' - u' is the rounding residual, stored as
      // e' / s * RESID_SCALE beside it
      P h[NP], hs[NP], e[NP], ro[NP], unused[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) h[p] = (qp[p] - gr.bg[p]) * iv[p];
      encode_cell<S>(gr.u_out + o, h, hs, raw.v);
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        e[p] = fmac(sc[p], hs[p], gr.bg[p]) - qp[p];
        ro[p] = e[p] * (iv[p] * lit<P>(RESID_SCALE));
      }
      encode_cell<RS>(reinterpret_cast<RS *>(gr.r) + o, ro, unused, rraw.v);
    }
    if (WRITE_V) store_cell<S>(gr.v + o, vn);
  }
  if (WRITE_U) {
    T qn[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) qn[f] = (f & 1) ? qp[f >> 1].y : qp[f >> 1].x;
    // one NaN test per cell: a NaN in any field makes the sum NaN
    T sum = qn[0];
#pragma unroll
    for (int f = 1; f < NV; ++f) sum += qn[f];
    nan |= sum != sum;
    if (rim) {  // tiles within HALF cells of an edge: the cell's ghost images for the next stage
      if constexpr (!DEV) {
        if constexpr (NP == 3) rim_images3<S>(gr.u_out, gr.L, i, j, qp[0], qp[1], qp[2], gr.p1, gr.p2);
        else rim_images<S>(gr.u_out, gr.L, i, j, qp[0], qp[NP - 1], gr.p1, gr.p2);
      }
      else {
        rim_images_raw<S>(gr.u_out, gr.L, i, j, raw, gr.p1, gr.p2);
        rim_images_raw<RS>(reinterpret_cast<RS *>(gr.r), gr.L, i, j, rraw, gr.p1, gr.p2);
      }
    }
    if (CFL) rate = fmax(rate, cfl_rate<T>(qn, a.p, gr.inv1, gr.inv2, i, j, dl1, dl2, cg));
  }
}

// Output row for slot R of a block: the row 3 behind the leading row, slot (R + 4) mod 7.
template <class S, unsigned M2, int R, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL, bool SC>
__device__ __forceinline__ void emit_row(const typename PairOf<typename Store<S>::C>::type vr[NP], int i, int j,
                                         int iend, const float4 &scv, const float4 &ivv,
                                         const KParams<typename Store<S>::C> &a, const GridRegs<S> &gr,
                                         const Roll<typename Store<S>::C> &s, bool full, bool rim, bool &nan,
                                         typename Store<S>::C &rate, const scheme::Geom<typename Store<S>::C> &cg)
{
  using T = typename Store<S>::C;
  Cell<T, NV> cell;
  typename PairOf<T>::type qc[NP];
  gather_row<T, M2, SC, (R + 4) % CH>(a, gr, s, cell, qc);
  finish_row<S, M2, READ_V, WRITE_V, WRITE_U, CFL, SC>(cell, qc, vr, i, j, iend, scv, ivv, a, gr, full, rim, nan, rate,
                                                       cg);
}

// Shared state of the chunk issue, read and written by thread 0 only.
struct Producer {
  int next_n;    // index of the next chunk to issue
  int c;         // chunk index within the tile (0 = warm-up)
  int done;      // the end-of-queue sentinel was issued
  TileSlot cur;  // the tile of that chunk
};
static_assert(sizeof(TileSlot) == 6 * sizeof(int) && sizeof(Producer) <= 12 * sizeof(int), "shared-memory tail");

// Grid of launch tile t: the last grid whose first tile is <= t (grids are in tile order).
__device__ __forceinline__ int grid_of_tile(const GridDesc *grids, int ngrids, int t)
{
  int lo = 0, hi = ngrids - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (grids[mid].tile0 <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Issues the next chunk of the CTA's sequence into its slot (free by the caller's check).
// `claim` (a register of the issuing thread) holds the queue position of the CTA's next tile:
// it is drawn when the last chunk of the current tile is issued, one chunk before it is
// needed, so the atomic's round trip is off the chunk's critical path.
template <class S, bool READ_V, bool READ_R, int W>
__device__ __forceinline__ void issue_chunk(Producer *ps, unsigned char *smem, uint64_t *full, TileSlot *slots,
                                            const GridDesc *grids, int ngrids, int ntiles, int nb, int tail,
                                            bool reverse, unsigned extra_bytes, int *queue, int &claim)
{
  using G = Geo<S, READ_V, READ_R, W>;
  if (ps->done) return;
  const int n = ps->next_n, s = n % G::NSLOT;
  if (ps->c == 0) {
    int t = claim;
    if (t >= ntiles) t = -1;
    else if (reverse) t = ntiles - 1 - t;
    TileSlot ts{t, 0, 0, 0, 0, 0};
    if (t >= 0) {
      const int g = grid_of_tile(grids, ngrids, t);
      const GridDesc &gd = grids[g];
      const TileGrid tg = tile_grid(gd.L, nb, W, tail);
      int q = t - gd.tile0;                // position of the tile in the grid's processing order
      if (reverse) q = tg.ntiles - 1 - q;
      const Band bd = band_rows(gd.L.n1, nb, tg.bands, q / tg.strips, reverse);
      ts = TileSlot{t, g, bd.i0, bd.iend, (q % tg.strips) * W, bd.nbt};
    }
    ps->cur = ts;
    slots[s] = ts;
  }
  if (ps->cur.tile < 0) {
    mbar_arrive(&full[s]);
    ps->done = 1;
  } else {
    const GridDesc &gd = grids[ps->cur.g];
    const int i0 = ps->cur.i0, j0 = ps->cur.j0, c = ps->c, last = ps->cur.nbt;
    const bool with_v = READ_V && c > 0;
    mbar_arrive_expect_tx(&full[s], G::U_BYTES + (with_v ? G::V_BYTES : 0u) + (READ_R ? G::U_BYTES : 0u) + extra_bytes);
    // box coordinates (group element, cell group, padded row): rows i0 - 4 + 7c ..,
    // columns j0 - 4 .. (padded column j0)
    tma_load_3d(smem + (size_t)s * G::SLOT, &gd.tm_u, &full[s], 0, j0 / G::G, i0 - 4 + CH * c + GT);
    // v of the 7 output rows of block c - 1
    if (with_v)
      tma_load_3d(smem + (size_t)s * G::SLOT + G::V_OFF, &gd.tm_v, &full[s], 0, (j0 + GL - G::VOFF) / G::G,
                  i0 + CH * (c - 1) + GT);
    // 16-bit storage: the rounding residual of the u box's cells
    if (READ_R)
      tma_load_3d(smem + (size_t)s * G::SLOT + G::R_OFF, &gd.tm_r, &full[s], 0, j0 / G::G, i0 - 4 + CH * c + GT);
    if (c == last) claim = atomicAdd(&queue[0], 1);  // the next tile's position, used one chunk later
    ps->c = c == last ? 0 : c + 1;
  }
  ps->next_n = n + 1;
}

// Loads the registers of grid g (every thread; the loads are uniform across the CTA).
template <class S, bool SC>
__device__ __forceinline__ void load_grid(const GridDesc &gd, const KParams<typename Store<S>::C> &a,
                                          GridRegs<S> &gr)
{
  using T = typename Store<S>::C;
  using P = typename PairOf<T>::type;
  gr.L = gd.L;
  gr.u_out = reinterpret_cast<S *>(gd.u_out);
  gr.v = reinterpret_cast<S *>(gd.v);
  gr.status = gd.status;
  gr.p1 = gd.p1;
  gr.p2 = gd.p2;
  const double dt = gd.dt ? *gd.dt : a.dt_dev ? *a.dt_dev : a.dt;
  // (R)(dt * gamma[i]), src/step.cpp:34
  gr.gdt = lit<P>(a.gamma * dt);
  if (SC) {
    gr.s1 = lit<P>(gd.inv1);
    gr.s2 = lit<P>(gd.inv2);
    gr.s11 = lit<P>(gd.inv11);
    gr.s22 = lit<P>(gd.inv22);
    gr.s12 = (T)gd.inv12;
    gr.inv1 = (T)gd.inv1;
    gr.inv2 = (T)gd.inv2;
    gr.delta1 = (T)gd.delta1;
    gr.delta2 = (T)gd.delta2;
  } else {
    gr.inv1 = a.ks.inv1;
    gr.inv2 = a.ks.inv2;
  }
  if constexpr (Store<S>::DEV) {
#pragma unroll
    for (int p = 0; p < NP; ++p) gr.bg[p] = make_float2(gd.dev.bg[2 * p], gd.dev.bg[2 * p + 1]);
    gr.scale = gd.dev.scale;
    gr.inv = gd.dev.inv;
    gr.r = reinterpret_cast<S *>(gd.dev.r_out);
    gr.tiles2 = gd.dev.tiles2;
  }
}

// Deviation storage: decodes the landed 7-row u box (padded rows prow0 .., box column 0 =
// padded column j0) and its residual box into FP32 cells dec ([row][BOXW][NV]): the state
// T = bg + s h - s r / RESID_SCALE, s of the tile of the interior cell each value images, so
// the stencil reads the state with its rounding compensated, not the 16-bit numbers.  Thread
// t decodes column t of every row and, for t below 7 (BOXW - NT), one cell of the columns
// beyond the strip, so the work is even across warps.
// A chunk whose 7 rows lie in one tile row (all but about one chunk in nine) reads each
// column's scales once.
template <class S, int BOXW, int NT>
__device__ __forceinline__ void decode_box(const S *box, const S *rbox, float *dec, int tx, int prow0, int j0,
                                           const GridRegs<S> &gr)
{
  using R = typename Resid<S>::type;
  constexpr int EXTRA = BOXW - NT;  // columns beyond one per thread
  const int n1 = gr.L.n1, n2 = gr.L.n2;
  const int i0 = prow0 - GT;
  const bool rows_inside = i0 >= 0 && i0 + CH <= n1;  // no ghost row in the box
  auto row_tile = [&](int r) { return ((rows_inside ? i0 + r : source_index(i0 + r, n1, gr.p1)) >> 6) * gr.tiles2; };
  auto col_tile = [&](int c) {
    const int j = j0 - GL + c;
    return (j >= 0 && j < n2 ? j : source_index(j, n2, gr.p2)) >> 6;
  };
  auto put = [&](int r, int c, float4 sc) {
    const float2 scp[2] = {make_float2(sc.x, sc.y), make_float2(sc.z, sc.w)};
    float2 h[NP], e[NP];
    load_cell<S>(box + (r * BOXW + c) * NV, h);
    load_cell<R>(reinterpret_cast<const R *>(rbox) + (r * BOXW + c) * NV, e);
#pragma unroll
    for (int p = 0; p < NP; ++p) h[p] = fmac(scp[p] * lit<float2>(-1.0 / RESID_SCALE), e[p], fmac(scp[p], h[p], gr.bg[p]));
    st_cell<float>(dec + (r * BOXW + c) * NV, h);
  };
  {
    const int tj = col_tile(tx);
    if (rows_inside && (i0 >> 6) == ((i0 + CH - 1) >> 6)) {
      const float4 sc = __ldg(gr.scale + (i0 >> 6) * gr.tiles2 + tj);
#pragma unroll
      for (int r = 0; r < CH; ++r) put(r, tx, sc);
    } else {
#pragma unroll
      for (int r = 0; r < CH; ++r) put(r, tx, __ldg(gr.scale + row_tile(r) + tj));
    }
  }
  if (tx < CH * EXTRA) {  // the EXTRA columns right of the strip, one cell per thread
    const int r = tx / EXTRA, c = NT + tx % EXTRA;
    put(r, c, __ldg(gr.scale + row_tile(r) + col_tile(c)));
  }
}

// Publishes a grid's NaN flag and CFL max (CTA-uniform call; warp-level reductions).
template <bool WRITE_U, bool CFL, class T>
__device__ __forceinline__ void flush_grid(Status *st, bool &nan, T &rate)
{
  const int lane = threadIdx.x & 31;
  if (WRITE_U) {
    if (__any_sync(0xffffffffu, nan) && lane == 0) atomicOr(&st->nan, 1u);
  }
  if (CFL) {
    double r = (double)rate;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    if (lane == 0 && r > 0.0) atomicMax(&st->smax, (unsigned long long)__double_as_longlong(r));
  }
  nan = false;
  rate = T(0);
}

// Per-thread position in the launch: the current tile, its grid's registers and the block.
template <class S>
struct TileState {
  using T = typename Store<S>::C;
  GridRegs<S> gr;
  int cur_g = -1;
  int i0 = 0, j0 = 0, b = -1;      // tile origin and block (-1: the warm-up chunk)
  int iend = 0, nbt = 0;           // the tile's rows end before iend; its blocks
  int tj = 0;                      // scale-tile column of the thread's column (16-bit storage)
  bool whole = false, rim = true;  // the tile lies inside the grid / within HALF cells of an edge
  scheme::Geom<T> cg{};            // the scheme's geometry of the thread's column
};

// Enters the tile of a chunk slot (warp-uniform call: flushes the previous grid's NaN flag
// and CFL max with warp collectives when the grid changes).
template <class S, bool WRITE_U, bool CFL, bool SC, int W>
__device__ __forceinline__ void enter_tile(TileState<S> &ts, const GridDesc *grids, const TileSlot &slot,
                                           const KParams<typename Store<S>::C> &a, bool &nan,
                                           typename Store<S>::C &rate)
{
  using T = typename Store<S>::C;
  const int g = slot.g;
  if (g != ts.cur_g) {
    if (ts.cur_g >= 0) flush_grid<WRITE_U, CFL>(ts.gr.status, nan, rate);
    load_grid<S, SC>(grids[g], a, ts.gr);
    ts.cur_g = g;
  }
  ts.i0 = slot.i0;
  ts.iend = slot.iend;
  ts.j0 = slot.j0;
  ts.nbt = slot.nbt;
  ts.b = -1;
  const int j = ts.j0 + (int)threadIdx.x;
  ts.whole = ts.iend - ts.i0 == CH * ts.nbt && ts.j0 + W <= ts.gr.L.n2;
  ts.cg = scheme::column_geom<T>(j, SC ? ts.gr.delta2 : a.ks.delta2);
  ts.rim = ts.i0 < HALF || ts.iend > ts.gr.L.n1 - HALF || ts.j0 < HALF || ts.j0 + W > ts.gr.L.n2 - HALF;
  if constexpr (Store<S>::DEV) ts.tj = min(j, ts.gr.L.n2 - 1) >> 6;
}

// The stencil work of one chunk: the warm-up chunk's 7 rows only feed the window and the
// accumulators; a block's 7 leading rows each complete the output row 3 behind.  base points
// at column j - 3 of the chunk's row 0 (the landed box, or its decoded copy); sbox is the
// chunk's slot (v and r boxes).
template <class S, unsigned M2, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL, bool SC, int W>
__device__ __forceinline__ void stencil_chunk(const typename Store<S>::C *base, const S *sbox, TileState<S> &ts,
                                              const KParams<typename Store<S>::C> &a,
                                              Roll<typename Store<S>::C> &st, bool &nan, typename Store<S>::C &rate)
{
  using T = typename Store<S>::C;
  using P = typename PairOf<T>::type;
  constexpr bool RR = Store<S>::DEV;  // the residual box of the landed u box
  using G = Geo<S, READ_V, RR, W>;
  constexpr int BW = Strip<W>::BW;
  const int tx = threadIdx.x;
  if (ts.b < 0) {
#pragma unroll
    for (int g2 = 0; g2 < ND12; ++g2)
#pragma unroll
      for (int q = 0; q < CH; ++q) st.x[g2][q] = T(0);
    // row i0 - 4 (box row 0) feeds no output row of the tile; rows i0 - 3 .. i0 - 1 feed the
    // window and the mixed derivatives only; rows i0 .. i0 + 2 are output rows
    lead_row<T, M2, 1, BW * NV, false>(base, a, st);
    lead_row<T, M2, 2, BW * NV, false>(base, a, st);
    lead_row<T, M2, 3, BW * NV, false>(base, a, st);
    lead_row<T, M2, 4, BW * NV>(base, a, st);
    lead_row<T, M2, 5, BW * NV>(base, a, st);
    lead_row<T, M2, 6, BW * NV>(base, a, st);
  } else {
    const int ib = ts.i0 + CH * ts.b, j = ts.j0 + tx;
    const S *sv = sbox + G::V_OFF / sizeof(S);
    // 16-bit storage: the scales of the output rows' tile, loaded once per chunk and again at
    // the row where the chunk crosses into the next tile row (CTA-uniform)
    float4 scv = make_float4(0.f, 0.f, 0.f, 0.f), ivv = scv;
    int next_tile_row = 1 << 30;
    if constexpr (Store<S>::DEV && WRITE_U) {
      const int r0 = min(ib, ts.gr.L.n1 - 1) >> 6;
      scv = __ldg(ts.gr.scale + r0 * ts.gr.tiles2 + ts.tj);
      ivv = __ldg(ts.gr.inv + r0 * ts.gr.tiles2 + ts.tj);
      if (((r0 + 1) << 6) < ts.gr.L.n1) next_tile_row = (r0 + 1) << 6;
    }
#define FG2_ROW(R)                                                                                         \
  {                                                                                                        \
    P vrow[NP];                                                                                            \
    if (READ_V) load_cell<S>(sv + (R * G::VBW + tx + G::VOFF) * NV, vrow);                                 \
    if (Store<S>::DEV && WRITE_U && ib + R == next_tile_row) {                                             \
      scv = __ldg(ts.gr.scale + (next_tile_row >> 6) * ts.gr.tiles2 + ts.tj);                              \
      ivv = __ldg(ts.gr.inv + (next_tile_row >> 6) * ts.gr.tiles2 + ts.tj);                                \
    }                                                                                                      \
    lead_row<T, M2, R, BW * NV>(base, a, st);                                                              \
    emit_row<S, M2, R, READ_V, WRITE_V, WRITE_U, CFL, SC>(vrow, ib + R, j, ts.iend, scv, ivv, a, ts.gr,       \
                                                          st, ts.whole, ts.rim, nan, rate, ts.cg);         \
  }
    if constexpr (rolled_rows()) {
#pragma unroll 1
      for (int R = 0; R < CH; ++R) {
        P vrow[NP];
        if (READ_V) load_cell<S>(sv + (R * G::VBW + tx + G::VOFF) * NV, vrow);
        if (Store<S>::DEV && WRITE_U && ib + R == next_tile_row) {
          scv = __ldg(ts.gr.scale + (next_tile_row >> 6) * ts.gr.tiles2 + ts.tj);
          ivv = __ldg(ts.gr.inv + (next_tile_row >> 6) * ts.gr.tiles2 + ts.tj);
        }
        Cell<T, NV> cell;
        P qc[NP];
        switch (R) {
#define FG2_FRONT(Q)                                                                                       \
  case Q:                                                                                                  \
    lead_row<T, M2, Q, BW * NV>(base, a, st);                                                              \
    gather_row<T, M2, SC, (Q + 4) % CH>(a, ts.gr, st, cell, qc);                                           \
    break;
          FG2_FRONT(0) FG2_FRONT(1) FG2_FRONT(2) FG2_FRONT(3) FG2_FRONT(4) FG2_FRONT(5) FG2_FRONT(6)
#undef FG2_FRONT
        }
        finish_row<S, M2, READ_V, WRITE_V, WRITE_U, CFL, SC>(cell, qc, vrow, ib + R, j, ts.iend, scv, ivv, a,
                                                             ts.gr, ts.whole, ts.rim, nan, rate, ts.cg);
      }
    } else {
      FG2_ROW(0) FG2_ROW(1) FG2_ROW(2) FG2_ROW(3) FG2_ROW(4) FG2_ROW(5) FG2_ROW(6)
    }
#undef FG2_ROW
  }
}

// Resident CTAs per SM the register budget is cut for (128-column strips; twice that for 64):
// 4 for three-field FP32 cells (at most 128 registers, no spills), 3 for four fields and for
// 16-bit storage, 2 for six-field FP32 cells; FP64 kernels are not bounded below one.
template <class S, int W>
__host__ __device__ constexpr int min_blocks()
{
  return sizeof(typename Store<S>::C) != 4 ? 128 / W
         : Store<S>::DEV                    ? 3 * (128 / W)
                                            : (NV > 4 ? 2 : NV == 3 ? 4 : 3) * (128 / W);
}

// Chunk loop.  Every thread waits (bounded) for its chunk itself; the one CTA barrier per
// chunk both agrees on a timeout (__syncthreads_or) and hands the consumed slot back to the
// issuing thread.  A thread whose wait ran out skips the chunk's work (its bookkeeping is
// not yet visible to it), and the CTA leaves together at that barrier.
//   FP32 / FP64 storage: wait for chunk n, stencil it from its slot, barrier, refill the slot.
//   16-bit storage: chunk n was decoded into dec[n & 1] during the previous chunk; stencil it,
//   wait for chunk n + 1 and decode it into the other copy, barrier, refill chunk n's slot.
template <class S, unsigned M2, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL, bool SC, int W>
__global__ void __launch_bounds__(W, min_blocks<S, W>()) substage_kernel(const GridDesc *__restrict__ grids, int ngrids, int ntiles,
                                                         const KParams<typename Store<S>::C> a, int *queue)
{
  using T = typename Store<S>::C;
  constexpr bool DEV = Store<S>::DEV;
  constexpr bool RR = DEV;  // 16-bit storage: the residual of every u box is loaded too
  using G = Geo<S, READ_V, RR, W>;
  constexpr int BW = Strip<W>::BW, NT = Strip<W>::NT;
  constexpr int NS = G::NSLOT;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + G::BAR_OFF);
  TileSlot *slots = reinterpret_cast<TileSlot *>(full + NS);
  Producer *ps = reinterpret_cast<Producer *>(slots + NS);

  int claim = 0;  // issuing thread: queue position of the CTA's next tile
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
    ps->next_n = 0;
    ps->c = 0;
    ps->done = 0;
    ps->cur = TileSlot{-1, 0, 0, 0, 0, 0};
    claim = atomicAdd(&queue[0], 1);
    for (int s = 0; s < NS; ++s)
      issue_chunk<S, READ_V, RR, W>(ps, smem, full, slots, grids, ngrids, ntiles, a.nb, a.tail, a.reverse != 0,
                                    a.wait_test_bytes, queue, claim);
  }
  __syncthreads();

  bool nan = false;
  T rate = T(0);
  const int tx = threadIdx.x;  // column within the strip
  TileState<S> ts;
  Roll<T> st;
  float *dec = reinterpret_cast<float *>(smem + G::DEC_OFF);
  auto slot = [&](int n) { return reinterpret_cast<const S *>(smem + (size_t)(n % NS) * G::SLOT); };
  auto parity = [&](int n) { return (uint32_t)((n / NS) & 1); };
  // padded row of the u box's row 0 for the thread's current tile and block
  auto box_row = [&]() { return ts.b < 0 ? ts.i0 - 4 + GT : ts.i0 + CH * ts.b + 3 + GT; };
  // the tile state for chunk n: a new tile after the last block of the previous one (tile < 0:
  // the end of the queue); returns false at the end
  auto advance = [&](int n) {
    if (ts.cur_g >= 0 && ts.b < ts.nbt - 1) {  // the next block of the current tile
      ++ts.b;
      return true;
    }
    const TileSlot &slot = slots[n % NS];
    if (slot.tile < 0) return false;
    enter_tile<S, WRITE_U, CFL, SC, W>(ts, grids, slot, a, nan, rate);
    return true;
  };
  bool failed = false;

  if constexpr (!DEV) {
    for (int n = 0;; ++n) {
      const bool landed = mbar_wait_bounded(&full[n % NS], parity(n), WAIT_NS);
      bool live = false;
      if (__all_sync(FULL, landed)) {
        live = advance(n);
        if (live)
          stencil_chunk<S, M2, READ_V, WRITE_V, WRITE_U, CFL, SC, W>(reinterpret_cast<const T *>(slot(n)) + (tx + GL - 3) * NV,
                                                                     slot(n), ts, a, st, nan, rate);
      }
      if (__syncthreads_or(!landed)) {
        failed = true;
        break;
      }
      if (!live) break;  // the end of the queue (the same chunk for every thread)
      if (threadIdx.x == 0)
        issue_chunk<S, READ_V, RR, W>(ps, smem, full, slots, grids, ngrids, ntiles, a.nb, a.tail, a.reverse != 0,
                                      a.wait_test_bytes, queue, claim);  // refill chunk n's slot
    }
  } else {
    // chunk 0: wait, decode
    bool landed = mbar_wait_bounded(&full[0], parity(0), WAIT_NS);
    bool live = false;
    if (__all_sync(FULL, landed)) {
      live = advance(0);
      if (live) decode_box<S, BW, NT>(slot(0), slot(0) + G::R_OFF / sizeof(S), dec, tx, box_row(), ts.j0, ts.gr);
    }
    failed = __syncthreads_or(!landed);
    for (int n = 0; live && !failed; ++n) {
      stencil_chunk<S, M2, READ_V, WRITE_V, WRITE_U, CFL, SC, W>(
          dec + (size_t)(n & 1) * (G::DEC_ONE / sizeof(float)) + (tx + GL - 3) * NV, slot(n), ts, a, st, nan, rate);
      landed = mbar_wait_bounded(&full[(n + 1) % NS], parity(n + 1), WAIT_NS);
      live = false;
      if (__all_sync(FULL, landed)) {
        live = advance(n + 1);
        if (live)
          decode_box<S, BW, NT>(slot(n + 1), slot(n + 1) + G::R_OFF / sizeof(S),
                                dec + (size_t)((n + 1) & 1) * (G::DEC_ONE / sizeof(float)), tx, box_row(),
                                ts.j0, ts.gr);
      }
      failed = __syncthreads_or(!landed);
      if (!failed && live && threadIdx.x == 0)
        issue_chunk<S, READ_V, RR, W>(ps, smem, full, slots, grids, ngrids, ntiles, a.nb, a.tail, a.reverse != 0,
                                      a.wait_test_bytes, queue, claim);  // refill chunk n's slot
    }
  }
  if (failed && threadIdx.x == 0) atomicOr(&a.status->error, ERR_TMA_TIMEOUT);

  if (ts.cur_g >= 0) flush_grid<WRITE_U, CFL>(ts.gr.status, nan, rate);

  __syncthreads();
  if (threadIdx.x == 0) {
    // after an error, let every load this CTA issued land before the CTA exits
    const int issued = ps->next_n;
    for (int s = 0; s < NS && s < issued; ++s) {
      const int last = s + ((issued - 1 - s) / NS) * NS;  // last chunk issued into slot s
      mbar_wait_bounded(&full[s], (uint32_t)((last / NS) & 1), WAIT_NS);
    }
    // the last CTA to finish resets the queue for the next launch
    __threadfence();
    if (atomicAdd(&queue[1], 1) == (int)gridDim.x - 1) {
      queue[0] = 0;
      queue[1] = 0;
      __threadfence();
    }
  }
}

}  // namespace sub
