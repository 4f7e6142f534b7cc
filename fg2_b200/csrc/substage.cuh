// fg2_b200/csrc/substage.cuh -- the fused RK3 substage kernel (included inside namespace fg2
// by kernels.cu, once per scheme).
//
// Work decomposition.  A tile is a strip of SW = 128 interior columns by TH = 35 rows of one
// simulation.  A persistent grid of CTAs drains a tile queue (an atomic counter that the
// last CTA to finish resets, so a launch needs no host-side reset and replays from a CUDA
// graph).  Each CTA has NCW = 2 warps; a thread owns the two columns t and t + 64 of the
// strip and evaluates both cells with one stream of pair instructions (packed FP32x2 on
// sm_100: add/mul/fma .f32x2).
//
// Data movement.  u streams through a ring of NSLOT shared-memory slots by TMA
// (cp.async.bulk.tensor.3d, no multicast): chunk 0 of a tile is the 7-row warm-up box
// u[i0-4 .. i0+3) x [j0-4, j0+132) (all fields), chunk b+1 the 7 leading rows u[i0+3+7b ..]
// of output block b; a box lands as [row][field][column].  v never enters shared memory:
// when a block's u chunk is issued, the same 7 rows of v are prefetched into L2
// (cp.async.bulk.prefetch.tensor), and each thread reads its v values with coalesced loads
// issued at the top of the row that updates them.  There is no producer warp: the warp that
// releases a slot last refills it.  Full mbarriers carry the TMA completion, empty
// mbarriers the releases; every wait is bounded (%globaltimer) and a timeout raises an
// error bit in the status block.
//
// Stencil.  Each thread walks its columns down the tile.  At every leading row L it loads
// the 7 values u(L, j-3..j+3) of each field from shared memory and computes the axis-2
// (contiguous) derivatives D2 and D22 of row L, pushes u(L, j) into a 7-row register window
// (the axis-1 stencil of row L-3 then needs no further loads), and feeds the mixed
// derivative by streaming accumulators: with delta_k(r) = u(r, j+k) - u(r, j-k),
// D12(r) = sum_k m_k (delta_k(r+k) - delta_k(r-k)), so delta_k(L) is added to row L-k and
// subtracted from row L+k (src/deriv.h:60-62 regrouped).  The output row L-3 then has all its
// derivatives in registers; the scheme's eqns() gives F, and the epilogue applies
// v <- F + beta v, u' <- u + gamma dt v (src/kick.cu:53, src/drift.cu:29), stores u' with
// its ghost images and v, flags NaNs and, on the last stage, folds the CFL rate into a max.
// Register slots are indexed by row mod 7 and the row loop is unrolled by 7, so the window
// never moves.
#pragma once

namespace sub {

constexpr int SW = 128;            // interior columns per tile (strip width)
constexpr int HW = SW / 2;         // distance between the two columns of a thread
constexpr int BW = SW + 2 * GL;    // TMA box width of u (halo 4 + 4; the stencil uses 3)
constexpr int CH = 7;              // rows per chunk = register window period
constexpr int NB = 5;              // output blocks per tile
constexpr int TH = NB * CH;        // output rows per tile
constexpr int NCW = 2;             // warps per CTA
constexpr int NT = NCW * 32;       // threads per CTA
static_assert(NT == HW, "one thread per column pair");

#ifndef FG2_NSLOT_F32
#define FG2_NSLOT_F32 2
#endif

template <class T>
struct Geo {
  static constexpr int NSLOT = sizeof(T) == 8 ? 2 : FG2_NSLOT_F32;
  static constexpr uint32_t U_BYTES = (uint32_t)(BW * CH * NV * sizeof(T));
  static constexpr uint32_t SLOT = (U_BYTES + 127) / 128 * 128;  // TMA destinations on 128 B
  static constexpr size_t BAR_OFF = (size_t)NSLOT * SLOT;
  // tail: full[NSLOT], empty[NSLOT] (mbarriers), rel[NSLOT], tile_of[NSLOT], producer state
  static constexpr size_t SMEM = BAR_OFF + 2 * NSLOT * sizeof(uint64_t) + 2 * NSLOT * sizeof(int) + 4 * sizeof(int) + 64;
  static_assert(SLOT % 128 == 0, "TMA shared-memory destinations must be 128-byte aligned");
  static_assert(BW <= 256 && CH <= 256, "TMA box dimensions");
  static_assert((BW * sizeof(T)) % 16 == 0 && (SW * sizeof(T)) % 16 == 0, "TMA rows must be 16-byte multiples");
};

// Tile t of a single grid: strip fastest, so horizontally adjacent tiles run together and
// share their halo columns through L2.
struct TileGrid {
  int strips, rows, ntiles;
};

__host__ __device__ inline TileGrid tile_grid(const Layout &L)
{
  TileGrid g;
  g.strips = (L.n2 + SW - 1) / SW;
  g.rows = (L.n1 + TH - 1) / TH;
  g.ntiles = g.strips * g.rows;
  return g;
}

// Per-thread rolling state.  Slot index = leading-row index mod 7.
template <class C>
struct Roll {
  C w[NV][CH];     // u(row, j), rows L-6 .. L
  C h2[NV][CH];    // D2 of each row
  C h22[NV][CH];   // D22 of each row
  C x[2][CH];      // D12 accumulators of u1, u2
};

__device__ __forceinline__ bool bounded_wait(uint64_t *bar, uint32_t parity, Status *st)
{
  if (mbar_wait_bounded(bar, parity, WAIT_NS)) return true;
  atomicOr(&st->error, ERR_TMA_TIMEOUT);
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Leading-row work for register slot R: loads row R of the chunk for both columns.
template <class T, unsigned M2, int R>
__device__ __forceinline__ void lead_row(const T *su, int tx, const Coef<typename PairOf<T>::type> &k,
                                         Roll<typename PairOf<T>::type> &s)
{
  using C = typename PairOf<T>::type;
  using PO = PairOf<T>;
  const T *p0 = su + R * (NV * BW) + tx + GL;
#pragma unroll
  for (int f = 0; f < NV; ++f) {
    const T *p = p0 + f * BW;
    const C c = PO::make(p[0], p[HW]);
    const C l1 = PO::make(p[-1], p[HW - 1]), r1 = PO::make(p[1], p[HW + 1]);
    const C l2 = PO::make(p[-2], p[HW - 2]), r2 = PO::make(p[2], p[HW + 2]);
    const C l3 = PO::make(p[-3], p[HW - 3]), r3 = PO::make(p[3], p[HW + 3]);
    s.w[f][R] = c;
    const C d1 = r1 - l1, d2 = r2 - l2, d3 = r3 - l3;
    s.h2[f][R] = fmac(k.a2[0], d1, fmac(k.a2[1], d2, k.a2[2] * d3));
    if (M2 & (1u << f))
      s.h22[f][R] = fmac(k.b2[0], c, fmac(k.b2[1], r1 + l1, fmac(k.b2[2], r2 + l2, k.b2[3] * (r3 + l3))));
    if (scheme::D12_FIELDS & (1u << f)) {
      const int g = f == scheme::U1 ? 0 : 1;
      // rows L+k get -m_k delta_k(L) (mn = -m), rows L-k get +m_k delta_k(L); row L-3 is
      // then complete.  The first contribution to row L+3 initialises its accumulator.
      s.x[g][(R + 3) % CH] = k.mn[2] * d3;
      s.x[g][(R + 2) % CH] = fmac(k.mn[1], d2, s.x[g][(R + 2) % CH]);
      s.x[g][(R + 1) % CH] = fmac(k.mn[0], d1, s.x[g][(R + 1) % CH]);
      s.x[g][(R + 6) % CH] = fmac(k.m[0], d1, s.x[g][(R + 6) % CH]);
      s.x[g][(R + 5) % CH] = fmac(k.m[1], d2, s.x[g][(R + 5) % CH]);
      s.x[g][(R + 4) % CH] = fmac(k.m[2], d3, s.x[g][(R + 4) % CH]);
    }
  }
}

// v values of output row i for both columns (coalesced loads, issued a row ahead of use).
template <class T, bool READ_V>
__device__ __forceinline__ void load_v(const T *v, const Layout &L, int i, int j,
                                       typename PairOf<T>::type vr[NV])
{
  if (!READ_V) return;
  const bool row_ok = i < L.n1, okx = row_ok && j < L.n2, oky = row_ok && j + HW < L.n2;
  const T *p = v + L.at(0, i, j);
#pragma unroll
  for (int f = 0; f < NV; ++f) {
    vr[f].x = okx ? __ldcs(p + f * L.FS) : T(0);
    vr[f].y = oky ? __ldcs(p + f * L.FS + HW) : T(0);
  }
}

// Output row for slot R of a block: the row 3 behind the leading row, slot (R + 4) mod 7.
template <class T, unsigned M2, int R, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL>
__device__ __forceinline__ void emit_row(const typename PairOf<T>::type vr[NV], int i, int j, const KParams<T> &a,
                                         const Layout &L, typename PairOf<T>::type gdt, T *u_out, T *v,
                                         const Roll<typename PairOf<T>::type> &s, bool &nan, T &rate)
{
  using C = typename PairOf<T>::type;
  constexpr int S0 = (R + 4) % CH;
  const C zero = lit<C>(0.0);
  Cell<C, NV> cell;
#pragma unroll
  for (int f = 0; f < NV; ++f) {
    const C c = s.w[f][S0];
    const C p1 = s.w[f][(S0 + 1) % CH], n1 = s.w[f][(S0 + 6) % CH];
    const C p2 = s.w[f][(S0 + 2) % CH], n2 = s.w[f][(S0 + 5) % CH];
    const C p3 = s.w[f][(S0 + 3) % CH], n3 = s.w[f][(S0 + 4) % CH];
    cell.q[f] = c;
    cell.d1[f] = fmac(a.k.a1[0], p1 - n1, fmac(a.k.a1[1], p2 - n2, a.k.a1[2] * (p3 - n3)));
    if (M2 & (1u << f)) {
      cell.d11[f] = fmac(a.k.b1[0], c, fmac(a.k.b1[1], p1 + n1, fmac(a.k.b1[2], p2 + n2, a.k.b1[3] * (p3 + n3))));
      cell.d22[f] = s.h22[f][S0];
    } else {
      cell.d11[f] = zero;
      cell.d22[f] = zero;
    }
    cell.d2[f] = s.h2[f][S0];
    cell.d12[f] = (scheme::D12_FIELDS & (1u << f)) ? s.x[f == scheme::U1 ? 0 : 1][S0] : zero;
  }
  if (i >= L.n1) return;
  C r[NV];
  scheme::eqns<M2>(cell, a.p, i, j, r, a.k.delta1);
  const bool okx = j < L.n2, oky = j + HW < L.n2;
  const long long o = L.at(0, i, j);
  C qn[NV];
#pragma unroll
  for (int f = 0; f < NV; ++f) {
    C vn = r[f];
    if (READ_V) vn = fmac(a.beta, vr[f], vn);
    if (WRITE_V) {
      if (okx) v[o + f * L.FS] = vn.x;
      if (oky) v[o + f * L.FS + HW] = vn.y;
    }
    qn[f] = fmac(gdt, vn, cell.q[f]);
    nan |= (okx && qn[f].x != qn[f].x) || (oky && qn[f].y != qn[f].y);
  }
  if (WRITE_U) {
    T qx[NV], qy[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) {
      qx[f] = qn[f].x;
      qy[f] = qn[f].y;
    }
    if (okx) store_images<T, T>(u_out, L, i, j, qx, a.p1, a.p2);
    if (oky) store_images<T, T>(u_out, L, i, j + HW, qy, a.p1, a.p2);
  }
  if (CFL) {
    const C cr = cfl_rate<C>(qn, a.p, a.k);
    if (okx) rate = fmax(rate, cr.x);
    if (oky) rate = fmax(rate, cr.y);
  }
}

// Shared state of the refill duty, handed from warp to warp through shared memory.
struct Producer {
  int next_n;  // index of the next chunk to issue
  int tile;    // tile of that chunk
  int c;       // chunk index within the tile (0 = warm-up)
  int done;    // the end-of-queue sentinel was issued
};

// Issues the next chunk of the CTA's sequence into its slot (free by the caller's check).
template <class T, bool READ_V>
__device__ __forceinline__ void issue_chunk(Producer *ps, unsigned char *smem, uint64_t *full, int *tile_of,
                                            const CUtensorMap *tm_u, const CUtensorMap *tm_v, int *queue,
                                            const TileGrid &tg)
{
  using G = Geo<T>;
  if (ps->done) return;
  const int n = ps->next_n, s = n % G::NSLOT;
  if (ps->c == 0) {
    int t = atomicAdd(&queue[0], 1);
    if (t >= tg.ntiles) t = -1;
    ps->tile = t;
    tile_of[s] = t;
  }
  if (ps->tile < 0) {
    mbar_arrive(&full[s]);
    ps->done = 1;
  } else {
    const int i0 = (ps->tile / tg.strips) * TH, j0 = (ps->tile % tg.strips) * SW;
    const int c = ps->c;
    mbar_arrive_expect_tx(&full[s], G::U_BYTES);
    // box coordinates (padded column, field, padded row): rows i0 - 4 + 7c .., columns j0 - 4 ..
    tma_load_3d(smem + (size_t)s * G::SLOT, tm_u, &full[s], j0, 0, i0 - 4 + CH * c + GT);
    // the v rows this chunk's output block updates, into L2 ahead of the threads' loads
    if (READ_V && c > 0) tma_prefetch_l2_3d(tm_v, j0 + GL, 0, i0 + CH * (c - 1) + GT);
    ps->c = c == NB ? 0 : c + 1;
  }
  ps->next_n = n + 1;
}

#ifndef FG2_MIN_CTAS
#define FG2_MIN_CTAS 1
#endif

template <class T, unsigned M2, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL>
__global__ void __launch_bounds__(NT, FG2_MIN_CTAS) substage_kernel(const __grid_constant__ CUtensorMap tm_u,
                                                      const __grid_constant__ CUtensorMap tm_v,
                                                      T *__restrict__ u_out, T *__restrict__ v, const Layout L,
                                                      const KParams<T> a, int *queue)
{
  using C = typename PairOf<T>::type;
  using G = Geo<T>;
  constexpr int NS = G::NSLOT;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + G::BAR_OFF);
  uint64_t *empty = full + NS;
  int *rel = reinterpret_cast<int *>(empty + NS);
  int *tile_of = rel + NS;
  Producer *ps = reinterpret_cast<Producer *>(tile_of + NS);
  const int lane = threadIdx.x & 31;
  const TileGrid tg = tile_grid(L);

  if (threadIdx.x == 0) {
    prefetch_tmap(&tm_u);
    if (READ_V) prefetch_tmap(&tm_v);
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
      rel[s] = 0;
    }
    fence_mbar_init();
    ps->next_n = 0;
    ps->tile = -1;
    ps->c = 0;
    ps->done = 0;
    for (int s = 0; s < NS; ++s) issue_chunk<T, READ_V>(ps, smem, full, tile_of, &tm_u, &tm_v, queue, tg);
  }
  __syncthreads();

  bool nan = false;
  T rate = T(0);
  const int tx = threadIdx.x;  // first column within the strip; the second is tx + 64
  const C gdt = lit<C>(a.gamma * (a.dt_dev ? *a.dt_dev : a.dt));  // (R)(dt * gamma[i]), src/step.cpp:34
  Roll<C> st;
  int n = 0;       // chunks consumed
  bool ok = true;

  // Release slot s of chunk n; the warp that releases last refills it.
  auto release = [&](int s) {
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&empty[s]);
      if (atomicAdd(&rel[s], 1) == NCW - 1) {
        rel[s] = 0;
        if (mbar_wait_bounded(&empty[s], (uint32_t)((n / NS) & 1), WAIT_NS))
          issue_chunk<T, READ_V>(ps, smem, full, tile_of, &tm_u, &tm_v, queue, tg);
        else
          atomicOr(&a.status->error, ERR_TMA_TIMEOUT);
      }
    }
  };

  while (ok) {
    int s = n % NS;
    if (!bounded_wait(&full[s], (uint32_t)((n / NS) & 1), a.status)) break;
    const int tile = tile_of[s];
    if (tile < 0) break;
    const int i0 = (tile / tg.strips) * TH;
    const int j = (tile % tg.strips) * SW + tx;
#pragma unroll
    for (int g = 0; g < 2; ++g)
#pragma unroll
      for (int q = 0; q < CH; ++q) st.x[g][q] = lit<C>(0.0);
    {  // warm-up chunk: rows i0-4 .. i0+2 only feed the window and the accumulators
      const T *su = reinterpret_cast<const T *>(smem + (size_t)s * G::SLOT);
      lead_row<T, M2, 0>(su, tx, a.k, st);
      lead_row<T, M2, 1>(su, tx, a.k, st);
      lead_row<T, M2, 2>(su, tx, a.k, st);
      lead_row<T, M2, 3>(su, tx, a.k, st);
      lead_row<T, M2, 4>(su, tx, a.k, st);
      lead_row<T, M2, 5>(su, tx, a.k, st);
      lead_row<T, M2, 6>(su, tx, a.k, st);
    }
    release(s);
    ++n;
    for (int b = 0; b < NB; ++b, ++n) {
      s = n % NS;
      if (!bounded_wait(&full[s], (uint32_t)((n / NS) & 1), a.status)) { ok = false; break; }
      const T *su = reinterpret_cast<const T *>(smem + (size_t)s * G::SLOT);
      const int ib = i0 + CH * b;
      C vr[NV];
#define FG2_ROW(R)                                                                                        \
  load_v<T, READ_V>(v, L, ib + R, j, vr);                                                                 \
  lead_row<T, M2, R>(su, tx, a.k, st);                                                                    \
  emit_row<T, M2, R, READ_V, WRITE_V, WRITE_U, CFL>(vr, ib + R, j, a, L, gdt, u_out, v, st, nan, rate);
      FG2_ROW(0) FG2_ROW(1) FG2_ROW(2) FG2_ROW(3) FG2_ROW(4) FG2_ROW(5) FG2_ROW(6)
#undef FG2_ROW
      release(s);
    }
  }

  if (WRITE_U) {
    if (__any_sync(0xffffffffu, nan) && lane == 0) atomicOr(&a.status->nan, 1u);
  }
  if (CFL) {
    double r = (double)rate;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    if (lane == 0 && r > 0.0) atomicMax(&a.status->smax, (unsigned long long)__double_as_longlong(r));
  }

  __syncthreads();
  if (threadIdx.x == 0) {
    // after an error, let every copy this CTA issued land before the CTA exits
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
