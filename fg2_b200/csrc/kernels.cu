// fg2_b200/csrc/kernels.cu -- device kernels of the B200 time step, compiled once per
// scheme (-I schemes/<name>), for sm_100a.
//
// The hot kernel is the fused RK3 substage (substage_kernel): one pass per stage that
//   1. stages a (TH + 6) x (TW + 8) x NVAR tile of u, halo included, from HBM into shared
//      memory with one TMA box load (cp.async.bulk.tensor.3d, completion on an mbarrier);
//   2. evaluates the 6th-order derivatives and the scheme's right-hand side per cell
//      (src/kick.cu:59-106 + src/deriv.h:39-63 + <scheme>/eqns.cuh);
//   3. applies the low-storage RK3 register update in the epilogue,
//      v <- F(u) + beta v (src/kick.cu:53) and u' <- u + gamma dt v (src/drift.cu:29),
//      flags NaNs (src/drift.cu:30), and writes the ghost images of the edge cells for the
//      next stage (the reference's separate bcond pass, src/bcond.cu:77-86);
//   4. optionally folds the CFL signal rate of u' into a running max (getdt).
// u is ping-ponged between two arrays so no stage overwrites a halo another tile reads.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdio>

#include "fg2b.h"
#include "kernels.h"
#include "ptx.cuh"

#include <state.h>
#include <eqns.cuh>
#include <bcond.cuh>
#include <Euler.cuh>

namespace fg2 {

constexpr int NV = scheme::NVAR;
constexpr uint64_t WAIT_NS = 2000000000ull;  // bound of every in-kernel wait (2 s)

// ---------------------------------------------------------------------------------------
// Parameters rounded to the compute type C.
template <class C>
struct KParams {
  Coef<C> k;
  Para<C> p;
  C beta;
  double gamma, dt;
  const double *dt_dev;
  int p1, p2;
  Status *status;
};

template <class C>
static KParams<C> make_params(const StageArgs &a)
{
  KParams<C> kp;
  // Delta = l / n is rounded to the state precision (src/config.cpp:39); the weights are
  // divided by it in double and rounded once.
  const double d1 = a.delta1, d2 = a.delta2;
  const double w1[3] = {45. / 60., -9. / 60., 1. / 60.};
  const double w2[4] = {-490. / 180., 270. / 180., -27. / 180., 2. / 180.};
  const double wm[3] = {270. / 720., -27. / 720., 2. / 720.};
  for (int q = 0; q < 3; ++q) {
    kp.k.a1[q] = (C)(w1[q] / d1);
    kp.k.a2[q] = (C)(w1[q] / d2);
    kp.k.m[q] = (C)(wm[q] / (d1 * d2));
  }
  for (int q = 0; q < 4; ++q) {
    kp.k.b1[q] = (C)(w2[q] / (d1 * d1));
    kp.k.b2[q] = (C)(w2[q] / (d2 * d2));
  }
  kp.k.delta1 = (C)d1;
  kp.k.delta2 = (C)d2;
  kp.k.inv1 = (C)(1.0 / d1);
  kp.k.inv2 = (C)(1.0 / d2);
  for (int q = 0; q < 8; ++q) kp.p.v[q] = (C)(a.para ? a.para[q] : 0.0);
  kp.beta = (C)a.beta;
  kp.gamma = a.gamma;
  kp.dt = a.dt;
  kp.dt_dev = a.dt_dev;
  kp.p1 = a.p1;
  kp.p2 = a.p2;
  kp.status = a.status;
  return kp;
}

// ---------------------------------------------------------------------------------------
// Ghost images of an interior cell (i, j): the cell itself plus, near an edge, the ghost
// positions the reference's bcond would copy it to (periodic wrap, zero-gradient mirror
// along axis 1, reflective mirror with sign flip along axis 2).
struct Images {
  int rows[3], cols[3];
  bool flip[3];
  int nr, nc;
};

__device__ __forceinline__ Images ghost_images(int i, int j, int n1, int n2, int p1, int p2)
{
  Images g;
  g.nr = 0;
  g.nc = 0;
  g.rows[g.nr++] = i;
  if (i < HALF) g.rows[g.nr++] = p1 ? i + n1 : -1 - i;
  if (i >= n1 - HALF) g.rows[g.nr++] = p1 ? i - n1 : 2 * n1 - 1 - i;
  g.cols[g.nc] = j;
  g.flip[g.nc++] = false;
  if (j < HALF) { g.cols[g.nc] = p2 ? j + n2 : -1 - j; g.flip[g.nc++] = !p2; }
  if (j >= n2 - HALF) { g.cols[g.nc] = p2 ? j - n2 : 2 * n2 - 1 - j; g.flip[g.nc++] = !p2; }
  return g;
}

template <class T, class C>
__device__ __forceinline__ void store_images(T *u, const Layout &L, int i, int j, const C q[NV], int p1, int p2)
{
  const bool edge = i < HALF || i >= L.n1 - HALF || j < HALF || j >= L.n2 - HALF;
  if (!edge) {
#pragma unroll
    for (int f = 0; f < NV; ++f) u[L.at(f, i, j)] = (T)q[f];
    return;
  }
  const Images g = ghost_images(i, j, L.n1, L.n2, p1, p2);
  for (int a = 0; a < g.nr; ++a)
    for (int b = 0; b < g.nc; ++b)
#pragma unroll
      for (int f = 0; f < NV; ++f) {
        const C x = g.flip[b] ? C(scheme::reflect_sign(f)) * q[f] : q[f];
        u[L.at(f, g.rows[a], g.cols[b])] = (T)x;
      }
}

template <class C>
__device__ __forceinline__ C cfl_rate(const C q[NV], const Para<C> &p, const Coef<C> &k)
{
  const C cs = scheme::sound_speed(q, p);
  return (fabs(q[scheme::U1]) + cs) * k.inv1 + (fabs(q[scheme::U2]) + cs) * k.inv2;
}

// ---------------------------------------------------------------------------------------
// Fused substage.  One CTA per TW x TH tile; NT threads, TW columns x (NT / TW) row groups.
template <class T, int TW, int TH, int NT>
struct SubstageCfg {
  static constexpr int BW = TW + 2 * GL;    // box width (columns j0-4 .. j0+TW+3)
  static constexpr int BH = TH + 2 * HALF;  // box height (rows i0-3 .. i0+TH+2)
  static constexpr int PLANE = BW * BH;
  static constexpr size_t TILE_BYTES = (size_t)NV * PLANE * sizeof(T);
  static constexpr size_t SMEM = TILE_BYTES + 16;
  static_assert(BW <= 256 && BH <= 256, "TMA box dimensions are limited to 256");
  static_assert((BW * sizeof(T)) % 16 == 0, "TMA box rows must be a multiple of 16 bytes");
  static_assert(TILE_BYTES % 8 == 0, "mbarrier alignment");
};

template <class T, int TW, int TH, int NT, bool READ_V, bool WRITE_V, bool WRITE_U, bool CFL>
__global__ void __launch_bounds__(NT) substage_kernel(const __grid_constant__ CUtensorMap tm, T *__restrict__ u_out,
                                                      T *__restrict__ v, const Layout L, const KParams<T> a)
{
  using C = T;
  using Cfg = SubstageCfg<T, TW, TH, NT>;
  constexpr int BW = Cfg::BW, PLANE = Cfg::PLANE;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *tile = reinterpret_cast<T *>(smem_raw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + Cfg::TILE_BYTES);

  const int i0 = blockIdx.y * TH, j0 = blockIdx.x * TW;
  if (threadIdx.x == 0) {
    prefetch_tmap(&tm);
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(bar, (uint32_t)Cfg::TILE_BYTES);
    // padded coordinates: column j0 - 4 + GL = j0, row i0 - 3 + GT = i0, all fields
    tma_load_3d(tile, &tm, bar, j0, i0, 0);
  }
  // every thread waits (bounded); the CTA then agrees on the outcome so that all threads
  // take the same path through the warp-collective epilogue
  const bool landed = mbar_wait_bounded(bar, 0, WAIT_NS);
  if (__syncthreads_or(!landed)) {
    if (threadIdx.x == 0) atomicOr(&a.status->error, ERR_TMA_TIMEOUT);
    mbar_wait_bounded(bar, 0, WAIT_NS);  // let the copy in flight land before exiting
    return;
  }

  const C gdt = (C)(a.gamma * (a.dt_dev ? *a.dt_dev : a.dt));  // (R)(dt * gamma[i]), src/step.cpp:34
  const unsigned m2 = scheme::d2_fields(a.p);
  const int tx = threadIdx.x % TW, ty = threadIdx.x / TW;
  constexpr int RG = NT / TW;
  const int j = j0 + tx;
  bool nan = false;
  C rate = C(0);

  for (int rr = ty; rr < TH; rr += RG) {
    const int i = i0 + rr;
    if (i >= L.n1 || j >= L.n2) continue;
    const T *c0 = tile + (rr + HALF) * BW + (tx + GL);
    Cell<C, NV> cell;
#pragma unroll
    for (int f = 0; f < NV; ++f) {
      const T *c = c0 + f * PLANE;
#define G(di, dj) ((C)c[(di) * BW + (dj)])
      cell.q[f] = G(0, 0);
      cell.d1[f] = a.k.a1[0] * (G(1, 0) - G(-1, 0)) + a.k.a1[1] * (G(2, 0) - G(-2, 0)) +
                   a.k.a1[2] * (G(3, 0) - G(-3, 0));
      cell.d2[f] = a.k.a2[0] * (G(0, 1) - G(0, -1)) + a.k.a2[1] * (G(0, 2) - G(0, -2)) +
                   a.k.a2[2] * (G(0, 3) - G(0, -3));
      if (m2 & (1u << f)) {
        cell.d11[f] = a.k.b1[0] * G(0, 0) + a.k.b1[1] * (G(1, 0) + G(-1, 0)) + a.k.b1[2] * (G(2, 0) + G(-2, 0)) +
                      a.k.b1[3] * (G(3, 0) + G(-3, 0));
        cell.d22[f] = a.k.b2[0] * G(0, 0) + a.k.b2[1] * (G(0, 1) + G(0, -1)) + a.k.b2[2] * (G(0, 2) + G(0, -2)) +
                      a.k.b2[3] * (G(0, 3) + G(0, -3));
      } else {
        cell.d11[f] = C(0);
        cell.d22[f] = C(0);
      }
      if (scheme::D12_FIELDS & (1u << f)) {
        cell.d12[f] = a.k.m[0] * (G(1, 1) - G(-1, 1) + G(-1, -1) - G(1, -1)) +
                      a.k.m[1] * (G(2, 2) - G(-2, 2) + G(-2, -2) - G(2, -2)) +
                      a.k.m[2] * (G(3, 3) - G(-3, 3) + G(-3, -3) - G(3, -3));
      } else {
        cell.d12[f] = C(0);
      }
#undef G
    }
    C r[NV];
    scheme::eqns(cell, a.p, i, j, r, a.k.delta1);

    const long long o = L.at(0, i, j);
    C qn[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) {
      C vn = r[f];
      if (READ_V) vn = fma(a.beta, (C)v[o + f * L.PS], r[f]);
      if (WRITE_V) v[o + f * L.PS] = (T)vn;
      qn[f] = fma(gdt, vn, cell.q[f]);
      nan |= qn[f] != qn[f];
    }
    if (WRITE_U) store_images<T, C>(u_out, L, i, j, qn, a.p1, a.p2);
    if (CFL) rate = fmax(rate, cfl_rate<C>(qn, a.p, a.k));
  }

  if (WRITE_U) {
    if (__any_sync(0xffffffffu, nan) && (threadIdx.x & 31) == 0) atomicOr(&a.status->nan, 1u);
  }
  if (CFL) {
    double r = (double)rate;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, s));
    if ((threadIdx.x & 31) == 0 && r > 0.0)
      atomicMax(&a.status->smax, (unsigned long long)__double_as_longlong(r));
  }
}

// Tile shapes per storage type.
constexpr int TW32 = 64, TH32 = 32, NT32 = 256;
constexpr int TW64 = 64, TH64 = 32, NT64 = 256;

TileShape substage_tile(int storage)
{
  if (storage == ST_F64) return {TW64, TH64, NT64, SubstageCfg<double, TW64, TH64, NT64>::SMEM};
  return {TW32, TH32, NT32, SubstageCfg<float, TW32, TH32, NT32>::SMEM};
}

CUresult encode_state_map(CUtensorMap *map, const void *base, const Layout &L, int storage)
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return CUDA_ERROR_NOT_FOUND;
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const TileShape ts = substage_tile(storage);
  const size_t elem = storage == ST_F64 ? 8 : (storage == ST_F32 ? 4 : 2);
  const CUtensorMapDataType dt = storage == ST_F64   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : storage == ST_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : storage == ST_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                     : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  cuuint64_t dims[3] = {(cuuint64_t)(L.n2 + 2 * GL), (cuuint64_t)(L.n1 + 2 * GT), (cuuint64_t)NV};
  cuuint64_t strides[2] = {(cuuint64_t)(L.P * elem), (cuuint64_t)(L.PS * elem)};
  cuuint32_t box[3] = {(cuuint32_t)(ts.tw + 2 * GL), (cuuint32_t)(ts.th + 2 * HALF), (cuuint32_t)NV};
  cuuint32_t estr[3] = {1, 1, 1};
  return encode(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

template <class T, int TW, int TH, int NT, bool RV, bool WV, bool WU, bool CF>
static cudaError_t run_substage(const CUtensorMap &tm, T *u_out, T *v, const Layout &L, const KParams<T> &kp,
                                cudaStream_t s)
{
  using Cfg = SubstageCfg<T, TW, TH, NT>;
  auto kern = substage_kernel<T, TW, TH, NT, RV, WV, WU, CF>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const dim3 grid((L.n2 + TW - 1) / TW, (L.n1 + TH - 1) / TH);
  kern<<<grid, NT, Cfg::SMEM, s>>>(tm, u_out, v, L, kp);
  return cudaGetLastError();
}

template <class T, int TW, int TH, int NT>
static cudaError_t substage_t(int kind, bool cfl, const CUtensorMap &tm, void *u_out, void *v, const Layout &L,
                              const StageArgs &a, cudaStream_t s)
{
  const KParams<T> kp = make_params<T>(a);
  T *uo = (T *)u_out, *vv = (T *)v;
  switch (kind) {
    case STAGE_FIRST: return run_substage<T, TW, TH, NT, false, true, true, false>(tm, uo, vv, L, kp, s);
    case STAGE_MID: return run_substage<T, TW, TH, NT, true, true, true, false>(tm, uo, vv, L, kp, s);
    case STAGE_LAST:
      return cfl ? run_substage<T, TW, TH, NT, true, false, true, true>(tm, uo, vv, L, kp, s)
                 : run_substage<T, TW, TH, NT, true, false, true, false>(tm, uo, vv, L, kp, s);
    case STAGE_KICK: return run_substage<T, TW, TH, NT, true, true, false, false>(tm, uo, vv, L, kp, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_substage(int storage, int kind, bool cfl, const CUtensorMap &u_in_map, void *u_out, void *v,
                            const Layout &L, const StageArgs &a, cudaStream_t s)
{
  if (storage == ST_F32) return substage_t<float, TW32, TH32, NT32>(kind, cfl, u_in_map, u_out, v, L, a, s);
  if (storage == ST_F64) return substage_t<double, TW64, TH64, NT64>(kind, cfl, u_in_map, u_out, v, L, a, s);
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------------------
// Ghost fill (the reference's bcond, src/bcond.cu:22-86): every ghost cell of the padded
// frame [-3, n1+3) x [-3, n2+3) copies its interior source; reflective columns flip the
// sign of the wall-normal velocity.  Sources are always interior cells, so one pass gives
// the reference's axis-1-then-axis-2 result, corners included.
template <class T>
__global__ void bcond_kernel(T *u, const Layout L, int p1, int p2)
{
  const int n1 = L.n1, n2 = L.n2;
  const long long wrow = n2 + 2 * HALF;
  const long long nrows = 2LL * HALF * wrow;  // ghost rows, full width
  const long long ncols = 2LL * HALF * n1;    // ghost columns of interior rows
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nrows + ncols) return;
  int r, c;
  if (idx < nrows) {
    const int gr = (int)(idx / wrow);
    c = (int)(idx % wrow) - HALF;
    r = gr < HALF ? gr - HALF : n1 + gr - HALF;
  } else {
    const long long k = idx - nrows;
    r = (int)(k / (2 * HALF));
    const int gc = (int)(k % (2 * HALF));
    c = gc < HALF ? gc - HALF : n2 + gc - HALF;
  }
  int rs = r, cs = c;
  bool flip = false;
  if (r < 0) rs = p1 ? r + n1 : -1 - r;
  else if (r >= n1) rs = p1 ? r - n1 : 2 * n1 - 1 - r;
  if (c < 0) { cs = p2 ? c + n2 : -1 - c; flip = !p2; }
  else if (c >= n2) { cs = p2 ? c - n2 : 2 * n2 - 1 - c; flip = !p2; }
#pragma unroll
  for (int f = 0; f < NV; ++f) {
    const T x = u[L.at(f, rs, cs)];
    u[L.at(f, r, c)] = (flip && scheme::reflect_sign(f) < 0) ? -x : x;
  }
}

// drift (src/drift.cu:23-32): u <- u + dt v over the interior, NaN flag.
template <class T>
__global__ void drift_kernel(T *u, const T *v, const Layout L, T dt, Status *st)
{
  const long long n = (long long)NV * L.n1 * L.n2;
  bool nan = false;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(k / ((long long)L.n1 * L.n2));
    const long long rem = k % ((long long)L.n1 * L.n2);
    const int i = (int)(rem / L.n2), j = (int)(rem % L.n2);
    const long long o = L.at(f, i, j);
    const T x = fma(dt, v[o], u[o]);
    u[o] = x;
    nan |= x != x;
  }
  if (__any_sync(0xffffffffu, nan) && (threadIdx.x & 31) == 0) atomicOr(&st->nan, 1u);
}

// Euler hook (src/kick.cu:121-126): per-cell operator-split update of the interior.
template <class T>
__global__ void euler_kernel(T *u, const Layout L, T dt, const Para<T> p, scheme::EulerArgs e, T d1, T d2)
{
  const long long n = (long long)L.n1 * L.n2;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / L.n2), j = (int)(k % L.n2);
    T q[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) q[f] = u[L.at(f, i, j)];
    scheme::first_order<T>(q, dt, i, j, p, e, d1, d2);
#pragma unroll
    for (int f = 0; f < NV; ++f) u[L.at(f, i, j)] = q[f];
  }
}

template <class T>
__global__ void fill_kernel(T *p, size_t n, T x)
{
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = x;
}

// host layout (rows i0 .. i0 + nrows, cells of NV interleaved values) -> device layout
template <class T, class H>
__global__ void scatter_kernel(T *u, const H *src, const Layout L, int i0, int nrows)
{
  const long long n = (long long)nrows * L.n2 * NV;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(k % NV);
    const long long cell = k / NV;
    const int i = i0 + (int)(cell / L.n2), j = (int)(cell % L.n2);
    u[L.at(f, i, j)] = (T)src[k];
  }
}

template <class T, class H>
__global__ void gather_kernel(H *dst, const T *u, const Layout L, int i0, int nrows)
{
  const long long n = (long long)nrows * L.n2 * NV;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(k % NV);
    const long long cell = k / NV;
    const int i = i0 + (int)(cell / L.n2), j = (int)(cell % L.n2);
    dst[k] = (H)u[L.at(f, i, j)];
  }
}

// getdt's reduction in FP64: max over cells of (|u1| + c_s) / Delta1 + (|u2| + c_s) / Delta2.
template <class T>
__global__ void signal_max_kernel(const T *u, const Layout L, const Para<double> p, double inv1, double inv2,
                                  Status *st)
{
  const long long n = (long long)L.n1 * L.n2;
  double m = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / L.n2), j = (int)(k % L.n2);
    double q[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) q[f] = (double)u[L.at(f, i, j)];
    const double cs = scheme::sound_speed<double>(q, p);
    m = fmax(m, (fabs(q[scheme::U1]) + cs) * inv1 + (fabs(q[scheme::U2]) + cs) * inv2);
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(&st->smax, (unsigned long long)__double_as_longlong(m));
}

// FP64 conserved sums with a fixed reduction order: block b sums rows b, b + B, ... in a
// fixed per-thread order, then a fixed shared-memory tree; the partials are reduced by
// one block in a fixed tree.
constexpr int SUM_THREADS = 256;
int sums_blocks(const Layout &L) { return L.n1 < 1024 ? L.n1 : 1024; }

template <class T>
__global__ void sums_kernel(const T *u, const Layout L, double *partials)
{
  __shared__ double red[4][SUM_THREADS];
  double acc[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x; i < L.n1; i += gridDim.x)
    for (int j = threadIdx.x; j < L.n2; j += blockDim.x) {
      double q[NV], c[4];
#pragma unroll
      for (int f = 0; f < NV; ++f) q[f] = (double)u[L.at(f, i, j)];
      scheme::conserved(q, c);
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] += c[k];
    }
#pragma unroll
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = SUM_THREADS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) partials[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void sums_final_kernel(const double *partials, int nb, double *out)
{
  __shared__ double red[4][SUM_THREADS];
  double acc[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] += partials[b * 4 + k];
#pragma unroll
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = SUM_THREADS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

__global__ void dt_update_kernel(Status *st, double courant, double dt_diff, double t_end)
{
  const double smax = __longlong_as_double((long long)st->smax);
  double dt = smax > 0.0 ? courant / smax : dt_diff;
  if (dt_diff > 0.0 && dt_diff < dt) dt = dt_diff;
  const double left = t_end - st->t;
  if (left < dt) dt = left > 0.0 ? left : 0.0;
  st->dt = dt;
  st->dt_next = dt;
  st->t += dt;
  st->smax = 0ull;
  st->steps += 1ull;
}

// ---------------------------------------------------------------------------------------
// launchers
static int grid_for(long long n, int threads)
{
  long long g = (n + threads - 1) / threads;
  if (g > 148LL * 32) g = 148LL * 32;
  return (int)(g < 1 ? 1 : g);
}

cudaError_t launch_bcond(int storage, void *u, const Layout &L, int p1, int p2, cudaStream_t s)
{
  const long long n = 2LL * HALF * (L.n2 + 2 * HALF) + 2LL * HALF * L.n1;
  const int g = (int)((n + 255) / 256);
  if (storage == ST_F32) bcond_kernel<float><<<g, 256, 0, s>>>((float *)u, L, p1, p2);
  else if (storage == ST_F64) bcond_kernel<double><<<g, 256, 0, s>>>((double *)u, L, p1, p2);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_drift(int storage, void *u, const void *v, const Layout &L, double dt, Status *st,
                         cudaStream_t s)
{
  const int g = grid_for((long long)NV * L.n1 * L.n2, 256);
  if (storage == ST_F32) drift_kernel<float><<<g, 256, 0, s>>>((float *)u, (const float *)v, L, (float)dt, st);
  else if (storage == ST_F64) drift_kernel<double><<<g, 256, 0, s>>>((double *)u, (const double *)v, L, dt, st);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_euler(int storage, void *u, const Layout &L, double dt, const double *para, double delta1,
                         double delta2, float r1, float r2, cudaStream_t s)
{
  const int g = grid_for((long long)L.n1 * L.n2, 256);
  const scheme::EulerArgs e{r1, r2};
  if (storage == ST_F32) {
    Para<float> p;
    for (int q = 0; q < 8; ++q) p.v[q] = (float)para[q];
    euler_kernel<float><<<g, 256, 0, s>>>((float *)u, L, (float)dt, p, e, (float)delta1, (float)delta2);
  } else if (storage == ST_F64) {
    Para<double> p;
    for (int q = 0; q < 8; ++q) p.v[q] = para[q];
    euler_kernel<double><<<g, 256, 0, s>>>((double *)u, L, dt, p, e, delta1, delta2);
  } else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_fill(int storage, void *p, size_t count, double value, cudaStream_t s)
{
  const int g = grid_for((long long)count, 256);
  if (storage == ST_F32) fill_kernel<float><<<g, 256, 0, s>>>((float *)p, count, (float)value);
  else if (storage == ST_F64) fill_kernel<double><<<g, 256, 0, s>>>((double *)p, count, value);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_scatter(int storage, void *u, const void *src, bool host_double, const Layout &L, int i0,
                           int nrows, cudaStream_t s)
{
  const int g = grid_for((long long)nrows * L.n2 * NV, 256);
  if (storage == ST_F32 && !host_double)
    scatter_kernel<float, float><<<g, 256, 0, s>>>((float *)u, (const float *)src, L, i0, nrows);
  else if (storage == ST_F64 && host_double)
    scatter_kernel<double, double><<<g, 256, 0, s>>>((double *)u, (const double *)src, L, i0, nrows);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_gather(int storage, void *dst, const void *u, bool host_double, const Layout &L, int i0,
                          int nrows, cudaStream_t s)
{
  const int g = grid_for((long long)nrows * L.n2 * NV, 256);
  if (storage == ST_F32 && !host_double)
    gather_kernel<float, float><<<g, 256, 0, s>>>((float *)dst, (const float *)u, L, i0, nrows);
  else if (storage == ST_F64 && host_double)
    gather_kernel<double, double><<<g, 256, 0, s>>>((double *)dst, (const double *)u, L, i0, nrows);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_signal_max(int storage, const void *u, const Layout &L, const double *para, double delta1,
                              double delta2, Status *st, cudaStream_t s)
{
  const int g = grid_for((long long)L.n1 * L.n2, 256);
  Para<double> p;
  for (int q = 0; q < 8; ++q) p.v[q] = para[q];
  if (storage == ST_F32)
    signal_max_kernel<float><<<g, 256, 0, s>>>((const float *)u, L, p, 1.0 / delta1, 1.0 / delta2, st);
  else if (storage == ST_F64)
    signal_max_kernel<double><<<g, 256, 0, s>>>((const double *)u, L, p, 1.0 / delta1, 1.0 / delta2, st);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_sums(int storage, const void *u, const Layout &L, double *partials, double *out, cudaStream_t s)
{
  const int nb = sums_blocks(L);
  if (storage == ST_F32) sums_kernel<float><<<nb, SUM_THREADS, 0, s>>>((const float *)u, L, partials);
  else if (storage == ST_F64) sums_kernel<double><<<nb, SUM_THREADS, 0, s>>>((const double *)u, L, partials);
  else return cudaErrorInvalidValue;
  sums_final_kernel<<<1, SUM_THREADS, 0, s>>>(partials, nb, out);
  return cudaGetLastError();
}

cudaError_t launch_dt_update(Status *st, double courant, double dt_diff, double t_end, cudaStream_t s)
{
  dt_update_kernel<<<1, 1, 0, s>>>(st, courant, dt_diff, t_end);
  return cudaGetLastError();
}

}  // namespace fg2
