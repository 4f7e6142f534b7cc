// fg2_b200/csrc/kernels.cu -- device kernels of the B200 time step, compiled once per
// scheme (-I schemes/<name>), for sm_100a.
//
// The hot kernel is the fused RK3 substage (substage_kernel): one pass per stage that
//   1. streams 7-row chunks of u (halo included) and v of a 128-column strip from HBM into
//      shared memory by TMA (cp.async.bulk.tensor.3d, completion on an mbarrier);
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
#include <cuda_bf16.h>
#include <cuda_fp16.h>
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
// Two cells per thread: the pair type of a storage type (packed FP32x2 for float).
template <class T>
struct PairOf;
template <>
struct PairOf<float> {
  using type = float2;
  static __host__ __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
};
template <>
struct PairOf<double> {
  using type = double2;
  static __host__ __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
};

// Storage types of the state arrays: the compute type C and, for 16-bit deviation storage
// (DEV), conversions of single values and of packed pairs.
template <class S>
struct Store {
  using C = S;
  static constexpr bool DEV = false;
};
template <>
struct Store<__half> {
  using C = float;
  using S2 = __half2;
  static constexpr bool DEV = true;
  static __device__ __forceinline__ float to(__half h) { return __half2float(h); }
  static __device__ __forceinline__ __half from(float x) { return __float2half_rn(x); }
  static __device__ __forceinline__ float2 to2(__half2 h) { return __half22float2(h); }
  static __device__ __forceinline__ __half2 from2(float2 x) { return __float22half2_rn(x); }
};
template <>
struct Store<__nv_bfloat16> {
  using C = float;
  using S2 = __nv_bfloat162;
  static constexpr bool DEV = true;
  static __device__ __forceinline__ float to(__nv_bfloat16 h) { return __bfloat162float(h); }
  static __device__ __forceinline__ __nv_bfloat16 from(float x) { return __float2bfloat16_rn(x); }
  static __device__ __forceinline__ float2 to2(__nv_bfloat162 h) { return __bfloat1622float2(h); }
  static __device__ __forceinline__ __nv_bfloat162 from2(float2 x) { return __float22bfloat162_rn(x); }
};

// Type of the rounding residual of a 16-bit state: FP16 for both storages (a BF16 state's
// residual e / s * RESID_SCALE is at most about 8, which FP16 holds to 11 bits where BF16
// would keep 8).
template <class S>
struct Resid {
  using type = S;
};
template <>
struct Resid<__nv_bfloat16> {
  using type = __half;
};

// Parameters of one substage launch, rounded to the storage precision T: the stencil
// weights both as scalars and broadcast to both lanes of a pair (so packed instructions read
// them straight from the constant bank), the scheme's parameters as scalars.
template <class T>
struct KParams {
  using P = typename PairOf<T>::type;
  Coef<P> k;   // packed stencil weights
  Coef<T> ks;  // scalar stencil weights
  Para<T> p;   // scheme parameters
  P beta2;     // the stage's beta on both lanes
  double gamma, dt;
  const double *dt_dev;  // device time step for grids without their own, or null: dt
  Status *status;        // launch errors
  int nb;                // output blocks of 7 rows per tile
  int tail;              // one-block bands that at least end each grid (0: none)
  int strip;             // strip width (columns per tile, threads per CTA)
  int reverse;           // tiles last first
  unsigned wait_test_bytes;  // extra bytes every chunk expects (timeout-path tests; 0 otherwise)
};

template <class T>
static typename PairOf<T>::type bc(double x)
{
  return PairOf<T>::make((T)x, (T)x);
}

// scaled: plain weights (Delta = 1), the grids' 1/Delta factors are applied in the kernel.
template <class T>
static KParams<T> make_params(const StageArgs &a, bool scaled)
{
  KParams<T> kp;
  // Delta = l / n is rounded to the state precision (src/config.cpp:39); the weights are
  // divided by it in double and rounded once.
  const double d1 = scaled ? 1.0 : a.delta1, d2 = scaled ? 1.0 : a.delta2;
  const double w1[3] = {45. / 60., -9. / 60., 1. / 60.};
  const double w2[4] = {-490. / 180., 270. / 180., -27. / 180., 2. / 180.};
  const double wm[3] = {270. / 720., -27. / 720., 2. / 720.};
  for (int q = 0; q < 3; ++q) {
    kp.ks.a1[q] = (T)(w1[q] / d1);
    kp.ks.a2[q] = (T)(w1[q] / d2);
    kp.ks.m[q] = (T)(wm[q] / (d1 * d2));
    kp.ks.mn[q] = (T)(-wm[q] / (d1 * d2));
  }
  for (int q = 0; q < 4; ++q) {
    kp.ks.b1[q] = (T)(w2[q] / (d1 * d1));
    kp.ks.b2[q] = (T)(w2[q] / (d2 * d2));
  }
  kp.ks.delta1 = (T)d1;
  kp.ks.delta2 = (T)d2;
  kp.ks.inv1 = (T)(1.0 / d1);
  kp.ks.inv2 = (T)(1.0 / d2);
  for (int q = 0; q < 3; ++q) {
    kp.k.a1[q] = bc<T>(kp.ks.a1[q]);
    kp.k.a2[q] = bc<T>(kp.ks.a2[q]);
    kp.k.m[q] = bc<T>(kp.ks.m[q]);
    kp.k.mn[q] = bc<T>(kp.ks.mn[q]);
  }
  for (int q = 0; q < 4; ++q) {
    kp.k.b1[q] = bc<T>(kp.ks.b1[q]);
    kp.k.b2[q] = bc<T>(kp.ks.b2[q]);
  }
  kp.k.delta1 = bc<T>(kp.ks.delta1);
  kp.k.delta2 = bc<T>(kp.ks.delta2);
  kp.k.inv1 = bc<T>(kp.ks.inv1);
  kp.k.inv2 = bc<T>(kp.ks.inv2);
  for (int q = 0; q < NPARA; ++q) kp.p.v[q] = (T)(a.para ? a.para[q] : 0.0);
  kp.beta2 = bc<T>(a.beta);
  kp.gamma = a.gamma;
  kp.dt = a.dt;
  kp.dt_dev = a.dt_dev;
  kp.status = a.status;
  kp.nb = a.nb > 0 ? a.nb : TILE_BLOCKS_DEFAULT;
  kp.tail = a.tail > 0 ? a.tail : 0;
  kp.strip = strip_width(a.strip);
  kp.reverse = a.reverse;
  kp.wait_test_bytes = a.wait_test_bytes;
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

// Only the ghost images of (i, j), not the cell itself (which the caller stores): the general
// case, any grid size.  Kept out of line: the fused kernel calls it only for grids narrower
// than two ghost widths, and inlined copies would crowd its instruction cache.
template <class T, class C>
__device__ __noinline__ void store_ghosts(T *u, const Layout L, int i, int j, const C *q, int p1, int p2)
{
  const bool edge = i < HALF || i >= L.n1 - HALF || j < HALF || j >= L.n2 - HALF;
  if (!edge) return;
  const Images g = ghost_images(i, j, L.n1, L.n2, p1, p2);
  for (int a = 0; a < g.nr; ++a)
    for (int b = 0; b < g.nc; ++b) {
      if (a == 0 && b == 0) continue;
#pragma unroll
      for (int f = 0; f < NV; ++f) {
        const C x = (g.flip[b] && scheme::reflect_sign(f) < 0) ? -q[f] : q[f];
        u[L.at(f, g.rows[a], g.cols[b])] = (T)x;
      }
    }
}

// CFL signal rate of a cell (the scheme's: (|u1| + c_s) / Delta1 + (|u2| + c_s) / Delta2 on a
// Cartesian grid, from the cell's position on a curvilinear one).
template <class C>
__device__ __forceinline__ C cfl_rate(const C q[NV], const Para<C> &p, C inv1, C inv2, int i, int j, C d1, C d2,
                                      const scheme::Geom<C> &cg)
{
  return scheme::signal_rate<C>(q, p, inv1, inv2, i, j, d1, d2, cg);
}

// 16-bit deviation storage codes hold at most DEV_MAX_FIELDS fields per cell; kernels for
// 16-bit arrays are only compiled for schemes within that.
constexpr bool DEV_OK = NV <= DEV_MAX_FIELDS;

#include "substage.cuh"

// ---------------------------------------------------------------------------------------
// Tensor maps: u with the halo box of one chunk, v with the interior box of one chunk.
namespace {
static_assert(sizeof(GridDesc) % 64 == 0 && alignof(GridDesc) == 64, "grid descriptors keep tensor-map alignment");
PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  return encode;
}

// Cells per 16-byte group: TMA boxes are built from whole groups, so the innermost box
// dimension (one group of interleaved cells, NV x 16 bytes) is a 16-byte multiple for any
// NVAR and the innermost coordinate is always 0.
int elem_bytes(int storage) { return storage == ST_F64 ? 8 : storage == ST_F32 ? 4 : 2; }
int group_cells(int storage) { return sub::group_of(elem_bytes(storage)); }

// Map over the padded array as (group element, cell group, padded row): box_cells x box_rows
// boxes land in shared memory as [row][cell][field]; the map covers ext_cells cells (whole
// groups) and ext_rows rows.
CUresult encode_map(CUtensorMap *map, const void *base, const Layout &L, int storage, int box_cells, int box_rows,
                    long long ext_cells, long long ext_rows)
{
  PFN_cuTensorMapEncodeTiled_v12000 encode = encoder();
  if (!encode) return CUDA_ERROR_NOT_FOUND;
  const size_t elem = elem_bytes(storage);
  const int G = group_cells(storage);
  const CUtensorMapDataType dt = storage == ST_F64   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : storage == ST_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : storage == ST_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                     : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  cuuint64_t dims[3] = {(cuuint64_t)(G * NV), (cuuint64_t)((ext_cells + G - 1) / G), (cuuint64_t)ext_rows};
  cuuint64_t strides[2] = {(cuuint64_t)(G * NV * elem), (cuuint64_t)(L.RS * elem)};
  cuuint32_t box[3] = {(cuuint32_t)(G * NV), (cuuint32_t)(box_cells / G), (cuuint32_t)box_rows};
  cuuint32_t estr[3] = {1, 1, 1};
  return encode(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}
}  // namespace

CUresult make_grid_desc(GridDesc *d, const void *u_in, void *u_out, void *v, const Layout &L, int storage, int p1,
                        int p2, double delta1, double delta2, const double *dt, Status *status, int tile0,
                        const DevCode *dev, int strip)
{
  const int sw = strip_width(strip);
  CUresult r = encode_map(&d->tm_u, u_in, L, storage, sw + 2 * GL, sub::CH, L.n2 + 2 * GL, L.n1 + 2 * GT);
  if (r != CUDA_SUCCESS) return r;
  // the v box starts GL % G cells left of the strip when a cell group is wider than GL
  const int G = group_cells(storage), vbw = (sw + GL % G + G - 1) / G * G;
  r = encode_map(&d->tm_v, v, L, storage, vbw, sub::CH, L.n2 + 2 * GL, L.n1 + 2 * GT);
  if (r != CUDA_SUCCESS) return r;
  if (dev && dev->r) {  // the input's rounding residual, in boxes like u's (halo included)
    r = encode_map(&d->tm_r, dev->r, L, resid_storage(storage), sw + 2 * GL, sub::CH, L.n2 + 2 * GL, L.n1 + 2 * GT);
    if (r != CUDA_SUCCESS) return r;
  } else {
    d->tm_r = d->tm_v;  // never read: only 16-bit stages load r
  }
  d->u_out = u_out;
  d->v = v;
  d->L = L;
  d->strips = sub::tile_grid(L, sub::NB_DEFAULT, sw).strips;
  d->tile0 = tile0;
  d->p1 = p1;
  d->p2 = p2;
  d->dt = dt;
  d->status = status;
  d->inv1 = 1.0 / delta1;
  d->inv2 = 1.0 / delta2;
  d->inv11 = 1.0 / (delta1 * delta1);
  d->inv22 = 1.0 / (delta2 * delta2);
  d->inv12 = 1.0 / (delta1 * delta2);
  d->delta1 = delta1;
  d->delta2 = delta2;
  if (dev) d->dev = *dev;
  else d->dev = DevCode{{0.f, 0.f, 0.f, 0.f}, nullptr, nullptr, 0, nullptr, nullptr};
  return CUDA_SUCCESS;
}

int strip_width(int strip) { return strip == 64 ? 64 : STRIP_DEFAULT; }

int substage_tiles(const Layout &L, int nb, int strip, int tail)
{
  return sub::tile_grid(L, nb > 0 ? nb : sub::NB_DEFAULT, strip_width(strip), tail > 0 ? tail : 0).ntiles;
}

int tile_bands(int n1, int nb, int tail, int reverse, int *out, int cap)
{
  if (n1 < 1 || nb < 0 || tail < 0) return -1;
  Layout L{};
  L.n1 = n1;
  L.n2 = 1;
  const int h = nb > 0 ? nb : sub::NB_DEFAULT;
  const sub::TileGrid g = sub::tile_grid(L, h, STRIP_DEFAULT, tail);
  const int nbands = g.bands + g.small;
  for (int q = 0; q < nbands && q < cap; ++q) {
    const sub::Band b = sub::band_rows(n1, h, g.bands, q, reverse != 0);
    out[3 * q] = b.i0;
    out[3 * q + 1] = b.iend;
    out[3 * q + 2] = b.nbt;
  }
  return nbands;
}

template <class S, unsigned M2, bool RV, bool WV, bool WU, bool CF, bool SC, int W>
static cudaError_t run_substage_w(const GridDesc *grids, int ngrids, int ntiles, const KParams<typename Store<S>::C> &kp,
                                  int max_ctas, int *queue, cudaStream_t s)
{
  using G = sub::Geo<S, RV, Store<S>::DEV, W>;  // 16-bit stages also load the residual box
  auto kern = sub::substage_kernel<S, M2, RV, WV, WU, CF, SC, W>;
  static int ctas_per_sm = 0, sms = 0;
  if (!ctas_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
    if (e != cudaSuccess) return e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, kern, W, G::SMEM)) != cudaSuccess)
      return e;
    if (ctas_per_sm < 1) return cudaErrorInvalidConfiguration;
  }
  if (ntiles < 1) return cudaSuccess;
  int grid = sms * (max_ctas > 0 && max_ctas < ctas_per_sm ? max_ctas : ctas_per_sm);
  if (grid > ntiles) grid = ntiles;
  kern<<<grid, W, G::SMEM, s>>>(grids, ngrids, ntiles, kp, queue);
  return cudaGetLastError();
}

// Single grids use the default strip; batch launches (SC) may take the narrower one.
template <class S, unsigned M2, bool RV, bool WV, bool WU, bool CF, bool SC>
static cudaError_t run_substage(const GridDesc *grids, int ngrids, int ntiles, const KParams<typename Store<S>::C> &kp,
                                int max_ctas, int *queue, cudaStream_t s)
{
  if constexpr (SC) {
    if (kp.strip == 64) return run_substage_w<S, M2, RV, WV, WU, CF, SC, 64>(grids, ngrids, ntiles, kp, max_ctas, queue, s);
  } else {
    if (kp.strip == 64) return cudaErrorInvalidValue;
  }
  return run_substage_w<S, M2, RV, WV, WU, CF, SC, STRIP_DEFAULT>(grids, ngrids, ntiles, kp, max_ctas, queue, s);
}

template <class S, unsigned M2, bool SC>
static cudaError_t substage_m(int kind, bool cfl, const GridDesc *g, int ng, int nt,
                              const KParams<typename Store<S>::C> &kp, int mc, int *queue, cudaStream_t s)
{
  switch (kind) {
    case STAGE_FIRST: return run_substage<S, M2, false, true, true, false, SC>(g, ng, nt, kp, mc, queue, s);
    case STAGE_MID: return run_substage<S, M2, true, true, true, false, SC>(g, ng, nt, kp, mc, queue, s);
    case STAGE_LAST:
      return cfl ? run_substage<S, M2, true, false, true, true, SC>(g, ng, nt, kp, mc, queue, s)
                 : run_substage<S, M2, true, false, true, false, SC>(g, ng, nt, kp, mc, queue, s);
    case STAGE_KICK: return run_substage<S, M2, true, true, false, false, SC>(g, ng, nt, kp, mc, queue, s);
  }
  return cudaErrorInvalidValue;
}

// The kernels are compiled for two sets of second-derivative fields: the scheme's default
// parameters' set, and all fields (correct for any parameters: an unused D11/D22 meets a
// zero coefficient).  FP64, the reference-precision path, always uses all fields.
template <class S, bool SC>
static cudaError_t substage_t(int kind, bool cfl, const GridDesc *g, int ng, int nt, const StageArgs &a, int *queue,
                              cudaStream_t s)
{
  using T = typename Store<S>::C;
  const KParams<T> kp = make_params<T>(a, SC);
  const unsigned need = scheme::d2_fields(a.para);
  if constexpr (sizeof(T) == 4) {
    if ((need & ~scheme::D2_DEFAULT) == 0)
      return substage_m<S, scheme::D2_DEFAULT, SC>(kind, cfl, g, ng, nt, kp, a.max_ctas, queue, s);
  }
  return substage_m<S, scheme::D2_ALL, SC>(kind, cfl, g, ng, nt, kp, a.max_ctas, queue, s);
}

template <class S>
static cudaError_t substage_s(int kind, bool cfl, bool scaled, const GridDesc *grids, int ngrids, int ntiles,
                              const StageArgs &a, int *queue, cudaStream_t s)
{
  return scaled ? substage_t<S, true>(kind, cfl, grids, ngrids, ntiles, a, queue, s)
                : substage_t<S, false>(kind, cfl, grids, ngrids, ntiles, a, queue, s);
}

cudaError_t launch_substage(int storage, int kind, bool cfl, bool scaled, const GridDesc *grids, int ngrids,
                            int ntiles, const StageArgs &a, int *queue, cudaStream_t s)
{
  switch (storage) {
    case ST_F32: return substage_s<float>(kind, cfl, scaled, grids, ngrids, ntiles, a, queue, s);
    case ST_F64: return substage_s<double>(kind, cfl, scaled, grids, ngrids, ntiles, a, queue, s);
    case ST_F16:
      if constexpr (!DEV_OK) return cudaErrorInvalidValue;
      else return substage_s<__half>(kind, cfl, scaled, grids, ngrids, ntiles, a, queue, s);
    case ST_BF16:
      if constexpr (!DEV_OK) return cudaErrorInvalidValue;
      else return substage_s<__nv_bfloat16>(kind, cfl, scaled, grids, ngrids, ntiles, a, queue, s);
  }
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

// drift (src/drift.cu:23-32): u <- u + dt v over the interior, NaN flag.  Interior rows
// are contiguous runs of n2 * NVAR elements.
template <class T>
__global__ void drift_kernel(T *u, const T *v, const Layout L, T dt, Status *st)
{
  const long long run = (long long)L.n2 * NV, n = run * L.n1;
  bool nan = false;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long o = L.at(0, (int)(k / run), 0) + k % run;
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

// Value of field f at interior cell (i, j), decoded for 16-bit deviation storage: the stored
// number's value S = bg + s h less the rounding residual e = s r / RESID_SCALE.
template <class S>
__device__ __forceinline__ double value_at(const S *u, const Layout &L, const DevCode &dc, int f, int i, int j)
{
  if constexpr (!Store<S>::DEV) {
    return (double)u[L.at(f, i, j)];
  } else {
    const float4 sc = __ldg(dc.scale + (i / SCALE_TILE) * dc.tiles2 + j / SCALE_TILE);
    const float sf = f == 0 ? sc.x : f == 1 ? sc.y : f == 2 ? sc.z : sc.w;
    const double x = (double)fmaf(sf, Store<S>::to(u[L.at(f, i, j)]), dc.bg[f]);
    if (!dc.r) return x;
    using R = typename Resid<S>::type;
    const double e = (double)Store<R>::to(reinterpret_cast<const R *>(dc.r)[L.at(f, i, j)]) * (double)sf / RESID_SCALE;
    return x - e;
  }
}

// getdt's reduction in FP64: max over cells of (|u1| + c_s) / Delta1 + (|u2| + c_s) / Delta2.
template <class T>
__global__ void signal_max_kernel(const T *u, const Layout L, const Para<double> p, double inv1, double inv2,
                                  double d1, double d2, Status *st, const DevCode dc)
{
  const long long n = (long long)L.n1 * L.n2;
  double m = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / L.n2), j = (int)(k % L.n2);
    double q[NV];
#pragma unroll
    for (int f = 0; f < NV; ++f) q[f] = value_at<T>(u, L, dc, f, i, j);
    if constexpr (scheme::CURVILINEAR) {
      m = fmax(m, scheme::signal_rate<double>(q, p, inv1, inv2, i, j, d1, d2, scheme::column_geom<double>(j, d2)));
    } else {
      const double cs = scheme::sound_speed<double>(q, p);
      m = fmax(m, (fabs(q[scheme::U1]) + cs) * inv1 + (fabs(q[scheme::U2]) + cs) * inv2);
    }
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
__global__ void sums_kernel(const T *u, const Layout L, double *partials, const DevCode dc)
{
  __shared__ double red[4][SUM_THREADS];
  double acc[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x; i < L.n1; i += gridDim.x)
    for (int j = threadIdx.x; j < L.n2; j += blockDim.x) {
      double q[NV], c[4];
#pragma unroll
      for (int f = 0; f < NV; ++f) q[f] = value_at<T>(u, L, dc, f, i, j);
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

// Deviation storage: FP32 cells (n1 x n2 x NV, no ghosts) -> 16-bit numbers, the
// substage kernel's encoding (h = (x - bg) / s of the cell's tile, rounded once).
template <class S>
__global__ void encode_kernel(S *u, const float *src, const Layout L, const DevCode dc, bool with_code)
{
  const long long n = (long long)L.n1 * L.n2 * NV;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(k % NV);
    const long long cell = k / NV;
    const int i = (int)(cell / L.n2), j = (int)(cell % L.n2);
    if (!with_code) {
      u[L.at(f, i, j)] = Store<S>::from(src[k]);
      continue;
    }
    const int t = (i / SCALE_TILE) * dc.tiles2 + j / SCALE_TILE;
    const float4 iv = __ldg(dc.inv + t), sc = __ldg(dc.scale + t);
    const float inv = f == 0 ? iv.x : f == 1 ? iv.y : f == 2 ? iv.z : iv.w;
    const float sf = f == 0 ? sc.x : f == 1 ? sc.y : f == 2 ? sc.z : sc.w;
    const S h = Store<S>::from((src[k] - dc.bg[f]) * inv);
    u[L.at(f, i, j)] = h;
    // the rounding residual e = S - x, kept as e / s * RESID_SCALE (the substage's encoding)
    if (dc.r) {
      const float e = fmaf(sf, Store<S>::to(h), dc.bg[f]) - src[k];
      using R = typename Resid<S>::type;
      reinterpret_cast<R *>(dc.r)[L.at(f, i, j)] = Store<R>::from(e * (inv * (float)RESID_SCALE));
    }
  }
}

// 16-bit numbers -> FP32 cells; with_code false: plain conversion (v).
template <class S>
__global__ void decode_kernel(float *dst, const S *u, const Layout L, const DevCode dc, bool with_code)
{
  const long long n = (long long)L.n1 * L.n2 * NV;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(k % NV);
    const long long cell = k / NV;
    const int i = (int)(cell / L.n2), j = (int)(cell % L.n2);
    dst[k] = with_code ? (float)value_at<S>(u, L, dc, f, i, j) : Store<S>::to(u[L.at(f, i, j)]);
  }
}

// Device-resident time steps of a batch: member k takes min(courant_k / smax_k, dt_diff_k),
// capped at t_end, exactly as dt_update_kernel does for one simulation.
__global__ void dt_update_batch_kernel(Status *st, const double2 *limits, int count, double t_end)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  Status &s = st[k];
  const double courant = limits[k].x, dt_diff = limits[k].y;
  const double smax = __longlong_as_double((long long)s.smax);
  double dt = smax > 0.0 ? courant / smax : dt_diff;
  if (dt_diff > 0.0 && dt_diff < dt) dt = dt_diff;
  const double left = t_end - s.t;
  if (left < dt) dt = left > 0.0 ? left : 0.0;
  s.dt = dt;
  s.dt_next = dt;
  s.t += dt;
  s.smax = 0ull;
  s.steps += 1ull;
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
  else if (storage == ST_F16) bcond_kernel<__half><<<g, 256, 0, s>>>((__half *)u, L, p1, p2);
  else if (storage == ST_BF16) bcond_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((__nv_bfloat16 *)u, L, p1, p2);
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
    for (int q = 0; q < NPARA; ++q) p.v[q] = (float)para[q];
    euler_kernel<float><<<g, 256, 0, s>>>((float *)u, L, (float)dt, p, e, (float)delta1, (float)delta2);
  } else if (storage == ST_F64) {
    Para<double> p;
    for (int q = 0; q < NPARA; ++q) p.v[q] = para[q];
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
  else if (storage == ST_F16 || storage == ST_BF16) return cudaMemsetAsync(p, 0, count * 2, s);  // 16-bit: h = 0
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_signal_max(int storage, const void *u, const Layout &L, const double *para, double delta1,
                              double delta2, Status *st, cudaStream_t s, const DevCode *dev)
{
  const int g = grid_for((long long)L.n1 * L.n2, 256);
  Para<double> p;
  for (int q = 0; q < NPARA; ++q) p.v[q] = para[q];
  const DevCode dc = dev ? *dev : DevCode{};
  const double i1 = 1.0 / delta1, i2 = 1.0 / delta2, d1 = delta1, d2 = delta2;
  switch (storage) {
    case ST_F32: signal_max_kernel<float><<<g, 256, 0, s>>>((const float *)u, L, p, i1, i2, d1, d2, st, dc); break;
    case ST_F64: signal_max_kernel<double><<<g, 256, 0, s>>>((const double *)u, L, p, i1, i2, d1, d2, st, dc); break;
    case ST_F16:
      if constexpr (!DEV_OK) return cudaErrorInvalidValue;
      else signal_max_kernel<__half><<<g, 256, 0, s>>>((const __half *)u, L, p, i1, i2, d1, d2, st, dc);
      break;
    case ST_BF16:
      if constexpr (!DEV_OK) return cudaErrorInvalidValue;
      else signal_max_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((const __nv_bfloat16 *)u, L, p, i1, i2, d1, d2, st, dc);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_sums(int storage, const void *u, const Layout &L, double *partials, double *out, cudaStream_t s,
                        const DevCode *dev)
{
  const int nb = sums_blocks(L);
  const DevCode dc = dev ? *dev : DevCode{};
  switch (storage) {
    case ST_F32: sums_kernel<float><<<nb, SUM_THREADS, 0, s>>>((const float *)u, L, partials, dc); break;
    case ST_F64: sums_kernel<double><<<nb, SUM_THREADS, 0, s>>>((const double *)u, L, partials, dc); break;
    case ST_F16:
      if constexpr (!DEV_OK) return cudaErrorInvalidValue;
      else sums_kernel<__half><<<nb, SUM_THREADS, 0, s>>>((const __half *)u, L, partials, dc);
      break;
    case ST_BF16:
      if constexpr (!DEV_OK) return cudaErrorInvalidValue;
      else sums_kernel<__nv_bfloat16><<<nb, SUM_THREADS, 0, s>>>((const __nv_bfloat16 *)u, L, partials, dc);
      break;
    default: return cudaErrorInvalidValue;
  }
  sums_final_kernel<<<1, SUM_THREADS, 0, s>>>(partials, nb, out);
  return cudaGetLastError();
}

cudaError_t launch_encode(int storage, void *u, const float *src, const Layout &L, const DevCode *dev, cudaStream_t s)
{
  const int g = grid_for((long long)L.n1 * L.n2 * NV, 256);
  const DevCode dc = dev ? *dev : DevCode{};
  if constexpr (!DEV_OK) return cudaErrorInvalidValue;
  else {
    if (storage == ST_F16) encode_kernel<__half><<<g, 256, 0, s>>>((__half *)u, src, L, dc, dev != nullptr);
    else if (storage == ST_BF16)
      encode_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((__nv_bfloat16 *)u, src, L, dc, dev != nullptr);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
}

cudaError_t launch_decode(int storage, float *dst, const void *u, const Layout &L, const DevCode *dev, cudaStream_t s)
{
  const int g = grid_for((long long)L.n1 * L.n2 * NV, 256);
  const DevCode dc = dev ? *dev : DevCode{};
  if constexpr (!DEV_OK) return cudaErrorInvalidValue;
  else {
    if (storage == ST_F16) decode_kernel<__half><<<g, 256, 0, s>>>(dst, (const __half *)u, L, dc, dev != nullptr);
    else if (storage == ST_BF16)
      decode_kernel<__nv_bfloat16><<<g, 256, 0, s>>>(dst, (const __nv_bfloat16 *)u, L, dc, dev != nullptr);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
}

cudaError_t launch_dt_update_batch(Status *st, const double2 *limits, int count, double t_end, cudaStream_t s)
{
  if (count < 1) return cudaSuccess;
  dt_update_batch_kernel<<<(count + 127) / 128, 128, 0, s>>>(st, limits, count, t_end);
  return cudaGetLastError();
}

cudaError_t launch_dt_update(Status *st, double courant, double dt_diff, double t_end, cudaStream_t s)
{
  dt_update_kernel<<<1, 1, 0, s>>>(st, courant, dt_diff, t_end);
  return cudaGetLastError();
}

}  // namespace fg2
