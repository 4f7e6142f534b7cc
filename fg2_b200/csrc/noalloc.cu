// fg2_b200/csrc/noalloc.cu -- FP64 conserved sums for callers that cannot allocate.
//
// fg2_sim_sums() reduces through partials the simulation handle allocated with cudaMalloc.
// Some callers cannot allocate device memory at the moment they want the sums: a host
// application whose own allocator has already reserved the GPU's memory (a framework that
// pre-reserves most of HBM), code that must not add an allocation to a real-time or
// budgeted loop, or a caller that has only a state array and no handle of this library.
// fg2_sums_noalloc() serves them: the caller passes the state array (input) and a device
// buffer of 4 doubles (output), and the only scratch is the file-scope array below, which
// every GPU that loads this library holds from load time until the process exits.
//
// Limits and sharing:
//   - at most NOALLOC_MAX_ROWS rows (n1); larger grids are rejected with FG2_ERR_ARG;
//   - every call writes the same scratch array, so calls that overlap on the GPU (two
//     streams, two threads, two host processes sharing a context) race; serialise them;
//   - each call overwrites every partial it reads, so nothing needs clearing between calls;
//   - the first call on a device resolves the array's device address (cudaGetSymbolAddress)
//     with that device current; make that first call before any stream capture.  The
//     address is kept per device and CUDA context: after the caller resets the device (a new
//     primary context) the next call resolves it again;
//   - `stream` must belong to the current device (checked).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fg2_b200.h"
#include "fg2b.h"
#include "kernels.h"

#include <state.h>
#include <eqns.cuh>

namespace fg2 {
namespace {

constexpr int NOALLOC_MAX_ROWS = FG2_NOALLOC_MAX_ROWS;
constexpr int NA_THREADS = 256;
constexpr int MAX_DEVICES = 64;

// One partial (rho, rho u1, rho u2, energy) per grid row: 16384 x 4 doubles = 512 KiB.
__device__ __align__(256) double noalloc_scratch[NOALLOC_MAX_ROWS * 4];

// Host-side cache of the array's device address per device, with the context it was
// resolved in.  In host code the name noalloc_scratch is only a host stand-in, never a
// device address.
double *g_scratch[MAX_DEVICES] = {};
CUcontext g_scratch_ctx[MAX_DEVICES] = {};
std::mutex g_scratch_mu;

// The calling thread's current CUDA context (driver entry point, resolved once).
CUcontext current_context()
{
  using Fn = CUresult (*)(CUcontext *);
  static Fn get = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get = (Fn)fn;
  });
  CUcontext c = nullptr;
  if (get && get(&c) != CUDA_SUCCESS) c = nullptr;
  return c;
}

// Block i sums row i: thread t takes columns t, t + 256, ... in order, then a fixed tree.
template <class T>
__global__ void __launch_bounds__(NA_THREADS) row_sums_kernel(const T *u, const Layout L, double *partials)
{
  __shared__ double red[4][NA_THREADS];
  const int i = blockIdx.x;
  double acc[4] = {0, 0, 0, 0};
  for (int j = threadIdx.x; j < L.n2; j += NA_THREADS) {
    double q[scheme::NVAR], c[4];
#pragma unroll
    for (int f = 0; f < scheme::NVAR; ++f) q[f] = (double)u[L.at(f, i, j)];
    scheme::conserved(q, c);
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] += c[k];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = NA_THREADS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) partials[i * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// One block adds the n1 row partials in a fixed order into out[4].
__global__ void __launch_bounds__(NA_THREADS) rows_final_kernel(const double *partials, int n1, double *out)
{
  __shared__ double red[4][NA_THREADS];
  double acc[4] = {0, 0, 0, 0};
  for (int r = threadIdx.x; r < n1; r += NA_THREADS)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] += partials[r * 4 + k];
#pragma unroll
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = NA_THREADS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

// Device address of the scratch array on the current device, resolved once per device.
int scratch_address(double **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error((int)e, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return set_error(FG2_ERR_ARG, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const CUcontext ctx = current_context();
  if (!g_scratch[dev] || g_scratch_ctx[dev] != ctx) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(e != cudaSuccess ? (int)e : FG2_ERR_ARG, "cudaGetSymbolAddress of the scratch array failed: %s",
                       cudaGetErrorString(e));
    g_scratch[dev] = (double *)p;
    g_scratch_ctx[dev] = current_context();  // the runtime call made the primary context current
  }
  *out = g_scratch[dev];
  return FG2_OK;
}

}  // namespace
}  // namespace fg2

extern "C" int fg2_sums_noalloc(const void *u, int n1, int n2, long long pitch, int storage, double *out,
                                void *stream)
{
  using namespace fg2;
  if (!u || !out) return set_error(FG2_ERR_ARG, "fg2_sums_noalloc: null array");
  if (n1 < 1 || n2 < 1) return set_error(FG2_ERR_ARG, "fg2_sums_noalloc: empty grid %d x %d", n1, n2);
  if (n1 > NOALLOC_MAX_ROWS)
    return set_error(FG2_ERR_ARG, "fg2_sums_noalloc: n1 = %d rows exceeds the scratch limit of %d rows", n1,
                     NOALLOC_MAX_ROWS);
  // pitch = row stride (element (f, i, j) at (i + 3) * pitch + (j + 4) * NVAR + f)
  if (pitch < ((long long)n2 + 2 * GL) * scheme::NVAR)
    return set_error(FG2_ERR_ARG, "fg2_sums_noalloc: pitch %lld too small for %d x %d", pitch, n1, n2);
  if (storage != ST_F32 && storage != ST_F64)
    return set_error(FG2_ERR_UNSUPPORTED, "fg2_sums_noalloc: storage %d not supported", storage);
  // an error left on this thread by earlier, unrelated work would otherwise be reported
  // as this call's launch failure
  (void)cudaGetLastError();
  cudaStream_t s = (cudaStream_t)stream;
  int cur = 0, sdev = 0;
  cudaError_t de = cudaGetDevice(&cur);
  if (de == cudaSuccess) de = cudaStreamGetDevice(s, &sdev);
  if (de != cudaSuccess) return set_error((int)de, "fg2_sums_noalloc: %s", cudaGetErrorString(de));
  if (sdev != cur)
    return set_error(FG2_ERR_ARG, "fg2_sums_noalloc: the stream belongs to device %d, the current device is %d", sdev,
                     cur);
  double *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  Layout L;
  L.n1 = n1;
  L.n2 = n2;
  L.RS = pitch;
  L.CS = scheme::NVAR;
  if (storage == ST_F32) row_sums_kernel<float><<<n1, NA_THREADS, 0, s>>>((const float *)u, L, scratch);
  else row_sums_kernel<double><<<n1, NA_THREADS, 0, s>>>((const double *)u, L, scratch);
  rows_final_kernel<<<1, NA_THREADS, 0, s>>>(scratch, n1, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error((int)e, "fg2_sums_noalloc launch: %s", cudaGetErrorString(e));
  return FG2_OK;
}
