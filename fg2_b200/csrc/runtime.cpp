// fg2_b200/csrc/runtime.cpp -- host runtime and C ABI (include/fg2_b200.h), compiled once
// per scheme with -I schemes/<name>.
//
// A simulation handle owns: two state arrays u[0], u[1] (ping-pong: a substage reads one
// and writes the other, so no tile overwrites a halo a neighbouring tile still reads), the
// RK3 register v, a tensor map per u array, a device status block and a stream.  The
// reference keeps the same state in namespace global (src/global.cpp:22-31) and allocates
// it in setup() (src/setup.cpp:60-87).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "sim.h"

#include <state.h>
#include <eqns.cuh>
#include <Euler.cuh>
#include <bcond.cuh>
#include <config.h>
#include <init.h>

using namespace fg2;

namespace {
thread_local char g_err[512] = "";
}  // namespace

int fg2::set_error(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

namespace fg2 {
namespace rt {

int cuda_status(cudaError_t e, const char *what)
{
  if (e == cudaSuccess) return FG2_OK;
  return fail((int)e, "%s: %s", what, cudaGetErrorString(e));
}

size_t elem_size(int storage) { return storage == ST_F64 ? 8 : storage == ST_F32 ? 4 : 2; }
size_t host_elem(int storage) { return storage == ST_F64 ? 8 : 4; }

const double RK_ALPHA[3] = {0.0, 1.0 / 3.0, 3.0 / 4.0};
const double RK_BETA[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
const double RK_GAMMA[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

namespace {
// 6th-order second-derivative symbol maximum (1088/180 per axis) and the RK3 real-axis
// stability bound: the explicit diffusive limit is dt <= c_d * 2.51 / (D (6.04/D1^2 + 6.04/D2^2)).
const double D2_SYMBOL = 1088.0 / 180.0;
const double RK3_REAL_LIMIT = 2.51;
}  // namespace

size_t array_elems(const fg2_sim *s) { return (size_t)s->L.elems(); }

// Delta = l / n in the state's precision (src/config.cpp:39: R Delta[] = {l1/n1, l2/n2}).
void compute_deltas(fg2_sim *s)
{
  if (s->storage == ST_F64) {
    s->delta1 = s->l1 / s->n1;
    s->delta2 = s->l2 / s->n2;
  } else {
    s->delta1 = (double)((float)s->l1 / (float)s->n1);
    s->delta2 = (double)((float)s->l2 / (float)s->n2);
  }
}

// parameters are parsed into R like the reference's atof -> R (src/para.cpp:34)
double round_para(const fg2_sim *s, double x) { return s->storage == ST_F64 ? x : (double)(float)x; }

// Tile height of the single-grid launches: the caller's, or the default (4 blocks of 7 rows)
// lowered for grids too small to give every resident CTA a tile (about 3 per SM), down to one
// block: a 512^2 grid then has 4 x 74 tiles instead of 4 x 19.  Results do not depend on it.
int tile_height(const fg2_sim *s)
{
  if (s->nb > 0) return s->nb;
  static int sms = 0;  // SMs of the first device seen (the same on every GPU of a node)
  if (!sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms < 1)
      sms = 148;
  }
  const int want = 3 * sms;
  int nb = TILE_BLOCKS_DEFAULT;
  while (nb > 1 && substage_tiles(s->L, nb) < want) --nb;
  return nb;
}

StageArgs stage_args(fg2_sim *s, int k, double dt, const double *dt_dev)
{
  StageArgs a;
  a.beta = RK_BETA[k];
  a.gamma = RK_GAMMA[k];
  a.dt = dt;
  a.dt_dev = dt_dev;
  a.delta1 = s->delta1;
  a.delta2 = s->delta2;
  a.para = s->para;
  a.p1 = s->p1;
  a.p2 = s->p2;
  a.status = s->status;
  a.wait_test_bytes = s->wait_test_bytes;
  a.nb = tile_height(s);
  a.tail = s->tail;
  a.max_ctas = s->max_ctas;
  return a;
}

const DevCode *dev_code_at(const fg2_sim *s, int k)
{
  if (!s->dev_storage) return nullptr;
  s->devk[k] = s->dev;
  s->devk[k].r = s->r[k];
  s->devk[k].r_out = s->r[1 - k];
  return &s->devk[k];
}

const DevCode *dev_code(const fg2_sim *s) { return dev_code_at(s, s->cur); }

// The two ping-pong descriptors (boundaries and Delta as configured); uploaded before any
// capture, since every path that launches a substage calls this first.
int ensure_descs(fg2_sim *s)
{
  if (s->desc_valid) return FG2_OK;
  for (int k = 0; k < 2; ++k)
    if (make_grid_desc(&s->desc_host[k], s->u[k], s->u[1 - k], s->v, s->L, s->storage, s->p1, s->p2, s->delta1,
                       s->delta2, nullptr, s->status, 0, dev_code_at(s, k)) != CUDA_SUCCESS)
      return fail(FG2_ERR_TMA, "cuTensorMapEncodeTiled failed");
  CK(cudaMemcpyAsync(s->desc, s->desc_host, 2 * sizeof(GridDesc), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->desc_valid = true;
  return FG2_OK;
}

// One substage of the state u[cur] into u[1 - cur] (kick: v only).
int launch_stage(fg2_sim *s, int kind, bool cfl, const StageArgs &a, const GridDesc *desc)
{
  StageArgs b = a;
  b.reverse = s->order;
  s->order ^= 1;
  CK(launch_substage(s->storage, kind, cfl, false, desc, 1, substage_tiles(s->L, b.nb, 0, b.tail), b, s->queue,
                             s->stream));
  return FG2_OK;
}


int ensure_config(fg2_sim *s)
{
  if (!s->configured) {
    const int p1 = s->p1, p2 = s->p2;
    if (s->storage == ST_F64) scheme::settings<double>(s->n1, s->n2, s->l1, s->l2, s->p1, s->p2);
    else scheme::settings<float>(s->n1, s->n2, s->l1, s->l2, s->p1, s->p2);
    if (s->p1 != p1 || s->p2 != p2) {  // a scheme that fixes its boundaries (src/config.cpp:26)
      s->ghosts_valid = false;
      drop_graph(s);
    }
    compute_deltas(s);
    s->configured = true;
  }
  return FG2_OK;
}

int do_bcond(fg2_sim *s)
{
  CK(launch_bcond(s->storage, s->u[s->cur], s->L, s->p1, s->p2, s->stream));
  // 16-bit storage: the residual's ghost cells image the same cells (the stencil reads T = S - e)
  if (s->dev_storage) CK(launch_bcond(resid_storage(s->storage), s->r[s->cur], s->L, s->p1, s->p2, s->stream));
  s->ghosts_valid = true;
  return FG2_OK;
}

int do_euler(fg2_sim *s, double dt)
{
  if (s->dev_storage) return fail(FG2_ERR_UNSUPPORTED, "the Euler hook needs FP32 or FP64 storage");
  if (!s->fixed_phases) {  // the reference's RANDOMIZE: two phases per Euler call
    s->r1 = (float)(6.2831853071795865 * s->forcing.uniform());
    s->r2 = (float)(6.2831853071795865 * s->forcing.uniform());
  }
  CK(launch_euler(s->storage, s->u[s->cur], s->L, dt, s->para, s->delta1, s->delta2, s->r1, s->r2, s->stream));
  s->ghosts_valid = false;
  s->smax_valid = false;
  return FG2_OK;
}

bool euler_active(const fg2_sim *s)
{
  Para<double> p;
  for (int q = 0; q < NPARA; ++q) p.v[q] = s->para[q];
  return scheme::euler_active<double>(p);
}

// One RK3 step: Euler hook, three fused substages.  dt_dev != null: device-resident dt.
int enqueue_step(fg2_sim *s, double dt, const double *dt_dev, bool cfl)
{
  int rc0 = ensure_descs(s);
  if (rc0) return rc0;
  if (euler_active(s)) {
    int rc = do_euler(s, dt);
    if (rc) return rc;
  }
  if (!s->ghosts_valid) {
    int rc = do_bcond(s);
    if (rc) return rc;
  }
  for (int k = 0; k < 3; ++k) {
    const StageArgs a = stage_args(s, k, dt, dt_dev);
    const int kind = k == 0 ? STAGE_FIRST : k == 1 ? STAGE_MID : STAGE_LAST;
    int rc = launch_stage(s, kind, cfl && k == 2, a, s->desc + s->cur);
    if (rc) return rc;
    s->cur = 1 - s->cur;
  }
  s->ghosts_valid = true;
  s->smax_valid = cfl;
  return FG2_OK;
}

double diffusive_dt(const fg2_sim *s)
{
  const double D = scheme::max_diffusivity(s->para);
  if (D <= 0.0) return 0.0;
  return s->c * RK3_REAL_LIMIT /
         (D * D2_SYMBOL * (1.0 / (s->delta1 * s->delta1) + 1.0 / (s->delta2 * s->delta2)));
}

int read_status(fg2_sim *s)
{
  CK(cudaMemcpyAsync(s->status_host, s->status, sizeof(Status), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  // a signal max folded into a stage that gave up or produced a NaN is not the state's
  if (s->status_host->error || s->status_host->nan) s->smax_valid = false;
  if (s->status_host->error) return fail(FG2_ERR_TIMEOUT, "a bounded in-kernel wait gave up (bits %u)", s->status_host->error);
  if (s->status_host->nan) return fail(FG2_ERR_NAN, "NaN in the state");
  return FG2_OK;
}

// Deviation storage: the codes of a host state (float, n1 x n2 x NVAR): per-field mean as
// background (0 for fields a reflecting wall negates), per 64 x 64 tile the largest
// deviation as scale (1 where the tile equals the background).  Uploaded to the device.
int set_codes(fg2_sim *s, const float *x)
{
  const int nv = scheme::NVAR, T = SCALE_TILE;
  for (int f = 0; f < 4; ++f) s->dev.bg[f] = 0.f;
  for (int f = 0; f < nv; ++f) {
    if (scheme::reflect_sign(f) < 0) continue;
    double sum = 0.0;
    for (size_t c = 0; c < (size_t)s->n1 * s->n2; ++c) sum += x[c * nv + f];
    s->dev.bg[f] = (float)(sum / ((double)s->n1 * s->n2));
  }
  std::vector<float4> sc((size_t)s->tiles1 * s->tiles2), iv(sc.size());
  for (int ti = 0; ti < s->tiles1; ++ti)
    for (int tj = 0; tj < s->tiles2; ++tj) {
      float m[4] = {0.f, 0.f, 0.f, 0.f};
      for (int i = ti * T; i < std::min(s->n1, (ti + 1) * T); ++i)
        for (int j = tj * T; j < std::min(s->n2, (tj + 1) * T); ++j)
          for (int f = 0; f < nv; ++f) m[f] = std::max(m[f], std::fabs(x[((size_t)i * s->n2 + j) * nv + f] - s->dev.bg[f]));
      for (int f = 0; f < 4; ++f)
        if (!(m[f] > 0.f) || !std::isfinite(m[f])) m[f] = 1.f;
      const size_t t = (size_t)ti * s->tiles2 + tj;
      sc[t] = make_float4(m[0], m[1], m[2], m[3]);
      iv[t] = make_float4(1.f / m[0], 1.f / m[1], 1.f / m[2], 1.f / m[3]);
    }
  CK(cudaMemcpyAsync(s->scale_dev, sc.data(), sc.size() * sizeof(float4), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->inv_dev, iv.data(), iv.size() * sizeof(float4), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  drop_graph(s);  // descriptors carry the background
  return FG2_OK;
}

// Deviation storage: host float cells <-> 16-bit device array through an FP32 device copy.
// The state u is coded with new codes on upload; v is plain 16-bit.
int transfer_dev(fg2_sim *s, void *dev_array, void *host, bool to_device)
{
  const bool is_u = dev_array != s->v;
  const size_t n = (size_t)s->n1 * s->n2 * scheme::NVAR;
  float *tmp = nullptr;
  CK(cudaMalloc(&tmp, n * sizeof(float)));
  std::unique_ptr<float, cudaError_t (*)(void *)> hold(tmp, cudaFree);
  if (to_device && is_u) {  // an upload of the state sets the background and scales first
    int rc = set_codes(s, (const float *)host);
    if (rc) return rc;
  }
  // the codes of the parity transferred, with its residual array
  const DevCode *dc = is_u ? dev_code_at(s, dev_array == s->u[0] ? 0 : 1) : nullptr;
  if (to_device) {
    CK(cudaMemcpyAsync(tmp, host, n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    CK(launch_encode(s->storage, dev_array, tmp, s->L, dc, s->stream));
  } else {
    CK(launch_decode(s->storage, tmp, dev_array, s->L, dc, s->stream));
    CK(cudaMemcpyAsync(host, tmp, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

// host array (rows of n2 cells x NVAR values) <-> device layout.  The device rows hold the
// same interleaved cells as the host rows, so a transfer is one strided 2D copy.
int transfer(fg2_sim *s, void *dev_array, void *host, bool to_device)
{
  if (s->dev_storage) return transfer_dev(s, dev_array, host, to_device);
  const size_t elem = elem_size(s->storage);
  if (host_elem(s->storage) != elem) return fail(FG2_ERR_UNSUPPORTED, "storage %d has no host transfer", s->storage);
  const size_t hrow = (size_t)s->n2 * scheme::NVAR * elem, drow = (size_t)s->L.RS * elem;
  char *d0 = (char *)dev_array + (size_t)s->L.at(0, 0, 0) * elem;
  if (to_device)
    CK(cudaMemcpy2DAsync(d0, drow, host, hrow, hrow, (size_t)s->n1, cudaMemcpyHostToDevice, s->stream));
  else
    CK(cudaMemcpy2DAsync(host, hrow, d0, drow, hrow, (size_t)s->n1, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

// Settings changed: the captured graphs and the descriptors are rebuilt on next use.
void drop_graph(fg2_sim *s)
{
  s->desc_valid = false;
  s->smax_valid = false;  // the signal max depends on the parameters, box and spacings too
  ++s->version;
  for (int b = 0; b < 2; ++b) {
    if (s->graph[b]) cudaGraphExecDestroy(s->graph[b]);
    s->graph[b] = nullptr;
  }
}

}  // namespace rt
}  // namespace fg2

using namespace fg2::rt;

extern "C" {

const char *fg2_scheme_name(void) { return scheme::NAME; }
int fg2_nvar(void) { return scheme::NVAR; }
const char *fg2_field_name(int f) { return (f >= 0 && f < scheme::NVAR) ? scheme::FIELD_NAMES[f] : nullptr; }
int fg2_eqns_flop(void) { return scheme::EQNS_FLOP; }
int fg2_para_count(void) { return scheme::NSLOT; }
const char *fg2_para_key(int k) { return (k >= 0 && k < scheme::NSLOT) ? scheme::PARA_KEYS[k].name : nullptr; }
const char *fg2_last_error(void) { return g_err; }
int fg2_tile_bands(int n1, int nb, int tail, int reverse, int *out, int cap)
{
  return tile_bands(n1, nb, tail, reverse, out, out ? cap : 0);
}

int fg2_setup_evaluate(const char *name, int n1, int n2, double l1, double l2, const double *para, uint64_t seed,
                       int storage, double *out)
{
  if (!name || !out || n1 < 1 || n2 < 1) return fail(FG2_ERR_ARG, "bad arguments");
  const bool single = storage != ST_F64;
  double p[NPARA] = {};
  for (int q = 0; q < scheme::NSLOT; ++q) {
    const double v = para ? para[q] : scheme::PARA_KEYS[q].def;
    p[scheme::PARA_KEYS[q].slot] = single ? (double)(float)v : v;  // parameters in R (src/para.cpp:34)
  }
  scheme::derive(p);
  int p1 = BC_PERIODIC, p2 = BC_PERIODIC;
  if (single) {  // the box in R, as fg2_sim_set_box keeps it for an FP32 state
    l1 = (double)(float)l1;
    l2 = (double)(float)l2;
    scheme::settings<float>(n1, n2, l1, l2, p1, p2);
  } else {
    scheme::settings<double>(n1, n2, l1, l2, p1, p2);
  }
  SetupCtx ctx{n1, n2, l1, l2, p, seed, single};
  std::unique_ptr<Setup> setup = scheme::pick(name, ctx);
  const size_t row = (size_t)n2 * scheme::NVAR;
  for (int i = 0; i < n1; ++i) {
    if (setup) setup->row(i, out + (size_t)i * row);
    else std::memset(out + (size_t)i * row, 0, row * sizeof(double));
  }
  return setup ? 1 : 0;
}

}  // extern "C"

namespace fg2 {
namespace rt {
namespace {

// A handle with the scheme's default parameters and its small device buffers (reduction
// scratch, tile queue, descriptors); the caller sets or allocates the arrays.
fg2_sim *new_handle(int n1, int n2, int storage, cudaStream_t stream, bool own_arrays)
{
  if (n1 < HALF || n2 < HALF) {
    fail(FG2_ERR_ARG, "grid %d x %d is smaller than the ghost width %d", n1, n2, HALF);
    return nullptr;
  }
  if (storage != ST_F32 && storage != ST_F64 && storage != ST_F16 && storage != ST_BF16) {
    fail(FG2_ERR_UNSUPPORTED, "unknown storage %d", storage);
    return nullptr;
  }
  if ((storage == ST_F16 || storage == ST_BF16) && scheme::NVAR > DEV_MAX_FIELDS) {
    fail(FG2_ERR_UNSUPPORTED, "16-bit deviation storage holds at most 4 fields per cell; scheme %s has %d",
         scheme::NAME, scheme::NVAR);
    return nullptr;
  }
  std::unique_ptr<fg2_sim> s(new fg2_sim);
  s->own_arrays = own_arrays;
  s->dev_storage = storage == ST_F16 || storage == ST_BF16;
  s->tiles1 = (n1 + SCALE_TILE - 1) / SCALE_TILE;
  s->tiles2 = (n2 + SCALE_TILE - 1) / SCALE_TILE;
  s->n1 = n1;
  s->n2 = n2;
  s->storage = storage;
  s->L = make_layout(n1, n2, scheme::NVAR);
  for (int q = 0; q < NPARA; ++q) s->para[q] = 0.0;
  for (int q = 0; q < scheme::NSLOT; ++q) s->para[scheme::PARA_KEYS[q].slot] = round_para(s.get(), scheme::PARA_KEYS[q].def);
  scheme::derive(s->para);
  if (stream) {
    s->stream = stream;
  } else {
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      fail(FG2_ERR_ALLOC, "stream creation failed");
      return nullptr;
    }
    s->own_stream = true;
  }
  if (cudaMalloc(&s->sums_partial, sizeof(double) * 4 * sums_blocks(s->L)) != cudaSuccess ||
      cudaMalloc(&s->sums_out, sizeof(double) * 4) != cudaSuccess || cudaMalloc(&s->queue, 2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&s->desc, 3 * sizeof(GridDesc)) != cudaSuccess ||
      cudaMemsetAsync(s->queue, 0, 2 * sizeof(int), s->stream) != cudaSuccess ||
      (s->dev_storage && (cudaMalloc(&s->scale_dev, sizeof(float4) * s->tiles1 * s->tiles2) != cudaSuccess ||
                          cudaMalloc(&s->inv_dev, sizeof(float4) * s->tiles1 * s->tiles2) != cudaSuccess))) {
    fail(FG2_ERR_ALLOC, "device allocation of the handle's buffers failed");
    fg2_sim_destroy(s.release());
    return nullptr;
  }
  if (s->dev_storage) {
    for (int f = 0; f < 4; ++f) s->dev.bg[f] = 0.f;
    s->dev.scale = s->scale_dev;
    s->dev.inv = s->inv_dev;
    s->dev.tiles2 = s->tiles2;
    const std::vector<float4> one((size_t)s->tiles1 * s->tiles2, make_float4(1.f, 1.f, 1.f, 1.f));
    if (cudaMemcpy(s->scale_dev, one.data(), one.size() * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->inv_dev, one.data(), one.size() * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess) {
      fail(FG2_ERR_ALLOC, "scale initialisation failed");
      fg2_sim_destroy(s.release());
      return nullptr;
    }
  }
  return s.release();
}

}  // namespace

fg2_sim *sim_create_in(int n1, int n2, int storage, cudaStream_t stream, void *u0, void *u1, void *v, void *r0,
                       void *r1, Status *status, Status *status_host)
{
  fg2_sim *s = new_handle(n1, n2, storage, stream, false);
  if (!s) return nullptr;
  s->u[0] = u0;
  s->u[1] = u1;
  s->v = v;
  s->status = status;
  s->status_host = status_host;
  if (s->dev_storage) {
    s->r[0] = r0;
    s->r[1] = r1;
  }
  return s;
}

int arrays_per_sim(int storage) { return storage == ST_F16 || storage == ST_BF16 ? 5 : 3; }

}  // namespace rt
}  // namespace fg2

extern "C" {

fg2_sim *fg2_sim_create(int n1, int n2, int storage, void *stream)
{
  std::unique_ptr<fg2_sim, void (*)(fg2_sim *)> s(new_handle(n1, n2, storage, (cudaStream_t)stream, true),
                                                  fg2_sim_destroy);
  if (!s) return nullptr;
  const size_t bytes = array_elems(s.get()) * elem_size(storage);
  if (cudaMalloc(&s->u[0], bytes) != cudaSuccess || cudaMalloc(&s->u[1], bytes) != cudaSuccess ||
      cudaMalloc(&s->v, bytes) != cudaSuccess ||
      (s->dev_storage && (cudaMalloc(&s->r[0], bytes) != cudaSuccess || cudaMalloc(&s->r[1], bytes) != cudaSuccess))) {
    fail(FG2_ERR_ALLOC, "device allocation of the state failed");
    return nullptr;
  }
  if (cudaMalloc(&s->status, sizeof(Status)) != cudaSuccess ||
      cudaMallocHost(&s->status_host, sizeof(Status)) != cudaSuccess) {
    fail(FG2_ERR_ALLOC, "status allocation failed");
    return nullptr;
  }
  // every array starts at -max like the reference (src/setup.cpp:80-83)
  const double lowest = storage == ST_F64 ? -std::numeric_limits<double>::max() : -std::numeric_limits<float>::max();
  if (launch_fill(storage, s->u[0], array_elems(s.get()), lowest, s->stream) != cudaSuccess ||
      launch_fill(storage, s->u[1], array_elems(s.get()), lowest, s->stream) != cudaSuccess ||
      launch_fill(storage, s->v, array_elems(s.get()), lowest, s->stream) != cudaSuccess ||
      (s->r[0] && cudaMemsetAsync(s->r[0], 0, bytes, s->stream) != cudaSuccess) ||
      (s->r[1] && cudaMemsetAsync(s->r[1], 0, bytes, s->stream) != cudaSuccess) ||
      cudaMemsetAsync(s->status, 0, sizeof(Status), s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess) {
    fail(FG2_ERR_ALLOC, "initial fill failed");
    return nullptr;
  }
  return s.release();
}

void fg2_sim_destroy(fg2_sim *s)
{
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  if (s->own_arrays) {
    cudaFree(s->u[0]);
    cudaFree(s->u[1]);
    cudaFree(s->v);
    cudaFree(s->r[0]);
    cudaFree(s->r[1]);
    cudaFree(s->status);
    cudaFreeHost(s->status_host);
  }
  cudaFree(s->sums_partial);
  cudaFree(s->sums_out);
  cudaFree(s->queue);
  cudaFree(s->desc);
  cudaFree(s->scale_dev);
  cudaFree(s->inv_dev);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

size_t fg2_sim_device_bytes(const fg2_sim *s)
{
  return s ? arrays_per_sim(s->storage) * array_elems(s) * elem_size(s->storage) : 0;
}
int fg2_sim_storage(const fg2_sim *s) { return s ? s->storage : -1; }

int fg2_sim_set_box(fg2_sim *s, double l1, double l2)
{
  if (!s || !(l1 > 0) || !(l2 > 0)) return fail(FG2_ERR_ARG, "box sizes must be positive");
  s->l1 = round_para(s, l1);
  s->l2 = round_para(s, l2);
  s->configured = false;
  drop_graph(s);
  return FG2_OK;
}

int fg2_sim_set_tiling(fg2_sim *s, int nb)
{
  if (!s || nb < 0 || nb > 64) return fail(FG2_ERR_ARG, "bad tile height %d", nb);
  if (nb != s->nb) drop_graph(s);
  s->nb = nb;
  return FG2_OK;
}

int fg2_sim_set_occupancy(fg2_sim *s, int ctas_per_sm)
{
  if (!s || ctas_per_sm < 0 || ctas_per_sm > 64) return fail(FG2_ERR_ARG, "bad occupancy %d", ctas_per_sm);
  if (ctas_per_sm != s->max_ctas) drop_graph(s);
  s->max_ctas = ctas_per_sm;
  return FG2_OK;
}

int fg2_sim_set_tail(fg2_sim *s, int tail)
{
  if (!s || tail < 0 || tail > 64) return fail(FG2_ERR_ARG, "bad tail band count %d", tail);
  if (tail != s->tail) drop_graph(s);
  s->tail = tail;
  return FG2_OK;
}

int fg2_sim_get_tail(const fg2_sim *s, int *tail)
{
  if (!s || !tail) return fail(FG2_ERR_ARG, "null argument");
  *tail = s->tail;
  return FG2_OK;
}

int fg2_sim_get_tiling(const fg2_sim *s, int *nb, int *ctas_per_sm)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  if (nb) *nb = tile_height(s);
  if (ctas_per_sm) *ctas_per_sm = s->max_ctas;
  return FG2_OK;
}

int fg2_sim_autotune(fg2_sim *s, int reps, double *best_ms)
{
  if (!s || reps < 1) return fail(FG2_ERR_ARG, "bad arguments");
  ensure_config(s);
  struct Cand {
    int nb, ctas, tail;
    double ms;
  };
  std::vector<Cand> cands;
  // tile height nb blocks of 7 rows; CTAs per SM: 0 = as many as fit, or 4, 8, 12 warps;
  // one-block tail bands: none, 1 or 3 (a tail only changes grids with more than one band)
  for (int nb : {1, 2, 3, 4, 5, 6, 8})
    for (int warps : {0, 4, 8, 12})
      for (int tail : {0, 1, 3})
        if (tail == 0 || (nb > 1 && substage_tiles(s->L, nb, 0, tail) != substage_tiles(s->L, nb)))
          cands.push_back({nb, warps * 32 / STRIP_DEFAULT, tail, 0.0});
  const int keep_nb = s->nb, keep_ctas = s->max_ctas, keep_tail = s->tail, keep_cur = s->cur;
  const bool keep_ghosts = s->ghosts_valid, keep_smax = s->smax_valid;
  // 16-bit storage: a step of dt = 0 re-encodes the state and its rounding residual, so
  // the state and the residual are kept aside and put back afterwards
  const size_t bytes = array_elems(s) * elem_size(s->storage);
  void *keep = nullptr;
  if (s->dev_storage) {
    CK(cudaMalloc(&keep, 2 * bytes));
    CK(cudaMemcpyAsync(keep, s->u[s->cur], bytes, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync((char *)keep + bytes, s->r[keep_cur], bytes, cudaMemcpyDeviceToDevice, s->stream));
  }
  std::unique_ptr<void, cudaError_t (*)(void *)> hold(keep, cudaFree);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto measure = [&](Cand &c) -> int {
    s->nb = c.nb;
    s->max_ctas = c.ctas;
    s->tail = c.tail;
    int r = FG2_OK;
    // two untimed steps, then 2 reps timed (dt = 0: u' = u + 0 v, bitwise)
    for (int q = 0; q < 2 && r == 0; ++q) r = enqueue_step(s, 0.0, nullptr, false);
    if (r) return r;
    if (cudaEventRecord(e0, s->stream) != cudaSuccess) return fail(FG2_ERR_ARG, "event record failed");
    for (int q = 0; q < 2 * reps && r == 0; ++q) r = enqueue_step(s, 0.0, nullptr, false);
    if (r) return r;
    float ms = 0.f;
    if (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return fail(FG2_ERR_ARG, "autotune timing failed");
    c.ms = ms / (2.0 * reps);
    return FG2_OK;
  };
  // the default tiling first: a step shorter than LAUNCH_BOUND_MS is bound by launch latency,
  // which no tiling changes and which hides the kernel's own time, so such grids keep the
  // default (its small-grid rule gives every resident CTA a tile)
  constexpr double LAUNCH_BOUND_MS = 0.05;
  Cand dflt{0, 0, 0, 0.0};
  int rc = measure(dflt);
  const bool launch_bound = rc == 0 && dflt.ms < LAUNCH_BOUND_MS;
  if (launch_bound) cands.assign(1, dflt);
  for (size_t i = 0; i < cands.size() && rc == 0 && !launch_bound; ++i) rc = measure(cands[i]);
  if (rc == 0 && !launch_bound) {  // the three best again, each scored by its faster measurement
    std::sort(cands.begin(), cands.end(), [](const Cand &x, const Cand &y) { return x.ms < y.ms; });
    for (size_t i = 0; i < 3 && i < cands.size() && rc == 0; ++i) {
      const double first = cands[i].ms;
      rc = measure(cands[i]);
      cands[i].ms = std::min(first, cands[i].ms);
    }
    std::sort(cands.begin(), cands.end(), [](const Cand &x, const Cand &y) { return x.ms < y.ms; });
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (keep) {
    CK(cudaMemcpyAsync(s->u[keep_cur], keep, bytes, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->r[keep_cur], (char *)keep + bytes, bytes, cudaMemcpyDeviceToDevice, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  // every stage of dt = 0 copied the state bitwise into the array it wrote, ghost images
  // included, so both arrays hold it; 16-bit storage got its own arrays back
  s->cur = keep_cur;
  s->ghosts_valid = s->dev_storage ? keep_ghosts : true;
  s->smax_valid = keep_smax;  // the state is unchanged
  s->nb = rc ? keep_nb : cands[0].nb;
  s->max_ctas = rc ? keep_ctas : cands[0].ctas;
  s->tail = rc ? keep_tail : cands[0].tail;
  drop_graph(s);
  if (rc) return rc;
  if (best_ms) *best_ms = cands[0].ms;
  return read_status(s);
}

int fg2_sim_set_courant(fg2_sim *s, double c)
{
  if (!s || !(c > 0)) return fail(FG2_ERR_ARG, "Courant number must be positive");
  s->c = round_para(s, c);
  drop_graph(s);
  return FG2_OK;
}

int fg2_sim_set_bcond(fg2_sim *s, int p1, int p2)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  s->p1 = p1 ? BC_PERIODIC : BC_WALL;
  s->p2 = p2 ? BC_PERIODIC : BC_WALL;
  s->ghosts_valid = false;
  drop_graph(s);
  return FG2_OK;
}

const char *fg2_sim_para(fg2_sim *s, const char *in)
{
  if (!s || !in) return nullptr;
  while (*in == '-') ++in;  // skip leading dashes (src/para.cpp:30)
  const char *eq = std::strchr(in, '=');
  if (!eq) { fail(FG2_ERR_ARG, "expected key=val"); return nullptr; }
  const std::string key(in, eq - in);
  for (int q = 0; q < scheme::NSLOT; ++q)
    if (key == scheme::PARA_KEYS[q].name) {
      const double val = round_para(s, std::atof(eq + 1));
      s->para[scheme::PARA_KEYS[q].slot] = val;
      scheme::derive(s->para);
      snprintf(s->para_msg, sizeof(s->para_msg), "%s = %g", key.c_str(), val);
      drop_graph(s);
      return s->para_msg;
    }
  fail(FG2_ERR_ARG, "unknown parameter '%s' for scheme %s", key.c_str(), scheme::NAME);
  return nullptr;
}

int fg2_sim_get_para(const fg2_sim *s, const char *key, double *val)
{
  if (!s || !key || !val) return fail(FG2_ERR_ARG, "null argument");
  for (int q = 0; q < scheme::NSLOT; ++q)
    if (!std::strcmp(key, scheme::PARA_KEYS[q].name)) {
      *val = s->para[scheme::PARA_KEYS[q].slot];
      return FG2_OK;
    }
  return fail(FG2_ERR_ARG, "unknown parameter '%s'", key);
}

int fg2_sim_config(fg2_sim *s)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  s->configured = false;
  drop_graph(s);
  return ensure_config(s);
}

int fg2_sim_init(fg2_sim *s, const char *name, uint64_t seed)
{
  if (!s || !name) return fail(FG2_ERR_ARG, "null argument");
  ensure_config(s);
  SetupCtx ctx{s->n1, s->n2, s->l1, s->l2, s->para, seed, s->storage != ST_F64};
  std::unique_ptr<Setup> setup = scheme::pick(name, ctx);
  const size_t ncell = (size_t)s->n2 * scheme::NVAR;
  std::vector<double> row(ncell, 0.0);
  const bool hd = s->storage == ST_F64;
  std::vector<unsigned char> host((size_t)s->n1 * ncell * host_elem(s->storage));
  for (int i = 0; i < s->n1; ++i) {
    if (setup) setup->row(i, row.data());
    if (hd) std::memcpy(host.data() + (size_t)i * ncell * 8, row.data(), ncell * 8);
    else {
      float *h = (float *)host.data() + (size_t)i * ncell;
      for (size_t k = 0; k < ncell; ++k) h[k] = (float)row[k];
    }
  }
  return fg2_sim_upload(s, host.data());
}

int fg2_sim_upload(fg2_sim *s, const void *host)
{
  if (!s || !host) return fail(FG2_ERR_ARG, "null argument");
  int rc = transfer(s, s->u[s->cur], const_cast<void *>(host), true);
  s->ghosts_valid = false;
  s->smax_valid = false;
  return rc;
}

int fg2_sim_download(fg2_sim *s, void *host)
{
  if (!s || !host) return fail(FG2_ERR_ARG, "null argument");
  return transfer(s, s->u[s->cur], host, false);
}

int fg2_sim_upload_v(fg2_sim *s, const void *host)
{
  if (!s || !host) return fail(FG2_ERR_ARG, "null argument");
  return transfer(s, s->v, const_cast<void *>(host), true);
}

int fg2_sim_download_v(fg2_sim *s, void *host)
{
  if (!s || !host) return fail(FG2_ERR_ARG, "null argument");
  return transfer(s, s->v, host, false);
}

int fg2_sim_set_dt_mode(fg2_sim *s, int mode)
{
  if (!s || (mode != FG2_DT_REFERENCE && mode != FG2_DT_CFL)) return fail(FG2_ERR_ARG, "bad dt mode");
  s->dt_mode = mode;
  return FG2_OK;
}

double fg2_sim_getdt(fg2_sim *s)
{
  if (!s) return 0.0;
  ensure_config(s);
  if (s->dt_mode == FG2_DT_REFERENCE) {
    // (E)c / (n1 / l1 + n2 / l2) with the quotients in R (src/getdt.cpp:26)
    if (s->storage == ST_F64) return s->c / (s->n1 / s->l1 + s->n2 / s->l2);
    const float den = (float)s->n1 / (float)s->l1 + (float)s->n2 / (float)s->l2;
    return (double)(float)s->c / (double)den;
  }
  // the last step() already took the signal max of the current state in its last stage;
  // otherwise (after an upload, a user drift, a fixed-dt run) one reduction pass takes it
  const bool reduce = !s->smax_valid;
  if ((reduce && (cudaMemsetAsync(&s->status->smax, 0, sizeof(unsigned long long), s->stream) != cudaSuccess ||
                  launch_signal_max(s->storage, s->u[s->cur], s->L, s->para, s->delta1, s->delta2, s->status,
                                    s->stream, dev_code(s)) != cudaSuccess)) ||
      cudaMemcpyAsync(s->status_host, s->status, sizeof(Status), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess) {
    fail(FG2_ERR_ARG, "getdt reduction failed");
    return 0.0;
  }
  s->smax_valid = true;
  unsigned long long bits = s->status_host->smax;
  double smax;
  std::memcpy(&smax, &bits, sizeof(smax));
  double dt = smax > 0 ? s->c / smax : std::numeric_limits<double>::infinity();
  const double dd = diffusive_dt(s);
  if (dd > 0 && dd < dt) dt = dd;
  return dt;
}

int fg2_sim_step(fg2_sim *s, double t, double dt)
{
  (void)t;  // passed to the equations by the reference but unused by them (src/kick.cu:98)
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  ensure_config(s);
  // with CFL time steps the last stage also takes the signal max of the new state, which the
  // next getdt() reads instead of a separate reduction pass
  const bool cfl = s->dt_mode != FG2_DT_REFERENCE;
  if (cfl) CK(cudaMemsetAsync(&s->status->smax, 0, sizeof(unsigned long long), s->stream));
  int rc = enqueue_step(s, dt, nullptr, cfl);
  if (rc) return rc;
  return read_status(s);
}

int fg2_sim_advance(fg2_sim *s, int nsteps, double dt, double t_end)
{
  if (!s || nsteps < 0) return fail(FG2_ERR_ARG, "bad arguments");
  ensure_config(s);
  const bool device_dt = !(dt > 0);
  if (device_dt && !s->smax_valid) {
    CK(cudaMemsetAsync(&s->status->smax, 0, sizeof(unsigned long long), s->stream));
    CK(launch_signal_max(s->storage, s->u[s->cur], s->L, s->para, s->delta1, s->delta2, s->status, s->stream,
                         dev_code(s)));
    s->smax_valid = true;
  }
  for (int n = 0; n < nsteps; ++n) {
    if (device_dt) CK(launch_dt_update(s->status, s->c, diffusive_dt(s), t_end, s->stream));
    int rc = enqueue_step(s, dt, device_dt ? &s->status->dt : nullptr, device_dt);
    if (rc) return rc;
  }
  return FG2_OK;
}

int fg2_sim_advance_graph(fg2_sim *s, int nsteps, double dt, double t_end)
{
  if (!s || nsteps < 0) return fail(FG2_ERR_ARG, "bad arguments");
  if (euler_active(s) && !s->fixed_phases)
    return fail(FG2_ERR_UNSUPPORTED, "per-step random forcing phases cannot be replayed from a graph");
  ensure_config(s);
  const bool device_dt = !(dt > 0);
  // bring the state to a point every replay starts from: valid ghosts and signal max
  if (!s->ghosts_valid || euler_active(s)) {
    int rc = fg2_sim_advance(s, 1, dt, t_end);
    if (rc) return rc;
    --nsteps;
  }
  if (device_dt && !s->smax_valid) {
    int rc = fg2_sim_advance(s, 1, dt, t_end);
    if (rc) return rc;
    --nsteps;
  }
  if (nsteps <= 0) return FG2_OK;
  int rcd = ensure_descs(s);
  if (rcd) return rcd;
  const int b = s->cur;
  if (s->graph[b] && (s->graph_dt[b] != dt || s->graph_tend[b] != t_end)) {
    cudaGraphExecDestroy(s->graph[b]);
    s->graph[b] = nullptr;
  }
  if (!s->graph[b]) {
    // two steps = six substages: the ping-pong parity returns to the start
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = fg2_sim_advance(s, 2, dt, t_end);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) return rc;
    CK(e);
    e = cudaGraphInstantiate(&s->graph[b], g, 0);
    cudaGraphDestroy(g);
    CK(e);
    s->graph_dt[b] = dt;
    s->graph_tend[b] = t_end;
  }
  for (int n = 0; n + 1 < nsteps; n += 2) CK(cudaGraphLaunch(s->graph[b], s->stream));
  if (nsteps & 1) return fg2_sim_advance(s, 1, dt, t_end);
  return FG2_OK;
}

int fg2_sim_stage(fg2_sim *s, int k, double dt)
{
  if (!s || k < 0 || k > 2) return fail(FG2_ERR_ARG, "bad arguments");
  ensure_config(s);
  if (!s->ghosts_valid) {
    int rc = do_bcond(s);
    if (rc) return rc;
  }
  int rc = ensure_descs(s);
  if (rc) return rc;
  const StageArgs a = stage_args(s, k, dt, nullptr);
  const int kind = k == 0 ? STAGE_FIRST : k == 1 ? STAGE_MID : STAGE_LAST;
  rc = launch_stage(s, kind, false, a, s->desc + s->cur);
  if (rc) return rc;
  s->cur = 1 - s->cur;
  s->smax_valid = false;
  return FG2_OK;
}

int fg2_sim_sync(fg2_sim *s)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  return read_status(s);
}

int fg2_sim_set_time(fg2_sim *s, double t)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  CK(cudaMemcpyAsync(&s->status->t, &t, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

double fg2_sim_time(fg2_sim *s)
{
  if (!s || read_status(s) < 0) return NAN;
  return s->status_host->t;
}

double fg2_sim_last_dt(fg2_sim *s)
{
  if (!s || read_status(s) < 0) return NAN;
  return s->status_host->dt_next;
}

int fg2_sim_test_stall_waits(fg2_sim *s, int bytes)
{
  if (!s || bytes < 0 || bytes > 4096) return fail(FG2_ERR_ARG, "bad arguments");
  s->wait_test_bytes = (unsigned)bytes;
  drop_graph(s);
  return FG2_OK;
}

void fg2_sim_clear_status(fg2_sim *s)
{
  if (!s) return;
  cudaMemsetAsync(s->status, 0, 2 * sizeof(unsigned), s->stream);
  cudaStreamSynchronize(s->stream);
}

int fg2_sim_kick(fg2_sim *s, double t, double beta)
{
  (void)t;
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  ensure_config(s);
  int rc = ensure_descs(s);
  if (rc) return rc;
  StageArgs a = stage_args(s, 0, 0.0, nullptr);
  a.beta = beta;
  rc = launch_stage(s, STAGE_KICK, false, a, s->desc + s->cur);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

int fg2_sim_drift(fg2_sim *s, double dt)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  if (s->dev_storage) return fail(FG2_ERR_UNSUPPORTED, "drift needs FP32 or FP64 storage");
  const double r = s->storage == ST_F64 ? dt : (double)(float)dt;
  CK(launch_drift(s->storage, s->u[s->cur], s->v, s->L, r, s->status, s->stream));
  s->ghosts_valid = false;
  s->smax_valid = false;
  return read_status(s);
}

int fg2_sim_bcond(fg2_sim *s)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  int rc = do_bcond(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

int fg2_sim_euler(fg2_sim *s, double dt)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  ensure_config(s);
  int rc = do_euler(s, dt);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

int fg2_sim_set_forcing_phases(fg2_sim *s, double r1, double r2)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  s->fixed_phases = true;
  s->r1 = (float)r1;
  s->r2 = (float)r2;
  drop_graph(s);
  return FG2_OK;
}

int fg2_sim_seed_forcing(fg2_sim *s, uint64_t seed)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  s->fixed_phases = false;
  s->forcing = Rng(seed);
  drop_graph(s);
  return FG2_OK;
}

int fg2_sim_sums(fg2_sim *s, double out[4])
{
  if (!s || !out) return fail(FG2_ERR_ARG, "null argument");
  CK(launch_sums(s->storage, s->u[s->cur], s->L, s->sums_partial, s->sums_out, s->stream, dev_code(s)));
  CK(cudaMemcpyAsync(out, s->sums_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FG2_OK;
}

void *fg2_sim_u(fg2_sim *s) { return s ? s->u[s->cur] : nullptr; }
void *fg2_sim_v(fg2_sim *s) { return s ? s->v : nullptr; }
void *fg2_sim_stream(fg2_sim *s) { return s ? (void *)s->stream : nullptr; }

int fg2_sim_layout(const fg2_sim *s, long long *pitch, long long *cell)
{
  if (!s) return fail(FG2_ERR_ARG, "null handle");
  if (pitch) *pitch = s->L.RS;
  if (cell) *cell = s->L.CS;
  return FG2_OK;
}

// .raw frames (src/io.cpp:24-76): int[6] {n1, n2, NVAR, sizeof(R), p1, p2}, E time,
// R[3] {l1, l2, c}, then n1 * n2 * NVAR values of R without ghosts.  E is double for
// R = float and long double for R = double (src/fg2.h:36-45).
int fg2_sim_dump(fg2_sim *s, const char *path, double time)
{
  if (!s || !path) return fail(FG2_ERR_ARG, "null argument");
  const bool hd = s->storage == ST_F64;
  const size_t he = host_elem(s->storage);
  std::vector<unsigned char> data((size_t)s->n1 * s->n2 * scheme::NVAR * he);
  int rc = fg2_sim_download(s, data.data());
  if (rc) return rc;
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(FG2_ERR_ARG, "cannot open %s", path);
  const int size[6] = {s->n1, s->n2, scheme::NVAR, (int)he, s->p1, s->p2};
  bool ok = std::fwrite(size, sizeof(int), 6, f) == 6;
  if (hd) {
    const long double t = time;
    const double info[3] = {s->l1, s->l2, s->c};
    ok = ok && std::fwrite(&t, sizeof(t), 1, f) == 1 && std::fwrite(info, sizeof(double), 3, f) == 3;
  } else {
    const float info[3] = {(float)s->l1, (float)s->l2, (float)s->c};
    ok = ok && std::fwrite(&time, sizeof(double), 1, f) == 1 && std::fwrite(info, sizeof(float), 3, f) == 3;
  }
  ok = ok && std::fwrite(data.data(), 1, data.size(), f) == data.size();
  std::fclose(f);
  return ok ? FG2_OK : fail(FG2_ERR_ARG, "short write to %s", path);
}

int fg2_sim_load(fg2_sim *s, const char *path, double *time)
{
  if (!s || !path) return fail(FG2_ERR_ARG, "null argument");
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(FG2_ERR_ARG, "cannot open %s", path);
  const bool hd = s->storage == ST_F64;
  const size_t he = host_elem(s->storage);
  int size[6];
  bool ok = std::fread(size, sizeof(int), 6, f) == 6;
  // compatibility check of src/io.cpp:32-33
  if (!ok || size[0] != s->n1 || size[1] != s->n2 || size[2] != scheme::NVAR || size[3] != (int)he) {
    std::fclose(f);
    return fail(FG2_ERR_ARG, "input data is not compatible with the setup");
  }
  double t = 0;
  if (hd) {
    long double lt;
    double info[3];
    ok = std::fread(&lt, sizeof(lt), 1, f) == 1 && std::fread(info, sizeof(double), 3, f) == 3;
    t = (double)lt;
    s->l1 = info[0]; s->l2 = info[1]; s->c = info[2];
  } else {
    float info[3];
    ok = std::fread(&t, sizeof(double), 1, f) == 1 && std::fread(info, sizeof(float), 3, f) == 3;
    s->l1 = info[0]; s->l2 = info[1]; s->c = info[2];
  }
  std::vector<unsigned char> data((size_t)s->n1 * s->n2 * scheme::NVAR * he);
  ok = ok && std::fread(data.data(), 1, data.size(), f) == data.size();
  std::fclose(f);
  if (!ok) return fail(FG2_ERR_ARG, "short read from %s", path);
  s->p1 = size[4] ? BC_PERIODIC : BC_WALL;
  s->p2 = size[5] ? BC_PERIODIC : BC_WALL;
  s->configured = false;
  drop_graph(s);
  if (time) *time = t;
  return fg2_sim_upload(s, data.data());
}

// The reference's solve() loop (src/solve.cpp:25-64): frames i+1 .. n evenly spaced up to
// t_final; each frame steps until its time (the last step shortened to land on it) and is
// dumped as <dir>/<frame, 4 digits>.raw (src/misc.cpp:57-62).  The time step is the
// handle's getdt mode: FG2_DT_REFERENCE takes getdt() on the host; FG2_DT_CFL keeps it on the
// device (graph replay, CFL rate folded into the last substage).  A NaN dumps the state as
// <dir>/****.raw and returns FG2_ERR_NAN, as the reference does before it aborts.
int fg2_sim_solve(fg2_sim *s, double t, double t_final, int i, int n, const char *dir, double *ms_per_step)
{
  if (!s || !dir || n <= i || !(t_final > t)) return fail(FG2_ERR_ARG, "bad solve arguments");
  ensure_config(s);
  auto path = [&](const char *leaf) { return std::string(dir) + "/" + leaf; };
  char leaf[64];
  cudaEvent_t c0 = nullptr, c1 = nullptr;
  CK(cudaEventCreate(&c0));
  CK(cudaEventCreate(&c1));
  std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> h0(c0, cudaEventDestroy), h1(c1, cudaEventDestroy);
  long long total_steps = 0;
  float total_ms = 0.f;
  const double dt_dump = (t_final - t) / (n - i);
  int rc = FG2_OK;
  if ((rc = fg2_sim_set_time(s, t)) != FG2_OK) return rc;
  while (i++ < n) {
    const double target = t_final - (n - i) * dt_dump;
    long long m = 0;
    CK(cudaEventRecord(c0, s->stream));
    if (s->dt_mode == FG2_DT_REFERENCE) {
      while (t < target) {
        const double dt = std::min(target - t, fg2_sim_getdt(s));
        if ((rc = fg2_sim_step(s, t, dt)) != FG2_OK) break;
        t = std::min(t + dt, target);
        ++m;
      }
    } else {
      // device-resident steps: the dt update caps the last step at the frame's time; chunks of
      // steps are sized from the last step until the device clock reaches the target
      while (rc == FG2_OK && t < target) {
        const double last = fg2_sim_last_dt(s);
        long long k = last > 0 ? (long long)std::ceil((target - t) / last) : 16;
        k = std::max(1LL, std::min(k, 4096LL));
        rc = fg2_sim_advance_graph(s, (int)k, 0.0, target);
        if (rc == FG2_OK) rc = fg2_sim_sync(s);
        t = fg2_sim_time(s);
        m += k;
        if (t >= target * (1.0 - 1e-15)) t = target;
      }
    }
    CK(cudaEventRecord(c1, s->stream));
    CK(cudaEventSynchronize(c1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c0, c1));
    total_ms += ms;
    total_steps += m;
    if (rc != FG2_OK) {
      fg2_sim_clear_status(s);
      fg2_sim_dump(s, path("****.raw").c_str(), t);
      break;
    }
    snprintf(leaf, sizeof(leaf), "%04d.raw", i);
    if ((rc = fg2_sim_dump(s, path(leaf).c_str(), t)) != FG2_OK) break;
  }
  if (ms_per_step) *ms_per_step = total_steps ? total_ms / total_steps : 0.0;
  return rc;
}

// ---- reference-mirror API over one process-wide simulation ------------------------------
static fg2_sim *g_sim = nullptr;
static void g_done(void) { fg2_sim_destroy(g_sim); g_sim = nullptr; }

fg2_sim *fg2_global(void) { return g_sim; }

size_t fg2_setup(int n1, int n2)
{
  if (g_sim) g_done();
  else std::atexit(g_done);  // the reference frees in an atexit hook (src/setup.cpp:24-34)
  g_sim = fg2_sim_create(n1, n2, ST_F32, nullptr);
  return g_sim ? fg2_sim_device_bytes(g_sim) : 0;
}

void fg2_config(void) { if (g_sim) fg2_sim_config(g_sim); }
const char *fg2_para(const char *in) { return g_sim ? fg2_sim_para(g_sim, in) : nullptr; }
void fg2_init(const char *name) { if (g_sim) fg2_sim_init(g_sim, name, 0); }

double fg2_load(const char *path)
{
  double t = 0;
  if (g_sim) fg2_sim_load(g_sim, path, &t);
  return t;
}

void fg2_dump(const char *path, double time) { if (g_sim) fg2_sim_dump(g_sim, path, time); }
double fg2_getdt(void) { return g_sim ? fg2_sim_getdt(g_sim) : 0.0; }
int fg2_step(double t, double dt) { return g_sim ? fg2_sim_step(g_sim, t, dt) : FG2_ERR_ARG; }

// The process-wide simulation's arrays as the reference's globals hold them: interior-origin
// pointers (element (f, i, j) at p[i * s + j * NVAR + f], ghosts at negative i, j) and the row
// stride s in elements (src/setup.cpp:64-72: global::u = base + HALF (s + NVAR)).  Here the
// interior starts one padding column further in, so the offset is 3 s + 4 NVAR.
static long long interior_offset(const fg2_sim *s) { return s->L.at(0, 0, 0); }
float *fg2_u(void) { return g_sim ? (float *)g_sim->u[g_sim->cur] + interior_offset(g_sim) : nullptr; }
float *fg2_v(void) { return g_sim ? (float *)g_sim->v + interior_offset(g_sim) : nullptr; }
long long fg2_s(void) { return g_sim ? g_sim->L.RS : 0; }

// kick/drift/bcond/Euler take interior-origin device pointers into arrays of the global
// layout, as the reference's do (src/fg2.h:81-84 called with global::u, global::v).
static float *array_base(const float *p) { return const_cast<float *>(p) - interior_offset(g_sim); }

void fg2_kick(float *v, const float *u, float t, float beta)
{
  (void)t;
  if (!g_sim || !v || !u) return;
  ensure_config(g_sim);
  v = array_base(v);
  u = array_base(u);
  // any arrays of the global layout: the descriptor is encoded for these pointers
  GridDesc &d = g_sim->desc_host[2];
  if (make_grid_desc(&d, u, nullptr, v, g_sim->L, g_sim->storage, g_sim->p1, g_sim->p2, g_sim->delta1, g_sim->delta2,
                     nullptr, g_sim->status, 0) != CUDA_SUCCESS) {
    fail(FG2_ERR_TMA, "cuTensorMapEncodeTiled failed");
    return;
  }
  if (cudaMemcpyAsync(g_sim->desc + 2, &d, sizeof(GridDesc), cudaMemcpyHostToDevice, g_sim->stream) != cudaSuccess)
    return;
  StageArgs a = stage_args(g_sim, 0, 0.0, nullptr);
  a.beta = beta;
  launch_stage(g_sim, STAGE_KICK, false, a, g_sim->desc + 2);
  cudaStreamSynchronize(g_sim->stream);
}

void fg2_drift(float *u, const float *v, float dt)
{
  if (!g_sim || !u || !v) return;
  u = array_base(u);
  v = array_base(v);
  launch_drift(g_sim->storage, u, v, g_sim->L, dt, g_sim->status, g_sim->stream);
  if (u == g_sim->u[g_sim->cur]) { g_sim->ghosts_valid = false; g_sim->smax_valid = false; }
  cudaStreamSynchronize(g_sim->stream);
}

void fg2_bcond(float *u, int p1, int p2)
{
  if (!g_sim || !u) return;
  u = array_base(u);
  launch_bcond(g_sim->storage, u, g_sim->L, p1 ? BC_PERIODIC : BC_WALL, p2 ? BC_PERIODIC : BC_WALL, g_sim->stream);
  cudaStreamSynchronize(g_sim->stream);
}

void fg2_Euler(float *u, float dt)
{
  if (!g_sim || !u) return;
  ensure_config(g_sim);
  u = array_base(u);
  if (u == g_sim->u[g_sim->cur]) { g_sim->ghosts_valid = false; g_sim->smax_valid = false; }
  if (!g_sim->fixed_phases) {
    g_sim->r1 = (float)(6.2831853071795865 * g_sim->forcing.uniform());
    g_sim->r2 = (float)(6.2831853071795865 * g_sim->forcing.uniform());
  }
  launch_euler(g_sim->storage, u, g_sim->L, dt, g_sim->para, g_sim->delta1, g_sim->delta2, g_sim->r1, g_sim->r2,
               g_sim->stream);
  cudaStreamSynchronize(g_sim->stream);
}

}  // extern "C"
