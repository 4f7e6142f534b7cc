// fg2_b200/csrc/batch.cpp -- many independent simulations of one scheme advanced together
// (C ABI fg2_batch_*, include/fg2_b200.h).
//
// The reference advances one grid per process (src/main.cpp:81-116, src/solve.cpp:25-64).
// A batch holds count members of any sizes in one device arena and advances all of them with
// one persistent substage launch per RK3 stage: the launch's tile queue runs over the tiles of
// every member (largest members first), each member described by a GridDesc (its tensor maps,
// arrays, boundaries, 1/Delta factors, time step and status block).  Every member is also an
// ordinary simulation handle (fg2_batch_member), so setup, transfers, sums, dumps and
// per-member status use the single-simulation API.  Members share the scheme parameters;
// box, boundaries and Courant number may differ.  With dt <= 0 every member takes its own
// device-resident CFL step, folded into its last substage; two steps are captured as a CUDA
// graph and replayed.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "sim.h"

#include <state.h>
#include <eqns.cuh>
#include <Euler.cuh>

using namespace fg2;
using namespace fg2::rt;

struct fg2_batch {
  int count = 0, storage = ST_F32;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void *arena = nullptr;           // u[0], u[1], v of every member
  size_t arena_bytes = 0;
  Status *status = nullptr;        // device, one per member
  Status *status_host = nullptr;   // pinned mirror
  std::vector<fg2_sim *> members;
  std::vector<int> order;          // members in tile order (smallest at both ends)
  long long cells = 0;
  GridDesc *desc = nullptr;        // device [2][count]: set 0 u[cur] -> u[1-cur], set 1 the reverse
  std::vector<GridDesc> desc_host;
  double2 *limits = nullptr;       // device: {courant, diffusive dt} per member
  std::vector<double2> limits_host;
  int *queue = nullptr;
  int ntiles = 0;
  // what the descriptors were built for
  bool desc_valid = false;
  bool desc_device_dt = false;
  int desc_nb = 0, desc_strip = 0;
  std::vector<unsigned> versions;
  std::vector<int> curs;
  // tiling (autotuned or set)
  int nb = TILE_BLOCKS_DEFAULT, max_ctas = 0, strip = STRIP_DEFAULT;
  int reverse = 0;  // tile order of the next substage launch (alternates)
  // the two-step graph and what it was captured for
  cudaGraphExec_t graph = nullptr;
  double graph_dt = 0, graph_tend = 0;
  int graph_nb = 0, graph_ctas = 0, graph_strip = 0;
  std::vector<double> graph_para;
};

namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

void drop_batch_graph(fg2_batch *b)
{
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

// Every member configured, all with the same scheme parameters (the launch's).
int check_members(fg2_batch *b)
{
  for (fg2_sim *m : b->members) ensure_config(m);
  const fg2_sim *m0 = b->members[0];
  for (fg2_sim *m : b->members)
    if (std::memcmp(m->para, m0->para, sizeof(m0->para)) != 0)
      return fail(FG2_ERR_ARG, "batch members have different scheme parameters");
  return FG2_OK;
}

// Descriptor sets for the members' current parities, tile order and dt mode.
int ensure_batch_descs(fg2_batch *b, bool device_dt)
{
  bool valid = b->desc_valid && b->desc_device_dt == device_dt && b->desc_nb == b->nb && b->desc_strip == b->strip;
  for (int k = 0; valid && k < b->count; ++k)
    valid = b->versions[k] == b->members[k]->version && b->curs[k] == b->members[k]->cur;
  if (valid) return FG2_OK;
  int tile0 = 0;
  for (int r = 0; r < b->count; ++r) {
    const int k = b->order[r];
    fg2_sim *m = b->members[k];
    const double *dt = device_dt ? &b->status[k].dt : nullptr;
    for (int set = 0; set < 2; ++set) {
      const int in = set == 0 ? m->cur : 1 - m->cur;
      if (make_grid_desc(&b->desc_host[(size_t)set * b->count + r], m->u[in], m->u[1 - in], m->v, m->L, m->storage,
                         m->p1, m->p2, m->delta1, m->delta2, dt, &b->status[k], tile0, dev_code_at(m, in),
                         b->strip) != CUDA_SUCCESS)
        return fail(FG2_ERR_TMA, "cuTensorMapEncodeTiled failed for batch member %d", k);
    }
    tile0 += substage_tiles(m->L, b->nb, b->strip);
    b->limits_host[k] = make_double2(m->c, diffusive_dt(m));
    b->versions[k] = m->version;
    b->curs[k] = m->cur;
  }
  b->ntiles = tile0;
  CK(cudaMemcpyAsync(b->desc, b->desc_host.data(), 2 * b->count * sizeof(GridDesc), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->limits, b->limits_host.data(), b->count * sizeof(double2), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  b->desc_valid = true;
  b->desc_device_dt = device_dt;
  b->desc_nb = b->nb;
  b->desc_strip = b->strip;
  return FG2_OK;
}

// One RK3 step of every member; `set` is the descriptor set of the first substage (the
// members' parity relative to the descriptors), flipped by the step.
int enqueue_batch_step(fg2_batch *b, double dt, bool device_dt, double t_end, int &set)
{
  const fg2_sim *m0 = b->members[0];
  if (device_dt) CK(launch_dt_update_batch(b->status, b->limits, b->count, t_end, b->stream));
  for (int k = 0; k < 3; ++k) {
    StageArgs a;
    a.beta = RK_BETA[k];
    a.gamma = RK_GAMMA[k];
    a.dt = device_dt ? 0.0 : dt;
    a.dt_dev = nullptr;
    a.delta1 = 1.0;
    a.delta2 = 1.0;
    a.para = m0->para;
    a.p1 = m0->p1;
    a.p2 = m0->p2;
    a.status = b->status;
    a.nb = b->nb;
    a.max_ctas = b->max_ctas;
    a.strip = b->strip;
    a.reverse = b->reverse;
    b->reverse ^= 1;
    const int kind = k == 0 ? STAGE_FIRST : k == 1 ? STAGE_MID : STAGE_LAST;
    CK(launch_substage(b->storage, kind, device_dt && k == 2, true, b->desc + (size_t)set * b->count, b->count,
                       b->ntiles, a, b->queue, b->stream));
    set = 1 - set;
  }
  return FG2_OK;
}

// Members' bookkeeping after n steps.
void finish_steps(fg2_batch *b, int n, bool device_dt)
{
  if (n <= 0) return;
  for (fg2_sim *m : b->members) {
    if (n & 1) m->cur = 1 - m->cur;
    m->ghosts_valid = true;
    m->smax_valid = device_dt;
  }
}

// Ghost cells and (device dt) signal maxima every step relies on.
int prepare_members(fg2_batch *b, bool device_dt)
{
  for (fg2_sim *m : b->members) {
    if (!m->ghosts_valid) {
      int rc = do_bcond(m);
      if (rc) return rc;
    }
    if (device_dt && !m->smax_valid) {
      CK(cudaMemsetAsync(&m->status->smax, 0, sizeof(unsigned long long), b->stream));
      CK(launch_signal_max(m->storage, m->u[m->cur], m->L, m->para, m->delta1, m->delta2, m->status, b->stream,
                           dev_code(m)));
      m->smax_valid = true;
    }
  }
  return FG2_OK;
}

bool any_euler(const fg2_batch *b)
{
  for (const fg2_sim *m : b->members)
    if (euler_active(m)) return true;
  return false;
}

int advance_plain(fg2_batch *b, int nsteps, double dt, double t_end)
{
  const bool device_dt = !(dt > 0);
  const bool euler = any_euler(b);
  int set = 0, done = 0, rc = 0;
  for (int n = 0; n < nsteps; ++n) {
    if (euler) {  // the operator-split update works on each member's current array
      finish_steps(b, done, device_dt);
      done = 0;
      set = 0;
      for (fg2_sim *m : b->members)
        if (euler_active(m) && (rc = do_euler(m, dt)) != 0) return rc;
    }
    if (n == 0 || euler) {
      if ((rc = prepare_members(b, device_dt)) != 0) return rc;
      if ((rc = ensure_batch_descs(b, device_dt)) != 0) return rc;
    }
    if ((rc = enqueue_batch_step(b, dt, device_dt, t_end, set)) != 0) return rc;
    ++done;
  }
  finish_steps(b, done, device_dt);
  return FG2_OK;
}

}  // namespace

extern "C" {

fg2_batch *fg2_batch_create(int count, const int *n1, const int *n2, int storage, void *stream)
{
  if (count < 1 || !n1 || !n2) {
    fail(FG2_ERR_ARG, "a batch needs at least one member");
    return nullptr;
  }
  if (storage != ST_F32 && storage != ST_F64 && storage != ST_F16 && storage != ST_BF16) {
    fail(FG2_ERR_UNSUPPORTED, "unknown storage %d", storage);
    return nullptr;
  }
  for (int k = 0; k < count; ++k)
    if (n1[k] < HALF || n2[k] < HALF) {
      fail(FG2_ERR_ARG, "member %d: grid %d x %d is smaller than the ghost width %d", k, n1[k], n2[k], HALF);
      return nullptr;
    }
  std::unique_ptr<fg2_batch, void (*)(fg2_batch *)> b(new fg2_batch, fg2_batch_destroy);
  b->count = count;
  b->storage = storage;
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
      fail(FG2_ERR_ALLOC, "stream creation failed");
      return nullptr;
    }
    b->own_stream = true;
  }
  const size_t elem = elem_size(storage);
  std::vector<size_t> bytes(count);
  for (int k = 0; k < count; ++k) {
    const Layout L = make_layout(n1[k], n2[k], scheme::NVAR);
    bytes[k] = align_up((size_t)L.elems() * elem, 256);
    b->arena_bytes += arrays_per_sim(storage) * bytes[k];
    b->cells += (long long)n1[k] * n2[k];
  }
  if (cudaMalloc(&b->arena, b->arena_bytes) != cudaSuccess || cudaMalloc(&b->status, count * sizeof(Status)) != cudaSuccess ||
      cudaMallocHost(&b->status_host, count * sizeof(Status)) != cudaSuccess ||
      cudaMalloc(&b->desc, 2 * (size_t)count * sizeof(GridDesc)) != cudaSuccess ||
      cudaMalloc(&b->limits, count * sizeof(double2)) != cudaSuccess || cudaMalloc(&b->queue, 2 * sizeof(int)) != cudaSuccess) {
    fail(FG2_ERR_ALLOC, "device allocation of the batch failed");
    return nullptr;
  }
  // every array starts at -max like the reference (src/setup.cpp:80-83)
  const double lowest = storage == ST_F64 ? -std::numeric_limits<double>::max() : -std::numeric_limits<float>::max();
  if (launch_fill(storage, b->arena, b->arena_bytes / elem, lowest, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->status, 0, count * sizeof(Status), b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->queue, 0, 2 * sizeof(int), b->stream) != cudaSuccess) {
    fail(FG2_ERR_ALLOC, "initial fill of the batch failed");
    return nullptr;
  }
  std::memset(b->status_host, 0, count * sizeof(Status));
  char *p = (char *)b->arena;
  const int na = arrays_per_sim(storage);
  for (int k = 0; k < count; ++k) {
    void *r = na > 3 ? p + 3 * bytes[k] : nullptr;  // 16-bit storage: the residuals of u[0], u[1]
    if (r && cudaMemsetAsync(r, 0, 2 * bytes[k], b->stream) != cudaSuccess) {
      fail(FG2_ERR_ALLOC, "initial fill of the batch failed");
      return nullptr;
    }
    fg2_sim *m = sim_create_in(n1[k], n2[k], storage, b->stream, p, p + bytes[k], p + 2 * bytes[k], r,
                               r ? p + 4 * bytes[k] : nullptr, &b->status[k], &b->status_host[k]);
    if (!m) return nullptr;
    b->members.push_back(m);
    p += na * bytes[k];
  }
  // tile order: the smallest members at both ends and the largest in the middle, so that
  // launches in either direction (they alternate) end on short tiles of small members and
  // the persistent CTAs finish together
  std::vector<int> by_size(count);
  for (int k = 0; k < count; ++k) by_size[k] = k;
  std::stable_sort(by_size.begin(), by_size.end(), [&](int x, int y) {
    return (long long)n1[x] * n2[x] < (long long)n1[y] * n2[y];
  });
  b->order.resize(count);
  for (int r = 0, front = 0, back = count - 1; r < count; ++r) b->order[(r & 1) ? back-- : front++] = by_size[r];
  b->desc_host.resize(2 * (size_t)count);
  b->limits_host.resize(count);
  b->versions.assign(count, 0);
  b->curs.assign(count, 0);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
    fail(FG2_ERR_ALLOC, "batch setup failed");
    return nullptr;
  }
  return b.release();
}

void fg2_batch_destroy(fg2_batch *b)
{
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_batch_graph(b);
  for (fg2_sim *m : b->members) fg2_sim_destroy(m);
  cudaFree(b->arena);
  cudaFree(b->status);
  cudaFreeHost(b->status_host);
  cudaFree(b->desc);
  cudaFree(b->limits);
  cudaFree(b->queue);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int fg2_batch_count(const fg2_batch *b) { return b ? b->count : 0; }
long long fg2_batch_cells(const fg2_batch *b) { return b ? b->cells : 0; }
size_t fg2_batch_device_bytes(const fg2_batch *b) { return b ? b->arena_bytes : 0; }
void *fg2_batch_stream(fg2_batch *b) { return b ? (void *)b->stream : nullptr; }

fg2_sim *fg2_batch_member(fg2_batch *b, int k)
{
  if (!b || k < 0 || k >= b->count) {
    fail(FG2_ERR_ARG, "no batch member %d", k);
    return nullptr;
  }
  return b->members[k];
}

int fg2_batch_set_box(fg2_batch *b, double l1, double l2)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  for (fg2_sim *m : b->members) {
    int rc = fg2_sim_set_box(m, l1, l2);
    if (rc) return rc;
  }
  return FG2_OK;
}

int fg2_batch_set_courant(fg2_batch *b, double c)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  for (fg2_sim *m : b->members) {
    int rc = fg2_sim_set_courant(m, c);
    if (rc) return rc;
  }
  return FG2_OK;
}

int fg2_batch_set_bcond(fg2_batch *b, int p1, int p2)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  for (fg2_sim *m : b->members) {
    int rc = fg2_sim_set_bcond(m, p1, p2);
    if (rc) return rc;
  }
  return FG2_OK;
}

const char *fg2_batch_para(fg2_batch *b, const char *kv)
{
  if (!b) return nullptr;
  const char *msg = nullptr;
  for (fg2_sim *m : b->members)
    if (!(msg = fg2_sim_para(m, kv))) return nullptr;
  drop_batch_graph(b);
  return msg;
}

int fg2_batch_config(fg2_batch *b)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  for (fg2_sim *m : b->members) {
    int rc = fg2_sim_config(m);
    if (rc) return rc;
  }
  drop_batch_graph(b);
  return FG2_OK;
}

int fg2_batch_set_time(fg2_batch *b, double t)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  for (fg2_sim *m : b->members) {
    int rc = fg2_sim_set_time(m, t);
    if (rc) return rc;
  }
  return FG2_OK;
}

int fg2_batch_set_tiling(fg2_batch *b, int nb, int ctas_per_sm)
{
  if (!b || nb < 1 || nb > 64 || ctas_per_sm < 0) return fail(FG2_ERR_ARG, "bad tiling %d / %d", nb, ctas_per_sm);
  if (nb != b->nb || ctas_per_sm != b->max_ctas) drop_batch_graph(b);
  b->nb = nb;
  b->max_ctas = ctas_per_sm;
  return FG2_OK;
}

int fg2_batch_get_tiling(const fg2_batch *b, int *nb, int *ctas_per_sm)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  if (nb) *nb = b->nb;
  if (ctas_per_sm) *ctas_per_sm = b->max_ctas;
  return FG2_OK;
}

int fg2_batch_set_strip(fg2_batch *b, int width)
{
  if (!b || (width != 64 && width != 128)) return fail(FG2_ERR_ARG, "strip width must be 64 or 128, not %d", width);
  if (width != b->strip) drop_batch_graph(b);
  b->strip = width;
  return FG2_OK;
}

int fg2_batch_get_strip(const fg2_batch *b) { return b ? b->strip : -1; }

int fg2_batch_advance(fg2_batch *b, int nsteps, double dt, double t_end, int use_graph)
{
  if (!b || nsteps < 0) return fail(FG2_ERR_ARG, "bad arguments");
  int rc = check_members(b);
  if (rc) return rc;
  if (nsteps == 0) return FG2_OK;
  const bool device_dt = !(dt > 0);
  if (any_euler(b)) {
    if (device_dt) return fail(FG2_ERR_UNSUPPORTED, "the Euler hook needs a fixed dt in a batch");
    return advance_plain(b, nsteps, dt, t_end);
  }
  if (!use_graph || nsteps < 2) return advance_plain(b, nsteps, dt, t_end);
  rc = prepare_members(b, device_dt);
  if (rc) return rc;
  rc = ensure_batch_descs(b, device_dt);
  if (rc) return rc;
  const std::vector<double> para(b->members[0]->para, b->members[0]->para + NPARA);
  if (b->graph && (b->graph_dt != dt || b->graph_tend != t_end || b->graph_nb != b->nb || b->graph_ctas != b->max_ctas ||
                   b->graph_strip != b->strip || b->graph_para != para))
    drop_batch_graph(b);
  if (!b->graph) {
    // two steps = six substages: the descriptor set returns to the start
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int set = 0;
    int rc1 = enqueue_batch_step(b, dt, device_dt, t_end, set);
    int rc2 = rc1 ? rc1 : enqueue_batch_step(b, dt, device_dt, t_end, set);
    const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (rc2) {
      if (g) cudaGraphDestroy(g);
      return rc2;
    }
    CK(ce);
    const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    b->graph_dt = dt;
    b->graph_tend = t_end;
    b->graph_nb = b->nb;
    b->graph_ctas = b->max_ctas;
    b->graph_strip = b->strip;
    b->graph_para = para;
  }
  for (int n = 0; n + 1 < nsteps; n += 2) CK(cudaGraphLaunch(b->graph, b->stream));
  finish_steps(b, nsteps & ~1, device_dt);
  if (nsteps & 1) return advance_plain(b, 1, dt, t_end);
  return FG2_OK;
}

int fg2_batch_sync(fg2_batch *b)
{
  if (!b) return fail(FG2_ERR_ARG, "null handle");
  CK(cudaMemcpyAsync(b->status_host, b->status, b->count * sizeof(Status), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  unsigned err = 0, nan = 0;
  for (int k = 0; k < b->count; ++k) {
    err |= b->status_host[k].error;
    nan |= b->status_host[k].nan;
    // a signal max folded into a stage that gave up or produced a NaN is not the state's
    if (b->status_host[k].error || b->status_host[k].nan) b->members[k]->smax_valid = false;
  }
  if (err) return fail(FG2_ERR_TIMEOUT, "a bounded in-kernel wait gave up (bits %u)", err);
  if (nan) return fail(FG2_ERR_NAN, "NaN in a batch member");
  return FG2_OK;
}

// Times steps of every candidate tiling with dt = 0 (u' = u + 0 v leaves every member's state
// unchanged; v is dead between steps) and keeps the fastest: every candidate once, then the
// three best again, each candidate scored by its faster measurement.
int fg2_batch_autotune(fg2_batch *b, int reps, double *best_ms)
{
  if (!b || reps < 1) return fail(FG2_ERR_ARG, "bad arguments");
  int rc = check_members(b);
  if (rc) return rc;
  struct Cand {
    int strip, nb, ctas;
    double ms;
  };
  std::vector<Cand> cands;
  // strip width 128 or 64 columns (4 or 2 warps per CTA); tile height nb blocks of 7 rows;
  // CTAs per SM: 0 = as many as fit (the occupancy limit), or capped at 4, 8 or 12 warps
  for (int strip : {128, 64})
    for (int nb : {1, 2, 3, 4, 5, 6, 8})
      for (int warps : {0, 4, 8, 12})
        cands.push_back({strip, nb, warps * 32 / strip, std::numeric_limits<double>::infinity()});
  const int keep_nb = b->nb, keep_ctas = b->max_ctas, keep_strip = b->strip;
  // 16-bit storage: a step of dt = 0 re-encodes the state and its rounding residual, so
  // the members' arrays are kept aside and put back afterwards
  void *keep = nullptr;
  if (b->members[0]->dev_storage) {
    CK(cudaMalloc(&keep, b->arena_bytes));
    CK(cudaMemcpyAsync(keep, b->arena, b->arena_bytes, cudaMemcpyDeviceToDevice, b->stream));
  }
  std::unique_ptr<void, cudaError_t (*)(void *)> hold(keep, cudaFree);
  std::vector<int> keep_cur;
  std::vector<char> keep_ghosts, keep_smax;
  for (fg2_sim *m : b->members) {
    keep_cur.push_back(m->cur);
    keep_ghosts.push_back(m->ghosts_valid);
    keep_smax.push_back(m->smax_valid);
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  rc = prepare_members(b, false);
  auto measure = [&](Cand &c) -> int {
    b->strip = c.strip;
    b->nb = c.nb;
    b->max_ctas = c.ctas;
    int r = ensure_batch_descs(b, false);
    int set = 0;
    // two untimed steps, then 2 reps timed (even counts leave the descriptor set at 0)
    for (int q = 0; q < 2 && r == 0; ++q) r = enqueue_batch_step(b, 0.0, false, 0.0, set);
    if (r) return r;
    if (cudaEventRecord(e0, b->stream) != cudaSuccess) return fail(FG2_ERR_ARG, "event record failed");
    for (int q = 0; q < 2 * reps && r == 0; ++q) r = enqueue_batch_step(b, 0.0, false, 0.0, set);
    if (r) return r;
    float ms = 0.f;
    if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return fail(FG2_ERR_ARG, "autotune timing failed");
    c.ms = std::min(c.ms, ms / (2.0 * reps));
    return FG2_OK;
  };
  for (size_t i = 0; i < cands.size() && rc == 0; ++i) rc = measure(cands[i]);
  if (rc == 0) {
    std::sort(cands.begin(), cands.end(), [](const Cand &x, const Cand &y) { return x.ms < y.ms; });
    for (size_t i = 0; i < 3 && i < cands.size() && rc == 0; ++i) rc = measure(cands[i]);
    std::sort(cands.begin(), cands.end(), [](const Cand &x, const Cand &y) { return x.ms < y.ms; });
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (keep) {
    CK(cudaMemcpyAsync(b->arena, keep, b->arena_bytes, cudaMemcpyDeviceToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    // the arrays are as they were, ghost cells included: so are the flags that describe them
    for (size_t k = 0; k < b->members.size(); ++k) {
      b->members[k]->cur = keep_cur[k];
      b->members[k]->ghosts_valid = keep_ghosts[k];
      b->members[k]->smax_valid = keep_smax[k];
    }
  }
  b->strip = rc ? keep_strip : cands[0].strip;
  b->nb = rc ? keep_nb : cands[0].nb;
  b->max_ctas = rc ? keep_ctas : cands[0].ctas;
  drop_batch_graph(b);
  b->desc_valid = false;
  if (rc) return rc;
  if (best_ms) *best_ms = cands[0].ms;
  return fg2_batch_sync(b);
}

}  // extern "C"
