// fg2_b200/csrc/sim.h -- the simulation handle and the runtime's internal helpers, shared by
// the single-simulation runtime (runtime.cpp) and the batch runtime (batch.cpp).  Host code.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>

#include "../../include/fg2_b200.h"
#include "fg2b.h"
#include "kernels.h"
#include "setup_common.h"

#define fail fg2::set_error

#define CK(expr)                                                   \
  do {                                                             \
    cudaError_t e_ = (expr);                                       \
    if (e_ != cudaSuccess) return fg2::rt::cuda_status(e_, #expr); \
  } while (0)

struct fg2_sim {
  bool own_arrays = true;   // u, v, status, status_host allocated by this handle
  int n1 = 0, n2 = 0, storage = fg2::ST_F32;
  fg2::Layout L{};
  void *u[2] = {nullptr, nullptr};
  void *v = nullptr;
  int cur = 0;  // u[cur] holds the state
  // substage descriptors: [0] u[0] -> u[1], [1] u[1] -> u[0], [2] the mirror API's kick
  fg2::GridDesc *desc = nullptr;   // device
  fg2::GridDesc desc_host[3];
  bool desc_valid = false;
  unsigned version = 0;       // bumped whenever settings that descriptors depend on change
  int order = 0;              // tile order of the next substage launch (alternates)
  int nb = 0;                 // tile height in blocks of 7 rows (0: the default)
  int max_ctas = 0;           // CTAs per SM of the persistent grid (0: as many as fit)
  int tail = 0;               // one-block tail bands ending the grid (0: none)
  unsigned wait_test_bytes = 0;  // timeout-path tests (fg2_sim_test_stall_waits)
  int *queue = nullptr;   // tile queue of the substage kernel (self-resetting)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  fg2::Status *status = nullptr;       // device
  fg2::Status *status_host = nullptr;  // pinned mirror
  double *sums_partial = nullptr, *sums_out = nullptr;
  double para[fg2::NPARA];  // runtime keys by slot, then the scheme's derived constants
  double l1 = 1.0, l2 = 1.0, c = 0.5;  // src/global.cpp:28
  int p1 = 1, p2 = 1;                  // src/global.cpp:29
  double delta1 = 0, delta2 = 0;
  bool configured = false;
  bool ghosts_valid = false;
  bool smax_valid = false;
  int dt_mode = FG2_DT_REFERENCE;
  fg2::Rng forcing{0x5eed5eedull};
  bool fixed_phases = false;
  float r1 = 0.f, r2 = 0.f;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // two-step graph per ping-pong parity
  double graph_dt[2] = {0, 0}, graph_tend[2] = {0, 0};
  char para_msg[256];
  // deviation storage (FP16 / BF16 arrays): per-field background and per-tile scales
  bool dev_storage = false;
  int tiles1 = 0, tiles2 = 0;
  float4 *scale_dev = nullptr, *inv_dev = nullptr;
  void *r[2] = {nullptr, nullptr};  // rounding residual of u[0] and of u[1] (16-bit numbers, layout of u)
  fg2::DevCode dev{};                // background and scales (shared by both parities)
  mutable fg2::DevCode devk[2]{};    // dev with the residual arrays of parity k: read r[k], write r[1 - k]
};

namespace fg2 {
namespace rt {

int cuda_status(cudaError_t e, const char *what);
size_t elem_size(int storage);
size_t host_elem(int storage);

// RK3 coefficients (src/step.cpp:24-26), evaluated in double as the reference's E.
extern const double RK_ALPHA[3], RK_BETA[3], RK_GAMMA[3];

size_t array_elems(const fg2_sim *s);
void compute_deltas(fg2_sim *s);
double round_para(const fg2_sim *s, double x);
StageArgs stage_args(fg2_sim *s, int k, double dt, const double *dt_dev);
int ensure_descs(fg2_sim *s);
int ensure_config(fg2_sim *s);
int do_bcond(fg2_sim *s);
int do_euler(fg2_sim *s, double dt);
bool euler_active(const fg2_sim *s);
double diffusive_dt(const fg2_sim *s);
int read_status(fg2_sim *s);
// The handle's deviation codes for kernels that decode the state u[cur] (null: plain storage),
// and for parity k: the residual of u[k] read, that of u[1 - k] written.
const fg2::DevCode *dev_code(const fg2_sim *s);
const fg2::DevCode *dev_code_at(const fg2_sim *s, int k);
void drop_graph(fg2_sim *s);
// A handle over caller-owned device memory: arrays u0, u1, v (and, for 16-bit storage, the
// residual arrays r0, r1 of u0 and u1, zero-filled) of the handle's layout and one status
// block (device) with its pinned host mirror; the handle frees none of them.
fg2_sim *sim_create_in(int n1, int n2, int storage, cudaStream_t stream, void *u0, void *u1, void *v, void *r0,
                       void *r1, Status *status, Status *status_host);
// Arrays per simulation in device memory: u[0], u[1], v, and r[0], r[1] for 16-bit storage.
int arrays_per_sim(int storage);

}  // namespace rt
}  // namespace fg2
