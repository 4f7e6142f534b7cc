// fg2_b200/csrc/kernels.h -- host-side launchers of the device kernels (kernels.cu),
// used by the runtime (runtime.cpp).  All launches are asynchronous on `stream`.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "fg2b.h"

namespace fg2 {

// Records the text of the last library error (read back by fg2_last_error) and returns code.
int set_error(int code, const char *fmt, ...);

// Scalar inputs of one substage launch (RK3 stage s: v <- F(u) + beta v,
// u_out <- u + gamma dt v), all in the host's double precision; each launcher rounds them
// to the compute type the way the reference rounds E-precision coefficients to R.
struct StageArgs {
  double beta;          // the stage's beta (src/step.cpp:25)
  double gamma;         // the stage's gamma (src/step.cpp:26)
  double dt;            // time step when dt_dev is null
  const double *dt_dev; // device-resident time step (graph-captured runs), or null
  double delta1, delta2;
  const double *para;   // scheme parameters by slot
  int p1, p2;           // boundary kind per axis (BC_PERIODIC / BC_WALL)
  Status *status;       // device status block
  int store_cols;       // interior columns covered by the bulk-store maps (store_cols())
};

enum StageKind : int {
  STAGE_FIRST = 0,  // beta = 0: v is written, not read
  STAGE_MID = 1,    // v read and written
  STAGE_LAST = 2,   // v read, not written (dead until the next step's first stage)
  STAGE_KICK = 3,   // the reference's kick(): v <- F(u) + beta v only, u untouched
};

// Tensor maps over one state array (all fields) in the device layout: u with the halo box
// of one row chunk of the fused substage kernel, v with its interior box, and the store map
// (interior box, extents ending at the interior) that bulk stores write through.  Return
// CUDA_SUCCESS or the driver's error.
CUresult encode_u_map(CUtensorMap *map, const void *base, const Layout &L, int storage);
CUresult encode_v_map(CUtensorMap *map, const void *base, const Layout &L, int storage);
CUresult encode_store_map(CUtensorMap *map, const void *base, const Layout &L, int storage);
int store_cols(const Layout &L, int storage);
int substage_tiles(const Layout &L);

// The four maps one substage launch uses: u read (halo box), v prefetched, u' stored, v stored.
struct StageMaps {
  const CUtensorMap *u_in, *v_in, *u_out, *v_out;
};

// One fused substage over a whole grid.  `queue` is the simulation's tile queue: two ints,
// zero before the first launch; every launch leaves them zero again.
cudaError_t launch_substage(int storage, int kind, bool cfl, const StageMaps &maps, void *u_out, void *v,
                            const Layout &L, const StageArgs &a, int *queue, cudaStream_t s);

cudaError_t launch_bcond(int storage, void *u, const Layout &L, int p1, int p2, cudaStream_t s);
cudaError_t launch_drift(int storage, void *u, const void *v, const Layout &L, double dt, Status *status,
                         cudaStream_t s);
cudaError_t launch_euler(int storage, void *u, const Layout &L, double dt, const double *para, double delta1,
                         double delta2, float r1, float r2, cudaStream_t s);
cudaError_t launch_fill(int storage, void *p, size_t count, double value, cudaStream_t s);
// max over the interior of (|u1| + c_s) / Delta1 + (|u2| + c_s) / Delta2, in double, as
// an atomic max into status->smax
cudaError_t launch_signal_max(int storage, const void *u, const Layout &L, const double *para, double delta1,
                              double delta2, Status *status, cudaStream_t s);
// FP64 sums of the conserved densities, deterministic: partials[nblocks * 4] then out[4]
int sums_blocks(const Layout &L);
cudaError_t launch_sums(int storage, const void *u, const Layout &L, double *partials, double *out,
                        cudaStream_t s);
// Device-resident time step: dt <- min(courant / smax, dt_diff, t_end - t), t <- t + dt
// (applied by the caller's order: the update runs before the step that uses dt and
// advances t by it), smax reset to 0 for the step's last stage to refill.
cudaError_t launch_dt_update(Status *status, double courant, double dt_diff, double t_end, cudaStream_t s);

}  // namespace fg2
