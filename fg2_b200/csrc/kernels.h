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
  Status *status;       // device status block (launch errors; per-grid blocks are in GridDesc)
  int nb = 0;           // tile height in blocks of 7 rows (0: the default)
  int tail = 0;         // the last rows of each grid as at least this many one-block tiles,
                        // so a launch's last tiles are short (0: none)
  int max_ctas = 0;     // CTAs per SM of the persistent grid (0: as many as fit)
  int strip = 0;        // strip width: 64 or 128 columns per tile (0: 128); one thread per
                        // column, so 2 or 4 warps per CTA; the descriptors must match it
  int reverse = 0;      // take the tiles last first (alternated from launch to launch, so a
                        // stage starts on the tiles the previous one wrote last, still in L2)
  unsigned wait_test_bytes = 0;  // tests of the timeout path: every chunk expects this many
                                 // bytes more than arrive, so every bounded wait runs out
};

enum StageKind : int {
  STAGE_FIRST = 0,  // beta = 0: v is written, not read
  STAGE_MID = 1,    // v read and written
  STAGE_LAST = 2,   // v read, not written (dead until the next step's first stage)
  STAGE_KICK = 3,   // the reference's kick(): v <- F(u) + beta v only, u untouched
};

// One grid of a substage launch, in device memory (the tensor maps keep CUtensorMap's
// 64-byte alignment).  A launch advances a list of grids in tile order: grid k owns launch
// tiles [tile0_k, tile0_k + tiles of grid k).
struct GridDesc {
  CUtensorMap tm_u;       // u (input): 7-row halo boxes of a strip
  CUtensorMap tm_v;       // v: 7-row interior boxes of a strip
  CUtensorMap tm_r;       // 16-bit storage: the rounding residual r, boxes like v's
  void *u_out;            // u' (written stages)
  void *v;                // v (read and/or written)
  Layout L;
  int strips;             // tile columns of this grid
  int tile0;              // its first launch tile
  int p1, p2;             // boundary kind per axis (BC_PERIODIC / BC_WALL)
  const double *dt;       // device time step of this grid, or null: the launch's
  Status *status;         // NaN flag and CFL max of this grid
  double inv1, inv2;      // 1 / Delta per axis (batch launches scale by these)
  double inv11, inv22, inv12;  // 1 / (Delta1 Delta1), 1 / (Delta2 Delta2), 1 / (Delta1 Delta2)
  double delta1, delta2;  // Delta1, Delta2 (curvilinear schemes place cells by them)
  DevCode dev;            // deviation-storage codes (FP16 / BF16 arrays)
};

// Fills a GridDesc (tensor maps over u_in and v encoded here).  Returns CUDA_SUCCESS or the
// driver's error.
// `strip` is the strip width the descriptors are for (box widths and tiles per row; 0: 128).
CUresult make_grid_desc(GridDesc *d, const void *u_in, void *u_out, void *v, const Layout &L, int storage, int p1,
                        int p2, double delta1, double delta2, const double *dt, Status *status, int tile0,
                        const DevCode *dev = nullptr, int strip = 0);
// Tile height of the substage kernel in blocks of 7 output rows, unless a launch sets nb.
constexpr int TILE_BLOCKS_DEFAULT = 4;
// Strip width of single-grid launches; batch launches may also use 64 (strip_width(64)).
constexpr int STRIP_DEFAULT = 128;
int strip_width(int strip);
// Tiles of one grid for a tile height of nb blocks of 7 rows, a strip width and a number of
// one-block tail bands (0: defaults, no tail bands).
int substage_tiles(const Layout &L, int nb = 0, int strip = 0, int tail = 0);
// Storage type of the rounding residual of a 16-bit state (FP16 for BF16 states too).
inline int resid_storage(int storage) { return storage == ST_BF16 ? ST_F16 : storage; }
// The row bands of a grid of n1 rows in the fused kernel's processing order (reverse: a
// reverse launch's), as (i0, iend, blocks) triples into out[3 cap]; returns the band count.
int tile_bands(int n1, int nb, int tail, int reverse, int *out, int cap);

// One fused substage over the grids of `grids` (device array of ngrids descriptors holding
// ntiles tiles in all).  `scaled`: the grids differ in Delta (stencil weights scaled per grid);
// otherwise a.delta1/a.delta2 are folded into the weights.  `queue` is the launch's tile
// queue: two ints, zero before the first launch; every launch leaves them zero again.
cudaError_t launch_substage(int storage, int kind, bool cfl, bool scaled, const GridDesc *grids, int ngrids,
                            int ntiles, const StageArgs &a, int *queue, cudaStream_t s);

cudaError_t launch_bcond(int storage, void *u, const Layout &L, int p1, int p2, cudaStream_t s);
cudaError_t launch_drift(int storage, void *u, const void *v, const Layout &L, double dt, Status *status,
                         cudaStream_t s);
cudaError_t launch_euler(int storage, void *u, const Layout &L, double dt, const double *para, double delta1,
                         double delta2, float r1, float r2, cudaStream_t s);
cudaError_t launch_fill(int storage, void *p, size_t count, double value, cudaStream_t s);
// max over the interior of (|u1| + c_s) / Delta1 + (|u2| + c_s) / Delta2, in double, as
// an atomic max into status->smax
cudaError_t launch_signal_max(int storage, const void *u, const Layout &L, const double *para, double delta1,
                              double delta2, Status *status, cudaStream_t s, const DevCode *dev = nullptr);
// FP64 sums of the conserved densities, deterministic: partials[nblocks * 4] then out[4]
int sums_blocks(const Layout &L);
cudaError_t launch_sums(int storage, const void *u, const Layout &L, double *partials, double *out,
                        cudaStream_t s, const DevCode *dev = nullptr);
// Deviation storage: interior cells of the FP32 cell array src (n1 x n2 x NVAR, no ghosts)
// encoded into the 16-bit array u with the codes dev; and back (dev null: v, plain 16-bit).
cudaError_t launch_encode(int storage, void *u, const float *src, const Layout &L, const DevCode *dev,
                          cudaStream_t s);
cudaError_t launch_decode(int storage, float *dst, const void *u, const Layout &L, const DevCode *dev,
                          cudaStream_t s);
// Device-resident time step: dt <- min(courant / smax, dt_diff, t_end - t), t <- t + dt
// (applied by the caller's order: the update runs before the step that uses dt and
// advances t by it), smax reset to 0 for the step's last stage to refill.
cudaError_t launch_dt_update(Status *status, double courant, double dt_diff, double t_end, cudaStream_t s);
// The same for the count members of a batch (status[k]; limits[k] = {courant, dt_diff}).
cudaError_t launch_dt_update_batch(Status *status, const double2 *limits, int count, double t_end, cudaStream_t s);

}  // namespace fg2
