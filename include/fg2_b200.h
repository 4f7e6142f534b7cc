/*
 * include/fg2_b200.h -- C ABI of the B200-native fg2 time step.
 *
 * One shared library per scheme, as the reference builds one binary per scheme directory
 * (Makefile:19-22, `make hydro` -> bin/hydro): libfg2_hydro.so, libfg2_hydro-isot.so and
 * libfg2_disk.so export the same symbols.  Plain C types only; device pointers are `void *`.
 *
 * Two layers:
 *   - the handle API (fg2_sim_*): explicit simulation objects, a caller-chosen CUDA stream,
 *     status codes instead of exit();
 *   - the reference-mirror API (fg2_setup ... fg2_Euler): the function contract of
 *     src/fg2.h:60-84 over one process-wide simulation, with the reference's argument
 *     meanings and return conventions.
 *
 * Status codes: 0 success; 1 a NaN appeared (the reference returns cudaErrorInvalidValue,
 * whose value is 1, src/step.cpp:38-40); other positive values are cudaError_t codes;
 * negative values are the FG2_ERR_* library errors below.
 *
 * Host arrays exchanged with the library use the reference's host layout without ghosts
 * (src/init.cpp:39-41, src/io.cpp:41-44): n1 * n2 cells in row-major order (axis 2
 * contiguous), NVAR interleaved values per cell, of type float (storage FG2_F32, FG2_F16,
 * FG2_BF16) or double (FG2_F64).
 */
#ifndef FG2_B200_H
#define FG2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FG2_OK 0
#define FG2_ERR_NAN 1         /* == cudaErrorInvalidValue, the reference's NaN status */
#define FG2_ERR_ARG (-1)      /* bad argument (size, key, mode) */
#define FG2_ERR_ALLOC (-2)    /* device or host allocation failed */
#define FG2_ERR_TMA (-3)      /* tensor-map encoding failed */
#define FG2_ERR_TIMEOUT (-4)  /* a bounded in-kernel wait gave up */
#define FG2_ERR_UNSUPPORTED (-5)

/* State storage precision. */
#define FG2_F32 0
#define FG2_F64 1
#define FG2_F16 2
#define FG2_BF16 3

/* getdt() modes. */
#define FG2_DT_REFERENCE 0 /* c / (n1/l1 + n2/l2), src/getdt.cpp:26 */
#define FG2_DT_CFL 1       /* FP64 reduction: c / max[(|u1|+cs)/D1 + (|u2|+cs)/D2], capped by the diffusive limit */

typedef struct fg2_sim fg2_sim;

/* ---- scheme description (compile-time plug-in, src/fg2.h:47-48, <scheme>/config.h) ---- */
const char *fg2_scheme_name(void);
int fg2_nvar(void);                 /* NVAR = sizeof(S) / sizeof(R), src/fg2.h:48 */
const char *fg2_field_name(int f);  /* field order of <scheme>/state.h */
int fg2_eqns_flop(void);            /* eqns_flop, src/hydro/config.h:19 */
int fg2_para_count(void);
const char *fg2_para_key(int k);    /* the para_<key> names of <scheme>/eqns.cuh */
const char *fg2_last_error(void);   /* text of the last library error (thread-local) */
/* Evaluate a named initial condition on the host (no device needed): fills out[n1*n2*NVAR]
 * in the host layout, in double.  para: the scheme's parameter values in the order of
 * fg2_para_key(), or NULL for the defaults.  storage: the precision of the state it is for
 * (FG2_F64: double; the others: the reference's setups compute in float, as src/init.cpp with
 * R = float does, and the parameters and box are rounded to float).  Returns 1 for a known
 * name, 0 for an unknown one (zeros, like the reference's pick() default), negative on bad
 * arguments. */
int fg2_setup_evaluate(const char *name, int n1, int n2, double l1, double l2, const double *para, uint64_t seed,
                       int storage, double *out);

/* ---- handle API ------------------------------------------------------------------------ */
/* setup() (src/setup.cpp:32-87): allocates u (two ping-pong arrays) and v on the current
 * device.  stream: a cudaStream_t, or NULL for a stream the handle owns.  NULL on failure. */
fg2_sim *fg2_sim_create(int n1, int n2, int storage, void *stream);
void fg2_sim_destroy(fg2_sim *s);
size_t fg2_sim_device_bytes(const fg2_sim *s);
int fg2_sim_storage(const fg2_sim *s);
/* global::l1/l2, c, p1/p2 (src/global.cpp:22-31; set by -l, -c, -b in src/main.cpp:48-57) */
int fg2_sim_set_box(fg2_sim *s, double l1, double l2);
int fg2_sim_set_courant(fg2_sim *s, double c);
int fg2_sim_set_bcond(fg2_sim *s, int p1, int p2);
/* Tile height of the fused kernel in blocks of 7 rows (0: the default, 4).  No counterpart in
 * the reference (its block shape came from setup()'s heuristic, src/setup.cpp:39-58); results
 * are bitwise the same for every height. */
int fg2_sim_set_tiling(fg2_sim *s, int nb);
/* CTAs per SM of the fused kernel's persistent grid (0: as many as fit), and the current
 * tiling (the tile height the launches use, after the default's small-grid rule). */
int fg2_sim_set_occupancy(fg2_sim *s, int ctas_per_sm);
int fg2_sim_get_tiling(const fg2_sim *s, int *nb, int *ctas_per_sm);
/* Tail bands: the last rows of the grid are cut into at least `tail` tiles of one block of 7
 * rows (0: none, the default), so that the last tiles of a launch's queue are short and the
 * persistent CTAs finish together.  Results are bitwise the same for every value. */
int fg2_sim_set_tail(fg2_sim *s, int tail);
int fg2_sim_get_tail(const fg2_sim *s, int *tail);
/* The row bands the fused kernel cuts a grid of n1 rows into for tile height nb (0: the
 * default) and `tail` tail bands, in the order a launch takes them (reverse != 0: the order
 * of the alternate launches, which lay the bands out from the last row up): band q covers
 * rows [out[3q], out[3q+1]) in out[3q+2] blocks of 7 rows.  Fills at most cap bands and
 * returns the band count (-1: bad arguments).  Host-only; no device work. */
int fg2_tile_bands(int n1, int nb, int tail, int reverse, int *out, int cap);
/* Times reps steps of each tiling candidate (tile height 1..8 blocks x occupancy cap: all
 * that fit, 4, 8 or 12 warps per SM x tail bands 0, 1, 3) on the simulation's own state with dt = 0 (the state
 * is left bitwise unchanged; 16-bit storage is kept aside and put back) and keeps the
 * fastest; best_ms (may be NULL) receives its time per step.  A grid whose step takes under
 * 0.05 ms with the default tiling is bound by launch latency and keeps the default.  The
 * successor, for one grid, of the reference's block-size heuristic (src/setup.cpp:39-58). */
int fg2_sim_autotune(fg2_sim *s, int reps, double *best_ms);
/* para() (src/para.cpp:25-40): "key=val" (leading dashes skipped); returns "key = val" in a
 * buffer owned by the handle, or NULL for an unknown key. */
const char *fg2_sim_para(fg2_sim *s, const char *keyval);
int fg2_sim_get_para(const fg2_sim *s, const char *key, double *val);
/* config() (src/config.cpp:24-42): scheme settings() then Delta1/Delta2 = l / n. */
int fg2_sim_config(fg2_sim *s);
/* init() (src/init.cpp:26-42): evaluate the named setup at cell centres on the host and
 * copy it to the device.  Unknown names give zeros, as the reference's pick() does.
 * `seed` seeds every random draw of the setup.  Names may carry options:
 * "turb:mach=0.3,kmin=2,kmax=16", "noise:sigma=0.01", "kh:w=0.01". */
int fg2_sim_init(fg2_sim *s, const char *name, uint64_t seed);
int fg2_sim_upload(fg2_sim *s, const void *host);   /* host array -> u */
int fg2_sim_download(fg2_sim *s, void *host);       /* u -> host array */
int fg2_sim_upload_v(fg2_sim *s, const void *host); /* host array -> v */
int fg2_sim_download_v(fg2_sim *s, void *host);     /* v -> host array */
/* getdt() (src/getdt.cpp:22-29) in the selected mode; FG2_DT_CFL synchronises. */
int fg2_sim_set_dt_mode(fg2_sim *s, int mode);
double fg2_sim_getdt(fg2_sim *s);
/* step() (src/step.cpp:22-43): Euler hook, then three fused RK3 substages; synchronises
 * and returns the status (1 on NaN). */
int fg2_sim_step(fg2_sim *s, double t, double dt);
/* nsteps steps enqueued on the stream without synchronising.  dt > 0: fixed dt.
 * dt <= 0: device-resident CFL time step (getdt fused into the last substage), advancing
 * the device clock toward t_end (steps past t_end do nothing). */
int fg2_sim_advance(fg2_sim *s, int nsteps, double dt, double t_end);
/* The same through a CUDA graph of two steps, captured on first use and replayed. */
int fg2_sim_advance_graph(fg2_sim *s, int nsteps, double dt, double t_end);
/* One fused RK3 substage k (0, 1, 2) of a step with time step dt, enqueued without
 * synchronising (src/step.cpp:30-35: bcond, kick, drift of stage k in one pass). */
int fg2_sim_stage(fg2_sim *s, int k, double dt);
int fg2_sim_sync(fg2_sim *s);                 /* wait; status of everything enqueued */
int fg2_sim_set_time(fg2_sim *s, double t);   /* device clock for device-resident runs */
double fg2_sim_time(fg2_sim *s);              /* device clock (synchronises) */
double fg2_sim_last_dt(fg2_sim *s);           /* last device-chosen dt (synchronises) */
void fg2_sim_clear_status(fg2_sim *s);        /* clear the sticky NaN / error words */
/* No counterpart in the reference.  For tests of the timeout path: with bytes > 0 every data
 * chunk of the substage kernel waits for `bytes` more than its copies deliver, so each bounded
 * in-kernel wait (2 s) runs out and the step returns FG2_ERR_TIMEOUT without faulting the GPU;
 * 0 restores normal operation. */
int fg2_sim_test_stall_waits(fg2_sim *s, int bytes);
/* The reference's building blocks on the handle's current arrays. */
int fg2_sim_kick(fg2_sim *s, double t, double beta); /* v <- F(u) + beta v  (src/kick.cu:108-114) */
int fg2_sim_drift(fg2_sim *s, double dt);            /* u <- u + dt v        (src/drift.cu:34-39) */
int fg2_sim_bcond(fg2_sim *s);                       /* ghost fill           (src/bcond.cu:77-86) */
int fg2_sim_euler(fg2_sim *s, double dt);            /* Euler hook           (src/kick.cu:128-138) */
/* Random phases of the stochastic forcing (src/hydro-isot/Euler.cuh:39-44).  After this
 * call every step uses (r1, r2); fg2_sim_seed_forcing returns to seeded per-step draws. */
int fg2_sim_set_forcing_phases(fg2_sim *s, double r1, double r2);
int fg2_sim_seed_forcing(fg2_sim *s, uint64_t seed);
/* FP64 sums of rho, rho u1, rho u2 and the energy density over the interior, in a fixed
 * reduction order (bitwise reproducible). */
int fg2_sim_sums(fg2_sim *s, double out[4]);
/* Current device arrays and their layout: element (f, i, j) at
 * base[(i + 3) * pitch + (j + 4) * cell + f], elements of the storage type; cells hold their
 * NVAR fields interleaved as in the host layout (cell = NVAR), pitch is the stride of a grid
 * row (a multiple of 32 cells, every row 128-byte aligned). */
void *fg2_sim_u(fg2_sim *s);
void *fg2_sim_v(fg2_sim *s);
int fg2_sim_layout(const fg2_sim *s, long long *pitch, long long *cell);
void *fg2_sim_stream(fg2_sim *s);
/* dump()/load() (src/io.cpp:24-76): the reference's .raw frame format. */
int fg2_sim_dump(fg2_sim *s, const char *path, double time);
int fg2_sim_load(fg2_sim *s, const char *path, double *time);
/* solve() (src/solve.cpp:25-64): frames i+1 .. n evenly spaced from t to t_final, each
 * stepped to its time and dumped as <dir>/%04d.raw; the time step follows the getdt mode
 * (FG2_DT_CFL: device-resident).  A NaN dumps <dir>/****.raw and returns FG2_ERR_NAN.
 * ms_per_step (optional): the device time per step. */
int fg2_sim_solve(fg2_sim *s, double t, double t_final, int i, int n, const char *dir, double *ms_per_step);

/* ---- batches of independent simulations --------------------------------------------------
 * No single counterpart in the reference, which advances one grid per process
 * (src/main.cpp:81-116).  A batch owns count members of any sizes (n1[k] x n2[k]) in one
 * device arena and advances them together: one persistent substage launch per RK3 stage over
 * the tiles of every member.  Members are ordinary handles (fg2_batch_member) for init,
 * upload/download, sums, time, dump/load and per-member status; they belong to the batch
 * (never fg2_sim_destroy them) and share its stream.  All members must hold the same scheme
 * parameters (fg2_batch_para sets them on every member); box, boundaries and Courant number
 * may differ per member. */
typedef struct fg2_batch fg2_batch;
fg2_batch *fg2_batch_create(int count, const int *n1, const int *n2, int storage, void *stream);
void fg2_batch_destroy(fg2_batch *b);
int fg2_batch_count(const fg2_batch *b);
long long fg2_batch_cells(const fg2_batch *b);     /* sum of n1[k] n2[k] */
size_t fg2_batch_device_bytes(const fg2_batch *b); /* the arena of u, u', v */
void *fg2_batch_stream(fg2_batch *b);
fg2_sim *fg2_batch_member(fg2_batch *b, int k);
int fg2_batch_set_box(fg2_batch *b, double l1, double l2);  /* every member */
int fg2_batch_set_courant(fg2_batch *b, double c);
int fg2_batch_set_bcond(fg2_batch *b, int p1, int p2);
const char *fg2_batch_para(fg2_batch *b, const char *kv);
int fg2_batch_config(fg2_batch *b);
int fg2_batch_set_time(fg2_batch *b, double t);
/* nsteps RK3 steps of every member.  dt > 0: that step for all; dt <= 0: each member's own
 * CFL step, device-resident, capped at t_end.  use_graph: replay two captured steps. */
int fg2_batch_advance(fg2_batch *b, int nsteps, double dt, double t_end, int use_graph);
int fg2_batch_sync(fg2_batch *b); /* wait; worst status over the members */
/* Tiling of the batch launches: tile height in blocks of 7 rows (nb), CTAs per SM
 * (0: as many as fit) and strip width (64 or 128 columns per tile, one thread per column:
 * 2 or 4 warps per CTA; default 128).  fg2_batch_autotune times steps of each candidate
 * (strip width x tile height x occupancy cap) on the batch's own members (with dt = 0, which
 * leaves every state unchanged) and keeps the fastest; the successor of the reference's
 * block-size heuristic (src/setup.cpp:39-58). */
int fg2_batch_set_tiling(fg2_batch *b, int nb, int ctas_per_sm);
int fg2_batch_get_tiling(const fg2_batch *b, int *nb, int *ctas_per_sm);
int fg2_batch_set_strip(fg2_batch *b, int width);
int fg2_batch_get_strip(const fg2_batch *b); /* 64 or 128 */
int fg2_batch_autotune(fg2_batch *b, int reps, double *best_ms);

/* ---- allocation-free sums ---------------------------------------------------------------
 * No counterpart in the reference.  The FP64 sums of fg2_sim_sums for callers that cannot
 * call cudaMalloc (their allocator already holds the GPU's memory, or the call sits in a
 * loop that must not allocate, or they hold a state array but no handle).  The caller
 * passes the state array u (device memory in the layout of fg2_sim_layout, storage FG2_F32
 * or FG2_F64) and out, a device buffer of 4 doubles.  The only scratch is a static device
 * array of FG2_NOALLOC_MAX_ROWS x 4 doubles (512 KiB) that every GPU loading this library
 * holds until the process exits; grids with more rows are rejected with FG2_ERR_ARG.  All
 * calls share that array, so calls that overlap on the GPU race.  The first call on a
 * device looks up the array's device address; make it before any stream capture.
 * Enqueued on `stream` without synchronising. */
#define FG2_NOALLOC_MAX_ROWS 16384
int fg2_sums_noalloc(const void *u, int n1, int n2, long long pitch, int storage, double *out,
                     void *stream);

/* ---- reference-mirror API (src/fg2.h:60-84) over one process-wide simulation ------------ */
size_t fg2_setup(int n1, int n2);          /* bytes of device memory, 0 on failure */
void fg2_config(void);
const char *fg2_para(const char *keyval);
void fg2_init(const char *name);
double fg2_load(const char *path);
void fg2_dump(const char *path, double time);
double fg2_getdt(void);
int fg2_step(double t, double dt);
/* The process-wide simulation's arrays as the reference's globals hold them
 * (src/setup.cpp:64-72, global::u, global::v, global::s): interior-origin device pointers,
 * element (f, i, j) at p[i * s + j * NVAR + f] with ghosts at negative i and j, and the row
 * stride s in elements.  The state ping-pongs between two arrays, so fg2_u() changes with
 * every step.  kick/drift/bcond/Euler take pointers of this form, as the reference's do. */
float *fg2_u(void);
float *fg2_v(void);
long long fg2_s(void);
void fg2_kick(float *v, const float *u, float t, float beta);
void fg2_drift(float *u, const float *v, float dt);
void fg2_bcond(float *u, int p1, int p2);
void fg2_Euler(float *u, float dt);
fg2_sim *fg2_global(void);                 /* the process-wide simulation (global::u, v, ...) */

#ifdef __cplusplus
}
#endif

#endif /* FG2_B200_H */
