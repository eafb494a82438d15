/*
 * hydrob200.h -- C ABI of the B200 shallow-water timestep library.
 *
 * Replaces the hot path of hydro-bench's hydro-cal solver: the per-edge flux
 * (CalculateFlux, cuda_native_impl/hydro-cal-src/src/functors.cu:787-792 and
 * :802-809) and the per-cell update (UpdateCell, functors.cu:794-799 and
 * :811-818) driven by the day/step loop of cuda_native_impl/benchmark.cu:87-96.
 * Every call returns an hb_status; nothing calls exit() (the reference's
 * CUDA_CHECK does, common.hpp:57-59).
 *
 * Arrays crossing this boundary are in the reference's own order and types:
 * per cell [CELL], per slot [4*CELL] with slot = 4*cell + j, per cell and day
 * [NDAYS*CELL] with index day*CELL + cell, rating tables [CELL*NHQ]
 * (cell.cpp:93-128).  The handle keeps its own renumbered copy on the device.
 */
#ifndef HYDROB200_H
#define HYDROB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    HB_OK = 0,
    HB_E_INVALID = 1,          /* bad argument */
    HB_E_BADMESH = 2,          /* mesh arrays inconsistent (neighbour index out of range, ...) */
    HB_E_CUDA = 3,             /* a CUDA call failed; hb_last_error_string() says which */
    HB_E_NONFINITE = 4,        /* a step produced NaN/Inf depth or velocity */
    HB_E_BARRIER_TIMEOUT = 5,  /* the persistent kernel's grid barrier gave up waiting */
    HB_E_IO = 6,               /* a deck file could not be read */
    HB_E_UNDEFINED_REF = 7,    /* a slot reached reference behaviour that reads undefined memory */
    HB_E_NOMEM = 8,
    HB_E_TOO_LARGE = 9         /* size beyond a fixed capacity */
} hb_status;

typedef enum { HB_VARIANT_H = 0, HB_VARIANT_F = 1 } hb_variant;
/* HB_FP64: the reference's fp64 kernels, bit for bit.  HB_FP32: the fp32 tree
 * (cuda_native_impl/fp32_src).  HB_SPLIT: no reference counterpart; fluxes,
 * velocities and depths in fp32, while water levels, beds and boundary levels
 * stay fp64, every depth formed as level minus bed is taken in fp64, and each
 * cell's depth update is Kahan-compensated.  Its device state is the fp32
 * quadruple {H, U, V, H_lo} (no Z; hb_get_state rebuilds Z in fp64). */
typedef enum { HB_FP64 = 0, HB_FP32 = 1, HB_SPLIT = 2 } hb_precision;
/* HB_LAYOUT_EDGE: two kernels per step, one thread per flux record then one
 * per cell, with the slots' terms of the cell sums passed through device
 * memory.  HB_LAYOUT_TILE: one kernel per step; the cells are grouped into
 * compact tiles of about tile_cells cells, and one CTA computes every flux of
 * its tile into shared memory and updates the tile's cells.  Both give the
 * same bits. */
typedef enum { HB_LAYOUT_EDGE = 0, HB_LAYOUT_TILE = 1 } hb_layout;

/* Host description of a mesh and its boundary tables, reference layout.
 * Mirrors what MeshView/CellView/SideView hold after FromHost
 * (mesh.hpp:114-141, cell.hpp:28-61, side.hpp:29-52). */
typedef struct hb_mesh_desc {
    int32_t cells;            /* CELL */
    int32_t ndays;            /* NDAYS: rows of the qt/dqt/zt/dzt tables */
    int32_t nhq;              /* NHQ: columns of zw/qw */
    int32_t steps_per_day;    /* MDT / DT (benchmark.cu:55); the loop runs kt = 1..steps_per_day-1 */
    double dt, hm1, hm2, jl;  /* DT, HM1, HM2, JL */
    const double *nac;        /* [4C] 1-based neighbour, 0 = none (stored as double, side.hpp:34) */
    const double *klas;       /* [4C] boundary code (double, side.hpp:32) */
    const double *side, *cosf, *sinf, *slcos, *slsin;   /* [4C] */
    const double *zbc, *zb1, *area, *fnc, *bfeat;       /* [C]; bfeat = BoundaryFeature (weir crest) */
    const int32_t *nhq1;      /* [C] rating-curve points used per cell */
    const double *zw, *qw;    /* [C*NHQ] */
    const double *qt, *dqt, *zt, *dzt;                   /* [NDAYS*C] */
} hb_mesh_desc;

typedef struct hb_handle hb_handle;

typedef struct hb_options {
    int32_t variant;          /* hb_variant */
    int32_t precision;        /* hb_precision */
    int32_t device;           /* CUDA device ordinal */
    int32_t renumber;         /* 1: reverse Cuthill-McKee cell order on the device (default), 0: input order */
    int32_t tile_config;      /* launch shape: 0 = the layout's default, k > 0 = entry k-1 of hb_launch_shapes() */
    int32_t layout;           /* hb_layout */
    int32_t tile_cells;       /* HB_LAYOUT_TILE: cells per tile, <= 1024; tiles hold up to 5*tile_cells/4.
                               * 0 = HB_FP32 / HB_SPLIT: balanced, about 512, sized so the tiles fill
                               * whole waves of the launch shape's resident CTAs on the device;
                               * HB_FP64: 256 */
    int32_t persistent;       /* HB_LAYOUT_EDGE with the default launch shape only.  1: a step sequence
                               * (hb_step, a captured graph) is one cooperative launch of resident CTAs that
                               * runs every step, flux records then cells, separated by grid barriers whose
                               * waits are bounded (hb_set_barrier_limit); 0: two launches per step.  Same
                               * bits either way.  Not for hb_autotune. */
} hb_options;

/* The compiled launch shapes: the layout each runs, threads per CTA, and
 * 100 * (flux or tile CTAs per SM) + (cell-update CTAs per SM, edge layout)
 * asked of the compiler; returns how many there are (tile_config = index + 1).
 * A handle takes only shapes of its own layout. */
int hb_launch_shapes(int32_t *layout, int32_t *threads, int32_t *min_blocks, int32_t capacity);
/* hb_launch_shapes without the layouts. */
int hb_tile_configs(int32_t *threads, int32_t *min_blocks, int32_t capacity);

/* Default options: variant H, fp64, device 0, renumbered. */
void hb_options_default(hb_options *opt);

/* Copy the mesh to the device (renumbered) and set the state to zero.
 * Replaces MeshView construction (benchmark.cu:52 -> cell.cpp:11-146, side.cpp:11-52). */
int hb_create(const hb_mesh_desc *mesh, const hb_options *opt, hb_handle **out);
int hb_destroy(hb_handle *h);

/* A batch of n independent scenarios (meshes of any sizes, their own DT, HM1,
 * HM2, JL and boundary tables) stepped together: every kernel launch covers
 * all of them, each CTA taking one scenario's records or cells from a segment
 * table.  No reference counterpart; the reference runs one mesh per process.
 * The calls below without _at address scenario 0; hb_step, hb_sync,
 * hb_capture_graph and hb_graph_launch advance every scenario, and
 * hb_position reports scenario 0's (kt, jt).  hb_step_host is single-mesh only. */
int hb_create_batch(const hb_mesh_desc *meshes, int32_t n, const hb_options *opt, hb_handle **out);
int hb_batch_size(hb_handle *h, int32_t *n);
/* Cells of scenario s and the device index of its first cell. */
int hb_scenario_cells(hb_handle *h, int32_t s, int32_t *cells, int32_t *first);
int hb_set_state_at(hb_handle *h, int32_t s, const double *H, const double *U, const double *V, const double *Z,
                    const double *W);
int hb_get_state_at(hb_handle *h, int32_t s, double *H, double *U, double *V, double *Z, double *W);
int hb_get_flux_at(hb_handle *h, int32_t s, double *F0, double *F1, double *F2, double *F3);
int hb_get_klas_at(hb_handle *h, int32_t s, double *klas);
int hb_get_permutation_at(hb_handle *h, int32_t s, int32_t *perm);

/* Launch shape of a handle (index + 1 into hb_tile_configs; 0 = default).
 * Changing it drops a captured graph. */
int hb_set_tile_config(hb_handle *h, int32_t tile_config);
int hb_get_tile_config(hb_handle *h, int32_t *tile_config);
/* Autotuner: times every launch shape over `steps` steps of this handle's own
 * mesh(es) from the current state (CUDA events on `stream`), restores the
 * state, fluxes, boundary codes, error bits and step counter afterwards, and
 * keeps the fastest shape (*best, as a tile_config).  ms_per_step[i] (i <
 * capacity) receives shape i+1's time.  Drops a captured graph if the shape
 * changes.  Needs steps + 1 steps of boundary tables beyond the position. */
int hb_autotune(hb_handle *h, int32_t steps, void *stream, float *ms_per_step, int32_t capacity, int32_t *best);

/* State in reference order, fp64 host arrays of [CELL]. W may be NULL. */
int hb_set_state(hb_handle *h, const double *H, const double *U, const double *V, const double *Z, const double *W);
int hb_get_state(hb_handle *h, double *H, double *U, double *V, double *Z, double *W);
/* The per-slot fluxes left by the last step, [4*CELL] each, and the current
 * boundary codes (KLAS=7 slots turn into 0 once breached, functors.cu:242). */
int hb_get_flux(hb_handle *h, double *F0, double *F1, double *F2, double *F3);
int hb_get_klas(hb_handle *h, double *klas);

/* Advance nsteps steps of the reference driver loop from its current
 * position (day jt, step kt); the first call starts at jt = 0, kt = 1.
 * `stream` is a cudaStream_t (NULL = the legacy default stream).  Returns
 * once the work is queued; hb_sync waits and reports device-side faults. */
int hb_step(hb_handle *h, int32_t nsteps, void *stream);
int hb_sync(hb_handle *h, void *stream);
/* Current position: steps taken so far, and the (kt, jt) of the next step. */
int hb_position(hb_handle *h, int64_t *steps_done, int32_t *kt, int32_t *jt);
int hb_set_position(hb_handle *h, int64_t steps_done);

/* End-to-end call with host buffers, for callers whose state lives on the
 * host (the reference driver keeps it in MeshData, benchmark.cu:66-84):
 * copies H, U, V, Z (reference order, [CELL] fp64) to the device, advances
 * nsteps steps, and copies H, U, V, Z, W back into the same buffers (W may be
 * NULL; arrays that follow one another in host memory, e.g. the rows of one
 * [4][CELL] or [5][CELL] block, move as one copy).  The
 * copies are asynchronous on `stream` (page-locked buffers make them truly
 * so); call hb_sync before reading the results. */
int hb_step_host(hb_handle *h, double *H, double *U, double *V, double *Z, double *W, int32_t nsteps, void *stream);

/* Capture nsteps steps as one CUDA graph owned by the handle; each replay
 * (hb_graph_launch) advances the boundary-table time like hb_step would. */
int hb_capture_graph(hb_handle *h, int32_t nsteps, void *stream);
int hb_graph_launch(hb_handle *h, void *stream);

/* Device-resident state pointers (renumbered order) for zero-copy use from
 * PyTorch: H, U, V, Z, W, fp64 (fp32 for HB_FP32).  H, U, V and Z are
 * interleaved per cell: element i of H is H[i * stride] (stride from *stride);
 * W is contiguous. */
int hb_device_state(hb_handle *h, void **H, void **U, void **V, void **Z, void **W, int32_t *stride);
/* Renumbering: perm[new] = old (cell ids, 0-based). */
int hb_get_permutation(hb_handle *h, int32_t *perm);
/* Write scenario s's state and last fluxes as the reference driver's --dump
 * file (cuda_native_impl/benchmark.cu:141-162): int32 CELL; H, U, V, Z;
 * SLCOS, SLSIN, SIDE (from `mesh`); FLUX0..3; values of the build's Real
 * type (float for HB_FP32, double otherwise), reference order. */
int hb_write_dump(hb_handle *h, int32_t s, const hb_mesh_desc *mesh, const char *path);
/* Checkpoint / resume (no reference counterpart): everything a run needs to
 * continue bit for bit -- the current state and W, the fluxes (codes that
 * leave fluxes unwritten keep the old ones), the per-slot boundary codes
 * (KLAS 7 slots breach), the device error bits and the step position -- in
 * one host buffer of hb_checkpoint_size bytes.  A checkpoint loads into a
 * handle of the same mesh(es) and options (precision, variant, layout,
 * tile_cells, renumbering); a captured graph stays valid. */
int hb_checkpoint_size(hb_handle *h, size_t *bytes);
int hb_checkpoint_save(hb_handle *h, void *buffer, size_t bytes);
int hb_checkpoint_load(hb_handle *h, const void *buffer, size_t bytes);

/* Halo exchange (no reference counterpart; the reference steps one mesh on
 * one GPU).  A mesh too large for one GPU is split into parts, each stepped
 * by its own handle over its cells plus a one-ring halo of its neighbours'
 * cells; after every step each halo cell takes the state its owner computed.
 * hb_halo_define registers a list of this handle's cells (reference order,
 * host memory) and returns its id.  hb_halo_pack copies the current state
 * record of every cell of a list, in list order, into `buf`; hb_halo_unpack
 * writes such records into the current state.  `buf` is device memory,
 * 16-byte aligned, of n * hb_state_record_bytes bytes; both calls are ordered
 * on `stream` after the handle's steps.  Single-mesh handles only. */
int hb_state_record_bytes(const hb_handle *h, int32_t *bytes);
int hb_halo_define(hb_handle *h, const int32_t *cells, int32_t n, int32_t *list);
int hb_halo_pack(hb_handle *h, int32_t list, void *buf, void *stream);
int hb_halo_unpack(hb_handle *h, int32_t list, const void *buf, void *stream);
/* Bound of every grid-barrier wait of a persistent handle (default 1 s of the
 * GPU's global timer, at most 10 s).  A wait that runs out sets the device
 * error bit of HB_E_BARRIER_TIMEOUT (hb_sync returns it) and every CTA leaves
 * the launch; the state is then partly stepped.  phantom_arrivals > 0 makes
 * every barrier also wait for that many arrivals that never come, so that the
 * bounded wait can be exercised without a fault; use 0. */
int hb_set_barrier_limit(hb_handle *h, int64_t timeout_ns, int32_t phantom_arrivals);

/* Sticky device error word (bit set of hb_status codes seen by kernels). */
int hb_device_errors(hb_handle *h, uint32_t *bits);

int hb_last_error(void);
const char *hb_last_error_string(void);
const char *hb_status_string(int status);

/* ---- reverse-mode adjoint (no reference counterpart) ----
 * Gradient of a gauge loss over a rollout with respect to the per-cell
 * Manning coefficient n (FNC = 9.81 n^2, mesh.cpp:364) and bed ZBC:
 *   L = sum over steps t = obs_every, 2 obs_every, ..., <= nsteps and gauge
 *       cells g of (H_t[g] - Hobs_t[g])^2,
 * for a rollout of nsteps steps from an initial level Z0 and velocities
 * (H0 = Z0 - ZBC where Z0 > ZBC, else H0 = HM1 and Z0 = ZBC + HM1,
 * mesh.cpp:350-361).  Branch choices (wet/dry, Osher's wave case, clamps,
 * fixed-point iteration counts) are those of the forward state.  The state is
 * checkpointed every checkpoint_every steps and each segment recomputed in
 * the backward pass.  Needs a single-mesh fp64 variant-H edge-layout handle,
 * not persistent, whose boundary codes are among KLAS 0, 1, 4, 10; the gauges
 * are distinct cells.  The rollout runs on the handle's own mesh and state
 * (its state is the rollout's end afterwards).  Checkpoints and gauge depths
 * are written by the rollout's own cell-update kernels. */
typedef struct hb_adjoint hb_adjoint;
int hb_adjoint_create(hb_handle *h, const int32_t *gauges, int32_t ngauges, int32_t obs_every, int32_t nsteps,
                      int32_t checkpoint_every, hb_adjoint **out);
int hb_adjoint_destroy(hb_adjoint *a);
/* Reference order [CELL]; either may be NULL (kept).  Rewrites the handle's FNC / ZBC. */
int hb_adjoint_set_parameters(hb_adjoint *a, const double *manning_n, const double *zbc);
int hb_adjoint_set_initial(hb_adjoint *a, const double *Z0, const double *U0, const double *V0);
/* [nobs][ngauges], nobs = nsteps / obs_every; row r is after step (r + 1) * obs_every. */
int hb_adjoint_set_observations(hb_adjoint *a, const double *obs);
/* The rollout and its loss; gauge_depths ([nobs][ngauges]) may be NULL. */
int hb_adjoint_forward(hb_adjoint *a, double *loss, double *gauge_depths, void *stream);
/* dL/dn and dL/dZBC of the last forward, reference order [CELL]; either may be NULL. */
int hb_adjoint_backward(hb_adjoint *a, double *grad_n, double *grad_zbc, void *stream);

/* ---- deck reader (cuda_native_impl/hydro-cal-src/src/mesh.cpp:5-533, cell.cpp:72-128) ---- */
typedef struct hb_deck hb_deck;
/* Read a hydro-cal text deck (BINFOR/, SOURCES/, BOUNDE/ under `root`). */
int hb_deck_load(const char *root, hb_deck **out);
/* Borrow the deck's mesh description (valid until hb_deck_free) and its
 * initial state (H, U, V, Z, W after preCalculate). */
int hb_deck_mesh(const hb_deck *d, hb_mesh_desc *mesh);
int hb_deck_state(const hb_deck *d, const double **H, const double **U, const double **V,
                  const double **Z, const double **W);
int hb_deck_free(hb_deck *d);

/* ---- result files in the reference's text formats (mesh.cpp:535-839) ----
 * hb_output_open creates (truncating) SIDE.OUT, H2U2V2.OUT, ZUV.OUT,
 * XY-TEC.DAT and TIMELOG.OUT in `dir` for the deck's mesh; hb_output_frame
 * appends one frame of a state (reference order, fp64 [CELL]) for day jt and
 * step kt as the reference's outputToFile(jt, kt) does (the first frame,
 * jt = 0 and kt = 1, also writes the geometry to SIDE.OUT).  The driver loop
 * writes the initial frame (0, 1), then one after the last step of every
 * NTOUTPUT-th day and after the last step (benchmark.cu:105-124). */
typedef struct hb_output hb_output;
int hb_output_open(const hb_deck *d, const char *dir, hb_output **out);
int hb_output_frame(hb_output *o, int32_t jt, int32_t kt, const double *H, const double *U, const double *V,
                    const double *Z);
int hb_output_close(hb_output *o);
/* NTOUTPUT of the deck (BINFOR/TIME.DAT). */
int hb_deck_ntoutput(const hb_deck *d, int32_t *ntoutput);

#ifdef __cplusplus
}
#endif
#endif
