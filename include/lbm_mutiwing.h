/*
 * lbm_mutiwing.h -- C ABI of the B200 implementation of the LBM_Mutiwing time
 * step: D2Q9 MRT collide-and-stream plus the implicit immersed-boundary
 * (bc_num = 4) interpolate / velocity-correct / spread cycle for moving
 * multi-airfoils, on one GPU.
 *
 * The reference (R-IFFERY/LBM_Mutiwing, Fortran 90 + OpenACC) keeps all state
 * in module globals and calls `evolution` once per lattice step.  Each entry
 * point below replaces one reference routine; the citation names it
 * (file:line in the reference project).  A Fortran host binds these with an
 * ISO_C_BINDING interface block, the way zmq_comm.f90:23-81 binds libzmq.
 *
 * Conventions
 *  - Status: 0 on success, negative on error; lbm_last_error() gives the text
 *    (the text an online driver sends back as "ERROR <msg>").  Nothing in the
 *    library exits or stops the process.
 *  - Ownership: the library owns all device memory; callers own host buffers.
 *  - Threading: calls on one handle are serialised by the caller; handles are
 *    independent.  Work is stream-ordered; calls that return host data
 *    synchronise before returning.
 *  - Arrays are row-major with x fastest: index (j-1)*nx + (i-1) holds the
 *    reference's mesh%f(i,j) etc.; distribution planes are 9 consecutive
 *    nx*ny planes in the reference's velocity order.
 */
#ifndef LBM_MUTIWING_H
#define LBM_MUTIWING_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* Storage / compute path. */
#define LBM_PRECISION_FP64 0   /* plain FP64, reference kernel order (the drop-in) */
#define LBM_PRECISION_FP32 1   /* fused pull kernel, FP32 deviation storage */

/* Motion source (driver.f90:10-31, LBM_MOTION_SOURCE). */
#define LBM_MOTION_FILE 1      /* per-step table built from motion_params.dat rows */
#define LBM_MOTION_STREAM 2    /* online smooth ramp between two rows (ZeroMQ STEP) */

/* LbmConfig.flags */
#define LBM_FLAG_NO_GRAPHS 1   /* launch every kernel directly (no CUDA graph replay) */
#define LBM_FLAG_SOLVE_STREAM 2  /* stream each wing's factor through shared memory in an 8-row substitution
                                    even when the wing fits whole (for testing) */
#define LBM_FLAG_SINGLE_STEPS 8   /* fused path: advance one step at a time instead of in two-step passes
                                     (the same results; for testing and comparison) */
#define LBM_FLAG_SOLVE_PANELS32 4  /* substitute in 32-row panels built by the factorisation, where every
                                      wing's panel data fit in shared memory (fewer dependent steps on the
                                      step's chain, a longer factorisation) */
#define LBM_FLAG_PASS_TALL_TILES 16   /* fused path: two-step passes over 64 x 12 tiles whatever the lattice
                                         size (by default from 32 Mi nodes on; the same results) */
#define LBM_FLAG_PASS_SHORT_TILES 32  /* fused path: two-step passes over 64 x 8 tiles whatever the lattice
                                         size (by default below 32 Mi nodes; the same results);
                                         LBM_FLAG_PASS_TALL_TILES wins when both are given */

/* lbm_step flags */
#define LBM_STEP_FIELDS 1      /* last step leaves rho, u, v, pre readable by lbm_get_fields */
#define LBM_STEP_ERR 2         /* last two steps keep u, u0 so lbm_err is available */

typedef struct LbmHandle LbmHandle;
typedef struct LbmBatch LbmBatch;

/* Runtime form of the reference's compile-time parameters
 * (main.f90:7-152, ini_mesh.f90:15-67). */
typedef struct LbmConfig {
    int32_t nx, ny;              /* lattice nodes: nint(W/scale)+1, nint(H/scale)+1 (ini_mesh.f90:22-23) */
    double scale;                /* lattice spacing in chords (mesh_max_scale, main.f90:32) */
    double uu;                   /* inflow lattice velocity UU (main.f90:12) */
    double re;                   /* Reynolds number on the chord (main.f90:106) */
    double ox, oy;               /* physical position of node (1,1) (ini_mesh.f90:36-37) */
    double s[9];                 /* MRT rates (ini_mesh.f90:59-67); s[7], s[8] <= 0 select 1/tau */
    int32_t wing_count;          /* wings (main.f90:18); 0 allowed (no immersed body) */
    double wing_x_origin;        /* main.f90:34 */
    double wing_x_spacing;       /* main.f90:35 */
    double wing_y_origin;        /* main.f90:36 */
    double xc, yc;               /* flow-centre offset (main.f90:114) */
    int32_t motion_source;       /* LBM_MOTION_FILE or LBM_MOTION_STREAM */
    int32_t precision;           /* LBM_PRECISION_* */
    int32_t device;              /* CUDA device ordinal */
    int32_t flags;               /* LBM_FLAG_* */
    int32_t reserved[6];
} LbmConfig;

/* Fill cfg with the reference defaults: 4001x2001 lattice, scale 0.01,
 * UU 0.01, Re 500, two wings at x 0.0 / 1.5, y 0.5, file motion, FP64. */
void lbm_config_default(LbmConfig* cfg);

/* Allocate and initialise one simulation: ini_mesh (ini_mesh.f90:1-80),
 * init (solution.f90:1-75) and read_boundary (airfoil.f90:207-242).
 * markers_xy: body-frame points (x, y) of all wings back to back, each wing a
 * closed loop with its first point repeated last; points_per_wing[w] >= 2. */
int lbm_create(const LbmConfig* cfg, const double* markers_xy, const int32_t* points_per_wing,
               LbmHandle** out);

/* Episode reset: reset_zmq_episode (driver.f90:205-258) -- fresh initial
 * state, empty band, cycle 1, force sums cleared. */
int lbm_reset(LbmHandle* h);

/* load_motion_table + build_motion_step_table (mode.f90:104-178, 388-412):
 * rows of 1 + 9*wing_count columns, non-decreasing time, absolute x and y. */
int lbm_set_motion_table(LbmHandle* h, const double* rows, int64_t nrows, int32_t ncols);

/* Online segment (driver.f90:174-186): motion between start_row and
 * target_row, each 1 + 9*wing_count values, interpolated per step as
 * lookup_stream_motion_row (mode.f90:414-449). */
int lbm_set_stream_rows(LbmHandle* h, const double* start_row, const double* target_row);

/* build_stream_target_row (mode.f90:287-325), host-side helper:
 * delta_row = (t, domega, dxv, dyv per wing). */
int lbm_build_stream_target_row(const LbmHandle* h, const double* start_row, double target_time,
                                const double* delta_row, double* target_row);

/* n_steps passes of evolution (solution.f90:272-422) for cycles
 * first_cycle .. first_cycle+n_steps-1, each followed by the move_mesh check
 * (main.f90:393-411).  force_rows (may be NULL) receives n_steps rows of
 * 4 + 12*wing_count doubles in the force_row layout of solution.f90:352-378.
 * Each row is also added to the running sums (latest_force_sum_row). */
int lbm_step(LbmHandle* h, int64_t first_cycle, int64_t n_steps, double* force_rows, int32_t flags);

/* Running force sums since the last reset (solution.f90:379-385). */
int lbm_get_sums(LbmHandle* h, double* sum_row, int32_t* sample_count, int32_t* row_len);
int lbm_reset_sums(LbmHandle* h);

/* rho, u, v, pre after the last step (any pointer may be NULL) -- the fields
 * output (solution.f90:132-241) reads.  The FP32 path needs LBM_STEP_FIELDS
 * on that step. */
int lbm_get_fields(LbmHandle* h, double* rho, double* u, double* v, double* pre);

/* output (solution.f90:132-241): every stride_x-th node of every
 * stride_y-th row, row by row, of u/UU, v/UU, the pressure and the vorticity
 * dv/dx - du/dy (centred inside, second-order one-sided on the border),
 * computed on the device; ((nx-1)/stride_x+1) x ((ny-1)/stride_y+1) values
 * each (any pointer may be NULL).  Needs the fields of the last step
 * (LBM_STEP_FIELDS on the FP32 path). */
int lbm_get_output(LbmHandle* h, int32_t stride_x, int32_t stride_y, double* u, double* v, double* pre,
                   double* vort);

/* erranalysis (solution.f90:77-130) on the fields of the last two steps. */
int lbm_err(LbmHandle* h, double* err);

/* No counterpart in the reference.  The same convergence error, on velocity
 * fields the caller owns in device memory (u, v current; u0, v0 previous;
 * node (i, j) at [j * pitch + i], 0 <= i < nx, 0 <= j < ny), computed
 * without allocating anything: for callers that cannot let a library
 * allocate device memory (the device handed to their own memory pool, or a
 * serving loop where an allocation would synchronise the device and stall
 * other streams).  Partial sums live in a fixed array inside the library,
 * sized for at most LBM_NOALLOC_MAX_ROWS lattice rows; a larger ny is
 * refused (-2).  Nothing has to start at zero: every partial sum a call reads
 * is written by the same call.  The array is shared by every call on a
 * device, so calls that overlap in time on one device race and must be
 * serialised by the caller.  The first call on each device looks the array
 * up (cudaGetSymbolAddress).  Kernels run on `stream` (a cudaStream_t, NULL
 * for the default stream) of `device`; every call then synchronises `stream`
 * and copies err to the host before it returns.  Returns 0, or -1 (bad
 * argument), -2 (too many rows), -3 (CUDA error) with the text in msg
 * (msg_cap bytes, may be NULL).  The caller's current device is kept. */
#define LBM_NOALLOC_MAX_ROWS 16384
int lbm_err_fields_noalloc(const double* u, const double* v, const double* u0, const double* v0,
                           int32_t nx, int32_t ny, int64_t pitch, int32_t device, void* stream,
                           double* err, char* msg, int32_t msg_cap);

/* Distributions f (9 planes, FP64) of the current state; set replaces them. */
int lbm_get_f(LbmHandle* h, double* f);
int lbm_set_f(LbmHandle* h, const double* f);

/* The rest of a checkpoint (saveflowfield / readflowfield,
 * solution.f90:1616-1851): the border populations f0 kept since set-up
 * (boundary_condition1 reads them; only move_mesh changes them) as
 * 9 x (2 ny + 2 nx) doubles -- population k at k * (2 ny + 2 nx) + e, e
 * running over the left column (j = 0 .. ny-1), the right column, the
 * bottom row (i = 0 .. nx-1) and the top row -- and the lattice shift count
 * movenum (move_mesh.f90).  Set replaces both. */
int lbm_get_border_f0(LbmHandle* h, double* f0, int32_t* movenum);
int lbm_set_border_f0(LbmHandle* h, const double* f0, int32_t movenum);

/* Band of the last step (adjoint_p, adjoint_wing_id; airfoil.f90:322-333):
 * 3 ints per node (i, j, wing), 1-based, in the reference's order. */
int lbm_get_band(LbmHandle* h, int32_t* n, int32_t* ij_wing, int32_t cap);

/* Marker points xb1, yb1 and segment midpoints xb2, yb2 of the last step. */
int lbm_get_markers(LbmHandle* h, double* xb1, double* yb1, double* xb2, double* yb2);

/* move_mesh (move_mesh.f90:1-336): shift the lattice one column (dr = +1/-1). */
int lbm_move_mesh(LbmHandle* h, int32_t dr);

/* Relative no-slip residual |X du - (ub - X u*)| / |ub - X u*| of the last step. */
int lbm_ibm_residual(LbmHandle* h, double* res);

/* Bit set of numerical warnings since the last call (band capacity, pivot
 * clamps, coupled wings); cleared on read. */
int lbm_status(LbmHandle* h, int32_t* bits);

/* Phase timers, the device-side counterpart of the reference's cpu_time
 * phase totals (main.f90:384-392, 443-456).  When enabled, every step records
 * CUDA events around its kernels; lbm_get_phase_times returns, in ms summed
 * over the timed steps: [0] move_boundary (markers and band), [1]
 * collide-stream (bulk kernel, or stream + moments + collide), [2] band
 * re-collision (FP64 path: none, the collide pass covers it; FP32 path: 0,
 * it is part of [4]), [3] far-field boundary, [4] immersed-boundary
 * right-hand side, substitution, spread and forces (FP32 path: with the band
 * re-collision and the cycle advance), [5] assembly and factorisation of
 * the immersed-boundary system, [6] the number of steps timed, and for the
 * FP32 path's two-step passes [7] their far-tile kernel (also in [1]), [8]
 * the passes timed and [9] the nodes of the far tiles they processed
 * (64 x 8 or 64 x 12 nodes a tile).  On the FP32 path phases 0, 3, 4 and 5 overlap phase 1; in a pass
 * [2] holds the step n + 1 ring and the near tiles.  Enabling (or disabling)
 * clears the totals.  n is the length of out (at most 10 values are
 * written). */
int lbm_set_timing(LbmHandle* h, int32_t enable);
int lbm_get_phase_times(LbmHandle* h, double* out, int32_t n);

/* The CUDA stream (cudaStream_t) the handle's step kernels are ordered on,
 * for callers that record their own events around lbm_step. */
void* lbm_stream(LbmHandle* h);

/* Device memory the handle holds, in bytes. */
int64_t lbm_device_bytes(const LbmHandle* h);

/* Free and total memory of a CUDA device (cudaMemGetInfo), for admitting new
 * episodes by the memory they would take: the online driver creates one
 * episode per RESET (reset_zmq_episode, driver.f90:205-258).  The caller's
 * current device is kept. */
int lbm_mem_info(int32_t device, int64_t* free_bytes, int64_t* total_bytes);

const char* lbm_last_error(const LbmHandle* h);
void lbm_destroy(LbmHandle* h);

/* Packed stepping of many resident episodes (the batched form of the
 * reference's per-episode evolution loop, driver.f90:322-363 once per
 * client): lbm_batch_step advances handle hs[i] by n_steps[i] steps from
 * first_cycle[i] exactly as lbm_step(hs[i], first_cycle[i], n_steps[i],
 * force_rows[i], flags[i]) would, bit for bit, but every kernel of a step is
 * one launch over all episodes still stepping.  FP32-path handles on the
 * batch's device only; each handle at most once; force_rows[i] may be NULL
 * (or force_rows itself), flags NULL means 0.  rcs (may be NULL) receives
 * each handle's status (nonzero: its lbm_last_error text); the call returns
 * 0, or -1 with lbm_batch_last_error naming the first failing episode.  The
 * handles' phase timers are not updated.  A batch object serves one call at
 * a time; handles must not be used by other threads during the call. */
int lbm_batch_create(int32_t device, LbmBatch** out);
int lbm_batch_step(LbmBatch* b, int32_t n, LbmHandle* const* hs, const int64_t* first_cycle,
                   const int64_t* n_steps, double* const* force_rows, const int32_t* flags, int32_t* rcs);
const char* lbm_batch_last_error(const LbmBatch* b);
void lbm_batch_destroy(LbmBatch* b);
int lbm_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
