/*
 * CPU FP64 oracle for the LBM_Mutiwing time step — TEST INFRASTRUCTURE ONLY.
 *
 * This header declares a sequential C++ restatement of the reference
 * Fortran solver's CPU semantics (OpenACC directives ignored, one MPI rank).
 * Only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark load it; the product library never links or calls it.
 *
 * Parity status: the reference cannot be compiled in this environment (no
 * Fortran compiler) and ships no golden vectors, so this restatement is
 * "parity unpinned" against the reference's own binary.  It is pinned
 * against known-answer tests derived from the reference's equations
 * (tests/test_oracle_kat.py) and against the reference's shipped fixtures
 * (boundary.dat geometry, motion_params.dat table) copied as data only.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field meanings as LbmConfig in include/lbm_mutiwing.h. */
typedef struct OraConfig {
    int32_t nx, ny;
    double scale;
    double uu;
    double re;
    double ox, oy;
    double s[9];            /* s[7], s[8] <= 0 selects 1/tau */
    int32_t wing_count;
    double wing_x_origin, wing_x_spacing, wing_y_origin;
    double xc, yc;
    int32_t motion_source;  /* 1 file table, 2 online stream */
} OraConfig;

void*  ora_create(const OraConfig* cfg, const double* markers_xy,
                  const int32_t* points_per_wing, int32_t nthreads);
void   ora_destroy(void* h);
int    ora_set_motion_table(void* h, const double* rows, int64_t nrows, int32_t ncols);
int    ora_set_stream_rows(void* h, const double* start_row, const double* target_row);
/* One pass of the offline loop body (main.f90:374-441) for cycle n:
 * erranalysis (n>=2), evolution, move_mesh check.  force_row receives
 * 4+12W doubles (may be NULL). */
int    ora_step(void* h, int64_t n, double* force_row);
double ora_err(void* h);
double ora_tau(void* h);
/* which: 0 rho 1 u 2 v 3 pre 4 u0 5 v0 6 gforce_x 7 gforce_y;
 *        100+k f plane k (0-based), 200+k f0 plane k.  out: nx*ny, x fastest. */
int    ora_get_field(void* h, int32_t which, double* out);
int    ora_set_f(void* h, const double* f);   /* overwrite f (9 planes) */
/* band list: ij_wing receives 3 ints per entry (i, j, wing), 1-based. */
int    ora_get_band(void* h, int32_t* n, int32_t* ij_wing, int32_t cap);
int    ora_get_markers(void* h, double* xb1, double* yb1, double* xb2, double* yb2);
int    ora_get_sums(void* h, double* sum_row, int32_t* sample_count, int32_t* row_len);
void   ora_reset_sums(void* h);
/* motion helpers restated from mode.f90 (for KATs) */
int    ora_stream_row(void* h, double t, double* row);
int    ora_build_stream_target_row(void* h, const double* start_row, double target_time,
                                   const double* delta_row, double* target_row);
void   ora_interpolate_triplet(double s0, double v0, double v1, double dt, double local_t,
                               double* s, double* v, double* a);
double ora_delta_phi(double r);
void   ora_inverse_m(double* minv81);
int    ora_move_mesh(void* h, int32_t dr);
/* IBM diagnostics of the last step: constraint residual |X(u*+du)-ub| / |ub-Xu*| */
double ora_ibm_residual(void* h);

#ifdef __cplusplus
}
#endif
#endif
