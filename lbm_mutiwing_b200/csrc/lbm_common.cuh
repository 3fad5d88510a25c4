// Shared device-side definitions: D2Q9 lattice, MRT moment basis, the
// immersed-boundary delta kernel and the device state passed to kernels.
//
// Reference mapping (R-IFFERY/LBM_Mutiwing):
//   velocity set / weights      D2Q9model.f90:5-32
//   MRT matrix M                solution.f90:17-25
//   delta kernel (smooth = 1)   boundary_condition.f90:1580-1600
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lbm {

constexpr int Q = 9;
constexpr double PAI = 3.1415926535897932384626433832795;  // main.f90:9

// Velocity set in the reference's order k = 1..9 (stored 0-based).
__host__ __device__ constexpr int ex(int k) {
    return k == 1 ? 1 : k == 3 ? -1 : k == 5 ? 1 : k == 6 ? -1 : k == 7 ? -1 : k == 8 ? 1 : 0;
}
__host__ __device__ constexpr int ey(int k) {
    return k == 2 ? 1 : k == 4 ? -1 : k == 5 ? 1 : k == 6 ? 1 : k == 7 ? -1 : k == 8 ? -1 : 0;
}

// Weights: single-precision literals 4.0/9.0, 1.0/9.0, 1.0/36.0 widened to
// FP64, exactly as D2Q9model.f90:24-32 stores them.
__host__ __device__ inline double weight(int k) {
    return k == 0 ? (double)(4.0f / 9.0f) : (k <= 4 ? (double)(1.0f / 9.0f) : (double)(1.0f / 36.0f));
}

// MRT matrix M (solution.f90:17-25), row-major M[row][q].
__host__ __device__ constexpr int mrt_m(int r, int q) {
    // rows: rho, e, eps, jx, qx, jy, qy, pxx, pxy
    return r == 0 ? 1
         : r == 1 ? (q == 0 ? -4 : q <= 4 ? -1 : 2)
         : r == 2 ? (q == 0 ? 4 : q <= 4 ? -2 : 1)
         : r == 3 ? ex(q)
         : r == 4 ? (q == 0 ? 0 : q <= 4 ? -2 * ex(q) : ex(q))
         : r == 5 ? ey(q)
         : r == 6 ? (q == 0 ? 0 : q <= 4 ? -2 * ey(q) : ey(q))
         : r == 7 ? (q == 0 ? 0 : q <= 4 ? (ex(q) != 0 ? 1 : -1) : 0)
         : (q <= 4 ? 0 : ex(q) * ey(q));
}

// Status bits written by kernels into DevState::status.
enum StatusBits : int {
    ST_BAND_OVERFLOW = 1,      // band list exceeded its capacity
    ST_BOX_OUTSIDE = 4,        // a segment box left the lattice
    ST_PIVOT_CLAMPED = 8,      // Cholesky pivot clamped (numerically singular IBM system)
    ST_WINGS_COUPLED = 16,     // two wings' supports share lattice nodes: the joint system was solved
    ST_COUPLED_NOCONV = 32,    // the joint solve of such wings did not reach its residual tolerance
    ST_MOTION = 64,            // no motion rows available
    ST_COPY_TIMEOUT = 128,     // a bulk shared-memory copy did not complete within its wait limit
};

constexpr int BOX_SLOTS = 36;   // a +-2.5 spacing box spans at most 6 x 6 nodes
constexpr int BAND_EMPTY = 0x7fffffff;

// delta kernel phi(r), smooth = 1 branch (boundary_condition.f90:1580-1600),
// evaluated with the same operation order (compile with -fmad=false).
__host__ __device__ inline double delta_phi(double disr) {
    const double a = fabs(disr);
    if (a <= 0.5) return 0.375 + 0.03125 * PAI - 0.25 * disr * disr;
    if (a <= 1.5 && a >= 0.5)
        return 0.25 + 0.125 * (1.0 - disr) * sqrt(-2.0 + 8.0 * disr - 4.0 * disr * disr) -
               0.125 * asin(sqrt(2.0) * (disr - 1.0));
    if (a <= 2.5 && a >= 1.5)
        return 1.0625 - 0.015625 * PAI - 0.75 * disr + 0.125 * disr * disr +
               0.0625 * (disr - 2.0) * sqrt(-14.0 + 16.0 * disr - 4.0 * disr * disr) +
               0.0625 * asin(sqrt(2.0) * (disr - 2.0));
    return 0.0;
}

// Per-wing motion state after apply_motion_row (mode.f90:180-218) plus the
// relative-body offsets (mode.f90:473-495).
struct WingMotion {
    double angle, omega, omgac, sa, sau, saac, sb, sbv, sbac;
    double extra_v, extra_s, extra_pos;
};

// Constants of the fused FP32 collision (deviation storage).
struct FusedConsts {
    float s1, s2, s4, s6, s7, s8;   // MRT rates of the non-conserved moments
    float k1, k2, wm1;              // deviation constants (rest-state moments)
};

// Everything a step kernel needs, passed by value.
struct DevState {
    // lattice
    int nx, ny, pitch;           // pitch: row stride in elements for planes and fields
    long long plane;             // pitch * ny
    double scale, uu, ox, oy;
    double s[9];                 // MRT rates
    double minv[81];             // M^-1 (Gauss-Jordan, solution.f90:1474-1529)
    int precision;               // 0 plain FP64, 1 fused FP32 deviation storage
    // plain FP64 path fields
    double* f;                   // 9 planes
    double* f0;                  // 9 planes
    double *rho, *u, *v, *u0, *v0, *pre, *gfx, *gfy;
    // fused path planes (deviation g = f - w) and border f0 store
    float* gA;
    float* gB;
    double* edge_f0;             // 9 x (2 ny + 2 nx): left, right, bottom, top
    double *fo_rho, *fo_u, *fo_v;        // optional output fields (fused path)
    double *fo_u0, *fo_v0;               // previous-step velocity (err)
    // band bookkeeping
    int* band_map;               // ny * pitch: BAND_EMPTY, claiming segment, or -(b + 2)
    unsigned* band_bits;         // fused path: one bit per node (pitched index) set for listed band nodes
    int band_cap;
    int* band_n;                 // [0] current band size, [1] previous band size
    int* band_ij;                // 2 * cap (i, j) 0-based
    int* band_wing;              // cap
    double *band_rho, *band_us, *band_vs, *band_du, *band_dv;   // cap each
    // markers
    int wing_count, npts, nseg;
    const int* wing_pstart;      // W
    const int* wing_sstart;      // W
    const int* wing_npts;        // W
    const int* seg_wing;         // nseg
    const double *xb0, *yb0;     // npts, body frame
    double *xb1, *yb1, *xb2, *yb2;
    int* box;                    // 4 * nseg: i1 i2 j1 j2 (1-based, inclusive)
    int* claim_cnt;              // nseg + 1: band-list offset of each segment's claims
    double *kx, *ky;             // 6 * nseg: delta values of each box column / row
    int* pb;                     // nseg * 36 band index per slot (-1 outside box)
    int* band_claimer;           // cap: segment that claimed each band node
    const int* rpos;             // nseg: position of each segment in its wing's RCM order
    int diag;                    // compute the no-slip residual this step
    int write_fields;            // fused path: this step writes rho, u, v fields
    double *rx, *ry;             // nseg right-hand sides, overwritten by solutions
    double *qx, *qy;             // nseg right-hand sides as built (residual diagnostic, joint solve)
    double* cg_work;             // 8 nseg: residual, preconditioned residual, direction, product (x then y)
    int* solve_count;            // wing blocks of the substitution done this step (joint solve)
    // banded Cholesky per wing (RCM order)
    const int* perm;             // nseg: local position -> global segment
    const int* wing_bw;          // W half bandwidths
    const long long* wing_lofs;  // W offsets into lband
    double* lband;               // sum_w nw*(bw+1), used when not in shared memory
    long long lband_total;       // doubles in lband
    double* piv_floor;           // W pivot floors of the last factorisation
    double* ymax;                // 2 W largest |y| of the last solve, per component (spread scale)
    int* ibm_flags;              // [0] two wings' supports share lattice nodes this step
    double* force_part;          // per-block partial force sums: blocks x W x 3
    int bw_max;                  // largest half bandwidth
    int nw_max;                  // largest segment count of a wing
    int factor_in_smem;          // a wing's banded factor fits in shared memory
    long long factor_smem_off;   // its byte offset in the factor kernel's shared memory
    double* linv;                // inverses of the factor's diagonal blocks, per wing and panel
    const long long* wing_linv_ofs;  // W offsets into linv
    int solve32;                 // the substitution runs in 32-row panels from the panel data in lq
    double* lq;                  // per wing and 32-row panel: MT, R, pivots (built by the factorisation)
    const long long* wing_qofs;  // W offsets into lq
    long long q32_doubles_max;   // largest wing's panel data (doubles)
    int solve_in_smem;           // the substitution copies the wing's factor to shared memory
    int solve_stream;            // otherwise it streams the factor through a ring of rows in shared memory
    long long solve_smem;        // dynamic shared memory of the substitution kernel (bytes)
    // configuration of wing placement
    double wing_x_origin, wing_x_spacing, wing_y_origin, xc, yc;
    // motion source
    int motion_source;           // 1 table, 2 stream
    int ncol;
    const double* step_table;    // step_rows x ncol
    long long step_rows;
    double motion_dt;
    double* stream_start;        // ncol
    double* stream_target;       // ncol
    WingMotion* wm;              // W, written by the IBM kernel each step
    // relative body state (zero unless coupled dynamics are enabled)
    double *rel_pos;             // W
    // step bookkeeping
    long long* cycle;            // device copy of the current cycle number
    long long* gcycle;           // cycle of the next geometry to build (advanced by the band list kernel)
    int* fin_count;              // fused path: blocks of the closing kernel done this step
    int slot_items;              // box slots (or G entries) per thread in the per-slot kernels
    double* force_rows;          // rows of 4 + 12 W, indexed by step within segment
    long long* row_index;        // step within segment
    int force_rows_cap;
    double* sum_row;             // 4 + 12 W
    int* sample_count;
    int* status;
    int movenum;                 // lattice shifts so far (move_mesh)
    double* wing_fm;             // 3 W raw per-wing Fx, Fy, M of the last step
    double* ibm_resid;           // [0] |X du - r|^2, [1] |r|^2
    FusedConsts fc;              // fused path: collision constants
    // two-step passes (fused path): lattice tiles of PASS_TX x pass_rows
    // nodes; a tile is flagged when it or a neighbour of it holds a band
    // node of this geometry set (its first step then needs the band's values)
    unsigned char* tile_flags;   // pass_ntx * pass_nty (null: not tracked)
    int* tile_list;              // the flagged tiles, compacted by the scan kernel
    int* tile_n;                 // [0] flagged tiles
    int pass_ntx, pass_nty, pass_rows;
};

__host__ __device__ inline long long pidx(const DevState& d, int i, int j) {
    return (long long)j * d.pitch + i;   // 0-based (i, j)
}

// Programmatic dependent launch (the chain of the immersed boundary): a
// kernel launched with programmatic stream serialization (launch_chained)
// may be scheduled while its predecessor in the stream still runs, once
// every block of the predecessor has called pdl_release(); pdl_wait() then
// holds it until the predecessor grid has completed and its writes are
// visible.  Both are no-ops for kernels launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Launches kernel k; chained: with programmatic stream serialization (the
// kernel must begin with pdl_wait() before it touches what its predecessor
// writes or reads).
template <class... P, class... A>
inline cudaError_t launch_chained(bool chained, void (*k)(P...), int grid, int block, size_t smem,
                                  cudaStream_t st, const A&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = chained ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

}  // namespace lbm
