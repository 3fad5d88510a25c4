// Host-side launch wrappers for the device kernels.
#pragma once
#include "lbm_common.cuh"

namespace lbm {

// plain FP64 path (kernels_fp64.cu)
void launch_plain_stream(const DevState& d, cudaStream_t st);
void launch_plain_moments(const DevState& d, cudaStream_t st);
void launch_plain_collide(const DevState& d, cudaStream_t st);
void launch_plain_shift(const DevState& d, int dr, cudaStream_t st);
// strided output fields u/UU, v/UU, pre, vorticity (4 planes of onx x ony)
void launch_output_fields(const DevState& d, int sx, int sy, double* out, cudaStream_t st);
// both paths
void launch_outer_bc(const DevState& d, cudaStream_t st);
void launch_err(const DevState& d, double* partial, double* out, cudaStream_t st);
int err_partial_count();

// fused FP32 path (kernels_fp32.cu)
FusedConsts fused_consts(const DevState& d);
// tmap (may be null): the CUtensorMap of d.gA's planes (fused_tensor_map);
// steps that write no fields then stage their pulls through shared memory
// by tensor loads
void launch_fused_bulk(const DevState& d, const FusedConsts& c, bool fields, const void* tmap, cudaStream_t st);
// Tensor map (a 128-byte CUtensorMap written to out) of the nine planes at
// base, for the tiled bulk kernel; 0 on success.
int fused_tensor_map(const DevState& d, const float* base, void* out);
bool is_bulk_kernel(const void* func);   // the bulk kernel (low priority in graphs)
bool is_far_field_kernel(const void* func);
void launch_fused_bc(const DevState& d, cudaStream_t st);   // far field of the fused path
void launch_fused_init(const DevState& d, cudaStream_t st);
void launch_fused_shift(const DevState& d, int dr, cudaStream_t st);
void launch_fused_export(const DevState& d, const float* g, double* f, cudaStream_t st);
void launch_fused_import(const DevState& d, const double* f, float* g, cudaStream_t st);

// Two-step pass n -> n + 2 of the fused path (kernels_fp32.cu).  Tile (tx,
// ty) covers the interior nodes [PASS_TX tx, PASS_TX tx + PASS_TX - 1] x
// [1 + PASS_TY ty, PASS_TY (ty + 1)]; its first step needs the tile and one
// ring of neighbours (R1), its pulls a second ring.
// Tiles of PASS_TX columns and, per handle, PASS_TY rows or PASS_TY_TALL
// rows: the taller tile recomputes a smaller share of its nodes (R1 against
// the tile) and runs three blocks per SM instead of four; it pays where the
// far tiles bound the pass (large lattices), the shorter one where the
// immersed-boundary chains do (PASS_TALL_NODES: the lattice size from which
// a handle takes the tall tiles).
#ifndef LBM_PASS_TX
#define LBM_PASS_TX 64
#endif
#ifndef LBM_PASS_TY
#define LBM_PASS_TY 8
#endif
#ifndef LBM_PASS_TY_TALL
#define LBM_PASS_TY_TALL 12
#endif
constexpr int PASS_TX = LBM_PASS_TX, PASS_TY = LBM_PASS_TY, PASS_TY_TALL = LBM_PASS_TY_TALL;
constexpr long long PASS_TALL_NODES = 32LL << 20;
// flagged tiles a support box can touch: its 6 nodes and the ring either
// side span 8 nodes in each direction
constexpr int pass_tiles_per_segment(int rows) { return ((8 + PASS_TX - 1) / PASS_TX + 1) * ((8 + rows - 1) / rows + 1); }
inline int pass_tiles_x(int nx) { return (nx + PASS_TX - 1) / PASS_TX; }
inline int pass_tiles_y(int ny, int rows) { return (ny - 2 + rows - 1) / rows; }
// whether R1 of tile (tx, ty) of `rows` rows holds a node of the lattice border
inline __host__ __device__ bool pass_border_tile(int tx, int ty, int nx, int ny, int rows) {
    const int x0 = tx * PASS_TX, y0 = 1 + ty * rows;
    return x0 - 1 <= 0 || x0 + PASS_TX >= nx - 1 || y0 - 1 <= 0 || y0 + rows >= ny - 1;
}
// The collision's constants as pairs (both lanes equal), for the paired
// FP32 instructions of the far tiles: in the kernel's parameters they are
// operands as they stand, instead of pairs rebuilt in registers at each use.
struct PassPairs {
    float2 m1, p2, m2, p3, m3, p4, m4, r4, r6, r9, r12, r36, wm1, mk1, k2, s1, s2, ms4, ms6, s7, s8;
};
PassPairs pass_pairs(const FusedConsts& c);
struct PassArgs {
    const float* P;              // planes of step n (read by the tensor map)
    const float* O;              // planes of step n + 1: band nodes of step n and the border
    float* Q;                    // planes of step n + 2
    const unsigned* bits0;       // band bits of step n's geometry
    const unsigned* bits1;       // band bits of step n + 1's geometry
    const unsigned char* flags0; // tile flags of step n's geometry
    const int* border_list;      // tiles whose R1 meets the border
    const int* band_list;        // flagged tiles of step n's geometry
    const int* band_n;           // their count
    int nborder, band_cap;       // border tiles; capacity of the flagged-tile list
    int nx, ny, pitch, ntx, nty;
    int rows;                    // tile rows: PASS_TY or PASS_TY_TALL
    long long plane;
    FusedConsts c;
    PassPairs k;
    int* status;
    int* far_tiles;              // counts the far tiles processed (null: not counted)
};
// Tensor map of the nine planes at base for the boxes of the pass kernels
// with tiles of `rows` rows (PASS_TY or PASS_TY_TALL).
int pass_tensor_map(const DevState& d, const float* base, int rows, void* out);
// far tiles (every tile not flagged and off the border), from P alone
void launch_pass_far(const PassArgs& a, const void* tmap, cudaStream_t st);
// the border tiles and the flagged tiles, after the band and the far field
// of step n have written their step n + 1 values to O
void launch_pass_near(const PassArgs& a, const void* tmap, cudaStream_t st);
// Step n + 1 values (from P) in O where the second step's immersed boundary
// and far field read them: the support boxes of step n + 1's geometry and
// one ring around them (d: that geometry), and the columns 1..3, nx-4..nx-2
// and rows 1, 2, ny-3, ny-2; band nodes of step n (bits0) are left to the
// band re-collision.
void launch_pass_ring(const DevState& d, const float* P, float* O, const unsigned* bits0, cudaStream_t st);
// raises the pass kernels' shared-memory limit (the calling thread's device)
cudaError_t pass_prepare();
bool is_pass_far_kernel(const void* func);
bool is_pass_near_kernel(const void* func);

// immersed boundary (ibm.cu)
// move_boundary: motion, markers, boxes, band list; geometry_done (may be
// null) is recorded once the boxes and kernel values exist
void launch_ibm_band(const DevState& d, cudaStream_t st, cudaEvent_t geometry_done);
// assembly and factorisation of G (needs the geometry only)
void launch_ibm_factor(const DevState& d, size_t factor_smem, cudaStream_t st);
// u*, right-hand side (needs the band list; on the plain path also the moments)
void launch_ibm_rhs(const DevState& d, bool fused, cudaStream_t st);
// substitution, spread, velocity correction, forces (needs rhs and factor);
// on the fused path also the band nodes' re-collision (fields: write rho,
// u, v there) and the cycle advance.  chained: the substitution, spread and
// closing kernel go out with programmatic stream serialization, each
// scheduled while its predecessor (the rhs first) still runs
void launch_ibm_solve(const DevState& d, bool fused, bool fields, cudaStream_t st, bool chained = false);
int ibm_finish_blocks(const DevState& d);
// kernels of a step's geometry (motion through factorisation)
bool is_geometry_kernel(const void* func);
bool is_factor_kernel(const void* func);
// banded L' D L'^T factorisation and substitution (ibm_solver.cu)
cudaError_t ibm_prepare(size_t factor_smem, size_t solve_smem);
// dynamic shared memory of the substitution kernel
size_t ibm_solve_smem(int nw_max, int bw_max, long long wing_storage_max, bool factor_in_smem);
// shared memory of the row ring when the factor is streamed, and whether
// its slot count is within the kernel's barrier table
size_t ibm_solve_ring_bytes(int bw);
bool ibm_solve_ring_fits(int bw);
// shared memory of the factorisation kernel ahead of the wing's storage
// (a multiple of 16 bytes)
size_t ibm_factor_staging_bytes(int bw_max);
void launch_ibm_factor_blocks(const DevState& d, size_t factor_smem, cudaStream_t st);
void launch_ibm_substitution(const DevState& d, size_t solve_smem, cudaStream_t st, bool chained = false);
// 32-row panel substitution: doubles of a wing's panel data, and the
// kernel's dynamic shared memory for the largest wing's panel data
long long ibm_panel32_storage(int nw, int bw);
size_t ibm_solve32_smem(long long q32_doubles_max, int nw_max, int bw_max);
constexpr int IBM_PANEL = 8;            // columns per factorisation panel
constexpr int IBM_MAX_BANDWIDTH = 160;  // staged panel rows and pair table stay within shared memory
// Banded storage of a wing's G: row p holds G(p, p - dd) at dd = 0..bw.
// The row stride covers bw + IBM_PANEL + 1 entries, so the entries past bw
// form a zero zone, and a zero row precedes row 0 and IBM_PANEL + bw zero
// rows follow the last: a panel's rows and columns can then be read without
// bounds tests (entries above the diagonal alias the previous row's zero
// zone).  The stride is even, so the diagonal-major accesses of a warp hit
// distinct shared-memory banks.
inline __host__ __device__ int ibm_ld(int bw) { return (bw + IBM_PANEL + 2) & ~1; }
inline __host__ __device__ long long ibm_wing_storage(int nw, int bw) {
    return (long long)(1 + nw + IBM_PANEL + bw) * ibm_ld(bw);
}
// Per panel of a wing's factor: the inverse of its unit lower diagonal block
// (row-major IBM_PANEL x IBM_PANEL) followed by the IBM_PANEL reciprocal
// pivots (zero past the last segment).
constexpr int IBM_PANEL_AUX = IBM_PANEL * IBM_PANEL + IBM_PANEL;
inline __host__ __device__ long long ibm_linv_storage(int nw) {
    return (long long)((nw + IBM_PANEL - 1) / IBM_PANEL) * IBM_PANEL_AUX;
}
void launch_step_advance(const DevState& d, cudaStream_t st);        // cycle += 1

// Packed launches: one grid covers the blocks of several episodes, block b
// running the kernel of episode e = max{e : boff[e] <= b} with local block
// index b - boff[e] (multi.cuh).  The fused path's kernels only; the bulk
// and closing kernels take the field flag from each episode's state.
enum MultiKernel : int {
    MK_GEOMETRY, MK_CLAIM, MK_COUNT, MK_SCAN, MK_LIST, MK_ASSEMBLE,   // geometry of a step
    MK_RHS, MK_SPREAD, MK_FINISH,                                      // immersed boundary
    MK_FACTOR_SMEM, MK_FACTOR_GLOBAL, MK_SOLVE32, MK_SOLVE_SMEM, MK_SOLVE_GLOBAL,  // banded solver
    MK_BULK1, MK_BULK2, MK_BULK4, MK_BC,   // lattice (bulk: 1, 2 or 4 node runs per block)
    MK_KINDS
};
struct MultiArgs {
    const DevState* const* ds;   // ne episode states (device memory)
    const int* boff;             // ne + 1 block offsets (device memory)
    int ne;
};
// blocks of one episode in the packed launch of k (0: none); -1 if k is not
// handled by that file
int multi_blocks_ibm(MultiKernel k, const DevState& d);
int multi_blocks_solver(MultiKernel k, const DevState& d);
int multi_blocks_fused(MultiKernel k, const DevState& d);
bool launch_multi_ibm(MultiKernel k, const MultiArgs& m, int blocks, cudaStream_t st);
bool launch_multi_solver(MultiKernel k, const MultiArgs& m, int blocks, size_t smem, cudaStream_t st);
bool launch_multi_fused(MultiKernel k, const MultiArgs& m, int blocks, cudaStream_t st);
bool is_bulk_multi_kernel(const void* func);
// packed kernels that take the middle priority (far field, geometry built
// ahead, factorisation), for the nodes of packed step graphs
bool is_far_field_multi_kernel(const void* func);
bool is_geometry_multi_kernel(const void* func);
bool is_factor_multi_kernel(const void* func);

}  // namespace lbm
