// Banded L' D L'^T factorisation and substitution for the immersed-boundary
// system G y = r of each wing (G = X X^T in reverse Cuthill-McKee order; see
// ibm.cu for how G arises from immersed_boundary_Wu,
// boundary_condition.f90:1558-1640).
//
// Blocked right-looking algorithm, PANEL = 8 columns at a time, one thread
// block per wing, the wing's banded matrix held in shared memory (brought in
// and written back with bulk copies).  Per panel p, two phases separated by
// block barriers:
//   B  every row below the panel (bw of them, one thread each) becomes
//      L'(i, p) = A(i, p) L_pp^-T D_p^-1 by an 8-step forward substitution;
//      a spare warp forms the inverse of L_pp for the substitution kernel;
//   A  the rank-8 update of the trailing window, in 4 x 4 register tiles by
//      warps 1.., while warp 0 updates the next panel's 8 x 8 diagonal block
//      first and one thread factors it in registers (look-ahead: the
//      sequential pivot chain of panel p + 1 overlaps panel p's update).
// The substitution applies each panel through its stored 8 x 8 inverse and
// reciprocal pivots and updates the rows below (forward) or above
// (backward) it, one warp per velocity component.
//
// The zero zones of the banded storage (entries past the bandwidth, rows past
// the last segment) make every panel-shaped read in bounds and zero where it
// falls outside the matrix, so the inner loops load without conditions.
#include <mutex>

#include "bulk_copy.cuh"
#include "lbm_kernels.h"
#include "multi.cuh"

namespace lbm {

constexpr int PANEL = IBM_PANEL;
constexpr int FACTOR_THREADS = 256;
constexpr int FACTOR_WARPS = FACTOR_THREADS / 32;
constexpr int SOLVE_THREADS = 64;
constexpr int SP = PANEL + 1;           // odd row stride of staged panel rows
constexpr int TILE = 4;                 // register tile of the trailing update
static_assert(IBM_MAX_BANDWIDTH <= FACTOR_THREADS - 32, "rows below a panel leave the last warp free");
static_assert(PANEL == 2 * TILE, "the next diagonal block is three tiles");

__device__ inline void solver_status(const DevState& d, int bit) { atomicOr(d.status, bit); }

// 1/x by Newton-Raphson (r <- r + r (1 - x r), twice) from the hardware
// approximation rcp.approx.ftz.f64; the relative error of the seed squares
// at each step, ending at the rounding level for the positive normal pivots
// met here.
__device__ inline double recip(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = __fma_rn(r, __fma_rn(-x, r, 1.0), r);
    r = __fma_rn(r, __fma_rn(-x, r, 1.0), r);
    return r;
}

// Packed lower triangle.
__host__ __device__ constexpr int tri(int x, int y) { return x * (x + 1) / 2 + y; }
// Row of packed index t.
__device__ inline int tri_row(int t) {
    int r = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > t) --r;
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    return r;
}
inline int round_tile(int n) { return (n + TILE - 1) / TILE * TILE; }

// One thread factors the diagonal block of the panel at k0 (np columns, the
// rest zero rows) held in storage and leaves the strictly lower part of its
// unit factor in Lpp and the reciprocal pivots (zero past np) in idp.
// Pivots not above fl are clamped to fl; returns whether any was.
__device__ inline bool factor_diagonal_block(const double* A, int ld, int k0, int np, double fl, double (*Lpp)[SP],
                                             double* idp) {
    double a[tri(PANEL, 0)];
#pragma unroll
    for (int x = 0; x < PANEL; ++x)
#pragma unroll
        for (int y = 0; y <= x; ++y) a[tri(x, y)] = A[(k0 + x) * ld + (x - y)];
    bool clamped = false;
#pragma unroll
    for (int c = 0; c < PANEL; ++c) {
        const bool live = c < np;
        double dc = a[tri(c, c)];
        const bool low = live && !(dc > fl);
        clamped |= low;
        dc = low ? fl : dc;
        double ic = recip(dc);
        ic = live ? ic : 0.0;
        idp[c] = ic;
        double l[PANEL];
#pragma unroll
        for (int x = c + 1; x < PANEL; ++x) l[x] = a[tri(x, c)] * ic;
#pragma unroll
        for (int x = c + 1; x < PANEL; ++x)
#pragma unroll
            for (int y = c + 1; y <= x; ++y) a[tri(x, y)] = a[tri(x, y)] - l[x] * a[tri(y, c)];
#pragma unroll
        for (int x = c + 1; x < PANEL; ++x) a[tri(x, c)] = l[x];
    }
#pragma unroll
    for (int x = 1; x < PANEL; ++x)
#pragma unroll
        for (int y = 0; y < x; ++y) Lpp[x][y] = a[tri(x, y)];
    return clamped;
}

// Substitution in panels of Q32 = 32 rows on the step's chain.  Per wing and
// panel q (rows k0 = 32 q ..), built by the factorisation kernel from the
// factor it holds: MT, the transposed inverse of the panel's unit lower
// diagonal block of L' (MT[c][l] = M[l][c], rows padded to 33 doubles);
// R, the coupling of the bw rows below the panel to the panel's columns
// (R[rb][c] = L'(k0 + np + rb, k0 + c), padded to 33); and the panel's
// reciprocal pivots.  Rows past the wing's last segment are identity in M
// and zero in R and the pivots.
constexpr int Q32 = 32, Q32P = 33;
__host__ __device__ inline int qpanels(int nw) { return (nw + Q32 - 1) / Q32; }
__host__ __device__ inline long long panel32_doubles(int bw) {
    return ((long long)Q32P * (Q32 + bw) + Q32 + 1) & ~1LL;   // even: 16-byte multiples
}
long long ibm_panel32_storage(int nw, int bw) { return qpanels(nw) * panel32_doubles(bw); }

// One warp builds panel q: lane c forms column c of M by block forward
// substitution over the panel's four factor panels, the entries off the
// 8 x 8 diagonal blocks from the banded storage A (row 0), the diagonal
// blocks through their stored inverses in aux.
__device__ __noinline__ void build_panel32(const double* A, int ld, const double* aux, int nw, int bw, int q,
                                           double* out, int lane) {
    const int k0 = q * Q32, np = min(Q32, nw - k0), c = lane;
    double x[Q32];
#pragma unroll
    for (int a8 = 0; a8 < Q32 / PANEL; ++a8) {
        double sv[PANEL];
#pragma unroll
        for (int i = 0; i < PANEL; ++i) {
            const int r = a8 * PANEL + i;
            double acc = (r == c) ? 1.0 : 0.0;
            if (r < np) {
                const double* row = A + (long long)(k0 + r) * ld;   // entry r - m: column k0 + m
#pragma unroll
                for (int m = 0; m < a8 * PANEL; ++m)
                    if (m >= c && r - m <= bw) acc = acc - row[r - m] * x[m];
            }
            sv[i] = acc;
        }
        const bool in_wing = a8 * PANEL < np;
        const double* Li = aux + (long long)(k0 / PANEL + a8) * IBM_PANEL_AUX;
#pragma unroll
        for (int i = 0; i < PANEL; ++i) {
            double v = sv[i];
            if (in_wing && a8 * PANEL + i < np) {
                v = 0.0;
#pragma unroll
                for (int k = 0; k < PANEL; ++k) v = v + Li[i * PANEL + k] * sv[k];
            }
            x[a8 * PANEL + i] = v;
        }
    }
    double* MT = out;
    double* R = out + Q32P * Q32;
    double* piv = R + Q32P * bw;
#pragma unroll
    for (int l = 0; l < Q32; ++l) MT[c * Q32P + l] = x[l];
    for (int rb = 0; rb < bw; ++rb) {
        const int dd = np + rb - c;   // row k0 + np + rb, column k0 + c
        const int i = k0 + np + rb;
        R[rb * Q32P + c] = (c < np && dd >= 1 && dd <= bw && i < nw) ? A[(long long)i * ld + dd] : 0.0;
    }
    const int k = k0 + lane;
    piv[lane] = k < nw ? aux[(long long)(k / PANEL) * IBM_PANEL_AUX + PANEL * PANEL + (k % PANEL)] : 0.0;
}

// Storage (ibm_wing_storage): row p of wing w at S + (p + 1) * ld, entry dd
// holding column p - dd.  On exit: L'(i, k) for every entry below the
// diagonal blocks, and per panel the inverse of its unit lower diagonal
// block and the reciprocal pivots in d.linv (the diagonal blocks of the
// storage are left as scratch).  Pivots below 1e-15 of the largest diagonal
// are clamped (numerically singular systems made by marker clusters finer
// than the lattice).  SMEM: the storage is worked on in shared memory (the
// template parameter lets every access compile to a shared-memory access).
template <bool SMEM>
__device__ __forceinline__ void ibm_factor_kernel_body(const DevState& d, const int bid_) {
    extern __shared__ __align__(16) double smem[];
    const int w = bid_;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], ld = ibm_ld(bw);
    const int bwr = (d.bw_max + TILE - 1) / TILE * TILE;
    double* Ps = smem;                        // [bwr][SP] rows below the panel, scaled (L')
    double* Pu = Ps + SP * bwr;               // [bwr][SP] unscaled (L' D)
    short2* tiles = reinterpret_cast<short2*>(Pu + SP * bwr);   // tiles of the remaining rows
    __shared__ double red[FACTOR_WARPS];
    __shared__ double Lpp[PANEL][SP];         // strictly lower part of the panel's unit lower block
    __shared__ double idp[PANEL];             // reciprocal pivots of the panel
    __shared__ uint64_t bar;
    const long long wsize = ibm_wing_storage(nw, bw);
    double* gS = d.lband + d.wing_lofs[w];
    double* S = gS;
    constexpr bool in_smem = SMEM;
    if (in_smem) {
        S = reinterpret_cast<double*>(reinterpret_cast<char*>(smem) + d.factor_smem_off);
        if (tid == 0) {
            mbar_init(&bar, 1);
            mbar_arrive_expect_tx(&bar, (uint32_t)(wsize * 8));
            bulk_load_all(S, gS, wsize * 8, &bar);
        }
    }
    double* A = S + ld;   // row 0
    double* aux = d.linv + d.wing_linv_ofs[w];
    for (int t = tid; t < 2 * SP * bwr; t += FACTOR_THREADS) Ps[t] = 0.0;   // rows past bw stay zero
    // the next diagonal block: entries (x, y), y <= x < b8; the remaining
    // rows of the trailing window in TILE x TILE tiles (X, Y), Y <= X,
    // X >= PANEL / TILE
    const int b8 = min(bw, PANEL), n8 = tri(b8, 0);
    const int nt = (bw + TILE - 1) / TILE;
    const int nrem = nt > PANEL / TILE ? tri(nt, 0) - tri(PANEL / TILE, 0) : 0;
    for (int t = tid; t < nrem; t += FACTOR_THREADS) {
        const int tt = t + tri(PANEL / TILE, 0), X = tri_row(tt);
        tiles[t] = make_short2((short)X, (short)(tt - tri(X, 0)));
    }
    int ex[2], ey[2];   // warp 0: entries lane and lane + 32 of the next diagonal block
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int t = min(lane + 32 * h, tri(PANEL, 0) - 1);
        ex[h] = tri_row(t);
        ey[h] = t - tri(ex[h], 0);
    }
    __syncthreads();
    if (in_smem) {
        const bool ok = mbar_wait(&bar, 0);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) solver_status(d, ST_COPY_TIMEOUT);
            mbar_wait(&bar, 0);   // let a late copy land before the block exits
            return;
        }
    }
    double mx = 0.0;
    for (int p = tid; p < nw; p += FACTOR_THREADS) mx = fmax(mx, A[p * ld]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    mx = 0.0;
    for (int k = 0; k < FACTOR_WARPS; ++k) mx = fmax(mx, red[k]);
    const double fl = mx > 0.0 ? 1e-15 * mx : 1.0;
    bool clamped = false;
    if (tid == 0) clamped = factor_diagonal_block(A, ld, 0, min(PANEL, nw), fl, Lpp, idp);
    __syncthreads();

    const int npan = (nw + PANEL - 1) / PANEL;
    for (int pan = 0; pan < npan; ++pan) {
        const int k0 = pan * PANEL, k1 = min(k0 + PANEL, nw);
        // B. rows below the panel: u = A(i, p) L_pp^-T, L'(i, p) = u / d
        // (past the last segment the rows and the pivots are zero)
        if (tid < bw) {
            const int rb = tid, i = k1 + rb;
            double* rw = A + i * ld + (i - k0);   // entry of column k0 + c at rw[-c]
            double u[PANEL], lo[tri(PANEL, 0)], ip[PANEL];
#pragma unroll
            for (int c = 0; c < PANEL; ++c) u[c] = rw[-c];
#pragma unroll
            for (int c = 1; c < PANEL; ++c)
#pragma unroll
                for (int k = 0; k < c; ++k) lo[tri(c, k)] = Lpp[c][k];
#pragma unroll
            for (int c = 0; c < PANEL; ++c) ip[c] = idp[c];
#pragma unroll
            for (int c = 1; c < PANEL; ++c)
#pragma unroll
                for (int k = 0; k < c; ++k) u[c] = u[c] - lo[tri(c, k)] * u[k];
#pragma unroll
            for (int c = 0; c < PANEL; ++c) {
                const double lv = u[c] * ip[c];
                Pu[rb * SP + c] = u[c];
                Ps[rb * SP + c] = lv;
                rw[-c] = lv;
            }
        } else if (warp == FACTOR_WARPS - 1 && lane < PANEL) {
            // inverse of the unit lower block, column lane, and the pivots
            const int l = lane;
            double x[PANEL];
#pragma unroll
            for (int k = 0; k < PANEL; ++k) {
                double s = (k == l) ? 1.0 : 0.0;
#pragma unroll
                for (int m = 0; m < k; ++m) s = s - Lpp[k][m] * x[m];
                x[k] = (k < l) ? 0.0 : s;
            }
            double* blk = aux + (long long)pan * IBM_PANEL_AUX;
#pragma unroll
            for (int k = 0; k < PANEL; ++k) blk[k * PANEL + l] = x[k];
            blk[PANEL * PANEL + l] = idp[l];
        }
        __syncthreads();
        if (pan + 1 == npan) break;   // later updates only touch the zero rows past the end
        // A. trailing update; warp 0 takes the next diagonal block first
        if (warp == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (lane + 32 * h >= n8) break;
                const int x = ex[h], y = ey[h];
                const double* pa = Ps + x * SP;
                const double* pb = Pu + y * SP;
                double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
                for (int c = 0; c < PANEL / 2; ++c) {
                    acc0 = acc0 + pa[c] * pb[c];
                    acc1 = acc1 + pa[c + PANEL / 2] * pb[c + PANEL / 2];
                }
                double* e = A + (k1 + x) * ld + (x - y);
                *e = *e - (acc0 + acc1);
            }
            __syncwarp();
            if (lane == 0) clamped |= factor_diagonal_block(A, ld, k1, min(PANEL, nw - k1), fl, Lpp, idp);
        } else {
          for (int t = tid - 32; t < nrem; t += FACTOR_THREADS - 32) {
            const short2 tl = tiles[t];
            const int x0 = TILE * tl.x, y0 = TILE * tl.y;
            double acc[TILE][TILE];
#pragma unroll
            for (int r = 0; r < TILE; ++r)
#pragma unroll
                for (int s = 0; s < TILE; ++s) acc[r][s] = 0.0;
#pragma unroll
            for (int c = 0; c < PANEL; ++c) {
                double pa[TILE], pb[TILE];
#pragma unroll
                for (int r = 0; r < TILE; ++r) {
                    pa[r] = Ps[(x0 + r) * SP + c];
                    pb[r] = Pu[(y0 + r) * SP + c];
                }
#pragma unroll
                for (int r = 0; r < TILE; ++r)
#pragma unroll
                    for (int s = 0; s < TILE; ++s) acc[r][s] = acc[r][s] + pa[r] * pb[s];
            }
#pragma unroll
            for (int r = 0; r < TILE; ++r)
#pragma unroll
                for (int s = 0; s < TILE; ++s) {
                    const int x = x0 + r, y = y0 + s;
                    if (x < bw && y <= x) {
                        double* e = A + (k1 + x) * ld + (x - y);
                        *e = *e - acc[r][s];
                    }
                }
          }
        }
        __syncthreads();
    }
    if (clamped) solver_status(d, ST_PIVOT_CLAMPED);
    if (d.solve32) {
        __syncthreads();   // the factor, the 8 x 8 inverses and the pivots are complete
        for (int q = warp; q < qpanels(nw); q += FACTOR_WARPS)
            build_panel32(A, ld, aux, nw, bw, q, d.lq + d.wing_qofs[w] + (long long)q * panel32_doubles(bw), lane);
    }
    if (in_smem) {
        fence_async_smem();
        __syncthreads();
        if (tid == 0) bulk_store_all(gS, S, wsize * 8);
    }
}
template <bool SMEM>
__global__ void __launch_bounds__(FACTOR_THREADS) ibm_factor_kernel(DevState d) { ibm_factor_kernel_body<SMEM>(d, blockIdx.x); }
template <bool SMEM>
__global__ void __launch_bounds__(FACTOR_THREADS) ibm_factor_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_factor_kernel_body<SMEM>(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Streaming of a wing's factor through shared memory when it does not fit
// whole: chunks of RING_ROWS consecutive rows (contiguous in global memory)
// are brought in by bulk copies into a ring of slots, each slot led by a
// zero row (the forward pass reads a little above the diagonal, which the
// banded layout keeps at zero in the previous row).  The forward pass needs
// the bw rows below the current panel, the backward pass the panel's own
// rows; the next chunk is in flight while the current ones are used.
constexpr int RING_ROWS = 16;
constexpr int RING_MAX_SLOTS = 16;
static_assert(RING_ROWS % PANEL == 0, "a panel's rows lie in one chunk");
__host__ __device__ inline int ring_slots(int bw) { return (bw + PANEL + RING_ROWS - 1) / RING_ROWS + 2; }
size_t ibm_solve_ring_bytes(int bw) { return (size_t)ring_slots(bw) * (RING_ROWS + 1) * ibm_ld(bw) * sizeof(double); }
bool ibm_solve_ring_fits(int bw) { return ring_slots(bw) <= RING_MAX_SLOTS; }

// ------------------------------------------------- joint solve of coupled wings
// When two wings' supports share lattice nodes, G has entries between their
// segments and the per-wing factors alone solve a different system from the
// reference's one dense system over all segments (boundary_condition.f90:
// 1609-1640).  The joint system G y = r is then solved by conjugate
// gradients preconditioned with the per-wing factors (G is symmetric
// positive definite, the preconditioner block diagonal), starting from the
// per-wing solution.  One warp per velocity component; products G p are
// formed as X (X^T p): a spread onto the band nodes with 64-bit fixed-point
// integer atomics (order-independent, so results are reproducible) and an
// interpolation back; dot products are lane-strided sums added by a fixed
// butterfly.  The iteration stops when the recursive residual is below
// CG_TOL of |r|, or after CG_MAXIT iterations (then ST_COUPLED_NOCONV).
constexpr int CG_MAXIT = 200;
constexpr double CG_TOL = 1e-13;

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// out = G in for one component; acc holds that component's band
// accumulators, zero on entry and left zero.
__device__ void cg_product(const DevState& d, const double* in, double* out, unsigned long long* acc, int lane) {
    double m = 0.0;
    for (int s = lane; s < d.nseg; s += 32) m = fmax(m, fabs(__ldcg(in + s)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e2 = 0;
    frexp(m > 0.0 ? 1024.0 * m : 1.0, &e2);
    const int e = 62 - e2;   // every contribution below 2^52 after scaling, as in the spread
    const int n = d.nseg * BOX_SLOTS;
    for (int t = lane; t < n; t += 32) {
        const int bi = d.pb[t];
        if (bi < 0) continue;
        const int s = t / BOX_SLOTS, slot = t % BOX_SLOTS;
        const double wv = d.kx[6 * s + slot / 6] * d.ky[6 * s + slot % 6];
        atomicAdd(acc + bi, (unsigned long long)__double2ll_rn(ldexp(wv * __ldcg(in + s), e)));
    }
    __syncwarp();
    for (int s = lane; s < d.nseg; s += 32) {
        double v = 0.0;
        for (int slot = 0; slot < BOX_SLOTS; ++slot) {
            const int bi = d.pb[s * BOX_SLOTS + slot];
            if (bi < 0) continue;
            const double wv = d.kx[6 * s + slot / 6] * d.ky[6 * s + slot % 6];
            v = v + wv * ldexp((double)(long long)__ldcg(acc + bi), -e);
        }
        out[s] = v;
    }
    __syncwarp();
    for (int t = lane; t < n; t += 32) {
        const int bi = d.pb[t];
        if (bi >= 0) __stcg(acc + bi, 0ull);
    }
    __syncwarp();
}

// out = D^-1 in for one component, D the block-diagonal part of G: each
// wing's forward and backward substitution with its banded factor and
// per-panel inverses read from global memory, one warp, z a shared-memory
// vector of at least nw_max + PANEL + bw_max doubles.
__device__ void cg_precondition(const DevState& d, const double* in, double* out, double* z, int lane) {
    const int li = lane & (PANEL - 1);
    for (int w = 0; w < d.wing_count; ++w) {
        const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], ld = ibm_ld(bw), s0 = d.wing_sstart[w];
        const int npan = (nw + PANEL - 1) / PANEL;
        const double* A = d.lband + d.wing_lofs[w] + ld;   // row 0
        const double* L = d.linv + d.wing_linv_ofs[w];
        const int* perm = d.perm + s0;
        for (int p = lane; p < nw + PANEL + bw; p += 32) z[p] = p < nw ? in[perm[p]] : 0.0;
        __syncwarp();
        for (int k0 = 0, pan = 0; k0 < nw; k0 += PANEL, ++pan) {   // L' D v = r
            const int np = min(PANEL, nw - k0);
            const double* Li = L + pan * IBM_PANEL_AUX;
            double w0 = 0.0, w1 = 0.0;
#pragma unroll
            for (int k = 0; k < PANEL / 2; ++k) {
                w0 = w0 + Li[li * PANEL + k] * z[k0 + k];
                w1 = w1 + Li[li * PANEL + k + PANEL / 2] * z[k0 + k + PANEL / 2];
            }
            const double wl = w0 + w1;
            double wc[PANEL];
#pragma unroll
            for (int c = 0; c < PANEL; ++c) wc[c] = __shfl_sync(0xffffffffu, wl, c);
            for (int rb = lane; rb < bw; rb += 32) {
                const int i = k0 + np + rb;
                const double* row = A + (long long)i * ld + (i - k0);
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int c = 0; c < PANEL / 2; ++c) {
                    a0 = a0 + row[-c] * wc[c];
                    a1 = a1 + row[-(c + PANEL / 2)] * wc[c + PANEL / 2];
                }
                z[i] -= a0 + a1;
            }
            if (lane < np) z[k0 + lane] = wl * Li[PANEL * PANEL + lane];
            __syncwarp();
        }
        for (int pan = npan - 1; pan >= 0; --pan) {   // L'^T y = v
            const int k0 = pan * PANEL;
            const double* Li = L + pan * IBM_PANEL_AUX;
            double y0 = 0.0, y1 = 0.0;
#pragma unroll
            for (int k = 0; k < PANEL / 2; ++k) {
                y0 = y0 + Li[k * PANEL + li] * z[k0 + k];
                y1 = y1 + Li[(k + PANEL / 2) * PANEL + li] * z[k0 + k + PANEL / 2];
            }
            const double yl = y0 + y1;
            double yc[PANEL];
#pragma unroll
            for (int c = 0; c < PANEL; ++c) yc[c] = __shfl_sync(0xffffffffu, yl, c);
            const int above = min(bw, k0);
            for (int r = lane; r < above; r += 32) {
                const int j = k0 - 1 - r;
                const double* col = A + (long long)k0 * ld + (k0 - j);   // L'(k0 + c, j) at col[c * (ld + 1)]
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int c = 0; c < PANEL / 2; ++c) {
                    a0 = a0 + col[c * (ld + 1)] * yc[c];
                    a1 = a1 + col[(c + PANEL / 2) * (ld + 1)] * yc[c + PANEL / 2];
                }
                z[j] -= a0 + a1;
            }
            if (lane < PANEL) z[k0 + lane] = yl;
            __syncwarp();
        }
        for (int p = lane; p < nw; p += 32) out[perm[p]] = z[p];
        __syncwarp();
    }
}

// The joint solve, warp `comp` for velocity component comp: y (rx or ry)
// holds the per-wing solution on entry and the joint one on exit; the
// right-hand side is qx or qy as the rhs kernel built it; the spread scale
// of every wing (ymax) is recomputed.  y was written by the other wing
// blocks, so it is read past the L1 cache (__ldcg).
__device__ void cg_joint_solve(const DevState& d, double* z, int comp, int lane) {
    const int n = d.nseg;
    double* y = comp ? d.ry : d.rx;
    const double* r0 = comp ? d.qy : d.qx;
    double* res = d.cg_work + (size_t)(4 * comp + 0) * n;
    double* zz = d.cg_work + (size_t)(4 * comp + 1) * n;
    double* p = d.cg_work + (size_t)(4 * comp + 2) * n;
    double* q = d.cg_work + (size_t)(4 * comp + 3) * n;
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(comp ? d.band_dv : d.band_du);
    cg_product(d, y, q, acc, lane);
    double rr0 = 0.0, rn = 0.0;
    for (int s = lane; s < n; s += 32) {
        const double rs = r0[s] - q[s];
        res[s] = rs;
        rr0 += r0[s] * r0[s];
        rn += rs * rs;
    }
    rr0 = warp_sum(rr0);
    rn = warp_sum(rn);
    __syncwarp();
    const double tol2 = CG_TOL * CG_TOL * rr0;
    double rz = 0.0;
    if (rn > tol2) {
        cg_precondition(d, res, zz, z, lane);
        for (int s = lane; s < n; s += 32) {
            p[s] = zz[s];
            rz += res[s] * zz[s];
        }
        rz = warp_sum(rz);
        __syncwarp();
    }
    int it = 0;
    for (; rn > tol2 && it < CG_MAXIT; ++it) {
        cg_product(d, p, q, acc, lane);
        double pq = 0.0;
        for (int s = lane; s < n; s += 32) pq += p[s] * q[s];
        pq = warp_sum(pq);
        if (!(pq > 0.0)) break;
        const double alpha = rz / pq;
        rn = 0.0;
        for (int s = lane; s < n; s += 32) {
            y[s] = __ldcg(y + s) + alpha * p[s];
            res[s] -= alpha * q[s];
            rn += res[s] * res[s];
        }
        rn = warp_sum(rn);
        __syncwarp();
        cg_precondition(d, res, zz, z, lane);
        double rz1 = 0.0;
        for (int s = lane; s < n; s += 32) rz1 += res[s] * zz[s];
        rz1 = warp_sum(rz1);
        const double beta = rz1 / rz;
        rz = rz1;
        for (int s = lane; s < n; s += 32) p[s] = zz[s] + beta * p[s];
        __syncwarp();
    }
    if (rn > tol2 && lane == 0) solver_status(d, ST_COUPLED_NOCONV);
    for (int w = 0; w < d.wing_count; ++w) {
        const int s0 = d.wing_sstart[w], nw = d.wing_npts[w] - 1;
        double ym = 0.0;
        for (int s = s0 + lane; s < s0 + nw; s += 32) ym = fmax(ym, fabs(__ldcg(y + s)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
        if (lane == 0) d.ymax[2 * w + comp] = ym;
    }
}

// Forward and backward substitution with the factor of wing w: warp 0 solves
// for the x component, warp 1 for the y component, on shared-memory copies
// of the per-panel inverses and pivots, of the factor (whole when it fits,
// else streamed through a ring of rows, else read from global memory) and
// of the right-hand sides.  Shared memory: [2 right-hand sides with zero
// tails][permutation][per-panel inverse blocks and pivots][factor or ring].
// Each lane updates rows lane and lane + 32 below or above a panel
// (bw <= 64) or loops.  SMEM: the factor is copied to shared memory whole.
template <bool SMEM>
__device__ __forceinline__ void ibm_solve_kernel_body(const DevState& d, const int bid_) {
    extern __shared__ __align__(16) double sm[];
    __shared__ uint64_t bar;
    __shared__ uint64_t sbar[RING_MAX_SLOTS];
    __shared__ uint32_t suse[RING_MAX_SLOTS];
    const int w = bid_;
    const int tid = threadIdx.x, lane = tid & 31, comp = tid >> 5;
    const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], ld = ibm_ld(bw), s0 = d.wing_sstart[w];
    const int npan = (nw + PANEL - 1) / PANEL;
    const int zlen = d.nw_max + PANEL + d.bw_max;
    double* z = sm + comp * zlen;
    int* perm = reinterpret_cast<int*>(sm + 2 * zlen);
    double* Lsh = reinterpret_cast<double*>(perm + ((d.nw_max + 3) & ~3));
    double* Sm = Lsh + ibm_linv_storage(d.nw_max);
    const double* gS = d.lband + d.wing_lofs[w];
    const long long lbytes = (long long)npan * IBM_PANEL_AUX * 8;
    const long long sbytes = SMEM ? ibm_wing_storage(nw, bw) * 8 : 0;
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, (uint32_t)(lbytes + sbytes));
        bulk_load_all(Lsh, d.linv + d.wing_linv_ofs[w], lbytes, &bar);
        if (sbytes) bulk_load_all(Sm, gS, sbytes, &bar);
    }
#pragma unroll 4
    for (int p = tid; p < nw; p += SOLVE_THREADS) perm[p] = d.perm[s0 + p];
    __syncthreads();
    double* rr = comp == 0 ? d.rx : d.ry;
#pragma unroll 8
    for (int p = lane; p < nw + PANEL + bw; p += 32) z[p] = p < nw ? rr[perm[p]] : 0.0;
    const bool ok = mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) solver_status(d, ST_COPY_TIMEOUT);
        mbar_wait(&bar, 0);
        return;
    }
    const double* A = (SMEM ? Sm : gS) + ld;   // row 0
    const int li = lane & (PANEL - 1);
    // the streamed form (not SMEM, the ring fits)
    const bool stream = !SMEM && d.solve_stream;
    const int NB = ring_slots(bw), nrows = nw + PANEL + bw;
    const int nq = (nrows + RING_ROWS - 1) / RING_ROWS;
    double* ring = Sm;
    auto rowp = [&](int i) -> const double* {   // row i (entry 0 = the diagonal)
        if (!stream) return A + (long long)i * ld;
        const int q = i / RING_ROWS;
        return ring + ((q % NB) * (RING_ROWS + 1) + 1 + (i - q * RING_ROWS)) * ld;
    };
    auto issue = [&](int q) {   // thread 0: chunk q into its slot
        const int s = q % NB;
        const int rows = min(RING_ROWS, nrows - q * RING_ROWS);
        const uint32_t bytes = (uint32_t)rows * ld * 8;
        fence_async_smem();
        mbar_arrive_expect_tx(&sbar[s], bytes);
        bulk_load_all(ring + (s * (RING_ROWS + 1) + 1) * ld, gS + (1 + (long long)q * RING_ROWS) * ld, bytes, &sbar[s]);
        suse[s] += 1;
    };
    auto wait_chunk = [&](int q) { return mbar_wait(&sbar[q % NB], (suse[q % NB] - 1) & 1); };
    auto drain = [&]() {   // every issued copy complete (bounded)
        bool all = true;
        for (int s = 0; s < NB; ++s)
            if (suse[s]) all &= mbar_wait(&sbar[s], (suse[s] - 1) & 1);
        return all;
    };
    int qi = 0;   // next chunk to issue (thread 0)
    if (stream) {
        for (int t = tid; t < NB * ld; t += SOLVE_THREADS) ring[(t / ld) * (RING_ROWS + 1) * ld + t % ld] = 0.0;
        if (tid < NB) {
            mbar_init(&sbar[tid], 1);
            suse[tid] = 0;
        }
        __syncthreads();
    }
    // L' D v = r: per panel w_p = Li_p z_p, v_p = w_p / d, rows below -= L' w_p
    for (int k0 = 0, pan = 0; k0 < nw; k0 += PANEL, ++pan) {
        const int np = min(PANEL, nw - k0);
        if (stream) {   // rows k0 + np .. k0 + np + bw - 1 resident, the next chunk in flight
            const int lo = (k0 + np) / RING_ROWS, hi = min(nq - 1, (k0 + np + bw - 1) / RING_ROWS);
            __syncthreads();
            if (tid == 0)
                for (; qi < nq && qi <= hi + 1 && qi - NB < lo; ++qi) issue(qi);
            __syncthreads();
            bool ok = true;
            for (int q = lo; q <= hi; ++q) ok &= wait_chunk(q);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) solver_status(d, ST_COPY_TIMEOUT);
                drain();
                return;
            }
        }
        const double* Li = Lsh + pan * IBM_PANEL_AUX;
        double zk[PANEL], lk[PANEL];
#pragma unroll
        for (int k = 0; k < PANEL; ++k) {
            zk[k] = z[k0 + k];
            lk[k] = Li[li * PANEL + k];
        }
        double w0 = 0.0, w1 = 0.0;
#pragma unroll
        for (int k = 0; k < PANEL / 2; ++k) {
            w0 = w0 + lk[k] * zk[k];
            w1 = w1 + lk[k + PANEL / 2] * zk[k + PANEL / 2];
        }
        const double wl = w0 + w1;
        double wc[PANEL];
#pragma unroll
        for (int c = 0; c < PANEL; ++c) wc[c] = __shfl_sync(0xffffffffu, wl, c);
        for (int rb0 = 0; rb0 < bw; rb0 += 32) {   // one row below the panel per lane
            const int rb = min(rb0 + lane, bw - 1);
            const int i = k0 + np + rb;
            const double* row = rowp(i) + (i - k0);
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int c = 0; c < PANEL / 2; ++c) {
                a0 = a0 + row[-c] * wc[c];
                a1 = a1 + row[-(c + PANEL / 2)] * wc[c + PANEL / 2];
            }
            if (rb0 + lane < bw) z[k0 + np + rb] -= a0 + a1;
        }
        if (lane < np) z[k0 + lane] = wl * Li[PANEL * PANEL + lane];
        __syncwarp();
    }
    // L'^T y = v: per panel (last first) y_p = Li_p^T v_p, rows above -= L'^T y_p
    int qb = (npan - 1) * PANEL / RING_ROWS;   // next chunk to issue, downwards (thread 0)
    if (stream) {   // no copy of the forward pass still in flight
        const bool ok = drain();
        if (__syncthreads_or(!ok)) {
            if (tid == 0) solver_status(d, ST_COPY_TIMEOUT);
            drain();
            return;
        }
    }
    for (int pan = npan - 1; pan >= 0; --pan) {
        const int k0 = pan * PANEL;
        if (stream) {   // the panel's rows (one chunk) resident, the chunk below in flight
            const int c = k0 / RING_ROWS;
            __syncthreads();
            if (tid == 0)
                for (; qb >= 0 && qb >= c - 1 && qb + NB > c; --qb) issue(qb);
            __syncthreads();
            const bool ok = wait_chunk(c);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) solver_status(d, ST_COPY_TIMEOUT);
                drain();
                return;
            }
        }
        const double* Li = Lsh + pan * IBM_PANEL_AUX;
        double vk[PANEL], lk[PANEL];
#pragma unroll
        for (int k = 0; k < PANEL; ++k) {
            vk[k] = z[k0 + k];
            lk[k] = Li[k * PANEL + li];
        }
        double y0 = 0.0, y1 = 0.0;
#pragma unroll
        for (int k = 0; k < PANEL / 2; ++k) {
            y0 = y0 + lk[k] * vk[k];
            y1 = y1 + lk[k + PANEL / 2] * vk[k + PANEL / 2];
        }
        const double yl = y0 + y1;
        double yc[PANEL];
#pragma unroll
        for (int c = 0; c < PANEL; ++c) yc[c] = __shfl_sync(0xffffffffu, yl, c);
        const int above = min(bw, k0);   // rows k0 - above .. k0 - 1
        for (int r0 = 0; r0 < above; r0 += 32) {   // one row above the panel per lane
            const int r = min(r0 + lane, above - 1);
            const int j = k0 - 1 - r;
            const double* col = rowp(k0) + (k0 - j);   // L'(k0 + c, j) at col[c * (ld + 1)]
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int c = 0; c < PANEL / 2; ++c) {
                a0 = a0 + col[c * (ld + 1)] * yc[c];
                a1 = a1 + col[(c + PANEL / 2) * (ld + 1)] * yc[c + PANEL / 2];
            }
            if (r0 + lane < above) z[k0 - 1 - r] -= a0 + a1;
        }
        if (lane < PANEL) z[k0 + lane] = yl;
        __syncwarp();
    }
    if (stream && !drain() && lane == 0) solver_status(d, ST_COPY_TIMEOUT);
    double ym = 0.0;
#pragma unroll 4
    for (int p = lane; p < nw; p += 32) {
        rr[perm[p]] = z[p];
        ym = fmax(ym, fabs(z[p]));
    }
    for (int o = 16; o > 0; o >>= 1) ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
    if (lane == 0) d.ymax[2 * w + comp] = ym;
    pdl_release();   // the spread may be scheduled (it waits for this grid to complete)
    // Supports of different wings share nodes: the last wing block to finish
    // (a per-episode counter after a fence; no block waits) solves the joint
    // system from the per-wing solutions, before the spread reads them.
    if (d.wing_count > 1 && __ldcg(d.ibm_flags) != 0) {
        __shared__ int last;
        __threadfence();
        __syncthreads();
        if (tid == 0) last = atomicAdd(d.solve_count, 1) == d.wing_count - 1;
        __syncthreads();
        if (!last) return;
        __threadfence();
        if (tid == 0) *d.solve_count = 0;
        cg_joint_solve(d, z, comp, lane);
    }
}
template <bool SMEM>
__global__ void __launch_bounds__(SOLVE_THREADS) ibm_solve_kernel(DevState d) {
    pdl_wait();
    ibm_solve_kernel_body<SMEM>(d, blockIdx.x);
}
template <bool SMEM>
__global__ void __launch_bounds__(SOLVE_THREADS) ibm_solve_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_solve_kernel_body<SMEM>(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Substitution in panels of 32 rows (wings whose panel data fit in shared
// memory): one block per wing, warp 0 for the x component, warp 1 for y.
// The wing's panel data (MT, R, pivots per panel) come in by one bulk copy.
// Forward, per panel: t = M z_p (lane l: a 32-term dot product over MT's
// column l), rows below -= R t, z_p = D^-1 t.  Backward, per panel, last
// first: v = z_p - R^T y_below (lane c pulls the solved rows below), y_p =
// M^T v.  14 dependent panel steps for a 200-segment wing instead of 50.
// The right-hand sides and solutions, ymax and the joint solve of coupled
// wings are as in the 8-row substitution.
__device__ __forceinline__ void ibm_solve32_body(const DevState& d, const int bid_) {
    extern __shared__ __align__(16) double sm[];
    __shared__ uint64_t bar;
    const int w = bid_;
    const int tid = threadIdx.x, lane = tid & 31, comp = tid >> 5;
    const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], s0 = d.wing_sstart[w];
    const int nq = qpanels(nw);
    const long long psz = panel32_doubles(bw);
    const int zlen = (d.nw_max + Q32 + d.bw_max + 1) & ~1;
    double* P = sm;
    double* z = sm + d.q32_doubles_max + comp * zlen;
    double* tb = sm + d.q32_doubles_max + 2 * zlen + comp * Q32;
    const long long bytes = (long long)nq * psz * 8;
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, (uint32_t)bytes);
        bulk_load_all(P, d.lq + d.wing_qofs[w], bytes, &bar);
    }
    const int* perm = d.perm + s0;
    double* rr = comp == 0 ? d.rx : d.ry;
    for (int p = lane; p < nw + Q32 + bw; p += 32) z[p] = p < nw ? rr[perm[p]] : 0.0;
    __syncthreads();
    const bool ok = mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) solver_status(d, ST_COPY_TIMEOUT);
        mbar_wait(&bar, 0);   // let a late copy land before the block exits
        return;
    }
    for (int q = 0; q < nq; ++q) {   // L' D v = r
        const int k0 = q * Q32, np = min(Q32, nw - k0);
        const double* MT = P + q * psz;
        const double* R = MT + Q32P * Q32;
        const double* piv = R + Q32P * bw;
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
#pragma unroll
        for (int c = 0; c < Q32; c += 4) {
            t0 = t0 + MT[c * Q32P + lane] * z[k0 + c];
            t1 = t1 + MT[(c + 1) * Q32P + lane] * z[k0 + c + 1];
            t2 = t2 + MT[(c + 2) * Q32P + lane] * z[k0 + c + 2];
            t3 = t3 + MT[(c + 3) * Q32P + lane] * z[k0 + c + 3];
        }
        const double tl = (t0 + t1) + (t2 + t3);
        tb[lane] = tl;
        __syncwarp();
        for (int rb = lane; rb < bw; rb += 32) {
            const double* Rr = R + rb * Q32P;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int c = 0; c < Q32; c += 4) {
                a0 = a0 + Rr[c] * tb[c];
                a1 = a1 + Rr[c + 1] * tb[c + 1];
                a2 = a2 + Rr[c + 2] * tb[c + 2];
                a3 = a3 + Rr[c + 3] * tb[c + 3];
            }
            z[k0 + np + rb] -= (a0 + a1) + (a2 + a3);
        }
        z[k0 + lane] = tl * piv[lane];   // zero past the last segment
        __syncwarp();
    }
    for (int q = nq - 1; q >= 0; --q) {   // L'^T y = v
        const int k0 = q * Q32, np = min(Q32, nw - k0);
        const double* MT = P + q * psz;
        const double* R = MT + Q32P * Q32;
        double a0 = 0.0, a1 = 0.0;
        int rb = 0;
        for (; rb + 1 < bw; rb += 2) {
            a0 = a0 + R[rb * Q32P + lane] * z[k0 + np + rb];
            a1 = a1 + R[(rb + 1) * Q32P + lane] * z[k0 + np + rb + 1];
        }
        if (rb < bw) a0 = a0 + R[rb * Q32P + lane] * z[k0 + np + rb];
        tb[lane] = z[k0 + lane] - (a0 + a1);
        __syncwarp();
        double y0 = 0.0, y1 = 0.0, y2 = 0.0, y3 = 0.0;
#pragma unroll
        for (int c = 0; c < Q32; c += 4) {
            y0 = y0 + MT[lane * Q32P + c] * tb[c];
            y1 = y1 + MT[lane * Q32P + c + 1] * tb[c + 1];
            y2 = y2 + MT[lane * Q32P + c + 2] * tb[c + 2];
            y3 = y3 + MT[lane * Q32P + c + 3] * tb[c + 3];
        }
        if (lane < np) z[k0 + lane] = (y0 + y1) + (y2 + y3);
        __syncwarp();
    }
    double ym = 0.0;
#pragma unroll 4
    for (int p = lane; p < nw; p += 32) {
        rr[perm[p]] = z[p];
        ym = fmax(ym, fabs(z[p]));
    }
    for (int o = 16; o > 0; o >>= 1) ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
    if (lane == 0) d.ymax[2 * w + comp] = ym;
    if (d.wing_count > 1 && __ldcg(d.ibm_flags) != 0) {
        __shared__ int last;
        __threadfence();
        __syncthreads();
        if (tid == 0) last = atomicAdd(d.solve_count, 1) == d.wing_count - 1;
        __syncthreads();
        if (!last) return;
        __threadfence();
        if (tid == 0) *d.solve_count = 0;
        cg_joint_solve(d, z, comp, lane);
    }
}
__global__ void __launch_bounds__(SOLVE_THREADS) ibm_solve32_kernel(DevState d) {
    pdl_wait();
    ibm_solve32_body(d, blockIdx.x);
}
__global__ void __launch_bounds__(SOLVE_THREADS) ibm_solve32_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_solve32_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}
size_t ibm_solve32_smem(long long q32_doubles_max, int nw_max, int bw_max) {
    const long long zlen = (nw_max + Q32 + bw_max + 1) & ~1;
    return (size_t)(q32_doubles_max + 2 * zlen + 2 * Q32) * sizeof(double);
}

size_t ibm_factor_staging_bytes(int bw_max) {
    const int nt = round_tile(bw_max) / TILE;
    const size_t rows = (size_t)2 * SP * round_tile(bw_max) * sizeof(double);   // a multiple of 16
    const size_t tl = (size_t)tri(nt, 0) * sizeof(short2);
    return rows + (tl + 15) / 16 * 16;
}

size_t ibm_solve_smem(int nw_max, int bw_max, long long wing_storage_max, bool factor_in_smem) {
    const size_t z = (size_t)2 * (nw_max + PANEL + bw_max) * sizeof(double);
    const size_t perm = (size_t)((nw_max + 3) & ~3) * sizeof(int);
    const size_t inv = (size_t)ibm_linv_storage(nw_max) * sizeof(double);
    return z + perm + inv + (factor_in_smem ? (size_t)wing_storage_max * sizeof(double) : 0);
}

// The dynamic shared-memory limit is a per-device property of each kernel,
// shared by every handle: it is raised once to the device's opt-in maximum
// (minus the kernel's static shared memory), never lowered, so handles of
// different sizes created in any order, from any thread, all launch.
static std::mutex g_prepare_mutex;
static unsigned long long g_prepared_devices = 0;

template <class K>
static cudaError_t raise_smem_limit(K kernel, int optin) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

cudaError_t ibm_prepare(size_t factor_smem, size_t solve_smem) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    if (factor_smem + 16 * 1024 > (size_t)optin || solve_smem + 1024 > (size_t)optin) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> lock(g_prepare_mutex);
    if (dev < 64 && (g_prepared_devices >> dev) & 1ULL) return cudaSuccess;
    e = raise_smem_limit(ibm_factor_kernel<true>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_factor_kernel<false>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_solve_kernel<true>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_solve_kernel<false>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_factor_kernel_multi<true>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_factor_kernel_multi<false>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_solve_kernel_multi<true>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_solve_kernel_multi<false>, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_solve32_kernel, optin);
    if (e == cudaSuccess) e = raise_smem_limit(ibm_solve32_kernel_multi, optin);
    if (e == cudaSuccess && dev < 64) g_prepared_devices |= 1ULL << dev;
    return e;
}

bool is_factor_multi_kernel(const void* func) {
    return func == reinterpret_cast<const void*>(ibm_factor_kernel_multi<true>) ||
           func == reinterpret_cast<const void*>(ibm_factor_kernel_multi<false>);
}

bool is_factor_kernel(const void* func) {
    return func == reinterpret_cast<const void*>(ibm_factor_kernel<true>) ||
           func == reinterpret_cast<const void*>(ibm_factor_kernel<false>);
}

void launch_ibm_factor_blocks(const DevState& d, size_t factor_smem, cudaStream_t st) {
    if (d.wing_count <= 0) return;
    if (d.factor_in_smem)
        ibm_factor_kernel<true><<<d.wing_count, FACTOR_THREADS, factor_smem, st>>>(d);
    else
        ibm_factor_kernel<false><<<d.wing_count, FACTOR_THREADS, factor_smem, st>>>(d);
}

void launch_ibm_substitution(const DevState& d, size_t solve_smem, cudaStream_t st, bool chained) {
    if (d.wing_count <= 0) return;
    if (d.solve32)
        launch_chained(chained, ibm_solve32_kernel, d.wing_count, SOLVE_THREADS, solve_smem, st, d);
    else if (d.solve_in_smem)
        launch_chained(chained, ibm_solve_kernel<true>, d.wing_count, SOLVE_THREADS, solve_smem, st, d);
    else
        launch_chained(chained, ibm_solve_kernel<false>, d.wing_count, SOLVE_THREADS, solve_smem, st, d);
}

// Packed launches: one block per wing of every episode; episodes whose
// factor (or substitution) does not take the kind's shared-memory form get
// no blocks in it.  The dynamic shared memory is the largest of the batch.
int multi_blocks_solver(MultiKernel k, const DevState& d) {
    switch (k) {
    case MK_FACTOR_SMEM: return d.factor_in_smem ? d.wing_count : 0;
    case MK_FACTOR_GLOBAL: return d.factor_in_smem ? 0 : d.wing_count;
    case MK_SOLVE32: return d.solve32 ? d.wing_count : 0;
    case MK_SOLVE_SMEM: return !d.solve32 && d.solve_in_smem ? d.wing_count : 0;
    case MK_SOLVE_GLOBAL: return !d.solve32 && !d.solve_in_smem ? d.wing_count : 0;
    default: return -1;
    }
}

bool launch_multi_solver(MultiKernel k, const MultiArgs& m, int nb, size_t smem, cudaStream_t st) {
    switch (k) {
    case MK_FACTOR_SMEM: ibm_factor_kernel_multi<true><<<nb, FACTOR_THREADS, smem, st>>>(m); return true;
    case MK_FACTOR_GLOBAL: ibm_factor_kernel_multi<false><<<nb, FACTOR_THREADS, smem, st>>>(m); return true;
    case MK_SOLVE32: ibm_solve32_kernel_multi<<<nb, SOLVE_THREADS, smem, st>>>(m); return true;
    case MK_SOLVE_SMEM: ibm_solve_kernel_multi<true><<<nb, SOLVE_THREADS, smem, st>>>(m); return true;
    case MK_SOLVE_GLOBAL: ibm_solve_kernel_multi<false><<<nb, SOLVE_THREADS, smem, st>>>(m); return true;
    default: return false;
    }
}

}  // namespace lbm
