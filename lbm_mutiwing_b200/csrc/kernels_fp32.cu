// Fused FP32 path: one pull-scheme kernel does streaming, moments and the MRT
// collision for every interior node (solution.f90:440-669 in one pass), on
// distributions stored in FP32 as deviations from the rest equilibrium,
// g_k = f_k - w_k (rho0 = 1, w_k the FP32-rounded weights of D2Q9model.f90).
//
// Layout in HBM: nine planes g[k][y][x] with a padded row pitch (multiple of
// 32 floats), three copies (a step reads one and writes another; a two-step
// pass also writes its first step's band and border values to the third).
// One step moves 9 reads + 9 writes of 4 bytes per node; a pass moves the
// same for two steps.
//
// Deviation form of the collision: with c = M w (only c0, c1, c2 are
// non-zero), m_dev = M g and rho = 1 + (m_dev,0 + W - 1), the post-collision
// deviation is m'_dev = m_dev + S (m_eq(rho, j) - c - m_dev), g' = M^-1 m'_dev.
// Bulk nodes carry no body force (the immersed-boundary force is non-zero
// only on band nodes), so j = (m_dev,3, m_dev,5) and m_eq needs no division.
// Band nodes are re-collided in FP64 by the immersed boundary's closing
// kernel with the corrected velocity and the Guo forcing term.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "bulk_copy.cuh"
#include "lbm_kernels.h"
#include "multi.cuh"

namespace lbm {

constexpr int BULK_TX = 256;   // one row per thread: short-lived blocks, 92% of copy bandwidth
constexpr int BULK_ROWS = 1;

FusedConsts fused_consts(const DevState& d) {
    double w0 = weight(0), w1 = weight(1), w5 = weight(5);
    double W = w0 + 4.0 * w1 + 4.0 * w5;
    double c1 = -4.0 * w0 - 4.0 * w1 + 8.0 * w5;
    double c2 = 4.0 * w0 - 8.0 * w1 + 4.0 * w5;
    FusedConsts c;
    c.s1 = (float)d.s[1]; c.s2 = (float)d.s[2]; c.s4 = (float)d.s[4];
    c.s6 = (float)d.s[6]; c.s7 = (float)d.s[7]; c.s8 = (float)d.s[8];
    c.k1 = (float)(2.0 + c1);
    c.k2 = (float)(1.0 - c2);
    c.wm1 = (float)(W - 1.0);
    return c;
}

// MRT collision on pulled deviations g (moments of the deviation,
// relaxation toward the equilibrium moments, back to populations); drho and
// (jx, jy) are the density deviation and momentum.  Every operation is an
// explicitly rounded IEEE add, multiply or fused multiply-add (a - b as
// fma(-1, b, a)), so the result does not depend on how the compiler would
// contract expressions: the lane type V is float (one node) or float2 (two
// nodes through the paired FP32 instructions of sm_100, each lane rounded
// as the float form), and every kernel gives the same bits.
template <class V>
struct Lanes;
template <>
struct Lanes<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float k(float x) { return x; }
};
template <>
struct Lanes<float2> {
    static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
    static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
    static __device__ __forceinline__ float2 k(float x) { return make_float2(x, x); }
};
template <class V, class K>
__device__ __forceinline__ void collide_lanes(const V g[9], const K& k, V o[9], V& drho, V& jx, V& jy) {
    using L = Lanes<V>;
    auto sub = [&](V a, V b) { return L::fma(k.m1(), b, a); };
    // moments of the deviation
    const V p13 = L::add(g[1], g[3]), p24 = L::add(g[2], g[4]);
    const V p57 = L::add(g[5], g[7]), p68 = L::add(g[6], g[8]);
    const V s14 = L::add(p13, p24), s58 = L::add(p57, p68);
    const V m0 = L::add(L::add(g[0], s14), s58);
    const V m1 = L::fma(k.p2(), s58, sub(L::mul(k.m4(), g[0]), s14));
    const V m2 = L::fma(k.p4(), g[0], L::fma(k.m2(), s14, s58));
    const V d13 = sub(g[1], g[3]), d24 = sub(g[2], g[4]);
    const V a5 = sub(g[5], g[7]), a6 = sub(g[6], g[8]);
    jx = sub(L::add(d13, a5), a6);
    const V m4 = sub(L::fma(k.m2(), d13, a5), a6);
    jy = L::add(L::add(d24, a5), a6);
    const V m6 = L::add(L::fma(k.m2(), d24, a5), a6);
    const V m7 = sub(p13, p24);
    const V m8 = sub(p57, p68);
    // relaxation toward the equilibrium moments (solution.f90:616-646)
    drho = L::add(m0, k.wm1());
    const V jxx = L::mul(jx, jx), jyy = L::mul(jy, jy), q = L::add(jxx, jyy);
    const V t1 = L::fma(k.p3(), q, L::fma(k.m2(), drho, k.mk1()));
    const V e1 = L::fma(k.s1(), sub(t1, m1), m1);
    const V t2 = L::fma(k.m3(), q, L::add(drho, k.k2()));
    const V e2 = L::fma(k.s2(), sub(t2, m2), m2);
    const V e4 = L::fma(k.ms4(), L::add(jx, m4), m4);
    const V e6 = L::fma(k.ms6(), L::add(jy, m6), m6);
    const V e7 = L::fma(k.s7(), sub(sub(jxx, jyy), m7), m7);
    const V e8 = L::fma(k.s8(), sub(L::mul(jx, jy), m8), m8);
    // back to populations: M^-1 = M^T diag(1/9, 1/36, 1/36, 1/6, 1/12, 1/6, 1/12, 1/4, 1/4)
    const V b0 = L::mul(m0, k.r9());
    const V b1 = L::mul(e1, k.r36()), b2 = L::mul(e2, k.r36());
    const V b3 = L::mul(jx, k.r6()), b4 = L::mul(e4, k.r12());
    const V b5 = L::mul(jy, k.r6()), b6 = L::mul(e6, k.r12());
    const V b7 = L::mul(e7, k.r4()), b8 = L::mul(e8, k.r4());
    const V rA = L::fma(k.m2(), b2, sub(b0, b1));   // axis populations, common part
    const V rD = L::add(L::fma(k.p2(), b1, b0), b2);  // diagonal populations, common part
    const V x34 = L::fma(k.m2(), b4, b3), y56 = L::fma(k.m2(), b6, b5);
    const V xd = L::add(b3, b4), yd = L::add(b5, b6);
    o[0] = L::fma(k.p4(), b2, L::fma(k.m4(), b1, b0));
    o[1] = L::add(L::add(rA, x34), b7);
    o[2] = sub(L::add(rA, y56), b7);
    o[3] = L::add(sub(rA, x34), b7);
    o[4] = sub(sub(rA, y56), b7);
    o[5] = L::add(L::add(L::add(rD, xd), yd), b8);
    o[6] = sub(L::add(sub(rD, xd), yd), b8);
    o[7] = L::add(sub(sub(rD, xd), yd), b8);
    o[8] = sub(sub(L::add(rD, xd), yd), b8);
}
// The constants of the collision for two nodes, from the kernel's parameters.
struct PairK {
    const PassPairs& k;
    __device__ float2 m1() const { return k.m1; }
    __device__ float2 p2() const { return k.p2; }
    __device__ float2 m2() const { return k.m2; }
    __device__ float2 p3() const { return k.p3; }
    __device__ float2 m3() const { return k.m3; }
    __device__ float2 p4() const { return k.p4; }
    __device__ float2 m4() const { return k.m4; }
    __device__ float2 r4() const { return k.r4; }
    __device__ float2 r6() const { return k.r6; }
    __device__ float2 r9() const { return k.r9; }
    __device__ float2 r12() const { return k.r12; }
    __device__ float2 r36() const { return k.r36; }
    __device__ float2 wm1() const { return k.wm1; }
    __device__ float2 mk1() const { return k.mk1; }
    __device__ float2 k2() const { return k.k2; }
    __device__ float2 s1() const { return k.s1; }
    __device__ float2 s2() const { return k.s2; }
    __device__ float2 ms4() const { return k.ms4; }
    __device__ float2 ms6() const { return k.ms6; }
    __device__ float2 s7() const { return k.s7; }
    __device__ float2 s8() const { return k.s8; }
};

PassPairs pass_pairs(const FusedConsts& c) {
    auto two = [](float x) { return make_float2(x, x); };
    PassPairs k;
    k.m1 = two(-1.0f); k.p2 = two(2.0f); k.m2 = two(-2.0f); k.p3 = two(3.0f); k.m3 = two(-3.0f);
    k.p4 = two(4.0f); k.m4 = two(-4.0f); k.r4 = two(0.25f); k.r6 = two(1.0f / 6.0f); k.r9 = two(1.0f / 9.0f);
    k.r12 = two(1.0f / 12.0f); k.r36 = two(1.0f / 36.0f); k.wm1 = two(c.wm1); k.mk1 = two(-c.k1);
    k.k2 = two(c.k2); k.s1 = two(c.s1); k.s2 = two(c.s2); k.ms4 = two(-c.s4); k.ms6 = two(-c.s6);
    k.s7 = two(c.s7); k.s8 = two(c.s8);
    return k;
}

// The constants of the collision for one node: literals and the rates of c.
struct ScalarK {
    const FusedConsts& c;
    __device__ float m1() const { return -1.0f; }
    __device__ float p2() const { return 2.0f; }
    __device__ float m2() const { return -2.0f; }
    __device__ float p3() const { return 3.0f; }
    __device__ float m3() const { return -3.0f; }
    __device__ float p4() const { return 4.0f; }
    __device__ float m4() const { return -4.0f; }
    __device__ float r4() const { return 0.25f; }
    __device__ float r6() const { return 1.0f / 6.0f; }
    __device__ float r9() const { return 1.0f / 9.0f; }
    __device__ float r12() const { return 1.0f / 12.0f; }
    __device__ float r36() const { return 1.0f / 36.0f; }
    __device__ float wm1() const { return c.wm1; }
    __device__ float mk1() const { return -c.k1; }
    __device__ float k2() const { return c.k2; }
    __device__ float s1() const { return c.s1; }
    __device__ float s2() const { return c.s2; }
    __device__ float ms4() const { return -c.s4; }
    __device__ float ms6() const { return -c.s6; }
    __device__ float s7() const { return c.s7; }
    __device__ float s8() const { return c.s8; }
};

__device__ __forceinline__ void fused_collide(const float g[9], const FusedConsts& c, float o[9], float& drho,
                                              float& jx, float& jy) {
    collide_lanes<float>(g, ScalarK{c}, o, drho, jx, jy);
}

// One interior node (i, j); nodes of the band list are left to the band
// re-collision, which runs concurrently and writes them.  EARLY: the band
// bit is tested before the nine pulls (one memory round trip ahead of
// them); otherwise it is loaded beside them and only gates the stores.
#ifndef BULK_EARLY_BAND_TEST
#define BULK_EARLY_BAND_TEST 1
#endif
template <bool FIELDS, bool EARLY>
__device__ __forceinline__ void fused_bulk_node(const float* __restrict__ gA, float* __restrict__ gB, int pitch,
                                                long long plane, const FusedConsts& c, double* __restrict__ fo_rho,
                                                double* __restrict__ fo_u, double* __restrict__ fo_v,
                                                const unsigned* __restrict__ bits, int i, int j) {
    const long long p = (long long)j * pitch + i;
    const unsigned word = __ldg(bits + (p >> 5));
    if (EARLY && ((word >> (p & 31)) & 1u)) return;
    float g[9], o[9], drho, jx, jy;
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = __ldg(gA + k * plane + p - ex(k) - (long long)ey(k) * pitch);
    fused_collide(g, c, o, drho, jx, jy);
    if (!EARLY && ((word >> (p & 31)) & 1u)) return;
#pragma unroll
    for (int k = 0; k < 9; ++k) gB[k * plane + p] = o[k];
    if (FIELDS) {
        const double rho = 1.0 + (double)drho;
        fo_rho[p] = rho;
        fo_u[p] = (double)jx / rho;
        fo_v[p] = (double)jy / rho;
    }
}
template <bool FIELDS>
__global__ void __launch_bounds__(BULK_TX) fused_bulk_kernel(const float* __restrict__ gA, float* __restrict__ gB,
                                                             int nx, int ny, int pitch, long long plane,
                                                             FusedConsts c, double* __restrict__ fo_rho,
                                                             double* __restrict__ fo_u, double* __restrict__ fo_v,
                                                             const unsigned* __restrict__ bits) {
    const int i = blockIdx.x * BULK_TX + threadIdx.x + 1;
    if (i > nx - 2) return;
    const int j0 = blockIdx.y * BULK_ROWS + 1;
#pragma unroll
    for (int r = 0; r < BULK_ROWS; ++r) {
        const int j = j0 + r;
        if (j > ny - 2) break;
        fused_bulk_node<FIELDS, BULK_EARLY_BAND_TEST != 0>(gA, gB, pitch, plane, c, fo_rho, fo_u, fo_v, bits, i, j);
    }
}
// Tiled form of the common step (no fields written): a block takes the
// nodes of 128 absolute columns [128 tx, 128 tx + 127] x TMA_TY interior
// rows; one thread issues nine tiled tensor loads, plane k's box starting at
// column 128 tx - 4 (16-byte aligned; out-of-range columns read as zero)
// and row y0 - ey(k), so box row r holds the pulls of interior row y0 + r
// and box column cc + 4 - ex(k) the pull of column 128 tx + cc.  The 136
// columns cover the +-1 shifts; the tiles either side share 8 columns (L2
// hits).  Every value is then read once from shared memory, collided and
// stored to the next planes.  Blocks stay short-lived (no persistent loop),
// so the immersed-boundary chain's blocks, at higher priority, are
// dispatched as bulk blocks retire.  Measured alone at 4001 x 2001: 96.7 us
// against 103.2 us for the one-node-per-thread form with global pulls.
#ifndef LBM_BULK_TILE_ROWS
#define LBM_BULK_TILE_ROWS 4
#endif
#ifndef LBM_BULK_TILE_THREADS
#define LBM_BULK_TILE_THREADS 256
#endif
constexpr int TMA_TX = 128, TMA_TY = LBM_BULK_TILE_ROWS, TMA_THREADS = LBM_BULK_TILE_THREADS;
constexpr int TMA_BOXW = TMA_TX + 8;
constexpr int TMA_CH = (TMA_TY * TMA_BOXW + 31) & ~31;   // floats per plane chunk, 128-byte multiple
constexpr size_t TMA_SMEM = 9 * TMA_CH * sizeof(float) + 128;
__global__ void __launch_bounds__(TMA_THREADS) fused_bulk_tma_kernel(const __grid_constant__ CUtensorMap tm,
                                                                     float* __restrict__ gB, int nx, int ny, int pitch,
                                                                     long long plane, FusedConsts c,
                                                                     const unsigned* __restrict__ bits, int ntx,
                                                                     int* status) {
    extern __shared__ unsigned char tma_raw[];
    __shared__ uint64_t bar;
    float* S = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(tma_raw) + 127) & ~(uintptr_t)127);
    const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
    const int x0 = tx * TMA_TX, y0 = 1 + ty * TMA_TY;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, (uint32_t)(9 * TMA_TY * TMA_BOXW * sizeof(float)));
#pragma unroll
        for (int k = 0; k < 9; ++k) tma_load_3d(S + k * TMA_CH, &tm, x0 - 4, y0 - ey(k), k, &bar);
    }
    __syncthreads();
    const bool ok = mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(status, ST_COPY_TIMEOUT);
        mbar_wait(&bar, 0);   // let a late copy land before the block exits
        return;
    }
#pragma unroll
    for (int n = threadIdx.x; n < TMA_TY * TMA_TX; n += TMA_THREADS) {
        const int r = n / TMA_TX, cc = n % TMA_TX, i = x0 + cc, j = y0 + r;
        if (i < 1 || i > nx - 2 || j > ny - 2) continue;
        const long long p = (long long)j * pitch + i;
        if ((__ldg(bits + (p >> 5)) >> (p & 31)) & 1u) continue;   // band nodes: the band re-collision
        float g[9], o[9], drho, jx, jy;
#pragma unroll
        for (int k = 0; k < 9; ++k) g[k] = S[k * TMA_CH + r * TMA_BOXW + cc + 4 - ex(k)];
        fused_collide(g, c, o, drho, jx, jy);
#pragma unroll
        for (int k = 0; k < 9; ++k) gB[k * plane + p] = o[k];
    }
}

// Tensor map of the nine planes at base (x: columns of the pitched rows, y:
// rows, z: planes) with the given box; 0 on success.
static int encode_plane_map(const DevState& d, const float* base, const cuuint32_t box[3], void* out) {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!enc) return -1;
    const cuuint64_t dims[3] = {(cuuint64_t)d.pitch, (cuuint64_t)d.ny, 9};
    const cuuint64_t strides[2] = {(cuuint64_t)d.pitch * sizeof(float), (cuuint64_t)d.plane * sizeof(float)};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = enc(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                           const_cast<float*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

int fused_tensor_map(const DevState& d, const float* base, void* out) {
    const cuuint32_t box[3] = {TMA_BOXW, TMA_TY, 1};
    return encode_plane_map(d, base, box, out);
}

// ------------------------------------------------------------ two-step passes
// One pass advances the interior n -> n + 2 with one read of step n's planes
// P and one write of step n + 2's planes Q (temporal blocking: half the HBM
// traffic of two steps).  A block takes a tile of PASS_TX x R nodes (R =
// PASS_TY or PASS_TY_TALL rows, a template parameter of the kernels): one
// thread issues nine tiled tensor loads of the tile and two rings of
// neighbours (box of PASS_TX + 8 columns from x0 - 4, 16-byte aligned, and
// R + 4 rows from y0 - 2; out-of-range parts read as zero), the block
// computes step n + 1 on the tile and one ring (R1) into shared memory, then
// step n + 2 on the tile from there.  Step n + 1 values that are not plain
// collisions -- band nodes of step n (immersed boundary) and the border (far
// field) -- come from O, where the band re-collision and the far field of
// step n put them; tiles whose R1 holds such nodes are the near tiles, run
// after those writers, every other tile (the far tiles) without waiting for
// them (it reads nothing but P).  Band nodes of step n + 1 and the border are left out of Q: the
// second step's band re-collision and far field write them.  Every node is
// computed by fused_collide, as in the one-step kernels, so a pass gives the
// bits of two steps.
// The block's shape for tiles of R rows: one column pair of R1 per thread,
// in whole warps; band-bit words of a tile row; the staged box (BOXW x BOXH)
// and its plane stride CH (a 128-byte multiple); R1 (MW x MH); the dynamic
// shared memory; the resident blocks per SM that it allows (the launch
// bounds then keep the registers within the same count).
template <int R>
struct PassShape {
    static constexpr int THREADS = ((R + 2) * (PASS_TX + 2) / 2 + 31) / 32 * 32;
    static constexpr int WORDS = PASS_TX / 32;
    static constexpr int BOXW = PASS_TX + 8, BOXH = R + 4;
    static constexpr int CH = (BOXH * BOXW + 31) & ~31;
    static constexpr int MW = PASS_TX + 2, MH = R + 2;
    static constexpr int MCH = MH * MW;
    static constexpr size_t SMEM = (size_t)(9 * CH + 9 * MCH) * sizeof(float) + 128;
    static constexpr int MINB = (227 * 1024) / (int)(SMEM + 1024) < 8 ? (227 * 1024) / (int)(SMEM + 1024) : 8;
    static_assert(BOXW <= 256 && BOXH <= 256, "tensor-map box extents");
    static_assert(WORDS * R <= THREADS, "a tile's band bits are staged one word per thread");
};
static_assert(PASS_TX % 32 == 0, "tiles start on 16-byte boundaries and on band-bit words");

// A near tile, one node per thread: step n + 1 values of border nodes and of
// step n's band nodes come from O, nodes outside the lattice are skipped.
template <int R>
__device__ __forceinline__ void pass_tile_near(const CUtensorMap* tm, const PassArgs& a, int t, float* Sin, float* Smid,
                                               uint64_t* bar) {
    using S = PassShape<R>;
    const int tx = t % a.ntx, ty = t / a.ntx;
    const int x0 = tx * PASS_TX, y0 = 1 + ty * R;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_arrive_expect_tx(bar, (uint32_t)(9 * S::BOXH * S::BOXW * sizeof(float)));
#pragma unroll
        for (int k = 0; k < 9; ++k) tma_load_3d(Sin + k * S::CH, tm, x0 - 4, y0 - 2, k, bar);
    }
    __syncthreads();
    const bool ok = mbar_wait(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(a.status, ST_COPY_TIMEOUT);
        mbar_wait(bar, 0);   // let a late copy land before the block exits
        return;
    }
    // step n + 1 on R1: node (x0 - 1 + mc, y0 - 1 + mr), box cell (mr + 1, mc + 3)
    for (int n = threadIdx.x; n < S::MH * S::MW; n += S::THREADS) {
        const int mr = n / S::MW, mc = n % S::MW;
        float o[9];
        {
            const int i = x0 - 1 + mc, j = y0 - 1 + mr;
            if (i < 0 || i > a.nx - 1 || j < 0 || j > a.ny - 1) continue;   // outside: never pulled
            const long long p = (long long)j * a.pitch + i;
            const bool border = i == 0 || j == 0 || i == a.nx - 1 || j == a.ny - 1;
            if (border || ((__ldg(a.bits0 + (p >> 5)) >> (p & 31)) & 1u)) {
#pragma unroll
                for (int k = 0; k < 9; ++k) Smid[k * S::MCH + n] = __ldcg(a.O + k * a.plane + p);
                continue;
            }
        }
        float g[9], drho, jx, jy;
#pragma unroll
        for (int k = 0; k < 9; ++k) g[k] = Sin[k * S::CH + (mr + 1 - ey(k)) * S::BOXW + mc + 3 - ex(k)];
        fused_collide(g, a.c, o, drho, jx, jy);
#pragma unroll
        for (int k = 0; k < 9; ++k) Smid[k * S::MCH + n] = o[k];
    }
    __syncthreads();
    // step n + 2 on the tile: node (x0 + cc, y0 + rr), R1 cell (rr + 1, cc + 1)
    for (int n = threadIdx.x; n < R * PASS_TX; n += S::THREADS) {
        const int rr = n / PASS_TX, cc = n % PASS_TX, i = x0 + cc, j = y0 + rr;
        if (i < 1 || i > a.nx - 2 || j > a.ny - 2) continue;
        const long long p = (long long)j * a.pitch + i;
        if ((__ldg(a.bits1 + (p >> 5)) >> (p & 31)) & 1u) continue;   // band nodes of step n + 1
        float g[9], o[9], drho, jx, jy;
#pragma unroll
        for (int k = 0; k < 9; ++k) g[k] = Smid[k * S::MCH + (rr + 1 - ey(k)) * S::MW + cc + 1 - ex(k)];
        fused_collide(g, a.c, o, drho, jx, jy);
#pragma unroll
        for (int k = 0; k < 9; ++k) a.Q[k * a.plane + p] = o[k];
    }
}

// A pair of horizontally adjacent values from shared memory at an even
// base index plus OFF: one 8-byte load when OFF is even, two otherwise.
template <int OFF>
__device__ __forceinline__ float2 lds_pair(const float* S, int even_base) {
    if (OFF % 2 == 0) return *reinterpret_cast<const float2*>(S + even_base + OFF);
    return make_float2(S[even_base + OFF], S[even_base + OFF + 1]);
}

// Far tiles, two nodes per thread through the paired FP32 instructions:
// every R1 node is interior and off step n's band, every tile node interior.
// Column pairs start at even offsets, so the pulls of the six directions
// with ex != 0, the step n + 1 stores and the step n + 2 stores are 8-byte
// accesses.  A block takes PASS_TPC consecutive tiles (near tiles among them
// are skipped): once the first step of a tile has read the staged planes,
// thread 0 issues the next tile's tensor loads into the same buffer, so they
// fly while the second step runs.  The band bits of step n + 1 of each tile
// (R rows x PassShape<R>::WORDS words) are staged beside its loads.
#ifndef LBM_PASS_TPC
#define LBM_PASS_TPC 2
#endif
constexpr int PASS_TPC = LBM_PASS_TPC;

template <int R>
__device__ __forceinline__ bool pass_far_tile(const PassArgs& a, int t) {
    return t < a.ntx * a.nty && !pass_border_tile(t % a.ntx, t / a.ntx, a.nx, a.ny, R) && !__ldg(a.flags0 + t);
}

// Thread 0 arms the barrier and issues tile t's loads; the first
// WORDS * R threads stage its band bits.
template <int R>
__device__ __forceinline__ void pass_issue_far(const CUtensorMap* tm, const PassArgs& a, int t, float* Sin,
                                               uint64_t* bar, unsigned* sbits) {
    using S = PassShape<R>;
    const int x0 = (t % a.ntx) * PASS_TX, y0 = 1 + (t / a.ntx) * R;
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(9 * S::BOXH * S::BOXW * sizeof(float)));
#pragma unroll
        for (int k = 0; k < 9; ++k) tma_load_3d(Sin + k * S::CH, tm, x0 - 4, y0 - 2, k, bar);
    }
    if (threadIdx.x < S::WORDS * R) {
        const long long w = ((long long)(y0 + threadIdx.x / S::WORDS) * a.pitch + x0) >> 5;
        sbits[threadIdx.x] = __ldg(a.bits1 + w + threadIdx.x % S::WORDS);
    }
}

template <int R>
__global__ void __launch_bounds__(PassShape<R>::THREADS, PassShape<R>::MINB)
    pass_far_kernel(const __grid_constant__ CUtensorMap tm, const PassArgs a) {
    using S = PassShape<R>;
    extern __shared__ unsigned char pass_raw[];
    __shared__ uint64_t bar;
    __shared__ unsigned sbits[2][S::WORDS * R];
    float* Sin = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(pass_raw) + 127) & ~(uintptr_t)127);
    float* Smid = Sin + 9 * S::CH;
    const int first = blockIdx.x * PASS_TPC, last = first + PASS_TPC;
    int t = first;
    while (t < last && !pass_far_tile<R>(a, t)) ++t;
    if (t >= last) return;   // near tiles only
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    pass_issue_far<R>(&tm, a, t, Sin, &bar, sbits[0]);
    __syncthreads();
    for (int it = 0; t < last; ++it) {
        if (a.far_tiles && threadIdx.x == 0) atomicAdd(a.far_tiles, 1);
        const int tx = t % a.ntx, ty = t / a.ntx;
        const int x0 = tx * PASS_TX, y0 = 1 + ty * R;
        int tn = t + 1;   // the block's next far tile (its flag loads overlap the wait)
        while (tn < last && !pass_far_tile<R>(a, tn)) ++tn;
        // thread 0 waits for the loads; the others hold at the block barrier,
        // which orders the staged planes for them, without taking issue slots
        bool ok = true;
        if (threadIdx.x == 0) ok = mbar_wait(&bar, it & 1);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicOr(a.status, ST_COPY_TIMEOUT);
                mbar_wait(&bar, it & 1);   // let a late copy land before the block exits
            }
            return;
        }
        // step n + 1 on R1: pair u = (mr, mc / 2), nodes (x0 - 1 + mc, y0 - 1 + mr)
        // and the next column; box cell (mr + 1, mc + 3)
        for (int u = threadIdx.x; u < S::MH * S::MW / 2; u += S::THREADS) {
            const int mr = u / (S::MW / 2), mc = 2 * (u % (S::MW / 2));
            float2 g[9], o[9], drho, jx, jy;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int base = k * S::CH + (mr + 1 - ey(k)) * S::BOXW + mc;
                switch (ex(k)) {   // ex is a constant per unrolled k
                case 1: g[k] = lds_pair<2>(Sin, base); break;
                case -1: g[k] = lds_pair<4>(Sin, base); break;
                default: g[k] = lds_pair<3>(Sin, base); break;
                }
            }
            collide_lanes<float2>(g, PairK{a.k}, o, drho, jx, jy);
#pragma unroll
            for (int k = 0; k < 9; ++k) *reinterpret_cast<float2*>(Smid + k * S::MCH + mr * S::MW + mc) = o[k];
        }
        __syncthreads();   // the staged planes are read: the next tile's loads may land
        if (tn < last) {
            if (threadIdx.x == 0) fence_async_smem();
            pass_issue_far<R>(&tm, a, tn, Sin, &bar, sbits[(it + 1) & 1]);
        }
        // step n + 2 on the tile: pair (rr, cc / 2), nodes (x0 + cc, y0 + rr)
        // and the next column; R1 cell (rr + 1, cc + 1)
        const unsigned* bits = sbits[it & 1];
        for (int u = threadIdx.x; u < R * PASS_TX / 2; u += S::THREADS) {
            const int rr = u / (PASS_TX / 2), cc = 2 * (u % (PASS_TX / 2));
            const unsigned word = bits[rr * S::WORDS + (cc >> 5)];
            const unsigned b0 = (word >> (cc & 31)) & 1u, b1 = (word >> ((cc & 31) + 1)) & 1u;
            if (b0 & b1) continue;   // both band nodes of step n + 1
            float2 g[9], o[9], drho, jx, jy;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int base = k * S::MCH + (rr + 1 - ey(k)) * S::MW + cc;
                switch (ex(k)) {
                case 1: g[k] = lds_pair<0>(Smid, base); break;
                case -1: g[k] = lds_pair<2>(Smid, base); break;
                default: g[k] = lds_pair<1>(Smid, base); break;
                }
            }
            collide_lanes<float2>(g, PairK{a.k}, o, drho, jx, jy);
            float* q = a.Q + (long long)(y0 + rr) * a.pitch + x0 + cc;
            if (!(b0 | b1)) {
#pragma unroll
                for (int k = 0; k < 9; ++k) *reinterpret_cast<float2*>(q + k * a.plane) = o[k];
            } else {
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    if (!b0) q[k * a.plane] = o[k].x;
                    if (!b1) q[k * a.plane + 1] = o[k].y;
                }
            }
        }
        __syncthreads();   // R1 values read: the next tile's first step may overwrite them
        t = tn;
    }
}

template <int R>
__global__ void __launch_bounds__(PassShape<R>::THREADS, PassShape<R>::MINB)
    pass_near_kernel(const __grid_constant__ CUtensorMap tm, const PassArgs a) {
    extern __shared__ unsigned char pass_raw[];
    __shared__ uint64_t bar;
    const int b = blockIdx.x;
    int t;
    if (b < a.nborder) {
        t = __ldg(a.border_list + b);
    } else {
        if (b - a.nborder >= min(__ldcg(a.band_n), a.band_cap)) return;
        t = __ldcg(a.band_list + (b - a.nborder));
        if (pass_border_tile(t % a.ntx, t / a.ntx, a.nx, a.ny, R)) return;   // taken by its border block
    }
    float* Sin = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(pass_raw) + 127) & ~(uintptr_t)127);
    pass_tile_near<R>(&tm, a, t, Sin, Sin + 9 * PassShape<R>::CH, &bar);
}

int pass_tensor_map(const DevState& d, const float* base, int rows, void* out) {
    if (rows != PASS_TY && rows != PASS_TY_TALL) return -1;
    const cuuint32_t box[3] = {(cuuint32_t)PASS_TX + 8, (cuuint32_t)rows + 4, 1};
    return encode_plane_map(d, base, box, out);
}

template <int R>
void launch_pass_far_rows(const PassArgs& a, const void* tmap, cudaStream_t st) {
    pass_far_kernel<R><<<(a.ntx * a.nty + PASS_TPC - 1) / PASS_TPC, PassShape<R>::THREADS, PassShape<R>::SMEM, st>>>(
        *reinterpret_cast<const CUtensorMap*>(tmap), a);
}
template <int R>
void launch_pass_near_rows(const PassArgs& a, const void* tmap, cudaStream_t st) {
    pass_near_kernel<R><<<a.nborder + a.band_cap, PassShape<R>::THREADS, PassShape<R>::SMEM, st>>>(
        *reinterpret_cast<const CUtensorMap*>(tmap), a);
}

void launch_pass_far(const PassArgs& a, const void* tmap, cudaStream_t st) {
    if (a.rows == PASS_TY_TALL)
        launch_pass_far_rows<PASS_TY_TALL>(a, tmap, st);
    else
        launch_pass_far_rows<PASS_TY>(a, tmap, st);
}

void launch_pass_near(const PassArgs& a, const void* tmap, cudaStream_t st) {
    if (a.rows == PASS_TY_TALL)
        launch_pass_near_rows<PASS_TY_TALL>(a, tmap, st);
    else
        launch_pass_near_rows<PASS_TY>(a, tmap, st);
}

template <int R>
cudaError_t pass_prepare_rows() {
    const int smem = (int)PassShape<R>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(pass_far_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pass_near_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}
cudaError_t pass_prepare() {
    const cudaError_t e = pass_prepare_rows<PASS_TY>();
    return e == cudaSuccess ? pass_prepare_rows<PASS_TY_TALL>() : e;
}

bool is_pass_far_kernel(const void* func) {
    return func == reinterpret_cast<const void*>(pass_far_kernel<PASS_TY>) ||
           func == reinterpret_cast<const void*>(pass_far_kernel<PASS_TY_TALL>);
}
bool is_pass_near_kernel(const void* func) {
    return func == reinterpret_cast<const void*>(pass_near_kernel<PASS_TY>) ||
           func == reinterpret_cast<const void*>(pass_near_kernel<PASS_TY_TALL>);
}

// Step n + 1 values for the second step's immersed boundary and far field:
// item t < 64 nseg is slot t % 64 of the 8 x 8 square around segment
// t / 64's support box (the box and one ring), then the columns 1..3,
// nx-4..nx-2 (rows 1..ny-2) and the rows 1, 2, ny-3, ny-2 (columns
// 4..nx-5).  Band nodes of step n are skipped (the band re-collision writes
// them), and so are nodes outside a segment's square.
__global__ void __launch_bounds__(256) pass_ring_kernel(const DevState d, const float* __restrict__ P,
                                                        float* __restrict__ O, const unsigned* __restrict__ bits0) {
    const long long nbox = 64LL * d.nseg, ncol = 6LL * (d.ny - 2), nrow = 4LL * (d.nx - 8);
    for (long long t = (long long)blockIdx.x * 256 + threadIdx.x; t < nbox + ncol + nrow;
         t += (long long)gridDim.x * 256) {
        int i, j;
        if (t < nbox) {
            const int s = (int)(t >> 6), a = (int)(t & 63) >> 3, c = (int)(t & 7);
            const int i1 = d.box[4 * s], i2 = d.box[4 * s + 1], j1 = d.box[4 * s + 2], j2 = d.box[4 * s + 3];
            if (i2 < i1 || j2 < j1 || a > i2 - i1 + 2 || c > j2 - j1 + 2) continue;
            i = i1 - 2 + a;   // box columns i1 - 1 .. i2 - 1 (0-based) and one ring
            j = j1 - 2 + c;
        } else if (t < nbox + ncol) {
            const int u = (int)(t - nbox), col = u / (d.ny - 2);
            i = col < 3 ? 1 + col : d.nx - 7 + col;   // 1, 2, 3, nx-4, nx-3, nx-2
            j = 1 + u % (d.ny - 2);
        } else {
            const int u = (int)(t - nbox - ncol), row = u / (d.nx - 8);
            j = row < 2 ? 1 + row : d.ny - 5 + row;   // 1, 2, ny-3, ny-2
            i = 4 + u % (d.nx - 8);
        }
        if (i < 1 || i > d.nx - 2 || j < 1 || j > d.ny - 2) continue;
        const long long p = (long long)j * d.pitch + i;
        if ((__ldg(bits0 + (p >> 5)) >> (p & 31)) & 1u) continue;
        float g[9], o[9], drho, jx, jy;
#pragma unroll
        for (int k = 0; k < 9; ++k) g[k] = __ldg(P + k * d.plane + p - ex(k) - (long long)ey(k) * d.pitch);
        fused_collide(g, d.fc, o, drho, jx, jy);
#pragma unroll
        for (int k = 0; k < 9; ++k) O[k * d.plane + p] = o[k];
    }
}

void launch_pass_ring(const DevState& d, const float* P, float* O, const unsigned* bits0, cudaStream_t st) {
    const long long n = 64LL * d.nseg + 6LL * (d.ny - 2) + 4LL * (d.nx - 8);
    const int grid = (int)std::min<long long>(1184, std::max<long long>(1, (n + 255) / 256));
    pass_ring_kernel<<<grid, 256, 0, st>>>(d, P, O, bits0);
}

// Packed form: an episode's interior nodes, row by row without the border
// columns, in runs of BULK_TX consecutive nodes (a warp may straddle two
// rows), so narrow lattices leave no thread idle; a block takes RUNS runs
// (1, 2 or 4: the batch engine times the three on a batch's first long call
// and keeps the fastest; every node is computed the same way in each).
// The episode's parameters are staged in shared memory by one thread, so
// the kernel fits the single-episode kernel's register budget (eight
// 256-thread blocks per SM).
struct BulkArgs {
    const float* gA;
    float* gB;
    double *fo_rho, *fo_u, *fo_v;
    const unsigned* bits;
    long long plane;
    int pitch, w, n, l, fields;
    FusedConsts c;
};
template <bool FIELDS, int RUNS>
__device__ __forceinline__ void fused_bulk_runs(const BulkArgs& a) {
#pragma unroll
    for (int r = 0; r < RUNS; ++r) {
        const int t = (a.l * RUNS + r) * BULK_TX + threadIdx.x;
        if (t >= a.n) break;
        const int jj = t / a.w;
        fused_bulk_node<FIELDS, false>(a.gA, a.gB, a.pitch, a.plane, a.c, a.fo_rho, a.fo_u, a.fo_v, a.bits,
                                       t - jj * a.w + 1, jj + 1);
    }
}
template <int RUNS>
__global__ void __launch_bounds__(BULK_TX, 8) fused_bulk_kernel_multi(MultiArgs m) {
    __shared__ BulkArgs a;
    if (threadIdx.x == 0) {
        const int e = multi_episode(m, blockIdx.x);
        const DevState& d = *m.ds[e];
        a.gA = d.gA;
        a.gB = d.gB;
        a.fo_rho = d.fo_rho;
        a.fo_u = d.fo_u;
        a.fo_v = d.fo_v;
        a.bits = d.band_bits;
        a.plane = d.plane;
        a.pitch = d.pitch;
        a.w = d.nx - 2;
        a.n = (d.nx - 2) * (d.ny - 2);
        a.l = blockIdx.x - m.boff[e];
        a.fields = d.write_fields && d.fo_rho;
        a.c = d.fc;
    }
    __syncthreads();
    if (a.fields)
        fused_bulk_runs<true, RUNS>(a);
    else
        fused_bulk_runs<false, RUNS>(a);
}

// Initial state (solution.f90:44-61): f = f0 = feq(1, UU, 0) on every node,
// both copies of the planes and the border f0 store.
__global__ void fused_init_kernel(DevState d) {
    const long long n = d.plane;
    const long long per = 2LL * d.ny + 2LL * d.nx;
    double fe[9];
    const double u1 = d.uu, v1 = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double eu = (double)ex(k) * u1 + (double)ey(k) * v1;
        double utwo = u1 * u1 + v1 * v1;
        fe[k] = weight(k) * 1.0 * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * utwo);
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            float g = (float)(fe[k] - weight(k));
            d.gA[k * n + t] = g;
            d.gB[k * n + t] = g;
        }
        if (t < per) {
#pragma unroll
            for (int k = 0; k < 9; ++k) d.edge_f0[k * per + t] = fe[k];
        }
    }
}

// move_mesh for the fused path: gB = gA shifted by one column (dr = +1 takes
// the right neighbour), and the border f0 store takes the shifted values as
// the reference's f0 does (move_mesh.f90:36-55).
__global__ void fused_shift_kernel(DevState d, int dr) {
    const long long per = 2LL * d.ny + 2LL * d.nx;
    const long long total = (long long)d.nx * d.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx), j = (int)(t / d.nx);
        const bool moved = dr == 1 ? (i <= d.nx - 2) : (i >= 1);
        const int src = moved ? i + dr : i;
        const long long p = pidx(d, i, j), q = pidx(d, src, j);
        for (int k = 0; k < 9; ++k) d.gB[k * d.plane + p] = d.gA[k * d.plane + q];
        if (moved) {
            long long e = -1;
            if (i == 0) e = j;
            else if (i == d.nx - 1) e = d.ny + j;
            if (e >= 0)
                for (int k = 0; k < 9; ++k) d.edge_f0[k * per + e] = (double)d.gA[k * d.plane + q] + weight(k);
            e = -1;
            if (j == 0) e = 2LL * d.ny + i;
            else if (j == d.ny - 1) e = 2LL * d.ny + d.nx + i;
            if (e >= 0)
                for (int k = 0; k < 9; ++k) d.edge_f0[k * per + e] = (double)d.gA[k * d.plane + q] + weight(k);
        }
    }
}

__global__ void fused_export_kernel(DevState d, const float* g, double* f) {
    const long long total = (long long)d.nx * d.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx), j = (int)(t / d.nx);
        const long long p = pidx(d, i, j);
        for (int k = 0; k < 9; ++k) f[k * total + t] = (double)g[k * d.plane + p] + weight(k);
    }
}

__global__ void fused_import_kernel(DevState d, const double* f, float* g) {
    const long long total = (long long)d.nx * d.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx), j = (int)(t / d.nx);
        const long long p = pidx(d, i, j);
        for (int k = 0; k < 9; ++k) g[k * d.plane + p] = (float)(f[k * total + t] - weight(k));
    }
}

bool is_bulk_kernel(const void* func) {
    return func == reinterpret_cast<const void*>(fused_bulk_kernel<false>) ||
           func == reinterpret_cast<const void*>(fused_bulk_kernel<true>) ||
           func == reinterpret_cast<const void*>(fused_bulk_tma_kernel);
}

void launch_fused_bulk(const DevState& d, const FusedConsts& c, bool fields, const void* tmap, cudaStream_t st) {
    if (tmap && !fields) {
        const int ntx = (d.nx + TMA_TX - 1) / TMA_TX, nty = (d.ny - 2 + TMA_TY - 1) / TMA_TY;
        fused_bulk_tma_kernel<<<ntx * nty, TMA_THREADS, TMA_SMEM, st>>>(
            *reinterpret_cast<const CUtensorMap*>(tmap), d.gB, d.nx, d.ny, d.pitch, d.plane, c, d.band_bits, ntx,
            d.status);
        return;
    }
    dim3 b(BULK_TX), g((d.nx - 2 + BULK_TX - 1) / BULK_TX, (d.ny - 2 + BULK_ROWS - 1) / BULK_ROWS);
    if (fields)
        fused_bulk_kernel<true><<<g, b, 0, st>>>(d.gA, d.gB, d.nx, d.ny, d.pitch, d.plane, c, d.fo_rho, d.fo_u, d.fo_v,
                                                 d.band_bits);
    else
        fused_bulk_kernel<false><<<g, b, 0, st>>>(d.gA, d.gB, d.nx, d.ny, d.pitch, d.plane, c, nullptr, nullptr, nullptr,
                                                  d.band_bits);
}
// ------------------------------------------------------------ far field
// boundary_condition1 (boundary_condition.f90:288-858) for the fused path:
// the same LODI update and edge populations as outer_bc_kernel, with the
// moment transforms written out (M f and M^-1 m = M^T diag(1/9, 1/36,
// 1/36, 1/6, 1/12, 1/6, 1/12, 1/4, 1/4) m), one reciprocal per density,
// and fused multiply-adds -- this path is compared with tolerances, and the
// kernel runs while the bulk kernel saturates memory, so its dependent
// arithmetic chain is kept short.
struct FarMom {
    double r, u, v;
};

__device__ __forceinline__ void border_f0(const DevState& d, int i, int j, double* f) {
    const long long per = 2LL * d.ny + 2LL * d.nx;
    const long long e = (i == 0) ? j : (i == d.nx - 1) ? d.ny + j : (j == 0) ? 2LL * d.ny + i : 2LL * d.ny + d.nx + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = d.edge_f0[k * per + e];
}

__device__ __forceinline__ void pulled_f0(const DevState& d, int i, int j, double* f) {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (double)d.gA[k * d.plane + pidx(d, i - ex(k), j - ey(k))] + weight(k);
}

__device__ __forceinline__ FarMom far_moments(const double* f) {
    const double r = (((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7]))) + f[8];
    const double jx = (f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7]);
    const double jy = (f[2] - f[4]) + (f[5] + f[6]) - (f[7] + f[8]);
    const double ir = 1.0 / r;
    return FarMom{r, jx * ir, jy * ir};
}

// LODI update of the left (side = 0) or right (side = 1) column at row j
// (boundary_condition.f90:413-441, 495-521)
__device__ FarMom far_lodi(const DevState& d, int side, int j, double* fnb) {
    const double cs = (double)sqrtf(3.0f) / 3.0;
    const int ib = side == 0 ? 0 : d.nx - 1, i1 = side == 0 ? 1 : d.nx - 2, i2 = side == 0 ? 2 : d.nx - 3;
    double fb[9], f2[9];
    border_f0(d, ib, j, fb);
    pulled_f0(d, i1, j, fnb);
    pulled_f0(d, i2, j, f2);
    const FarMom b = far_moments(fb), m1 = far_moments(fnb), m2 = far_moments(f2);
    const double sg = side == 0 ? -1.0 : 1.0;   // one-sided difference toward the inside
    const double rhox = sg * (3.0 * b.r - 4.0 * m1.r + m2.r) * 0.5;
    const double ux = sg * (3.0 * b.u - 4.0 * m1.u + m2.u) * 0.5;
    const double vx = sg * (3.0 * b.v - 4.0 * m1.v + m2.v) * 0.5;
    double lx1 = 0.0, lx2 = 0.0, lx3 = 0.0;
    if (side == 0) {
        lx1 = (b.u - cs) * (cs * cs * rhox - cs * b.r * ux);
        lx2 = (b.u < 0.0) ? b.u * vx : 0.0;
    } else {
        lx2 = (b.u >= 0.0) ? b.u * vx : 0.0;
        lx3 = (b.u + cs) * (cs * cs * rhox + cs * b.r * ux);
    }
    FarMom o;
    o.r = b.r - (lx1 + lx3) * 1.5;
    o.u = b.u + (lx1 - lx3) / (2.0 * cs * o.r);
    o.v = b.v - lx2;
    return o;
}

__device__ __forceinline__ void far_meq(const FarMom& m, double* t) {
    const double jx = m.r * m.u, jy = m.r * m.v, ir = 1.0 / m.r;
    const double q = (jx * jx + jy * jy) * ir;
    t[0] = m.r; t[1] = -2.0 * m.r + 3.0 * q; t[2] = m.r - 3.0 * q;
    t[3] = jx; t[4] = -jx; t[5] = jy; t[6] = -jy;
    t[7] = (jx * jx - jy * jy) * ir; t[8] = jx * jy * ir;
}

// edge populations f = M^-1 [m_eq(edge) + (I - S)(M f0(nbr) - m_eq(nbr))]
__device__ void far_edge(const DevState& d, int ie, int je, const FarMom& e, const double* fn, const FarMom& nb) {
    double t1[9], t2[9], m[9];
    far_meq(e, t1);
    far_meq(nb, t2);
    const double s14 = (fn[1] + fn[3]) + (fn[2] + fn[4]), s58 = (fn[5] + fn[7]) + (fn[6] + fn[8]);
    const double d13 = fn[1] - fn[3], d24 = fn[2] - fn[4], a5 = fn[5] - fn[7], a6 = fn[6] - fn[8];
    m[0] = (fn[0] + s14) + s58;
    m[1] = -4.0 * fn[0] - s14 + 2.0 * s58;
    m[2] = 4.0 * fn[0] - 2.0 * s14 + s58;
    m[3] = d13 + a5 - a6;
    m[4] = -2.0 * d13 + a5 - a6;
    m[5] = d24 + a5 + a6;
    m[6] = -2.0 * d24 + a5 + a6;
    m[7] = (fn[1] + fn[3]) - (fn[2] + fn[4]);
    m[8] = (fn[5] + fn[7]) - (fn[6] + fn[8]);
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = t1[k] + (1.0 - d.s[k]) * (m[k] - t2[k]);
    const double b0 = m[0] * (1.0 / 9.0), b1 = m[1] * (1.0 / 36.0), b2 = m[2] * (1.0 / 36.0);
    const double b3 = m[3] * (1.0 / 6.0), b4 = m[4] * (1.0 / 12.0), b5 = m[5] * (1.0 / 6.0);
    const double b6 = m[6] * (1.0 / 12.0), b7 = m[7] * 0.25, b8 = m[8] * 0.25;
    const double rA = b0 - b1 - 2.0 * b2, rD = b0 + 2.0 * b1 + b2;
    const double x34 = b3 - 2.0 * b4, y56 = b5 - 2.0 * b6, xd = b3 + b4, yd = b5 + b6;
    double o[9];
    o[0] = b0 - 4.0 * b1 + 4.0 * b2;
    o[1] = rA + x34 + b7; o[2] = rA + y56 - b7; o[3] = rA - x34 + b7; o[4] = rA - y56 - b7;
    o[5] = rD + xd + yd + b8; o[6] = rD - xd + yd - b8; o[7] = rD - xd - yd + b8; o[8] = rD + xd - yd - b8;
    const long long p = pidx(d, ie, je);
#pragma unroll
    for (int k = 0; k < 9; ++k) d.gB[k * d.plane + p] = (float)(o[k] - weight(k));
    if (d.write_fields && d.fo_rho) {
        d.fo_rho[p] = e.r;
        d.fo_u[p] = e.u;
        d.fo_v[p] = e.v;
    }
}

// One thread per border node: [left j=1..ny-2][right j=1..ny-2][top i][bottom i];
// the corners of the top and bottom rows take the LODI state of the column
// node inside them, as the reference's edge order left -> right -> top ->
// bottom leaves it.
// border nodes per thread: one alone, slot_items in packed launches
__host__ __device__ inline int far_field_grid(const DevState& d) {
    const int n = 2 * (d.ny - 2) + 2 * d.nx, per = 64 * d.slot_items;
    return (n + per - 1) / per;
}
__device__ __forceinline__ void fused_bc_node(const DevState& d, int t) {
    const int nl = d.ny - 2;
    double fn[9];
    if (t < 2 * nl) {
        const int side = t < nl ? 0 : 1, j = 1 + (side == 0 ? t : t - nl);
        const FarMom e = far_lodi(d, side, j, fn);
        far_edge(d, side == 0 ? 0 : d.nx - 1, j, e, fn, far_moments(fn));
        return;
    }
    t -= 2 * nl;
    if (t < 2 * d.nx) {
        const bool top = t < d.nx;
        const int i = top ? t : t - d.nx;
        const int je = top ? d.ny - 1 : 0, jn = top ? d.ny - 2 : 1;
        FarMom nb;
        if (i == 0 || i == d.nx - 1) {
            double fc[9];
            nb = far_lodi(d, i == 0 ? 0 : 1, jn, fc);
            border_f0(d, i, jn, fn);   // the corner column node's own populations
        } else {
            pulled_f0(d, i, jn, fn);
            nb = far_moments(fn);
        }
        far_edge(d, i, je, FarMom{nb.r, 0.0, 0.0}, fn, nb);
    }
}
__device__ __forceinline__ void fused_bc_kernel_body(const DevState& d, const int bid_) {
    const int n = 2 * (d.ny - 2) + 2 * d.nx, stride = far_field_grid(d) * 64;
    for (int t = bid_ * 64 + threadIdx.x; t < n; t += stride) fused_bc_node(d, t);
}
__global__ void __launch_bounds__(64) fused_bc_kernel(DevState d) { fused_bc_kernel_body(d, blockIdx.x); }
__global__ void __launch_bounds__(64) fused_bc_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    fused_bc_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

void launch_fused_bc(const DevState& d, cudaStream_t st) { fused_bc_kernel<<<far_field_grid(d), 64, 0, st>>>(d); }

void launch_fused_init(const DevState& d, cudaStream_t st) { fused_init_kernel<<<1184, 256, 0, st>>>(d); }
void launch_fused_shift(const DevState& d, int dr, cudaStream_t st) { fused_shift_kernel<<<1184, 256, 0, st>>>(d, dr); }
void launch_fused_export(const DevState& d, const float* g, double* f, cudaStream_t st) {
    fused_export_kernel<<<1184, 256, 0, st>>>(d, g, f);
}
void launch_fused_import(const DevState& d, const double* f, float* g, cudaStream_t st) {
    fused_import_kernel<<<1184, 256, 0, st>>>(d, f, g);
}

// ------------------------------------------------------------ packed launches
int multi_blocks_fused(MultiKernel k, const DevState& d) {
    switch (k) {
    case MK_BULK1:
    case MK_BULK2:
    case MK_BULK4: {
        const int per = k == MK_BULK1 ? 1 : k == MK_BULK2 ? 2 : 4;
        const long long runs = ((long long)(d.nx - 2) * (d.ny - 2) + BULK_TX - 1) / BULK_TX;
        return (int)((runs + per - 1) / per);
    }
    case MK_BC: return far_field_grid(d);
    default: return -1;
    }
}

bool launch_multi_fused(MultiKernel k, const MultiArgs& m, int blocks, cudaStream_t st) {
    switch (k) {
    case MK_BULK1: fused_bulk_kernel_multi<1><<<blocks, BULK_TX, 0, st>>>(m); return true;
    case MK_BULK2: fused_bulk_kernel_multi<2><<<blocks, BULK_TX, 0, st>>>(m); return true;
    case MK_BULK4: fused_bulk_kernel_multi<4><<<blocks, BULK_TX, 0, st>>>(m); return true;
    case MK_BC: fused_bc_kernel_multi<<<blocks, 64, 0, st>>>(m); return true;
    default: return false;
    }
}

bool is_far_field_multi_kernel(const void* func) { return func == reinterpret_cast<const void*>(fused_bc_kernel_multi); }

bool is_bulk_multi_kernel(const void* func) {
    return func == reinterpret_cast<const void*>(fused_bulk_kernel_multi<1>) ||
           func == reinterpret_cast<const void*>(fused_bulk_kernel_multi<2>) ||
           func == reinterpret_cast<const void*>(fused_bulk_kernel_multi<4>);
}

bool is_far_field_kernel(const void* func) { return func == reinterpret_cast<const void*>(fused_bc_kernel); }

}  // namespace lbm
