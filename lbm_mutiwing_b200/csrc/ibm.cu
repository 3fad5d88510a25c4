// Implicit velocity-correction immersed boundary step (bc_num = 4), on the
// device in FP64, as short kernels on two streams.
//
// Reference: move_boundary (airfoil.f90:244-338) and immersed_boundary_Wu
// (boundary_condition.f90:1512-1736), with the motion lookup of mode.f90.
//
// The reference builds dense delta matrices xx1 (segments x band) and
// xx2 = xx1^T diag(arc_l), forms A = xx1 xx2 with cublasDgemm and solves
// A c = ub - xx1 u* with cuSOLVER LU.  Because A = X X^T D and the spread is
// du = X^T D c, the arc lengths cancel: du = X^T y with (X X^T) y = ub - X u*.
// Here X is kept sparse: segment s touches only the nodes of its support box
// (at most 6 x 6), and the smoothed delta kernel is a product
// phi(rx) phi(ry), so a segment needs 6 + 6 kernel values (kx, ky) and
//   G(a, c) = [sum_i kx_a(i) kx_c(i)] [sum_j ky_a(j) ky_c(j)]
// over the common node columns i and rows j of the two boxes.  G is
// assembled per wing in a banded layout after a reverse Cuthill-McKee
// ordering fixed at set-up (rigid wings keep their pairwise distances) and
// factored as L' D L'^T, panel by panel, one thread block per wing.  G
// depends on the geometry only, so assembly and factorisation run on a side
// stream while the band list and the right-hand side are built.
//
// Kernels of one step (main chain | side chain):
//   geometry   motion, markers, midpoints, support boxes, kernel values,
//              clearing of the previous band             (move_boundary)
//   claim      lowest segment index claims each box node   | assemble  G
//   count      claims per segment                          | factor    L' D L'^T
//   scan       band-list offsets, coupled-wing check       |
//   list       band list in the reference's order (segment, i, j), band
//              bit plane; advances the geometry's cycle counter
// then, plain FP64 path:
//   ustar      u*, rho at band nodes; zeroed spread accumulators
//   rhs        r = ub - X u* (one warp per segment)
//   solve      forward and backward substitution (waits for the factor)
//   spread     du = X^T y with fixed-point integer atomics
//   finish     du, body force, per-block force partials
//   forces     per-wing force and moment, force row
// or, FP32 path (beside the bulk kernel):
//   rhs        u* from the pulled distributions at each box node, r = ub - X u*
//   solve, spread as above
//   close      du, band-node re-collision, force partials; the last block
//              writes the force row and advances the cycle counter
//
// Determinism: the band list is built in first-claimant order from an
// atomicMin claim pass plus a prefix sum; the spread rounds every
// contribution once to a 64-bit fixed-point number and adds integers
// (associative, hence order-independent); all other sums use fixed trees.
// Results are identical from run to run.
//
// The box scan compares node distances against 2.5 spacings: marker,
// midpoint and node coordinates are formed with explicitly rounded
// multiplies and adds in the reference's order so that band membership
// matches it.
#include <cstdio>

#include "lbm_kernels.h"
#include "multi.cuh"

namespace lbm {

constexpr int MAX_WINGS = 16;
constexpr int FINISH_THREADS = 256;
constexpr int BORDER_GAP = 3;           // support boxes keep this many nodes off the border

__device__ inline void set_status(const DevState& d, int bit) { atomicOr(d.status, bit); }

// Grids.  The per-slot kernels (claims, spread) and the assembly of G loop
// over d.slot_items items per thread, and the motion kernel clears the
// previous band in a loop.  One episode uses one item per thread (its
// latency-bound chains want the most threads); packed batches use several,
// so a step dispatches a few thousand blocks of immersed-boundary work
// instead of tens of thousands, which would hold up the bulk kernel's
// dispatch (they run at higher priority).  Results do not depend on it.
__host__ __device__ inline int grid_of(long long n, int threads) { return (int)(n <= 0 ? 1 : (n + threads - 1) / threads); }
__host__ __device__ inline int geometry_grid(const DevState& d) {
    return grid_of(d.npts > 12 * d.nseg ? d.npts : 12 * d.nseg, 128);
}
__host__ __device__ inline int slot_grid(const DevState& d) {
    return grid_of((long long)d.nseg * BOX_SLOTS, 256 * d.slot_items);
}
__host__ __device__ inline int assemble_grid(const DevState& d) { return grid_of(d.lband_total, 256 * d.slot_items); }
// rhs: one warp per segment, 128-thread blocks
__host__ __device__ inline int rhs_grid(const DevState& d) { return grid_of(32LL * d.nseg, 128 * d.slot_items); }

// Exactly rounded FP64 steps for the marker and box arithmetic.
__device__ inline double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double add(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double sub(double a, double b) { return __dsub_rn(a, b); }
// node coordinate ox + scale * (i - 1) as the reference rounds it
__device__ inline double node_x(double o, double scale, int i) { return add(o, mul(scale, (double)(i - 1))); }

// smooth ramp functions of the online motion (mode.f90:220-261)
__device__ inline double smooth_r(double x) {
    if (x < 0.0) return 0.0;
    if (x <= 1.0) return 0.5 * x * x + (cos(2.0 * PAI * x) - 1.0) / (4.0 * PAI * PAI);
    return x - 0.5;
}
__device__ inline double smooth_h(double x) {
    if (x < 0.0) return 0.0;
    if (x <= 1.0) return x - sin(2.0 * PAI * x) / (2.0 * PAI);
    return 1.0;
}
__device__ inline double smooth_d(double x) {
    if (x >= 0.0 && x <= 1.0) return 1.0 - cos(2.0 * PAI * x);
    return 0.0;
}
// interpolate_motion_triplet (mode.f90:263-285)
__device__ inline void triplet(double s0, double v0, double v1, double dt, double lt, double& s,
                               double& v, double& a) {
    double dv = v1 - v0;
    if (dt <= 1.0e-14) {
        s = (v0 + dv) * lt + s0;
        v = v0 + dv;
        a = 0.0;
        return;
    }
    double x = lt / dt;
    s = dv * dt * smooth_r(x) + v0 * lt + s0;
    v = dv * smooth_h(x) + v0;
    a = dv / dt * smooth_d(x);
}

// time of the current step (force rows) and of the geometry being built
// (solution.f90:292); the geometry runs one step ahead of the flow on its
// own counter, which the band list kernel advances
__device__ inline double step_time(const DevState& d) {
    return mul((double)(*d.cycle - 1), mul(d.scale, d.uu));
}
__device__ inline double geometry_time(const DevState& d) {
    return mul((double)(*d.gcycle - 1), mul(d.scale, d.uu));
}

// mode + apply_motion_row for wing w at the current cycle (mode.f90:451-471,
// 180-218, 414-449) and update_body_extra_from_rel (mode.f90:473-495),
// whose relative motion is zero unless rigid-body dynamics are enabled.
__device__ WingMotion wing_motion(const DevState& d, int w) {
    const double time = geometry_time(d);
    double v[9];
    if (d.motion_source == 2) {
        const double t1 = d.stream_start[0], t2 = d.stream_target[0], dt = t2 - t1;
        const int col = 1 + 9 * w;
        if (time <= t1 + 1.0e-12) {
            for (int c = 0; c < 9; ++c) v[c] = d.stream_start[col + c];
        } else {
            double lt = fmin(fmax(time - t1, 0.0), fmax(dt, 0.0));
            for (int t = 0; t < 3; ++t)
                triplet(d.stream_start[col + 3 * t], d.stream_start[col + 3 * t + 1],
                        d.stream_target[col + 3 * t + 1], dt, lt, v[3 * t], v[3 * t + 1], v[3 * t + 2]);
        }
    } else {
        long long idx = llround(time / d.motion_dt) + 1;
        idx = idx < 1 ? 1 : (idx > d.step_rows ? d.step_rows : idx);
        const double* row = d.step_table + (idx - 1) * d.ncol + 1 + 9 * w;
        for (int c = 0; c < 9; ++c) v[c] = row[c];
    }
    WingMotion m;
    m.angle = v[0]; m.omega = v[1]; m.omgac = v[2];
    m.sa = v[3]; m.sau = v[4]; m.saac = v[5];
    m.sb = v[6]; m.sbv = v[7]; m.sbac = v[8];
    if (d.motion_source == 1) {
        m.sa = m.sa - (d.wing_x_origin + (double)w * d.wing_x_spacing);
        m.sb = m.sb - d.wing_y_origin;
    }
    double ap = 0.0;
    for (int k = 0; k <= w; ++k) ap = add(ap, d.rel_pos[k]);
    m.extra_v = 0.0;
    m.extra_s = 0.0;
    m.extra_pos = ap;
    return m;
}

__device__ inline int wing_of_point(const DevState& d, int p) {
    int w = 0;
    while (w + 1 < d.wing_count && p >= d.wing_pstart[w + 1]) ++w;
    return w;
}

// marker point p of wing w (airfoil.f90:260-264)
__device__ inline void marker(const DevState& d, const WingMotion& m, int w, int p, double& x, double& y) {
    double ca, sn;
    sincos(m.angle, &sn, &ca);
    x = add(mul(ca, d.xb0[p]), mul(sn, d.yb0[p]));
    x = add(add(add(add(x, d.wing_x_origin), mul((double)w, d.wing_x_spacing)), m.sa), d.xc);
    x = sub(add(x, m.extra_s / (1.0 / d.scale)), mul((double)d.movenum, d.scale));
    y = add(-mul(sn, d.xb0[p]), mul(ca, d.yb0[p]));
    y = add(add(add(y, d.wing_y_origin), m.sb), d.yc);
}

// ---------------------------------------------------------------- kernels
// move_boundary part 1: markers, midpoints, support boxes (airfoil.f90:288-321),
// separable delta values (boundary_condition.f90:1580-1603), and the clearing
// of the previous band (airfoil.f90:276-284).  Twelve threads per segment:
// thread (s, axis, k) scans its axis for the box and evaluates the kernel at
// the box's k-th node column or row.
__device__ __forceinline__ void ibm_geometry_kernel_body(const DevState& d, const int bid_) {
    const int t = bid_ * blockDim.x + threadIdx.x;
    if (t < d.wing_count) d.wm[t] = wing_motion(d, t);
    if (t < d.npts) {
        const int w = wing_of_point(d, t);
        const WingMotion m = wing_motion(d, w);
        double x, y;
        marker(d, m, w, t, x, y);
        d.xb1[t] = x;
        d.yb1[t] = y;
    }
    if (t < d.nseg * 12) {
        const int s = t / 12, q = t % 12, axis = q / 6, k = q % 6;
        const int w = d.seg_wing[s];
        const WingMotion m = wing_motion(d, w);
        const int p = d.wing_pstart[w] + (s - d.wing_sstart[w]);
        double xa, ya, xb, yb;
        marker(d, m, w, p + 1, xb, yb);
        marker(d, m, w, p, xa, ya);
        const double c2 = axis == 0 ? mul(0.5, add(xb, xa)) : mul(0.5, add(yb, ya));
        const double o = axis == 0 ? d.ox : d.oy;
        const int n = axis == 0 ? d.nx : d.ny;
        int lo = (int)(add((c2 - o) / d.scale, 1.0));
        for (int i = lo; i >= 1; --i)
            if (fabs((node_x(o, d.scale, i) - c2) / d.scale) > 2.5) { lo = i + 1; break; }
        int hi = (int)(add((c2 - o) / d.scale, 1.0));
        for (int i = hi; i <= n; ++i)
            if (fabs((node_x(o, d.scale, i) - c2) / d.scale) > 2.5) { hi = i - 1; break; }
        // the far-field boundary reads the moments of the first three rows
        // and columns, which must stay outside every support box
        if (lo < 1 + BORDER_GAP || hi > n - BORDER_GAP || hi - lo > 5 || hi < lo) {
            if (k == 0) set_status(d, ST_BOX_OUTSIDE);
            lo = 1; hi = 0;   // empty box
        }
        (axis == 0 ? d.kx : d.ky)[6 * s + k] =
            (lo + k <= hi) ? delta_phi(fabs((node_x(o, d.scale, lo + k) - c2) / d.scale)) : 0.0;
        if (k == 0) {
            d.box[4 * s + 2 * axis] = lo;
            d.box[4 * s + 2 * axis + 1] = hi;
            (axis == 0 ? d.xb2 : d.yb2)[s] = c2;
        }
    }
    const int nclear = d.band_n[0], stride = geometry_grid(d) * 128;
    for (int b = t; b < nclear; b += stride) {
        const long long p = pidx(d, d.band_ij[2 * b], d.band_ij[2 * b + 1]);
        d.band_map[p] = BAND_EMPTY;
        if (d.band_bits) atomicAnd(d.band_bits + (p >> 5), ~(1u << (p & 31)));
        if (d.precision == 0) { d.gfx[p] = 0.0; d.gfy[p] = 0.0; }
    }
    if (d.tile_flags) {   // set again by the count kernel
        const int nwords = (d.pass_ntx * d.pass_nty + 3) >> 2;
        for (int b = t; b < nwords; b += stride) reinterpret_cast<unsigned*>(d.tile_flags)[b] = 0u;
    }
    if (t == 0 && d.wing_count > 0 && d.motion_source == 1 && d.step_rows <= 0) set_status(d, ST_MOTION);
    if (t == 0) d.ibm_flags[0] = 0;   // set again by the count kernel when supports share nodes
}
__global__ void ibm_geometry_kernel(DevState d) { ibm_geometry_kernel_body(d, blockIdx.x); }
__global__ void ibm_geometry_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_geometry_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

__device__ inline bool box_empty(const DevState& d, int s) {
    return d.box[4 * s + 1] < d.box[4 * s] || d.box[4 * s + 3] < d.box[4 * s + 2];
}

// claims: lowest segment index wins (airfoil.f90:322-333)
__device__ __forceinline__ void ibm_claim_kernel_body(const DevState& d, const int bid_) {
    const int n = d.nseg * BOX_SLOTS, stride = slot_grid(d) * 256;
    for (int t = bid_ * 256 + threadIdx.x; t < n; t += stride) {
        const int s = t / BOX_SLOTS, slot = t % BOX_SLOTS;
        if (box_empty(d, s)) continue;
        const int i = d.box[4 * s] + slot / 6, j = d.box[4 * s + 2] + slot % 6;
        if (i <= d.box[4 * s + 1] && j <= d.box[4 * s + 3]) atomicMin(&d.band_map[pidx(d, i - 1, j - 1)], s);
    }
}
__global__ void ibm_claim_kernel(DevState d) { ibm_claim_kernel_body(d, blockIdx.x); }
__global__ void ibm_claim_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_claim_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Flags the pass tiles whose R1 (the tile and one ring) holds node (i, j)
// (0-based): tx with x0 - 1 <= i <= x0 + PASS_TX, ty with y0 - 1 <= j <=
// y0 + R (x0 = PASS_TX tx, y0 = 1 + R ty, R = d.pass_rows).
__device__ inline void flag_pass_tiles(const DevState& d, int i, int j) {
    const int R = d.pass_rows;
    const int tx0 = max(0, (i + PASS_TX - 1) / PASS_TX - 1), tx1 = min(d.pass_ntx - 1, (i + 1) / PASS_TX);
    const int ty0 = max(0, (j + R - 2) / R - 1), ty1 = min(d.pass_nty - 1, j / R);
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) d.tile_flags[ty * d.pass_ntx + tx] = 1;
}

// Claims per segment, and the coupling test: a box node claimed by a
// segment of another wing lies in the supports of both wings, so G has
// entries between them and the wings are solved jointly (the lowest segment
// index claims a node, hence every shared node is seen from the higher
// wing's side).  One warp per segment, a box slot per lane: every node's
// claimer is loaded at once and counted by a ballot.  Each claimed node
// flags the pass tiles around it.
__device__ __forceinline__ void ibm_count_kernel_body(const DevState& d, const int bid_) {
    const int s = (bid_ * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= d.nseg) return;
    int c = 0;
    bool shared = false;
    if (!box_empty(d, s)) {
        const int w = d.seg_wing[s];
        const int i1 = d.box[4 * s], i2 = d.box[4 * s + 1], j1 = d.box[4 * s + 2], j2 = d.box[4 * s + 3];
        for (int slot0 = 0; slot0 < BOX_SLOTS; slot0 += 32) {
            const int slot = slot0 + lane, i = i1 + slot / 6, j = j1 + slot % 6;
            bool mine = false;
            if (slot < BOX_SLOTS && i <= i2 && j <= j2) {
                const int bm = d.band_map[pidx(d, i - 1, j - 1)];
                mine = bm == s;
                shared |= bm != s && bm >= 0 && bm < d.nseg && d.seg_wing[bm] != w;
                if (mine && d.tile_flags) flag_pass_tiles(d, i - 1, j - 1);
            }
            c += __popc(__ballot_sync(0xffffffffu, mine));
        }
    }
    if (lane == 0) d.claim_cnt[s] = c;
    if (__any_sync(0xffffffffu, shared) && lane == 0) {
        d.ibm_flags[0] = 1;
        set_status(d, ST_WINGS_COUPLED);
    }
}
__global__ void ibm_count_kernel(DevState d) { ibm_count_kernel_body(d, blockIdx.x); }
__global__ void ibm_count_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_count_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Exclusive scan of the claim counts (one block) and the band size.
__device__ __forceinline__ void ibm_scan_kernel_body(const DevState& d, const int bid_) {
    __shared__ int wsum[32];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int per = (d.nseg + nt - 1) / nt;
    const int lo = min(d.nseg, tid * per), hi = min(d.nseg, lo + per);
    int lsum = 0;
    for (int s = lo; s < hi; ++s) lsum += d.claim_cnt[s];
    int x = lsum;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    int base = 0, tot = 0;
    for (int k = 0; k < (nt >> 5); ++k) {
        if (k < warp) base += wsum[k];
        tot += wsum[k];
    }
    int run = base + x - lsum;
    for (int s = lo; s < hi; ++s) {
        const int c = d.claim_cnt[s];
        d.claim_cnt[s] = run;
        run += c;
    }
    __syncthreads();
    if (tid == 0) {
        const int nb = min(tot, d.band_cap);
        if (tot > d.band_cap) set_status(d, ST_BAND_OVERFLOW);
        d.band_n[0] = nb;
        d.claim_cnt[d.nseg] = nb;
    }
    if (!d.tile_flags) return;
    // the flagged pass tiles in index order (the same scan over the flags)
    const int ntl = d.pass_ntx * d.pass_nty, tper = (ntl + nt - 1) / nt;
    const int t0 = min(ntl, tid * tper), t1 = min(ntl, t0 + tper);
    int tl = 0;
    for (int u = t0; u < t1; ++u) tl += d.tile_flags[u];
    x = tl;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();   // wsum is free again
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    int tb = 0, ttot = 0;
    for (int k = 0; k < (nt >> 5); ++k) {
        if (k < warp) tb += wsum[k];
        ttot += wsum[k];
    }
    int at = tb + x - tl;
    for (int u = t0; u < t1; ++u)
        if (d.tile_flags[u]) d.tile_list[at++] = u;
    if (tid == 0) d.tile_n[0] = ttot;
}
__global__ void __launch_bounds__(1024) ibm_scan_kernel(DevState d) { ibm_scan_kernel_body(d, blockIdx.x); }
__global__ void __launch_bounds__(1024) ibm_scan_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_scan_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Band list in the reference's order (segment, then i, then j) and the
// band_map encoding -(b + 2); a node still holding its claimer's index is
// never confused with another segment's index, so encoding as we go is safe.
// One warp per segment, a box slot per lane: slot a * 6 + c is node
// (i1 + a, j1 + c), so a claimed slot's place is its segment's offset plus
// the claimed slots before it (a ballot prefix).  The geometry's cycle
// counter moves on (the motion kernel read it before).
__device__ __forceinline__ void ibm_list_kernel_body(const DevState& d, const int bid_) {
    const int s = (bid_ * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s == 0 && lane == 0) *d.gcycle += 1;
    if (s >= d.nseg || box_empty(d, s)) return;
    const int nb = d.band_n[0];
    const int w = d.seg_wing[s];
    const int i1 = d.box[4 * s], i2 = d.box[4 * s + 1], j1 = d.box[4 * s + 2], j2 = d.box[4 * s + 3];
    int b = d.claim_cnt[s];
    for (int slot0 = 0; slot0 < BOX_SLOTS; slot0 += 32) {
        const int slot = slot0 + lane, i = i1 + slot / 6, j = j1 + slot % 6;
        long long p = 0;
        bool mine = false;
        if (slot < BOX_SLOTS && i <= i2 && j <= j2) {
            p = pidx(d, i - 1, j - 1);
            mine = d.band_map[p] == s;
        }
        const unsigned ball = __ballot_sync(0xffffffffu, mine);
        const int bi = b + __popc(ball & ((1u << lane) - 1u));
        if (mine && bi < nb) {
            d.band_ij[2 * bi] = i - 1;
            d.band_ij[2 * bi + 1] = j - 1;
            d.band_wing[bi] = w;
            d.band_claimer[bi] = s;
            d.band_map[p] = -(bi + 2);
            if (d.band_bits) atomicOr(d.band_bits + (p >> 5), 1u << (p & 31));
        }
        b += __popc(ball);
    }
}
__global__ void ibm_list_kernel(DevState d) { ibm_list_kernel_body(d, blockIdx.x); }
__global__ void ibm_list_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_list_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Plain path: u*, rho at band nodes from the moment fields
// (solution.f90:510-554), and the spread accumulators zeroed.  The FP32 path
// evaluates u* inside its rhs kernel instead.
__global__ void ibm_ustar_kernel(DevState d) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.band_n[0]) return;
    const long long p = pidx(d, d.band_ij[2 * b], d.band_ij[2 * b + 1]);
    reinterpret_cast<unsigned long long*>(d.band_du)[b] = 0ull;
    reinterpret_cast<unsigned long long*>(d.band_dv)[b] = 0ull;
    d.band_rho[b] = d.rho[p];
    d.band_us[b] = d.u[p];
    d.band_vs[b] = d.v[p];
}

// r = ub - X u* (boundary_condition.f90:1540-1555, 1609-1629) and the band
// index of each (segment, slot); one warp per segment, slots 0..35 over the
// lanes, summed by a fixed butterfly.
__device__ __forceinline__ void ibm_rhs_kernel_body(const DevState& d, const int bid_) {
    const int s = (bid_ * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= d.nseg) return;
    const int nb = d.band_n[0];
    const int i1 = d.box[4 * s], i2 = d.box[4 * s + 1], j1 = d.box[4 * s + 2], j2 = d.box[4 * s + 3];
    double bu = 0.0, bv = 0.0;
    for (int slot = lane; slot < BOX_SLOTS; slot += 32) {
        const int a = slot / 6, c = slot % 6;
        const int i = i1 + a, j = j1 + c;
        int bi = -1;
        if (i <= i2 && j <= j2) {
            const int bm = d.band_map[pidx(d, i - 1, j - 1)];
            bi = (bm <= -2) ? -(bm + 2) : -1;
            if (bi >= nb) bi = -1;
            if (bi < 0) {
                set_status(d, ST_BAND_OVERFLOW);
            } else {
                const double wv = d.kx[6 * s + a] * d.ky[6 * s + c];
                bu = bu + wv * d.band_us[bi];
                bv = bv + wv * d.band_vs[bi];
            }
        }
        d.pb[s * BOX_SLOTS + slot] = bi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        bu += __shfl_xor_sync(0xffffffffu, bu, o);
        bv += __shfl_xor_sync(0xffffffffu, bv, o);
    }
    if (lane == 0) {
        const int w = d.seg_wing[s];
        const WingMotion m = d.wm[w];
        const int p = d.wing_pstart[w] + (s - d.wing_sstart[w]);
        double sn, cs;
        sincos(m.angle, &sn, &cs);
        const double xs = d.xb0[p + 1] + d.xb0[p], ys = d.yb0[p + 1] + d.yb0[p];
        const double ub = d.uu * (-(m.omega * sn * 0.5 * xs) + m.omega * cs * 0.5 * ys + m.sau) + m.extra_v;
        const double vb = d.uu * (-(m.omega * cs * 0.5 * xs) - m.omega * sn * 0.5 * ys + m.sbv);
        d.rx[s] = ub - bu;
        d.ry[s] = vb - bv;
        d.qx[s] = ub - bu;   // kept for the residual diagnostic
        d.qy[s] = vb - bv;
    }
}
__global__ void ibm_rhs_kernel(DevState d) { ibm_rhs_kernel_body(d, blockIdx.x); }

// rho and u* of a band node from its pulled distributions (fused path;
// band nodes are interior nodes: boxes keep off the border), as the
// moments of solution.f90:510-554.
__device__ __forceinline__ void pulled_moments(const DevState& d, long long p, double f[9], double& rho, double& us,
                                               double& vs) {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (double)d.gA[k * d.plane + p - ex(k) - (long long)ey(k) * d.pitch] + weight(k);
    double trho = 0.0, tu = 0.0, tv = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        trho = trho + f[k];
        tu = tu + (double)ex(k) * f[k];
        tv = tv + (double)ey(k) * f[k];
    }
    rho = trho;
    us = tu / trho;
    vs = tv / trho;
}

// Fused path: the rhs with u* evaluated at each box node from the pulled
// distributions (no separate u* pass), clearing the spread accumulators of
// the band nodes it meets (every listed node lies in its claimer's box).
__device__ __forceinline__ void ibm_rhs_fused_seg(const DevState& d, const int s, const int lane) {
    const int nb = d.band_n[0];
    const int i1 = d.box[4 * s], i2 = d.box[4 * s + 1], j1 = d.box[4 * s + 2], j2 = d.box[4 * s + 3];
    double bu = 0.0, bv = 0.0;
    for (int slot = lane; slot < BOX_SLOTS; slot += 32) {
        const int a = slot / 6, c = slot % 6;
        const int i = i1 + a, j = j1 + c;
        int bi = -1;
        if (i <= i2 && j <= j2) {
            const long long p = pidx(d, i - 1, j - 1);
            const int bm = d.band_map[p];
            bi = (bm <= -2) ? -(bm + 2) : -1;
            if (bi >= nb) bi = -1;
            if (bi < 0) {
                set_status(d, ST_BAND_OVERFLOW);
            } else {
                double f[9], rho, us, vs;
                pulled_moments(d, p, f, rho, us, vs);
                reinterpret_cast<unsigned long long*>(d.band_du)[bi] = 0ull;
                reinterpret_cast<unsigned long long*>(d.band_dv)[bi] = 0ull;
                const double wv = d.kx[6 * s + a] * d.ky[6 * s + c];
                bu = bu + wv * us;
                bv = bv + wv * vs;
            }
        }
        d.pb[s * BOX_SLOTS + slot] = bi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        bu += __shfl_xor_sync(0xffffffffu, bu, o);
        bv += __shfl_xor_sync(0xffffffffu, bv, o);
    }
    if (lane == 0) {
        const int w = d.seg_wing[s];
        const WingMotion m = d.wm[w];
        const int p = d.wing_pstart[w] + (s - d.wing_sstart[w]);
        double sn, cs;
        sincos(m.angle, &sn, &cs);
        const double xs = d.xb0[p + 1] + d.xb0[p], ys = d.yb0[p + 1] + d.yb0[p];
        const double ub = d.uu * (-(m.omega * sn * 0.5 * xs) + m.omega * cs * 0.5 * ys + m.sau) + m.extra_v;
        const double vb = d.uu * (-(m.omega * cs * 0.5 * xs) - m.omega * sn * 0.5 * ys + m.sbv);
        d.rx[s] = ub - bu;
        d.ry[s] = vb - bv;
        d.qx[s] = ub - bu;   // kept for the residual diagnostic
        d.qy[s] = vb - bv;
    }
}
__device__ __forceinline__ void ibm_rhs_fused_body(const DevState& d, const int bid_) {
    const int stride = rhs_grid(d) * 4;   // warps of the grid
    for (int s = (bid_ * 128 + threadIdx.x) >> 5; s < d.nseg; s += stride) ibm_rhs_fused_seg(d, s, threadIdx.x & 31);
}
// the substitution after it may be scheduled at once (its block holds much
// shared memory and so finds an SM while this kernel runs)
__global__ void ibm_rhs_fused_kernel(DevState d) {
    pdl_release();
    ibm_rhs_fused_body(d, blockIdx.x);
}
__global__ void ibm_rhs_fused_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_rhs_fused_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// G(a, c) = Sx(a, c) Sy(a, c), the delta kernel being separable.
__device__ inline double gram(const DevState& d, int a, int c) {
    const int ai1 = d.box[4 * a], ai2 = d.box[4 * a + 1], aj1 = d.box[4 * a + 2], aj2 = d.box[4 * a + 3];
    const int ci1 = d.box[4 * c], ci2 = d.box[4 * c + 1], cj1 = d.box[4 * c + 2], cj2 = d.box[4 * c + 3];
    double sx = 0.0, sy = 0.0;
    for (int i = max(ai1, ci1); i <= min(ai2, ci2); ++i) sx = sx + d.kx[6 * a + i - ai1] * d.kx[6 * c + i - ci1];
    for (int j = max(aj1, cj1); j <= min(aj2, cj2); ++j) sy = sy + d.ky[6 * a + j - aj1] * d.ky[6 * c + j - cj1];
    return sx * sy;
}

// Banded G per wing in RCM order (layout of ibm_wing_storage): row p of
// wing w starts at lband[lofs_w + (p + 1) * ld]; entry dd holds G(p, p - dd).
// Every slot of the storage is written, zero zones included.
__device__ __forceinline__ void ibm_assemble_kernel_body(const DevState& d, const int bid_) {
    const long long total = d.lband_total, stride = (long long)assemble_grid(d) * 256;
    for (long long t = bid_ * 256LL + threadIdx.x; t < total; t += stride) {
        int w = 0;
        while (w + 1 < d.wing_count && t >= d.wing_lofs[w + 1]) ++w;
        const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], ld = ibm_ld(bw), s0 = d.wing_sstart[w];
        const long long r = t - d.wing_lofs[w];
        const int p = (int)(r / ld) - 1, dd = (int)(r % ld), q = p - dd;
        d.lband[t] = (p >= 0 && p < nw && q >= 0 && dd <= bw) ? gram(d, d.perm[s0 + p], d.perm[s0 + q]) : 0.0;
    }
}
__global__ void ibm_assemble_kernel(DevState d) { ibm_assemble_kernel_body(d, blockIdx.x); }
__global__ void ibm_assemble_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_assemble_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// blocks of the finish and closing kernels (as ibm_finish_blocks)
__device__ __forceinline__ int ibm_finish_blocks_dev(const DevState& d) {
    return (int)max(1LL, ((long long)d.band_cap + FINISH_THREADS - 1) / FINISH_THREADS);
}

// Fixed-point exponent shared by the spread and the finish kernels: every
// contribution is below 2^(62 - 10) in magnitude after scaling, so sums of up
// to 1024 of them cannot overflow.
__device__ inline int spread_exponent(const DevState& d) {
    double ym = 0.0;
    for (int w = 0; w < 2 * d.wing_count; ++w) ym = fmax(ym, d.ymax[w]);
    int e2 = 0;
    frexp(ym > 0.0 ? 1024.0 * ym : 1.0, &e2);
    return 62 - e2;
}

// du = X^T y: every (segment, slot) contribution is rounded once to a 64-bit
// fixed-point number and added with an integer atomic.
__device__ __forceinline__ void ibm_spread_kernel_body(const DevState& d, const int bid_) {
    const int n = d.nseg * BOX_SLOTS, stride = slot_grid(d) * 256;
    const int e = spread_exponent(d);
    for (int t = bid_ * 256 + threadIdx.x; t < n; t += stride) {
        const int bi = d.pb[t];
        if (bi < 0) continue;
        const int s = t / BOX_SLOTS, slot = t % BOX_SLOTS;
        const double wv = d.kx[6 * s + slot / 6] * d.ky[6 * s + slot % 6];
        atomicAdd(reinterpret_cast<unsigned long long*>(d.band_du) + bi,
                  (unsigned long long)__double2ll_rn(ldexp(wv * d.rx[s], e)));
        atomicAdd(reinterpret_cast<unsigned long long*>(d.band_dv) + bi,
                  (unsigned long long)__double2ll_rn(ldexp(wv * d.ry[s], e)));
    }
}
__global__ void ibm_spread_kernel(DevState d) {
    pdl_wait();
    ibm_spread_kernel_body(d, blockIdx.x);
}
__global__ void ibm_spread_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    ibm_spread_kernel_body(*m.ds[e], blockIdx.x - __ldg(m.boff + e));
}

// Plain path: du back to FP64, velocity correction and body force fields,
// and per-block partial sums of each wing's force and moment over the
// block's contiguous slice of the band list (each wing owns a contiguous
// range: claim order).  The FP32 path does this in its closing kernel.
__device__ __forceinline__ void ibm_finish_kernel_body(const DevState& d, const int bid_) {
    constexpr int NWARP = FINISH_THREADS / 32;
    __shared__ double red[NWARP][3];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = d.band_n[0];
    const int b = bid_ * FINISH_THREADS + tid;
    const int e = spread_exponent(d);
    double t1 = 0.0, t2 = 0.0;
    int myw = -1;
    double x0 = 0.0, y0 = 0.0;
    if (b < nb) {
        const double du = ldexp((double)reinterpret_cast<long long*>(d.band_du)[b], -e);
        const double dv = ldexp((double)reinterpret_cast<long long*>(d.band_dv)[b], -e);
        d.band_du[b] = du;
        d.band_dv[b] = dv;
        const int i = d.band_ij[2 * b], j = d.band_ij[2 * b + 1];
        const double rh = d.band_rho[b];
        t1 = 2.0 * rh * du;
        t2 = 2.0 * rh * dv;
        {
            const long long p = pidx(d, i, j);
            d.u[p] = d.band_us[b] + du;
            d.v[p] = d.band_vs[b] + dv;
            d.gfx[p] = t1;
            d.gfy[p] = t2;
        }
        myw = d.band_wing[b];
        const WingMotion m = d.wm[myw];
        const double xw = d.xc + d.wing_x_origin + (double)myw * d.wing_x_spacing + m.sa;
        const double yw = d.yc + d.wing_y_origin + m.sb;
        x0 = (d.ox + d.scale * (double)i - xw) / d.scale - m.extra_pos;
        y0 = (d.oy + d.scale * (double)j - yw) / d.scale;
    }
    const int b0 = bid_ * FINISH_THREADS;
    const int b1 = min(nb, b0 + FINISH_THREADS) - 1;
    const int wlo = b0 < nb ? d.band_wing[b0] : 0, whi = b0 < nb ? d.band_wing[b1] : -1;
    for (int w = 0; w < d.wing_count; ++w) {
        double* out = d.force_part + ((long long)bid_ * d.wing_count + w) * 3;
        if (w < wlo || w > whi) {
            if (tid < 3) out[tid] = 0.0;
            continue;
        }
        double fx = 0.0, fy = 0.0, mz = 0.0;
        if (myw == w) {
            fx = -t1;
            fy = -t2;
            mz = -x0 * t2 + y0 * t1;
        }
        for (int o = 16; o > 0; o >>= 1) {
            fx += __shfl_down_sync(0xffffffffu, fx, o);
            fy += __shfl_down_sync(0xffffffffu, fy, o);
            mz += __shfl_down_sync(0xffffffffu, mz, o);
        }
        if (lane == 0) { red[warp][0] = fx; red[warp][1] = fy; red[warp][2] = mz; }
        __syncthreads();
        if (tid < 3) {
            double v = 0.0;
            for (int k = 0; k < NWARP; ++k) v += red[k][tid];
            out[tid] = v;
        }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(FINISH_THREADS) ibm_finish_kernel(DevState d) { ibm_finish_kernel_body(d, blockIdx.x); }

// Per-wing force and moment from the block partials (in block order), the
// no-slip residual when diagnostics are on, and the force row; run by one
// block of 256 threads.  The partials come from other blocks: they are read
// through L2.
__device__ __forceinline__ void force_row_body(const DevState& d) {
    const int nblocks = (int)max(1LL, ((long long)d.band_cap + FINISH_THREADS - 1) / FINISH_THREADS);
    constexpr int STAGE = 1536;   // partial sums staged per pass (12 KB)
    __shared__ double fm[MAX_WINGS][3];
    __shared__ double red[8][2];
    __shared__ double part[STAGE];
    const int tid = threadIdx.x, W = d.wing_count;
    // partials are loaded in parallel (every load of a pass issued before
    // any is used), then added in block order
    const int per = W > 0 ? STAGE / (3 * W) : nblocks;   // blocks per pass (at least 32: W <= 16)
    double v = 0.0;
    for (int k0 = 0; k0 < nblocks; k0 += per) {
        const int nk = min(per, nblocks - k0), n = nk * 3 * W;
        const double* src = d.force_part + (long long)k0 * W * 3;
        double r[STAGE / 256];
#pragma unroll
        for (int q = 0; q < STAGE / 256; ++q) {
            const int t = tid + q * 256;
            r[q] = t < n ? __ldcg(src + t) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < STAGE / 256; ++q) {
            const int t = tid + q * 256;
            if (t < n) part[t] = r[q];
        }
        __syncthreads();
        if (tid < 3 * W)
            for (int k = 0; k < nk; ++k) v += part[k * 3 * W + tid];
        __syncthreads();
    }
    if (tid < 3 * W) fm[tid / 3][tid % 3] = v;
    if (d.diag) {
        double e2 = 0.0, r2 = 0.0;
        for (int s = tid; s < d.nseg; s += blockDim.x) {
            double ax = 0.0, ay = 0.0;
            for (int slot = 0; slot < BOX_SLOTS; ++slot) {
                const int bi = d.pb[s * BOX_SLOTS + slot];
                if (bi < 0) continue;
                const double wv = d.kx[6 * s + slot / 6] * d.ky[6 * s + slot % 6];
                ax = ax + wv * d.band_du[bi];
                ay = ay + wv * d.band_dv[bi];
            }
            e2 += (ax - d.qx[s]) * (ax - d.qx[s]) + (ay - d.qy[s]) * (ay - d.qy[s]);
            r2 += d.qx[s] * d.qx[s] + d.qy[s] * d.qy[s];
        }
        for (int o = 16; o > 0; o >>= 1) {
            e2 += __shfl_down_sync(0xffffffffu, e2, o);
            r2 += __shfl_down_sync(0xffffffffu, r2, o);
        }
        if ((tid & 31) == 0) { red[tid >> 5][0] = e2; red[tid >> 5][1] = r2; }
    }
    __syncthreads();
    // force normalisation and force row (solution.f90:330-385): thread 0
    // assembles the row in shared memory, then one thread per column writes
    // it and adds it to the running sums
    __shared__ double rowv[4 + 12 * MAX_WINGS];
    const int rl = 4 + 12 * W;
    if (tid == 0) {
        if (d.diag) {
            double a = 0.0, b = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += red[k][0]; b += red[k][1]; }
            d.ibm_resid[0] = a;
            d.ibm_resid[1] = b;
        }
        const double uu = d.uu, sc = d.scale;
        double fx = 0.0, fy = 0.0, mt = 0.0;
        rowv[0] = step_time(d);
        int col = 1;
        for (int w = 0; w < W; ++w) {
            const double Fx = 2.0 * fm[w][0] / (uu * uu * (1.0 / sc));
            const double Fy = 2.0 * fm[w][1] / (uu * uu * (1.0 / sc));
            const double Mz = -(2.0 * fm[w][2] / (uu * uu * (1.0 / (sc * sc))));
            rowv[col] = Fx; rowv[col + 1] = Fy; rowv[col + 2] = Mz;
            col += 3;
        }
        for (int w = 0; w < W; ++w) { fx = fx + rowv[1 + 3 * w]; fy = fy + rowv[2 + 3 * w]; }
        for (int w = 0; w < W; ++w) mt = mt + rowv[3 + 3 * w];
        rowv[col] = fx; rowv[col + 1] = fy; rowv[col + 2] = mt;
        *d.sample_count += 1;
    }
    if (tid < W) {   // one thread per wing: its motion columns
        const int w = tid, col = 4 + 3 * W + 9 * w;
        const WingMotion m = d.wm[w];
        const double sc = d.scale;
        rowv[col] = add(add(add(d.wing_x_origin, mul((double)w, d.wing_x_spacing)), m.sa), m.extra_s / (1.0 / sc));
        rowv[col + 1] = m.sau; rowv[col + 2] = m.saac;
        rowv[col + 3] = add(d.wing_y_origin, m.sb);
        rowv[col + 4] = m.sbv; rowv[col + 5] = m.sbac;
        rowv[col + 6] = m.angle; rowv[col + 7] = m.omega; rowv[col + 8] = m.omgac;
    }
    if (tid < 3 * W) d.wing_fm[tid] = fm[tid / 3][tid % 3];
    __syncthreads();
    const long long ri = *d.row_index;
    double* row = (d.force_rows && ri < d.force_rows_cap) ? d.force_rows + ri * rl : nullptr;
    for (int c = tid; c < rl; c += blockDim.x) {
        if (row) row[c] = rowv[c];
        d.sum_row[c] = d.sum_row[c] + rowv[c];
    }
}
__global__ void __launch_bounds__(256) ibm_forces_kernel(DevState d) { force_row_body(d); }

__global__ void step_advance_kernel(DevState d) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *d.cycle += 1;
        *d.row_index += 1;
    }
}

// Band node re-collision in FP64 with the corrected velocity (ut, vt) and the
// body force (gx, gy) = 2 rho du (solution.f90:599-655 with
// boundary_condition.f90:1645-1659); f holds the pulled distributions.
template <bool FIELDS>
__device__ __forceinline__ void band_recollide(const DevState& d, long long p, const double f[9], double rt, double ut,
                                               double vt, double gx, double gy) {
    double temp[9], temp1[9], fp[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) sum = sum + (double)mrt_m(r, q) * f[q];
        temp1[r] = sum;
    }
    const double* s = d.s;
    temp[0] = 0.0;
    temp[1] = -(2.0 * rt) + 3.0 * (rt * ut * rt * ut + rt * vt * rt * vt);
    temp[2] = rt - 3.0 * (rt * ut * rt * ut + rt * vt * rt * vt);
    temp[3] = 0.0;
    temp[4] = -(rt * ut);
    temp[5] = 0.0;
    temp[6] = -(rt * vt);
    temp[7] = (rt * ut * rt * ut - rt * vt * rt * vt);
    temp[8] = (rt * ut * rt * vt);
    fp[0] = 0.0;
    fp[1] = 6.0 * (1.0 - 0.5 * s[1]) * (ut * gx + vt * gy);
    fp[2] = -(6.0 * (1.0 - 0.5 * s[2]) * (ut * gx + vt * gy));
    fp[3] = gx;
    fp[4] = -((1.0 - 0.5 * s[4]) * gx);
    fp[5] = gy;
    fp[6] = -((1.0 - 0.5 * s[6]) * gy);
    fp[7] = 2.0 * (1.0 - 0.5 * s[7]) * (ut * gx - vt * gy);
    fp[8] = (1.0 - 0.5 * s[8]) * (ut * gy + vt * gx);
#pragma unroll
    for (int k = 0; k < 9; ++k) temp[k] = temp1[k] + (temp[k] - temp1[k]) * s[k] + fp[k];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) sum = sum + d.minv[r * 9 + q] * temp[q];
        d.gB[r * d.plane + p] = (float)(sum - weight(r));
    }
    if (FIELDS && d.fo_rho) {
        d.fo_rho[p] = rt;
        d.fo_u[p] = ut;
        d.fo_v[p] = vt;
    }
}

// Fused path, after the spread, one thread per band node: du back to FP64,
// rho and u* from the pulled distributions (the values the rhs used), the
// node's re-collision, and the block's partial force and moment sums per
// wing (as ibm_finish_kernel).  The last block to finish (a device-wide
// counter per episode) reduces the partials in block order, writes the
// force row and sums (force_row_body) and advances the cycle counter, so
// the chain ends in this one kernel.
// Virtual block vb: band nodes vb * 256 .. vb * 256 + 255 and their partial
// sums (the partition of ibm_finish_kernel whatever the grid).
template <bool FIELDS>
__device__ __forceinline__ void ibm_close_vblock(const DevState& d, const int bid_) {
    constexpr int NWARP = FINISH_THREADS / 32;
    __shared__ double red[NWARP][3];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = d.band_n[0];
    const int b = bid_ * FINISH_THREADS + tid;
    const int e = spread_exponent(d);
    double t1 = 0.0, t2 = 0.0;
    int myw = -1;
    double x0 = 0.0, y0 = 0.0;
    if (b < nb) {
        const double du = ldexp((double)reinterpret_cast<long long*>(d.band_du)[b], -e);
        const double dv = ldexp((double)reinterpret_cast<long long*>(d.band_dv)[b], -e);
        d.band_du[b] = du;
        d.band_dv[b] = dv;
        const int i = d.band_ij[2 * b], j = d.band_ij[2 * b + 1];
        const long long p = pidx(d, i, j);
        double f[9], rh, us, vs;
        pulled_moments(d, p, f, rh, us, vs);
        t1 = 2.0 * rh * du;
        t2 = 2.0 * rh * dv;
        if (i != 0 && j != 0 && i != d.nx - 1 && j != d.ny - 1) band_recollide<FIELDS>(d, p, f, rh, us + du, vs + dv, t1, t2);
        myw = d.band_wing[b];
        const WingMotion m = d.wm[myw];
        const double xw = d.xc + d.wing_x_origin + (double)myw * d.wing_x_spacing + m.sa;
        const double yw = d.yc + d.wing_y_origin + m.sb;
        x0 = (d.ox + d.scale * (double)i - xw) / d.scale - m.extra_pos;
        y0 = (d.oy + d.scale * (double)j - yw) / d.scale;
    }
    const int b0 = bid_ * FINISH_THREADS;
    const int b1 = min(nb, b0 + FINISH_THREADS) - 1;
    const int wlo = b0 < nb ? d.band_wing[b0] : 0, whi = b0 < nb ? d.band_wing[b1] : -1;
    for (int w = 0; w < d.wing_count; ++w) {
        double* out = d.force_part + ((long long)bid_ * d.wing_count + w) * 3;
        if (w < wlo || w > whi) {
            if (tid < 3) out[tid] = 0.0;
            continue;
        }
        double fx = 0.0, fy = 0.0, mz = 0.0;
        if (myw == w) {
            fx = -t1;
            fy = -t2;
            mz = -x0 * t2 + y0 * t1;
        }
        for (int o = 16; o > 0; o >>= 1) {
            fx += __shfl_down_sync(0xffffffffu, fx, o);
            fy += __shfl_down_sync(0xffffffffu, fy, o);
            mz += __shfl_down_sync(0xffffffffu, mz, o);
        }
        if (lane == 0) { red[warp][0] = fx; red[warp][1] = fy; red[warp][2] = mz; }
        __syncthreads();
        if (tid < 3) {
            double v = 0.0;
            for (int k = 0; k < NWARP; ++k) v += red[k][tid];
            out[tid] = v;
        }
        __syncthreads();
    }
}
// A block takes virtual blocks bid, bid + grid, ... (one alone, slot_items
// in packed launches).
__host__ __device__ inline int close_grid(const DevState& d) {
    const int nvb = (int)(d.band_cap > 0 ? (d.band_cap + FINISH_THREADS - 1) / FINISH_THREADS : 1);
    return (nvb + d.slot_items - 1) / d.slot_items;
}
template <bool FIELDS>
__device__ __forceinline__ void ibm_close_body(const DevState& d, const int bid_) {
    __shared__ int last;
    const int tid = threadIdx.x, grid = close_grid(d), nvb = ibm_finish_blocks_dev(d);
    for (int vb = bid_; vb < nvb; vb += grid) ibm_close_vblock<FIELDS>(d, vb);
    // the last block of the episode closes the step
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(d.fin_count, 1) == grid - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    force_row_body(d);
    __syncthreads();
    if (tid == 0) {
        *d.fin_count = 0;
        *d.cycle += 1;
        *d.row_index += 1;
    }
}
template <bool FIELDS>
__global__ void __launch_bounds__(FINISH_THREADS) ibm_close_kernel(DevState d) {
    pdl_wait();
    ibm_close_body<FIELDS>(d, blockIdx.x);
}
__global__ void __launch_bounds__(FINISH_THREADS) ibm_close_kernel_multi(MultiArgs m) {
    const int e = multi_episode(m, blockIdx.x);
    const DevState& d = *m.ds[e];
    if (d.write_fields)
        ibm_close_body<true>(d, blockIdx.x - __ldg(m.boff + e));
    else
        ibm_close_body<false>(d, blockIdx.x - __ldg(m.boff + e));
}

// ------------------------------------------------------------ host side
static inline int blocks(long long n, int t) { return (int)std::max<long long>(1, (n + t - 1) / t); }

int ibm_finish_blocks(const DevState& d) { return blocks(d.band_cap, FINISH_THREADS); }

bool is_geometry_multi_kernel(const void* func) {
    for (const void* k : {reinterpret_cast<const void*>(ibm_geometry_kernel_multi),
                          reinterpret_cast<const void*>(ibm_claim_kernel_multi),
                          reinterpret_cast<const void*>(ibm_count_kernel_multi),
                          reinterpret_cast<const void*>(ibm_scan_kernel_multi),
                          reinterpret_cast<const void*>(ibm_list_kernel_multi),
                          reinterpret_cast<const void*>(ibm_assemble_kernel_multi)})
        if (func == k) return true;
    return is_factor_multi_kernel(func);
}

bool is_geometry_kernel(const void* func) {
    for (const void* k : {reinterpret_cast<const void*>(ibm_geometry_kernel), reinterpret_cast<const void*>(ibm_claim_kernel),
                          reinterpret_cast<const void*>(ibm_count_kernel), reinterpret_cast<const void*>(ibm_scan_kernel),
                          reinterpret_cast<const void*>(ibm_list_kernel), reinterpret_cast<const void*>(ibm_assemble_kernel)})
        if (func == k) return true;
    return is_factor_kernel(func);
}

void launch_ibm_band(const DevState& d, cudaStream_t st, cudaEvent_t geometry_done) {
    ibm_geometry_kernel<<<geometry_grid(d), 128, 0, st>>>(d);
    if (geometry_done) cudaEventRecord(geometry_done, st);
    ibm_claim_kernel<<<slot_grid(d), 256, 0, st>>>(d);
    ibm_count_kernel<<<blocks(32LL * d.nseg, 128), 128, 0, st>>>(d);
    ibm_scan_kernel<<<1, 1024, 0, st>>>(d);
    ibm_list_kernel<<<blocks(32LL * d.nseg, 128), 128, 0, st>>>(d);
}

void launch_ibm_factor(const DevState& d, size_t factor_smem, cudaStream_t st) {
    ibm_assemble_kernel<<<assemble_grid(d), 256, 0, st>>>(d);
    launch_ibm_factor_blocks(d, factor_smem, st);
}

void launch_ibm_rhs(const DevState& d, bool fused, cudaStream_t st) {
    if (fused) {
        ibm_rhs_fused_kernel<<<rhs_grid(d), 128, 0, st>>>(d);
        return;
    }
    ibm_ustar_kernel<<<blocks(d.band_cap, 128), 128, 0, st>>>(d);
    ibm_rhs_kernel<<<blocks(32LL * d.nseg, 128), 128, 0, st>>>(d);
}

void launch_ibm_solve(const DevState& d, bool fused, bool fields, cudaStream_t st, bool chained) {
    launch_ibm_substitution(d, (size_t)d.solve_smem, st, chained);
    launch_chained(chained, ibm_spread_kernel, slot_grid(d), 256, 0, st, d);
    const int nbk = ibm_finish_blocks(d);
    if (fused) {
        if (fields)
            launch_chained(chained, ibm_close_kernel<true>, close_grid(d), FINISH_THREADS, 0, st, d);
        else
            launch_chained(chained, ibm_close_kernel<false>, close_grid(d), FINISH_THREADS, 0, st, d);
        return;
    }
    ibm_finish_kernel<<<nbk, FINISH_THREADS, 0, st>>>(d);
    ibm_forces_kernel<<<1, 256, 0, st>>>(d);
}

void launch_step_advance(const DevState& d, cudaStream_t st) { step_advance_kernel<<<1, 32, 0, st>>>(d); }

// ------------------------------------------------------------ packed launches
// (fused path: u* in the rhs from the pulled distributions; the closing
// kernel re-collides the band nodes, writes the force row and advances the
// cycle)
int multi_blocks_ibm(MultiKernel k, const DevState& d) {
    switch (k) {
    case MK_GEOMETRY: return geometry_grid(d);
    case MK_CLAIM: return slot_grid(d);
    case MK_COUNT: return blocks(32LL * d.nseg, 128);
    case MK_SCAN: return 1;
    case MK_LIST: return blocks(32LL * d.nseg, 128);
    case MK_ASSEMBLE: return assemble_grid(d);
    case MK_RHS: return rhs_grid(d);
    case MK_SPREAD: return slot_grid(d);
    case MK_FINISH: return close_grid(d);
    default: return -1;
    }
}

bool launch_multi_ibm(MultiKernel k, const MultiArgs& m, int nb, cudaStream_t st) {
    switch (k) {
    case MK_GEOMETRY: ibm_geometry_kernel_multi<<<nb, 128, 0, st>>>(m); return true;
    case MK_CLAIM: ibm_claim_kernel_multi<<<nb, 256, 0, st>>>(m); return true;
    case MK_COUNT: ibm_count_kernel_multi<<<nb, 128, 0, st>>>(m); return true;
    case MK_SCAN: ibm_scan_kernel_multi<<<nb, 1024, 0, st>>>(m); return true;
    case MK_LIST: ibm_list_kernel_multi<<<nb, 128, 0, st>>>(m); return true;
    case MK_ASSEMBLE: ibm_assemble_kernel_multi<<<nb, 256, 0, st>>>(m); return true;
    case MK_RHS: ibm_rhs_fused_kernel_multi<<<nb, 128, 0, st>>>(m); return true;
    case MK_SPREAD: ibm_spread_kernel_multi<<<nb, 256, 0, st>>>(m); return true;
    case MK_FINISH: ibm_close_kernel_multi<<<nb, FINISH_THREADS, 0, st>>>(m); return true;
    default: return false;
    }
}

}  // namespace lbm
