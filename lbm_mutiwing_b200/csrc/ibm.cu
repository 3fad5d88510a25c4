// Implicit velocity-correction immersed boundary step (bc_num = 4), on the
// device in FP64, one thread block per simulation.
//
// Reference: move_boundary (airfoil.f90:244-338) and immersed_boundary_Wu
// (boundary_condition.f90:1512-1736), with the motion lookup of mode.f90.
//
// The reference builds dense delta matrices xx1 (segments x band) and
// xx2 = xx1^T diag(arc_l), forms A = xx1 xx2 with cublasDgemm and solves
// A c = ub - xx1 u* with cuSOLVER LU.  Because A = X X^T D and the spread is
// du = X^T D c, the arc lengths cancel: du = X^T y with (X X^T) y = ub - X u*.
// Here X is kept sparse (each segment's 6 x 6 support box), G = X X^T is
// assembled in a per-wing banded layout after a reverse Cuthill-McKee
// ordering fixed at set-up (rigid wings keep their pairwise distances), and
// factored by a banded Cholesky, one warp per wing.
//
// Determinism: the band list is built in the reference's first-claimant
// order (segment, then i, then j) from an atomicMin claim pass plus a prefix
// sum; the spread sums each band node's contributions in ascending segment
// order; force sums use a fixed reduction tree.  Results are identical from
// run to run.
//
// Built with -fmad=false: the box scan compares node distances against 2.5
// spacings with the reference's rounding.
#include <cstdio>

#include "lbm_kernels.h"

namespace lbm {

constexpr int IBM_THREADS = 512;
constexpr int IBM_WARPS = IBM_THREADS / 32;
constexpr int MAX_WINGS = 16;

int ibm_threads() { return IBM_THREADS; }

struct IbmShared {
    WingMotion wm[MAX_WINGS];
    double xbase[MAX_WINGS], ybase[MAX_WINGS];
    int scan[IBM_THREADS];
    double red[IBM_WARPS][MAX_WINGS][3];
    double fm[MAX_WINGS][3];
    int nb;
};

__device__ inline void set_status(const DevState& d, int bit) { atomicOr(d.status, bit); }

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

// mode + apply_motion_row for wing w at the current cycle (mode.f90:451-471,
// 180-218, 414-449).
__device__ void wing_motion(const DevState& d, int w, double time, WingMotion& m) {
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
    m.angle = v[0]; m.omega = v[1]; m.omgac = v[2];
    m.sa = v[3]; m.sau = v[4]; m.saac = v[5];
    m.sb = v[6]; m.sbv = v[7]; m.sbac = v[8];
    if (d.motion_source == 1) {
        m.sa = m.sa - (d.wing_x_origin + (double)w * d.wing_x_spacing);
        m.sb = m.sb - d.wing_y_origin;
    }
}

__device__ inline int wing_of_point(const DevState& d, int p) {
    int w = 0;
    while (w + 1 < d.wing_count && p >= d.wing_pstart[w + 1]) ++w;
    return w;
}

// ------------------------------------------------------------------ phases
// move_boundary: motion, markers, band rebuild.
__device__ void phase_band(const DevState& d, IbmShared& sh) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long cycle = *d.cycle;
    const double time = (double)(cycle - 1) * (d.scale * d.uu);
    if (tid < d.wing_count) {
        WingMotion m;
        wing_motion(d, tid, time, m);
        // update_body_extra_from_rel (mode.f90:473-495); relative motion is
        // zero unless rigid-body dynamics are enabled.
        double av = 0.0, as = 0.0, ap = 0.0;
        for (int w = 0; w <= tid; ++w) { ap = ap + d.rel_pos[w]; }
        m.extra_v = av; m.extra_s = as; m.extra_pos = ap;
        sh.wm[tid] = m;
        d.wm[tid] = m;
    }
    if (tid == 0 && d.motion_source == 1 && d.step_rows <= 0) set_status(d, ST_MOTION);
    __syncthreads();
    // markers (airfoil.f90:254-265)
    for (int p = tid; p < d.npts; p += nt) {
        int w = wing_of_point(d, p);
        const WingMotion& m = sh.wm[w];
        double ca = cos(m.angle), sn = sin(m.angle);
        d.xb1[p] = ca * d.xb0[p] + sn * d.yb0[p] + d.wing_x_origin + (double)w * d.wing_x_spacing + m.sa +
                   d.xc + m.extra_s / (1.0 / d.scale) - (double)d.movenum * d.scale;
        d.yb1[p] = -(sn * d.xb0[p]) + ca * d.yb0[p] + d.wing_y_origin + m.sb + d.yc;
    }
    // clear the previous band (airfoil.f90:276-284)
    const int nb_old = d.band_n[0];
    for (int b = tid; b < nb_old; b += nt) {
        int i = d.band_ij[2 * b], j = d.band_ij[2 * b + 1];
        long long p = pidx(d, i, j);
        d.band_map[p] = BAND_EMPTY;
        if (d.precision == 0) { d.gfx[p] = 0.0; d.gfy[p] = 0.0; }
    }
    __syncthreads();
    // midpoints (airfoil.f90:267-270) and support boxes (:288-321)
    for (int s = tid; s < d.nseg; s += nt) {
        int w = d.seg_wing[s];
        int p = d.wing_pstart[w] + (s - d.wing_sstart[w]);
        double x2 = 0.5 * (d.xb1[p + 1] + d.xb1[p]);
        double y2 = 0.5 * (d.yb1[p + 1] + d.yb1[p]);
        d.xb2[s] = x2;
        d.yb2[s] = y2;
        int i1 = (int)((x2 - d.ox) / d.scale + 1.0);
        for (int i = i1; i >= 1; --i) {
            double t = d.ox + (double)(i - 1) * d.scale;
            if (fabs((t - x2) / d.scale) > 2.5) { i1 = i + 1; break; }
        }
        int i2 = (int)((x2 - d.ox) / d.scale + 1.0);
        for (int i = i2; i <= d.nx; ++i) {
            double t = d.ox + (double)(i - 1) * d.scale;
            if (fabs((t - x2) / d.scale) > 2.5) { i2 = i - 1; break; }
        }
        int j2 = (int)((y2 - d.oy) / d.scale + 1.0);
        for (int i = j2; i <= d.ny; ++i) {
            double t = d.oy + (double)(i - 1) * d.scale;
            if (fabs((t - y2) / d.scale) > 2.5) { j2 = i - 1; break; }
        }
        int j1 = (int)((y2 - d.oy) / d.scale + 1.0);
        for (int i = j1; i >= 1; --i) {
            double t = d.oy + (double)(i - 1) * d.scale;
            if (fabs((t - y2) / d.scale) > 2.5) { j1 = i + 1; break; }
        }
        if (i1 < 1 || j1 < 1 || i2 > d.nx || j2 > d.ny || i2 - i1 > 5 || j2 - j1 > 5 || i2 < i1 || j2 < j1) {
            set_status(d, ST_BOX_OUTSIDE);
            i1 = 1; i2 = 0; j1 = 1; j2 = 0;   // empty box
        }
        d.box[4 * s] = i1; d.box[4 * s + 1] = i2; d.box[4 * s + 2] = j1; d.box[4 * s + 3] = j2;
    }
    __syncthreads();
    // claim: lowest segment index wins (airfoil.f90:322-333)
    for (int t = tid; t < d.nseg * BOX_SLOTS; t += nt) {
        int s = t / BOX_SLOTS, slot = t % BOX_SLOTS;
        int i = d.box[4 * s] + slot / 6, j = d.box[4 * s + 2] + slot % 6;
        if (i <= d.box[4 * s + 1] && j <= d.box[4 * s + 3]) atomicMin(&d.band_map[pidx(d, i - 1, j - 1)], s);
    }
    __syncthreads();
    for (int s = tid; s < d.nseg; s += nt) {
        int c = 0;
        for (int i = d.box[4 * s]; i <= d.box[4 * s + 1]; ++i)
            for (int j = d.box[4 * s + 2]; j <= d.box[4 * s + 3]; ++j)
                c += (d.band_map[pidx(d, i - 1, j - 1)] == s);
        d.claim_cnt[s] = c;
    }
    __syncthreads();
    // exclusive prefix sum over segments
    const int per = (d.nseg + nt - 1) / nt;
    int lsum = 0;
    for (int s = tid * per; s < min(d.nseg, (tid + 1) * per); ++s) lsum += d.claim_cnt[s];
    sh.scan[tid] = lsum;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        int v = tid >= off ? sh.scan[tid - off] : 0;
        __syncthreads();
        sh.scan[tid] += v;
        __syncthreads();
    }
    int run = sh.scan[tid] - lsum;
    for (int s = tid * per; s < min(d.nseg, (tid + 1) * per); ++s) {
        int c = d.claim_cnt[s];
        d.claim_cnt[s] = run;
        run += c;
    }
    if (tid == nt - 1) {
        int nb = sh.scan[nt - 1];
        if (nb > d.band_cap) { set_status(d, ST_BAND_OVERFLOW); nb = d.band_cap; }
        sh.nb = nb;
    }
    __syncthreads();
    const int nb = sh.nb;
    for (int s = tid; s < d.nseg; s += nt) {
        int b = d.claim_cnt[s];
        int w = d.seg_wing[s];
        for (int i = d.box[4 * s]; i <= d.box[4 * s + 1]; ++i)
            for (int j = d.box[4 * s + 2]; j <= d.box[4 * s + 3]; ++j)
                if (d.band_map[pidx(d, i - 1, j - 1)] == s) {
                    if (b < nb) {
                        d.band_ij[2 * b] = i - 1;
                        d.band_ij[2 * b + 1] = j - 1;
                        d.band_wing[b] = w;
                    }
                    ++b;
                }
    }
    __syncthreads();
    for (int b = tid; b < nb; b += nt) d.band_map[pidx(d, d.band_ij[2 * b], d.band_ij[2 * b + 1])] = -(b + 2);
    if (tid == 0) d.band_n[0] = nb;
    __syncthreads();
}

// u* and rho at band nodes: fields of the plain path, or the moments of the
// pulled distributions of the fused path.
template <bool FUSED>
__device__ void phase_ustar(const DevState& d, int nb) {
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int i = d.band_ij[2 * b], j = d.band_ij[2 * b + 1];
        const long long p = pidx(d, i, j);
        if (!FUSED) {
            d.band_rho[b] = d.rho[p];
            d.band_us[b] = d.u[p];
            d.band_vs[b] = d.v[p];
        } else {
            double trho = 0.0, tu = 0.0, tv = 0.0;
            const bool border = i == 0 || j == 0 || i == d.nx - 1 || j == d.ny - 1;
            const long long per = 2LL * d.ny + 2LL * d.nx;
            for (int k = 0; k < 9; ++k) {
                double t;
                if (border) {
                    long long e = (i == 0) ? j : (i == d.nx - 1) ? d.ny + j : (j == 0) ? 2LL * d.ny + i
                                                                                        : 2LL * d.ny + d.nx + i;
                    t = d.edge_f0[k * per + e];
                } else {
                    t = (double)d.gA[k * d.plane + p - ex(k) - (long long)ey(k) * d.pitch] + weight(k);
                }
                trho = trho + t;
                tu = tu + (double)ex(k) * t;
                tv = tv + (double)ey(k) * t;
            }
            d.band_rho[b] = trho;
            d.band_us[b] = tu / trho;
            d.band_vs[b] = tv / trho;
        }
    }
}

// Delta weights per (segment, slot), band index per slot, cover lists,
// right-hand sides r = ub - X u* (boundary_condition.f90:1540-1629).
__device__ void phase_weights_rhs(const DevState& d, IbmShared& sh, int nb) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int b = tid; b < nb; b += nt) d.cover_n[b] = 0;
    __syncthreads();
    for (int t = tid; t < d.nseg * BOX_SLOTS; t += nt) {
        int s = t / BOX_SLOTS, slot = t % BOX_SLOTS;
        int i = d.box[4 * s] + slot / 6, j = d.box[4 * s + 2] + slot % 6;
        double wv = 0.0;
        int bi = -1;
        if (i <= d.box[4 * s + 1] && j <= d.box[4 * s + 3]) {
            int bm = d.band_map[pidx(d, i - 1, j - 1)];
            bi = (bm <= -2) ? -(bm + 2) : -1;
            if (bi < 0 || bi >= nb) {
                bi = -1;
                set_status(d, ST_BAND_OVERFLOW);
            } else {
                double x0 = d.ox + d.scale * (double)(i - 1);
                double y0 = d.oy + d.scale * (double)(j - 1);
                double k1 = delta_phi(fabs((x0 - d.xb2[s]) / d.scale));
                double k2 = delta_phi(fabs((y0 - d.yb2[s]) / d.scale));
                wv = k1 * k2;
                int pos = atomicAdd(&d.cover_n[bi], 1);
                if (pos < MAX_COVER) d.cover_list[(long long)bi * MAX_COVER + pos] = t;
                else set_status(d, ST_COVER_OVERFLOW);
            }
        }
        d.pw[t] = wv;
        d.pb[t] = bi;
    }
    __syncthreads();
    for (int s = tid; s < d.nseg; s += nt) {
        const int w = d.seg_wing[s];
        const WingMotion& m = sh.wm[w];
        const int p = d.wing_pstart[w] + (s - d.wing_sstart[w]);
        const double sn = sin(m.angle), cs = cos(m.angle);
        const double xs = d.xb0[p + 1] + d.xb0[p], ys = d.yb0[p + 1] + d.yb0[p];
        const double ub = d.uu * (-(m.omega * sn * 0.5 * xs) + m.omega * cs * 0.5 * ys + m.sau) + m.extra_v;
        const double vb = d.uu * (-(m.omega * cs * 0.5 * xs) - m.omega * sn * 0.5 * ys + m.sbv);
        double bu = 0.0, bv = 0.0;
        for (int slot = 0; slot < BOX_SLOTS; ++slot) {
            int bi = d.pb[s * BOX_SLOTS + slot];
            if (bi < 0) continue;
            double wv = d.pw[s * BOX_SLOTS + slot];
            bu = bu + wv * d.band_us[bi];
            bv = bv + wv * d.band_vs[bi];
        }
        d.rx[s] = ub - bu;
        d.ry[s] = vb - bv;
        d.qx[s] = ub - bu;   // keep r for the residual diagnostic
        d.qy[s] = vb - bv;
    }
    __syncthreads();
}

// G(a, c) = sum over the common support of segments a and c.
__device__ inline double gram(const DevState& d, int a, int c) {
    const int ai1 = d.box[4 * a], ai2 = d.box[4 * a + 1], aj1 = d.box[4 * a + 2], aj2 = d.box[4 * a + 3];
    const int ci1 = d.box[4 * c], ci2 = d.box[4 * c + 1], cj1 = d.box[4 * c + 2], cj2 = d.box[4 * c + 3];
    const int i1 = max(ai1, ci1), i2 = min(ai2, ci2), j1 = max(aj1, cj1), j2 = min(aj2, cj2);
    double g = 0.0;
    for (int i = i1; i <= i2; ++i)
        for (int j = j1; j <= j2; ++j)
            g = g + d.pw[a * BOX_SLOTS + (i - ai1) * 6 + (j - aj1)] * d.pw[c * BOX_SLOTS + (i - ci1) * 6 + (j - cj1)];
    return g;
}

// Banded G per wing in RCM order: L[w][p][dd] holds G(p, p - dd).
__device__ void phase_assemble(const DevState& d, double* lband) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int w = 0; w < d.wing_count; ++w) {
        const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], s0 = d.wing_sstart[w];
        double* L = lband + d.wing_lofs[w];
        const int tot = nw * (bw + 1);
        for (int t = tid; t < tot; t += nt) {
            int p = t / (bw + 1), dd = t % (bw + 1), q = p - dd;
            L[t] = (q >= 0) ? gram(d, d.perm[s0 + p], d.perm[s0 + q]) : 0.0;
        }
    }
    __syncthreads();
}

// Banded Cholesky and two triangular solves for wing w, one warp.
__device__ void wing_factor_solve(const DevState& d, double* lband, int w, bool factor) {
    const int lane = threadIdx.x & 31;
    const int nw = d.wing_npts[w] - 1, bw = d.wing_bw[w], s0 = d.wing_sstart[w];
    const int ld = bw + 1;
    double* L = lband + d.wing_lofs[w];
    if (factor) {
        double maxdiag = 0.0;
        for (int p = lane; p < nw; p += 32) maxdiag = fmax(maxdiag, L[p * ld]);
        for (int o = 16; o > 0; o >>= 1) maxdiag = fmax(maxdiag, __shfl_xor_sync(0xffffffffu, maxdiag, o));
        const double floor_piv = 1e-15 * maxdiag;
        for (int k = 0; k < nw; ++k) {
            double dkk = L[k * ld];
            if (!(dkk > floor_piv)) {
                dkk = floor_piv > 0.0 ? floor_piv : 1.0;
                if (lane == 0) set_status(d, ST_PIVOT_CLAMPED);
            }
            const double lkk = sqrt(dkk);
            const int m = min(bw, nw - 1 - k);
            __syncwarp();
            for (int r = lane; r < m; r += 32) {
                const int i = k + 1 + r;
                L[i * ld + (i - k)] = L[i * ld + (i - k)] / lkk;
            }
            __syncwarp();
            if (lane == 0) L[k * ld] = lkk;
            const int P = m * (m + 1) / 2;
            for (int t = lane; t < P; t += 32) {
                int r1 = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
                while (r1 * (r1 + 1) / 2 > t) --r1;
                while ((r1 + 1) * (r1 + 2) / 2 <= t) ++r1;
                const int r2 = t - r1 * (r1 + 1) / 2;
                const int i = k + 1 + r1, j = k + 1 + r2;
                L[i * ld + (i - j)] = L[i * ld + (i - j)] - L[i * ld + (i - k)] * L[j * ld + (j - k)];
            }
            __syncwarp();
        }
    }
    // forward: L z = r (RCM order, z held in qx/qy work arrays as zx/zy)
    double* zx = d.zx + s0;
    double* zy = d.zy + s0;
    for (int p = lane; p < nw; p += 32) {
        zx[p] = d.rx[d.perm[s0 + p]];
        zy[p] = d.ry[d.perm[s0 + p]];
    }
    __syncwarp();
    for (int k = 0; k < nw; ++k) {
        const double lkk = L[k * ld];
        const double ax = zx[k] / lkk, ay = zy[k] / lkk;
        const int m = min(bw, nw - 1 - k);
        __syncwarp();
        for (int r = lane; r < m; r += 32) {
            const int i = k + 1 + r;
            const double lik = L[i * ld + (i - k)];
            zx[i] = zx[i] - lik * ax;
            zy[i] = zy[i] - lik * ay;
        }
        if (lane == 0) { zx[k] = ax; zy[k] = ay; }
        __syncwarp();
    }
    // backward: L^T y = z
    for (int k = nw - 1; k >= 0; --k) {
        const double lkk = L[k * ld];
        const double ax = zx[k] / lkk, ay = zy[k] / lkk;
        const int m = min(bw, k);
        __syncwarp();
        for (int r = lane; r < m; r += 32) {
            const int j = k - 1 - r;
            const double lkj = L[k * ld + (k - j)];
            zx[j] = zx[j] - lkj * ax;
            zy[j] = zy[j] - lkj * ay;
        }
        if (lane == 0) { zx[k] = ax; zy[k] = ay; }
        __syncwarp();
    }
    for (int p = lane; p < nw; p += 32) {
        d.rx[d.perm[s0 + p]] = zx[p];
        d.ry[d.perm[s0 + p]] = zy[p];
    }
    __syncwarp();
}

// du = X^T y, summed per band node in ascending (segment, slot) order.
__device__ void phase_spread(const DevState& d, int nb) {
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        int n = min(d.cover_n[b], MAX_COVER);
        int* lst = d.cover_list + (long long)b * MAX_COVER;
        for (int a = 1; a < n; ++a) {   // insertion sort: run-to-run deterministic order
            int v = lst[a], c = a - 1;
            while (c >= 0 && lst[c] > v) { lst[c + 1] = lst[c]; --c; }
            lst[c + 1] = v;
        }
        double sx = 0.0, sy = 0.0;
        int w0 = -1;
        bool coupled = false;
        for (int a = 0; a < n; ++a) {
            int t = lst[a], s = t / BOX_SLOTS;
            double wv = d.pw[t];
            sx = sx + wv * d.rx[s];
            sy = sy + wv * d.ry[s];
            int w = d.seg_wing[s];
            if (w0 < 0) w0 = w; else if (w != w0) coupled = true;
        }
        if (coupled) set_status(d, ST_WINGS_COUPLED);
        d.band_du[b] = sx;
        d.band_dv[b] = sy;
    }
}

// Velocity correction, body force, per-wing force and moment, force row.
template <bool FUSED>
__device__ void phase_finish(const DevState& d, IbmShared& sh, int nb) {
    const int tid = threadIdx.x, nt = blockDim.x, W = d.wing_count;
    double acc[MAX_WINGS][3];
    for (int w = 0; w < W; ++w) acc[w][0] = acc[w][1] = acc[w][2] = 0.0;
    for (int b = tid; b < nb; b += nt) {
        const int i = d.band_ij[2 * b], j = d.band_ij[2 * b + 1];
        const double rh = d.band_rho[b], du = d.band_du[b], dv = d.band_dv[b];
        const double t1 = 2.0 * rh * du, t2 = 2.0 * rh * dv;
        if (!FUSED) {
            long long p = pidx(d, i, j);
            d.u[p] = d.band_us[b] + du;
            d.v[p] = d.band_vs[b] + dv;
            d.gfx[p] = t1;
            d.gfy[p] = t2;
        }
        const int w = d.band_wing[b];
        const WingMotion& m = sh.wm[w];
        double x0 = (d.ox + d.scale * (double)i - (d.xc + d.wing_x_origin + (double)w * d.wing_x_spacing + m.sa)) / d.scale -
                    m.extra_pos;
        double y0 = (d.oy + d.scale * (double)j - (d.yc + d.wing_y_origin + m.sb)) / d.scale;
        for (int ww = 0; ww < W; ++ww) {   // register-resident accumulators
            if (ww == w) {
                acc[ww][0] = acc[ww][0] - t1;
                acc[ww][1] = acc[ww][1] - t2;
                acc[ww][2] = acc[ww][2] - x0 * t2 + y0 * t1;
            }
        }
    }
    const int lane = tid & 31, warp = tid >> 5;
    for (int w = 0; w < W; ++w)
        for (int c = 0; c < 3; ++c) {
            double v = acc[w][c];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) sh.red[warp][w][c] = v;
        }
    // no-slip residual diagnostic |X du - r|^2 and |r|^2
    double e2 = 0.0, r2 = 0.0;
    for (int s = tid; s < d.nseg; s += nt) {
        double ax = 0.0, ay = 0.0;
        for (int slot = 0; slot < BOX_SLOTS; ++slot) {
            int bi = d.pb[s * BOX_SLOTS + slot];
            if (bi < 0) continue;
            ax = ax + d.pw[s * BOX_SLOTS + slot] * d.band_du[bi];
            ay = ay + d.pw[s * BOX_SLOTS + slot] * d.band_dv[bi];
        }
        e2 += (ax - d.qx[s]) * (ax - d.qx[s]) + (ay - d.qy[s]) * (ay - d.qy[s]);
        r2 += d.qx[s] * d.qx[s] + d.qy[s] * d.qy[s];
    }
    for (int o = 16; o > 0; o >>= 1) {
        e2 += __shfl_down_sync(0xffffffffu, e2, o);
        r2 += __shfl_down_sync(0xffffffffu, r2, o);
    }
    __shared__ double res_s[IBM_WARPS][2];
    if (lane == 0) { res_s[warp][0] = e2; res_s[warp][1] = r2; }
    __syncthreads();
    if (tid < W * 3) {
        int w = tid / 3, c = tid % 3;
        double v = 0.0;
        for (int k = 0; k < (nt >> 5); ++k) v += sh.red[k][w][c];
        sh.fm[w][c] = v;
    }
    __syncthreads();
    if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (nt >> 5); ++k) { a += res_s[k][0]; b += res_s[k][1]; }
        d.ibm_resid[0] = a;
        d.ibm_resid[1] = b;
        // force normalisation and force row (solution.f90:330-385)
        const double uu = d.uu, sc = d.scale;
        const long long cycle = *d.cycle;
        const double time = (double)(cycle - 1) * (sc * uu);
        const long long ri = *d.row_index;
        const int rl = 4 + 12 * W;
        double* row = (d.force_rows && ri < d.force_rows_cap) ? d.force_rows + ri * rl : nullptr;
        double fx = 0.0, fy = 0.0, mt = 0.0;
        double rowv[4 + 12 * MAX_WINGS];
        rowv[0] = time;
        int col = 1;
        for (int w = 0; w < W; ++w) {
            double Fx = 2.0 * sh.fm[w][0] / (uu * uu * (1.0 / sc));
            double Fy = 2.0 * sh.fm[w][1] / (uu * uu * (1.0 / sc));
            double Mz = -(2.0 * sh.fm[w][2] / (uu * uu * (1.0 / (sc * sc))));
            d.wing_fm[3 * w] = sh.fm[w][0];
            d.wing_fm[3 * w + 1] = sh.fm[w][1];
            d.wing_fm[3 * w + 2] = sh.fm[w][2];
            rowv[col] = Fx; rowv[col + 1] = Fy; rowv[col + 2] = Mz;
            col += 3;
        }
        for (int w = 0; w < W; ++w) { fx = fx + rowv[1 + 3 * w]; fy = fy + rowv[2 + 3 * w]; }
        for (int w = 0; w < W; ++w) mt = mt + rowv[3 + 3 * w];
        rowv[col] = fx; rowv[col + 1] = fy; rowv[col + 2] = mt;
        col += 3;
        for (int w = 0; w < W; ++w) {
            const WingMotion& m = sh.wm[w];
            rowv[col] = d.wing_x_origin + (double)w * d.wing_x_spacing + m.sa + m.extra_s / (1.0 / sc);
            rowv[col + 1] = m.sau; rowv[col + 2] = m.saac;
            rowv[col + 3] = d.wing_y_origin + m.sb;
            rowv[col + 4] = m.sbv; rowv[col + 5] = m.sbac;
            rowv[col + 6] = m.angle; rowv[col + 7] = m.omega; rowv[col + 8] = m.omgac;
            col += 9;
        }
        for (int c = 0; c < rl; ++c) {
            if (row) row[c] = rowv[c];
            d.sum_row[c] = d.sum_row[c] + rowv[c];
        }
        *d.sample_count += 1;
    }
}

template <bool FUSED>
__device__ void phase_solve(const DevState& d, IbmShared& sh, double* lband) {
    const int nb = d.band_n[0];
    phase_ustar<FUSED>(d, nb);
    __syncthreads();
    phase_weights_rhs(d, sh, nb);
    phase_assemble(d, lband);
    const int warp = threadIdx.x >> 5;
    for (int w = warp; w < d.wing_count; w += IBM_WARPS) wing_factor_solve(d, lband, w, true);
    __syncthreads();
    phase_spread(d, nb);
    __syncthreads();
    phase_finish<FUSED>(d, sh, nb);
}

__global__ void __launch_bounds__(IBM_THREADS) ibm_band_kernel(DevState d) {
    __shared__ IbmShared sh;
    phase_band(d, sh);
}

__global__ void __launch_bounds__(IBM_THREADS) ibm_solve_plain_kernel(DevState d, int band_in_smem) {
    __shared__ IbmShared sh;
    extern __shared__ double dyn[];
    if (threadIdx.x < d.wing_count) sh.wm[threadIdx.x] = d.wm[threadIdx.x];
    __syncthreads();
    phase_solve<false>(d, sh, band_in_smem ? dyn : d.lband);
}

__global__ void __launch_bounds__(IBM_THREADS) ibm_full_fused_kernel(DevState d, int band_in_smem) {
    __shared__ IbmShared sh;
    extern __shared__ double dyn[];
    phase_band(d, sh);
    phase_solve<true>(d, sh, band_in_smem ? dyn : d.lband);
}

__global__ void step_advance_kernel(DevState d) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *d.cycle += 1;
        *d.row_index += 1;
    }
}

void launch_ibm_band(const DevState& d, cudaStream_t st) {
    ibm_band_kernel<<<1, IBM_THREADS, 0, st>>>(d);
}
void launch_ibm_solve(const DevState& d, size_t smem, bool band_in_smem, cudaStream_t st) {
    ibm_solve_plain_kernel<<<1, IBM_THREADS, smem, st>>>(d, band_in_smem ? 1 : 0);
}
void launch_ibm_full(const DevState& d, size_t smem, bool band_in_smem, cudaStream_t st) {
    ibm_full_fused_kernel<<<1, IBM_THREADS, smem, st>>>(d, band_in_smem ? 1 : 0);
}
void launch_step_advance(const DevState& d, cudaStream_t st) { step_advance_kernel<<<1, 32, 0, st>>>(d); }

cudaError_t ibm_set_smem_limit(size_t bytes) {
    cudaError_t e = cudaFuncSetAttribute(ibm_solve_plain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(ibm_full_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace lbm
