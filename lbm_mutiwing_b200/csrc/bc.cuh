// Far-field boundary condition (boundary_condition1, the live part of
// boundary_condition.f90:288-858) for both storage paths.
//
// Sequential CPU semantics of the reference, evaluated in parallel:
//  * left/right columns, j = 2..Ny-1: a LODI characteristic update of
//    rho, u, v (:413-441 left, :495-521 right) from the column's own moments
//    and one-sided x-differences of the two interior neighbours;
//  * top/bottom rows, every i: rho copied from the row inside, u = v = 0
//    (:655-661, :782-788) -- the rows' own LODI update and the corner
//    precompute are overwritten before use and are not evaluated;
//  * every border node: f = M^-1 [ m_eq(edge) + (I - S)(M f0(nbr) - m_eq(nbr)) ]
//    with m_eq built from j^2/rho (:443-481, :524-565, :681-716, :808-843).
// Edge order left -> right -> top -> bottom matters only at the corners of the
// top and bottom rows, whose inside neighbours are left/right column nodes;
// those threads recompute the column's LODI update themselves.
// The column's own moments are those physical_variables computed from the
// border f0, which streaming never writes (solution.f90:450-466, 510-554).
#pragma once
#include "lbm_common.cuh"

namespace lbm {

struct Mom {
    double r, u, v;
};

__device__ inline double bc_cs() {
    // cs = sqrt(3.0)/3.0d0 with a REAL(4) literal under the sqrt (:303)
    return (double)sqrtf(3.0f) / 3.0;
}

// Border f0 of node (i, j) from the plain path's f0 planes or the fused
// path's edge store.
template <class Acc>
__device__ inline Mom border_moments(const Acc& a, int i, int j) {
    double trho = 0.0, tu = 0.0, tv = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double t = a.f0(i, j, k);
        trho = trho + t;
        tu = tu + (double)ex(k) * t;
        tv = tv + (double)ey(k) * t;
    }
    return Mom{trho, tu / trho, tv / trho};
}

template <class Acc>
__device__ inline Mom lodi_left(const Acc& a, int j) {
    const double cs = bc_cs();
    Mom b = border_moments(a, 0, j);
    Mom m1 = a.moments(1, j), m2 = a.moments(2, j);
    double rhox = (-(3.0 * b.r) + 4.0 * m1.r - m2.r) * 0.5;
    double ux = (-(3.0 * b.u) + 4.0 * m1.u - m2.u) * 0.5;
    double vx = (-(3.0 * b.v) + 4.0 * m1.v - m2.v) * 0.5;
    double lx1 = (b.u - cs) * (cs * cs * rhox - cs * b.r * ux);
    double lx2 = (b.u < 0.0) ? b.u * vx : 0.0;
    double lx3 = 0.0;
    Mom o;
    o.r = b.r - (lx1 + lx3) * 1.5;
    o.u = b.u + (lx1 - lx3) / (2.0 * cs * o.r);
    o.v = b.v - lx2;
    return o;
}

template <class Acc>
__device__ inline Mom lodi_right(const Acc& a, int j) {
    const double cs = bc_cs();
    const int n = a.d.nx - 1;
    Mom b = border_moments(a, n, j);
    Mom m1 = a.moments(n - 1, j), m2 = a.moments(n - 2, j);
    double rhox = (3.0 * b.r - 4.0 * m1.r + m2.r) * 0.5;
    double ux = (3.0 * b.u - 4.0 * m1.u + m2.u) * 0.5;
    double vx = (3.0 * b.v - 4.0 * m1.v + m2.v) * 0.5;
    double lx1 = 0.0;
    double lx2 = (b.u >= 0.0) ? b.u * vx : 0.0;
    double lx3 = (b.u + cs) * (cs * cs * rhox + cs * b.r * ux);
    Mom o;
    o.r = b.r - (lx1 + lx3) * 1.5;
    o.u = b.u + (lx1 - lx3) / (2.0 * cs * o.r);
    o.v = b.v - lx2;
    return o;
}

__device__ inline void meq_bc(double rh, double uu, double vv, double* t) {
    double jx = rh * uu, jy = rh * vv;
    t[0] = rh;
    t[1] = -(2.0 * rh) + 3.0 * (jx * jx + jy * jy) / rh;
    t[2] = rh - 3.0 * (jx * jx + jy * jy) / rh;
    t[3] = jx;
    t[4] = -jx;
    t[5] = jy;
    t[6] = -jy;
    t[7] = (jx * jx - jy * jy) / rh;
    t[8] = (jx * jy) / rh;
}

// f(edge) from the edge state and the inside neighbour (matmulvoc order).
template <class Acc>
__device__ inline void edge_f(const Acc& a, int ie, int je, Mom e, int in, int jn, Mom nb) {
    const DevState& d = a.d;
    double t1[9], t2[9], f0n[9], t3[9], out[9];
    meq_bc(e.r, e.u, e.v, t1);
    meq_bc(nb.r, nb.u, nb.v, t2);
#pragma unroll
    for (int k = 0; k < 9; ++k) f0n[k] = a.f0(in, jn, k);
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) sum = sum + (double)mrt_m(r, q) * f0n[q];
        t3[r] = sum;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) t3[k] = t1[k] + (1.0 - d.s[k]) * (t3[k] - t2[k]);
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) sum = sum + d.minv[r * 9 + q] * t3[q];
        out[r] = sum;
    }
    a.write_f(ie, je, out);
    a.write_fields(ie, je, e);
}

// One thread per border node: [left j=1..ny-2][right j=1..ny-2][top i][bottom i].
template <class Acc>
__global__ void outer_bc_kernel(Acc a) {
    const DevState& d = a.d;
    const int nl = d.ny - 2;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nl) {
        int j = 1 + t;
        Mom e = lodi_left(a, j);
        edge_f(a, 0, j, e, 1, j, a.moments(1, j));
        return;
    }
    t -= nl;
    if (t < nl) {
        int j = 1 + t;
        Mom e = lodi_right(a, j);
        edge_f(a, d.nx - 1, j, e, d.nx - 2, j, a.moments(d.nx - 2, j));
        return;
    }
    t -= nl;
    if (t < 2 * d.nx) {
        const bool top = t < d.nx;
        const int i = top ? t : t - d.nx;
        const int je = top ? d.ny - 1 : 0;
        const int jn = top ? d.ny - 2 : 1;
        Mom nb = (i == 0) ? lodi_left(a, jn) : (i == d.nx - 1) ? lodi_right(a, jn) : a.moments(i, jn);
        Mom e{nb.r, 0.0, 0.0};
        edge_f(a, i, je, e, i, jn, nb);
    }
}

}  // namespace lbm
