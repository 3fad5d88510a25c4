// Plain FP64 path: one kernel per reference routine, in the reference's order
// (streaming -> physical_variables -> [IBM] -> colission -> boundary), with
// full-grid FP64 fields laid out like mesh_dat (main.f90:161-179) but with a
// padded row pitch.  Built with -fmad=false so every multiply and add rounds
// separately, as in the reference's source order.
//
// Also the plain path's far-field kernel, the convergence residual, the
// lattice shift and the output fields of both paths.
#include "bc.cuh"
#include "lbm_kernels.h"

namespace lbm {

// ------------------------------------------------------------ accessors
struct PlainAcc {
    DevState d;
    __device__ double f0(int i, int j, int k) const { return d.f0[k * d.plane + pidx(d, i, j)]; }
    __device__ Mom moments(int i, int j) const {
        long long p = pidx(d, i, j);
        return Mom{d.rho[p], d.u[p], d.v[p]};
    }
    __device__ void write_f(int i, int j, const double* f) const {
        long long p = pidx(d, i, j);
#pragma unroll
        for (int k = 0; k < 9; ++k) d.f[k * d.plane + p] = f[k];
    }
    __device__ void write_fields(int i, int j, Mom m) const {
        long long p = pidx(d, i, j);
        d.rho[p] = m.r;
        d.u[p] = m.u;
        d.v[p] = m.v;
    }
};

// ------------------------------------------------------------ plain kernels
// streaming (solution.f90:440-481): f0(i,j,k) = f(i-ex, j-ey, k), interior.
__global__ void plain_stream_kernel(DevState d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx - 2 || j > d.ny - 2) return;
    long long p = pidx(d, i, j);
#pragma unroll
    for (int k = 0; k < 9; ++k) d.f0[k * d.plane + p] = d.f[k * d.plane + p - ex(k) - (long long)ey(k) * d.pitch];
}

// physical_variables (solution.f90:483-583), every node.
__global__ void plain_moments_kernel(DevState d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= d.nx || j >= d.ny) return;
    long long p = pidx(d, i, j);
    d.u0[p] = d.u[p];
    d.v0[p] = d.v[p];
    bool border = i == 0 || j == 0 || i == d.nx - 1 || j == d.ny - 1;
    double trho = 0.0, tu = 0.0, tv = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double t = d.f0[k * d.plane + p];
        if (!border) d.f[k * d.plane + p] = t;
        trho = trho + t;
        tu = tu + (double)ex(k) * t;
        tv = tv + (double)ey(k) * t;
    }
    d.rho[p] = trho;
    d.pre[p] = trho / 3.0;
    d.u[p] = tu / trho;
    d.v[p] = tv / trho;
}

// colission (solution.f90:585-669), interior, MRT with Guo forcing.
__global__ void plain_collide_kernel(DevState d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx - 2 || j > d.ny - 2) return;
    long long p = pidx(d, i, j);
    double temp[9], temp1[9], fp[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) temp[k] = d.f[k * d.plane + p];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) sum = sum + (double)mrt_m(r, q) * temp[q];
        temp1[r] = sum;
    }
    const double ut = d.u[p], vt = d.v[p], rt = d.rho[p];
    temp[0] = 0.0;
    temp[1] = -(2.0 * rt) + 3.0 * (rt * ut * rt * ut + rt * vt * rt * vt);
    temp[2] = rt - 3.0 * (rt * ut * rt * ut + rt * vt * rt * vt);
    temp[3] = 0.0;
    temp[4] = -(rt * ut);
    temp[5] = 0.0;
    temp[6] = -(rt * vt);
    temp[7] = (rt * ut * rt * ut - rt * vt * rt * vt);
    temp[8] = (rt * ut * rt * vt);
    const double gx = d.gfx[p], gy = d.gfy[p];
    const double* s = d.s;
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
        d.f[r * d.plane + p] = sum;
    }
}

// Deterministic two-pass sums for erranalysis (solution.f90:77-130):
// block b reduces a fixed row range; the second pass adds partials in order.
constexpr int ERR_BLOCKS = 296;

template <bool FUSED>
__global__ void err_partial_kernel(DevState d, double* partial) {
    __shared__ double s1[256], s2[256];
    const double* u = FUSED ? d.fo_u : d.u;
    const double* v = FUSED ? d.fo_v : d.v;
    const double* u0 = FUSED ? d.fo_u0 : d.u0;
    const double* v0 = FUSED ? d.fo_v0 : d.v0;
    double a = 0.0, b = 0.0;
    const long long n_in = (long long)(d.nx - 2) * (d.ny - 2);
    for (long long t = blockIdx.x * 256LL + threadIdx.x; t < n_in; t += 256LL * gridDim.x) {
        int i = 1 + (int)(t % (d.nx - 2)), j = 1 + (int)(t / (d.nx - 2));
        long long p = pidx(d, i, j);
        double du = u[p] - u0[p], dv = v[p] - v0[p];
        a = a + du * du + dv * dv;
        b = b + u[p] * u[p] + v[p] * v[p];
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s1[threadIdx.x] += s1[threadIdx.x + w];
            s2[threadIdx.x] += s2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = s1[0];
        partial[2 * blockIdx.x + 1] = s2[0];
    }
}

__global__ void err_final_kernel(const double* partial, int nb, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < nb; ++k) {
        a += partial[2 * k];
        b += partial[2 * k + 1];
    }
    out[0] = sqrt(a) / (sqrt(b) + 1e-30);
}

// move_mesh single-rank path (move_mesh.f90:29-58, 185-214): shift f, u, v,
// rho by one column.  The plain path shifts its full fields; the fused path
// shifts the distribution planes and the border store.
__global__ void plain_shift_kernel(DevState d, int dr) {
    // one thread per (row j); sequential over k within the row keeps the
    // in-place semantics of the reference's two loops exactly.
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.ny) return;
    const int klo = dr == 1 ? 0 : 1, khi = dr == 1 ? d.nx - 2 : d.nx - 1, src = dr == 1 ? 1 : -1;
    if (dr == 1) {
        for (int k = klo; k <= khi; ++k) {
            long long p = pidx(d, k, j), q = pidx(d, k + src, j);
            for (int c = 0; c < 9; ++c) d.f0[c * d.plane + p] = d.f[c * d.plane + q];
            d.u0[p] = d.u[q]; d.v0[p] = d.v[q]; d.pre[p] = d.rho[q];
        }
    } else {
        for (int k = khi; k >= klo; --k) {
            long long p = pidx(d, k, j), q = pidx(d, k + src, j);
            for (int c = 0; c < 9; ++c) d.f0[c * d.plane + p] = d.f[c * d.plane + q];
            d.u0[p] = d.u[q]; d.v0[p] = d.v[q]; d.pre[p] = d.rho[q];
        }
    }
    for (int k = klo; k <= khi; ++k) {
        long long p = pidx(d, k, j);
        for (int c = 0; c < 9; ++c) d.f[c * d.plane + p] = d.f0[c * d.plane + p];
        d.u[p] = d.u0[p]; d.v[p] = d.v0[p]; d.rho[p] = d.pre[p];
    }
}

void launch_plain_stream(const DevState& d, cudaStream_t st) {
    dim3 b(128), g((d.nx - 2 + 127) / 128, d.ny - 2);
    plain_stream_kernel<<<g, b, 0, st>>>(d);
}
void launch_plain_moments(const DevState& d, cudaStream_t st) {
    dim3 b(128), g((d.nx + 127) / 128, d.ny);
    plain_moments_kernel<<<g, b, 0, st>>>(d);
}
void launch_plain_collide(const DevState& d, cudaStream_t st) {
    dim3 b(128), g((d.nx - 2 + 127) / 128, d.ny - 2);
    plain_collide_kernel<<<g, b, 0, st>>>(d);
}
void launch_outer_bc(const DevState& d, cudaStream_t st) {
    int n = 2 * (d.ny - 2) + 2 * d.nx;
    if (d.precision == 0)
        outer_bc_kernel<PlainAcc><<<(n + 127) / 128, 128, 0, st>>>(PlainAcc{d});
    else
        launch_fused_bc(d, st);   // the fused path's own form (kernels_fp32.cu)
}
void launch_err(const DevState& d, double* partial, double* out, cudaStream_t st) {
    if (d.precision == 0)
        err_partial_kernel<false><<<ERR_BLOCKS, 256, 0, st>>>(d, partial);
    else
        err_partial_kernel<true><<<ERR_BLOCKS, 256, 0, st>>>(d, partial);
    err_final_kernel<<<1, 32, 0, st>>>(partial, ERR_BLOCKS, out);
}
int err_partial_count() { return ERR_BLOCKS; }
void launch_plain_shift(const DevState& d, int dr, cudaStream_t st) {
    plain_shift_kernel<<<(d.ny + 127) / 128, 128, 0, st>>>(d, dr);
}

// output (solution.f90:132-241): at every sx-th node of every sy-th row,
// u/UU, v/UU, the pressure and the vorticity dv/dx - du/dy with centred
// differences inside and second-order one-sided ones on the border rows and
// columns (:197-211), in the reference's operation order.  The fused path's
// pressure is rho/3 of the streamed populations inside and the border
// store's sum / 3 on the border, as its field export gives it.
__global__ void output_fields_kernel(DevState d, int sx, int sy, int onx, int ony, double* out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long per = (long long)onx * ony;
    if (t >= per) return;
    const int oi = (int)(t % onx), oj = (int)(t / onx);
    const int i = oi * sx, j = oj * sy;
    const bool fused = d.precision != 0;
    const double* U = fused ? d.fo_u : d.u;
    const double* V = fused ? d.fo_v : d.v;
    auto u = [&](int a, int b) { return U[pidx(d, a, b)]; };
    auto v = [&](int a, int b) { return V[pidx(d, a, b)]; };
    const double uu = d.uu, sc = d.scale;
    double dvx, duy;
    if (i == d.nx - 1)
        dvx = (1.5 * v(i, j) - 2.0 * v(i - 1, j) + 0.5 * v(i - 2, j)) / (uu * sc);
    else if (i == 0)
        dvx = (-1.5 * v(i, j) + 2.0 * v(i + 1, j) - 0.5 * v(i + 2, j)) / (uu * sc);
    else
        dvx = (v(i + 1, j) - v(i - 1, j)) / (uu * 2.0 * sc);
    if (j == d.ny - 1)
        duy = (1.5 * u(i, j) - 2.0 * u(i, j - 1) + 0.5 * u(i, j - 2)) / (uu * sc);
    else if (j == 0)
        duy = (-1.5 * u(i, j) + 2.0 * u(i, j + 1) - 0.5 * u(i, j + 2)) / (uu * sc);
    else
        duy = (u(i, j + 1) - u(i, j - 1)) / (uu * 2.0 * sc);
    double pre;
    if (!fused) {
        pre = d.pre[pidx(d, i, j)];
    } else if (i == 0 || j == 0 || i == d.nx - 1 || j == d.ny - 1) {
        const long long eper = 2LL * d.ny + 2LL * d.nx;
        const long long e = (i == 0) ? j : (i == d.nx - 1) ? d.ny + j : (j == 0) ? 2LL * d.ny + i
                                                                               : 2LL * d.ny + d.nx + i;
        double s = 0.0;
        for (int k = 0; k < 9; ++k) s = s + d.edge_f0[k * eper + e];
        pre = s / 3.0;
    } else {
        pre = d.fo_rho[pidx(d, i, j)] / 3.0;
    }
    out[t] = u(i, j) / uu;
    out[per + t] = v(i, j) / uu;
    out[2 * per + t] = pre;
    out[3 * per + t] = dvx - duy;
}

void launch_output_fields(const DevState& d, int sx, int sy, double* out, cudaStream_t st) {
    const int onx = (d.nx - 1) / sx + 1, ony = (d.ny - 1) / sy + 1;
    const long long n = (long long)onx * ony;
    output_fields_kernel<<<(int)((n + 255) / 256), 256, 0, st>>>(d, sx, sy, onx, ony, out);
}

}  // namespace lbm
