// Convergence error of caller-owned velocity fields, computed without any
// allocation.
//
// Some callers cannot let a library allocate device memory: a host solver
// that has handed the whole device to its own memory pool, or a serving loop
// in which a cudaMalloc / cudaFree (which may synchronise the device) would
// stall the streams of the other episodes.  lbm_err_fields_noalloc computes
// the reference's erranalysis (solution.f90:77-130),
//   err = sqrt(sum |u - u0|^2) / (sqrt(sum |u|^2) + 1e-30)
// over the interior nodes, on fields that the caller owns, with its partial
// sums in a fixed array compiled into this library.
//
// Scratch: one pair (sum |u - u0|^2, sum |u|^2) per interior lattice row and
// the result slot, for at most LBM_NOALLOC_MAX_ROWS lattice rows; larger
// lattices are refused with an error.  Every slot a call reads is written
// earlier in the same call, so nothing relies on the array starting at zero.
// The array is one per device and shared by all calls on that device: calls
// that overlap in time on one device (two host threads, or two streams not
// ordered by events) race on it, so the caller must serialise them.
//
// The address of the array is looked up once per device, on the first call
// for that device.  Every call synchronises the caller's stream and copies
// the result to the host before it returns.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/lbm_mutiwing.h"

namespace {

constexpr int MAX_DEVICES = 64;
constexpr int SCRATCH_DOUBLES = 2 * LBM_NOALLOC_MAX_ROWS + 2;   // row pairs, then the result

static __device__ __align__(256) double g_err_scratch[SCRATCH_DOUBLES];

std::mutex g_setup_mutex;
double* g_scratch_ptr[MAX_DEVICES] = {};

// One warp per interior row j: lane-strided sums over the row's interior
// nodes, then a fixed shuffle tree; the pair goes to rows[2 (j - 1)].
__global__ void err_rows_kernel(const double* __restrict__ u, const double* __restrict__ v,
                                const double* __restrict__ u0, const double* __restrict__ v0, int nx, int ny,
                                long long pitch, double* rows) {
    const int lane = threadIdx.x & 31;
    const int j = 1 + (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    if (j > ny - 2) return;   // whole warps leave together
    const long long r = (long long)j * pitch;
    double a = 0.0, b = 0.0;
    for (int i = 1 + lane; i <= nx - 2; i += 32) {
        const double uu = u[r + i], vv = v[r + i];
        const double du = uu - u0[r + i], dv = vv - v0[r + i];
        a = a + du * du + dv * dv;
        b = b + uu * uu + vv * vv;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
        rows[2 * (j - 1)] = a;
        rows[2 * (j - 1) + 1] = b;
    }
}

// One warp adds the row pairs in a fixed order and writes err to result.
__global__ void err_rows_final_kernel(const double* rows, int nrows, double* result) {
    const int lane = threadIdx.x;
    double a = 0.0, b = 0.0;
    for (int k = lane; k < nrows; k += 32) {
        a += rows[2 * k];
        b += rows[2 * k + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) result[0] = sqrt(a) / (sqrt(b) + 1e-30);
}

int report(char* msg, int32_t cap, int code, const char* text, cudaError_t e = cudaSuccess) {
    if (msg && cap > 0) {
        if (e != cudaSuccess)
            snprintf(msg, (size_t)cap, "%s: %s", text, cudaGetErrorString(e));
        else
            snprintf(msg, (size_t)cap, "%s", text);
    }
    return code;
}

}  // namespace

extern "C" int lbm_err_fields_noalloc(const double* u, const double* v, const double* u0, const double* v0,
                                      int32_t nx, int32_t ny, int64_t pitch, int32_t device, void* stream,
                                      double* err, char* msg, int32_t msg_cap) {
    if (msg && msg_cap > 0) msg[0] = '\0';
    if (!u || !v || !u0 || !v0 || !err) return report(msg, msg_cap, -1, "null field or result pointer");
    if (nx < 3 || ny < 3 || pitch < nx) return report(msg, msg_cap, -1, "need nx >= 3, ny >= 3 and pitch >= nx");
    if (ny > LBM_NOALLOC_MAX_ROWS) {
        char t[160];
        snprintf(t, sizeof t, "ny = %d exceeds the %d lattice rows of the built-in scratch", (int)ny,
                 LBM_NOALLOC_MAX_ROWS);
        return report(msg, msg_cap, -2, t);
    }
    if (device < 0 || device >= MAX_DEVICES) return report(msg, msg_cap, -1, "device index out of range");
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return report(msg, msg_cap, -3, "cudaGetDevice", e);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return report(msg, msg_cap, -3, "cudaSetDevice", e);
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[device]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_err_scratch);
            if (e != cudaSuccess) {
                cudaSetDevice(prev);
                return report(msg, msg_cap, -3, "cudaGetSymbolAddress of the scratch array", e);
            }
            g_scratch_ptr[device] = static_cast<double*>(p);
        }
        scratch = g_scratch_ptr[device];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nrows = ny - 2;
    const int threads = 256, blocks = (nrows * 32 + threads - 1) / threads;
    err_rows_kernel<<<blocks, threads, 0, st>>>(u, v, u0, v0, nx, ny, (long long)pitch, scratch);
    err_rows_final_kernel<<<1, 32, 0, st>>>(scratch, nrows, scratch + 2 * LBM_NOALLOC_MAX_ROWS);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(err, scratch + 2 * LBM_NOALLOC_MAX_ROWS, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return report(msg, msg_cap, -3, "convergence-error kernels", e);
    return 0;
}
