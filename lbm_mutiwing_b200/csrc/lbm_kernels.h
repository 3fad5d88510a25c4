// Host-side launch wrappers for the device kernels.
#pragma once
#include "lbm_common.cuh"

namespace lbm {

// plain FP64 path (kernels_fp64.cu)
void launch_plain_stream(const DevState& d, cudaStream_t st);
void launch_plain_moments(const DevState& d, cudaStream_t st);
void launch_plain_collide(const DevState& d, cudaStream_t st);
void launch_plain_shift(const DevState& d, int dr, cudaStream_t st);
// both paths
void launch_outer_bc(const DevState& d, cudaStream_t st);
void launch_err(const DevState& d, double* partial, double* out, cudaStream_t st);
int err_partial_count();

// fused FP32 path (kernels_fp32.cu)
struct FusedConsts {
    float s1, s2, s4, s6, s7, s8;   // MRT rates of the non-conserved moments
    float k1, k2, wm1;              // deviation constants (rest-state moments)
};
FusedConsts fused_consts(const DevState& d);
void launch_fused_bulk(const DevState& d, const FusedConsts& c, bool fields, cudaStream_t st);
void launch_fused_band(const DevState& d, bool fields, cudaStream_t st);
void launch_fused_init(const DevState& d, cudaStream_t st);
void launch_fused_shift(const DevState& d, int dr, cudaStream_t st);
void launch_fused_export(const DevState& d, const float* g, double* f, cudaStream_t st);
void launch_fused_import(const DevState& d, const double* f, float* g, cudaStream_t st);

// immersed boundary (ibm.cu)
void launch_ibm_band(const DevState& d, cudaStream_t st);            // move_boundary
void launch_ibm_solve(const DevState& d, size_t smem, bool band_in_smem, cudaStream_t st);
void launch_ibm_full(const DevState& d, size_t smem, bool band_in_smem, cudaStream_t st);
void launch_step_advance(const DevState& d, cudaStream_t st);        // cycle += 1
int ibm_threads();

}  // namespace lbm
