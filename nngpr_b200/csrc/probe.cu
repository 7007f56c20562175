// FMA-rate probes (FP32 and FP64): the denominators of the roofline fractions of the kernels
// here that are bound by a SIMT pipe.  Each thread runs 8 independent FMA chains of `iters`
// steps (16 flops per step); the sum is written out so nothing is eliminated.  The caller times
// the launch.
#include "common.cuh"

namespace nngp {

__global__ void __launch_bounds__(256) fma_probe_kernel(float *out, int64_t iters, float a, float b) {
    float v0 = threadIdx.x * 1e-3f, v1 = v0 + 1.f, v2 = v0 + 2.f, v3 = v0 + 3.f;
    float v4 = v0 + 4.f, v5 = v0 + 5.f, v6 = v0 + 6.f, v7 = v0 + 7.f;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            v0 = fmaf(v0, a, b); v1 = fmaf(v1, a, b); v2 = fmaf(v2, a, b); v3 = fmaf(v3, a, b);
            v4 = fmaf(v4, a, b); v5 = fmaf(v5, a, b); v6 = fmaf(v6, a, b); v7 = fmaf(v7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = v0 + v1 + v2 + v3 + v4 + v5 + v6 + v7;
}

__global__ void __launch_bounds__(256) fma_probe_f64_kernel(double *out, int64_t iters, double a, double b) {
    double v0 = threadIdx.x * 1e-3, v1 = v0 + 1.0, v2 = v0 + 2.0, v3 = v0 + 3.0;
    double v4 = v0 + 4.0, v5 = v0 + 5.0, v6 = v0 + 6.0, v7 = v0 + 7.0;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            v0 = fma(v0, a, b); v1 = fma(v1, a, b); v2 = fma(v2, a, b); v3 = fma(v3, a, b);
            v4 = fma(v4, a, b); v5 = fma(v5, a, b); v6 = fma(v6, a, b); v7 = fma(v7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = v0 + v1 + v2 + v3 + v4 + v5 + v6 + v7;
}

}  // namespace nngp

extern "C" nngp_status nngp_fma_probe(float *out, int64_t iters, int32_t blocks, void *stream) {
    using namespace nngp;
    set_error("");
    if (!out || iters <= 0 || blocks <= 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "fma_probe: bad arguments");
    fma_probe_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out, iters, 0.999999f, 1e-6f);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}

extern "C" nngp_status nngp_fma_probe_f64(double *out, int64_t iters, int32_t blocks, void *stream) {
    using namespace nngp;
    set_error("");
    if (!out || iters <= 0 || blocks <= 0) return fail(NNGP_ERR_INVALID_ARGUMENT, "fma_probe_f64: bad arguments");
    fma_probe_f64_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out, iters, 0.999999, 1e-6);
    NNGP_CUDA_TRY(cudaGetLastError());
    return NNGP_OK;
}
