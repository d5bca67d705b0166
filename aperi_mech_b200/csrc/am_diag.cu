// am_diag.cu -- measured FP32 and FP64 FMA throughput of the current device.
//
// The element kernels of this library are bound by FP32 issue or by the FP64 pipe,
// not by HBM, so their compute roofline needs a measured denominator beside the
// measured copy bandwidth. k_fma_peak runs eight independent FMA chains per thread
// over a grid of eight 256-thread blocks per SM (sixteen warps per scheduler, enough
// to hide the FMA latency), nothing but FMAs in the loop; the host times one launch
// with CUDA events after a warm-up launch.
#include <cuda_runtime.h>

#include <string>

#include "../../include/aperi_b200.h"

namespace am {
void set_free_error(const std::string& msg);  // am_context.cu
}

namespace {

static __device__ double g_fma_sink;

constexpr int kChains = 8;
constexpr int kUnroll = 16;

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(int iters, T seed) {
    T a[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = seed + T(threadIdx.x + i);
    const T m = T(0.9999999), c = T(1e-7);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < kUnroll; ++k)
#pragma unroll
            for (int i = 0; i < kChains; ++i) a[i] = fma(a[i], m, c);
    }
    T s = T(0);
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += a[i];
    if (s == T(-1.25)) g_fma_sink = static_cast<double>(s);  // never true; keeps the chains live
}

int fail(int code, const std::string& msg) {
    am::set_free_error(msg);
    return code;
}

}  // namespace

extern "C" int am_measure_fma_peak(int32_t fp64, void* cuda_stream, double* flops_per_s) {
    am::set_free_error("");
    if (flops_per_s == nullptr) return fail(AM_EINVAL, "null output pointer");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("device query: ") + cudaGetErrorString(e));
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    const unsigned grid = static_cast<unsigned>(8 * sms);
    const int iters = fp64 ? 1024 : 2048;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
        e = cudaEventRecord(e0, s);
        if (fp64)
            k_fma_peak<double><<<grid, 256, 0, s>>>(iters, 1.0);
        else
            k_fma_peak<float><<<grid, 256, 0, s>>>(iters, 1.0f);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("FMA peak kernel: ") + cudaGetErrorString(e));
    const double flop = 2.0 * kChains * kUnroll * static_cast<double>(iters) * 256.0 * grid;
    *flops_per_s = flop / (static_cast<double>(ms) * 1e-3);
    return AM_OK;
}
