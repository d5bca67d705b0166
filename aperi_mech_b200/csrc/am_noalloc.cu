// am_noalloc.cu -- Tet4 internal force for callers that cannot allocate device memory.
//
// Some callers run where cudaMalloc is off limits: a host framework that owns all
// device memory through its own pool and forbids foreign allocations, or code that
// must not add allocation latency or synchronization to a step it already
// schedules. am_tet4_internal_force_noalloc serves them: the caller passes every
// input and output as device pointers, and the per-element force slots (the only
// scratch the computation needs) live in a fixed file-scope device array.
//
// The array holds the force slots of at most AM_NOALLOC_MAX_TETS tets (4 slots per
// tet, 3 doubles each: 16 MiB), which every GPU that loads this library keeps until the process exits.
// Every call shares it: the element pass overwrites each slot it uses before the
// gather pass reads it, so nothing needs clearing between calls, but two calls
// that overlap on the GPU (different streams, or different threads without
// ordering) race on the array and must be serialized by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/aperi_b200.h"
#include "am_math.cuh"

namespace am {
void set_free_error(const std::string& msg);  // am_context.cu
}

namespace {

constexpr int64_t kNoAllocMaxSlots = 4 * static_cast<int64_t>(AM_NOALLOC_MAX_TETS);  // 16 MiB of FP64 slots
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_slots[kNoAllocMaxSlots * 3];

// Device address of g_noalloc_slots, looked up once per device. In host code the
// symbol name is only a host-side stand-in, so kernels must receive this address.
double* g_slot_addr[kMaxDevices] = {nullptr};
std::mutex g_slot_mutex;

// One thread per tet, reading row-major N x 3 coordinate and displacement arrays.
template <int MAT>
__global__ void __launch_bounds__(256) k_tet4_force_aos(int64_t num_elems, const int32_t* __restrict__ conn,
                                                         const double* __restrict__ X, const double* __restrict__ U,
                                                         double lambda, double mu, double* __restrict__ slots) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= num_elems) return;
    int32_t n[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) n[a] = conn[4 * e + a];
    double J[9], D[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            J[i * 3 + j] = X[3 * n[j + 1] + i] - X[3 * n[0] + i];
            D[i * 3 + j] = U[3 * n[j + 1] + i] - U[3 * n[0] + i];
        }
    const double det = am::det3(J);
    double Ji[9];
    am::cof_inv3(J, Ji, det);
    const double w = det / 6.0;
    double H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) H[i * 3 + j] = D[i * 3 + 0] * Ji[0 * 3 + j] + D[i * 3 + 1] * Ji[1 * 3 + j] + D[i * 3 + 2] * Ji[2 * 3 + j];
    double P[9];
    am::stress<double>(MAT, lambda, mu, H, P);
    double f[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double q = w * (Ji[k * 3 + 0] * P[i * 3 + 0] + Ji[k * 3 + 1] * P[i * 3 + 1] + Ji[k * 3 + 2] * P[i * 3 + 2]);
            f[(k + 1) * 3 + i] = -q;
            f[i] += q;
        }
    double* out = slots + 12 * e;
#pragma unroll
    for (int k = 0; k < 12; ++k) out[k] = f[k];
}

__global__ void __launch_bounds__(256) k_gather_aos(int64_t num_nodes, const int32_t* __restrict__ node_ptr,
                                                     const int32_t* __restrict__ node_slots,
                                                     const double* __restrict__ slots, double* __restrict__ f) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= num_nodes) return;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int32_t p = node_ptr[i]; p < node_ptr[i + 1]; ++p) {
        const int64_t s = node_slots[p];
        fx += slots[3 * s + 0];
        fy += slots[3 * s + 1];
        fz += slots[3 * s + 2];
    }
    f[3 * i + 0] = fx;
    f[3 * i + 1] = fy;
    f[3 * i + 2] = fz;
}

int fail(int code, const std::string& msg) {
    am::set_free_error(msg);  // readable through am_last_error(NULL)
    return code;
}

// First call on a device: look up the array's device address with that device current.
int slot_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(AM_ERANGE, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    if (g_slot_addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_slots);
        if (e != cudaSuccess || p == nullptr)
            return fail(AM_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_slot_addr[dev] = static_cast<double*>(p);
    }
    *out = g_slot_addr[dev];
    return AM_OK;
}

}  // namespace

extern "C" {

int am_tet4_internal_force_noalloc(int32_t material, double lambda, double mu, int64_t num_nodes,
                                   int64_t num_elems, const double* coords, const double* u, const int32_t* conn,
                                   const int32_t* node_ptr, const int32_t* node_slots, double* f,
                                   void* cuda_stream) {
    am::set_free_error("");
    if (material < AM_LINEAR_ELASTIC || material > AM_ELASTIC_SVK) return fail(AM_EINVAL, "unknown material");
    if (num_nodes <= 0 || num_elems < 0) return fail(AM_EINVAL, "num_nodes must be positive, num_elems >= 0");
    if (!coords || !u || !f || !node_ptr || (num_elems > 0 && (!conn || !node_slots)))
        return fail(AM_EINVAL, "null device pointer");
    if (num_elems > AM_NOALLOC_MAX_TETS)
        return fail(AM_ERANGE, "am_tet4_internal_force_noalloc: " + std::to_string(num_elems) +
                                   " tets exceed the fixed scratch of AM_NOALLOC_MAX_TETS = " +
                                   std::to_string(AM_NOALLOC_MAX_TETS) + " tets");
    double* slots = nullptr;
    const int rc = slot_address(&slots);
    if (rc != AM_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    if (num_elems > 0) {
        const unsigned grid = static_cast<unsigned>((num_elems + 255) / 256);
        switch (material) {
            case AM_LINEAR_ELASTIC: k_tet4_force_aos<0><<<grid, 256, 0, s>>>(num_elems, conn, coords, u, lambda, mu, slots); break;
            case AM_NEO_HOOKEAN: k_tet4_force_aos<1><<<grid, 256, 0, s>>>(num_elems, conn, coords, u, lambda, mu, slots); break;
            default: k_tet4_force_aos<2><<<grid, 256, 0, s>>>(num_elems, conn, coords, u, lambda, mu, slots); break;
        }
    }
    k_gather_aos<<<static_cast<unsigned>((num_nodes + 255) / 256), 256, 0, s>>>(num_nodes, node_ptr, node_slots, slots, f);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return AM_OK;
}

}  // extern "C"
