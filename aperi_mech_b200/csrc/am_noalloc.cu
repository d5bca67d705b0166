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
//
// A second file-scope word pair holds the status of the most recent call on the
// device (first error code and its element or node index): det J <= 0, J <= 0 for
// neo-Hookean, or a node -> slot CSR entry outside the call's 4 num_elems slots.
// Each call clears it (stream-ordered) before its kernels run; am_noalloc_status
// reads it back. It is shared exactly like the slots.
#include <cuda.h>
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
// {status code, element or node index} of the most recent call on this device
static __device__ __align__(8) int g_noalloc_status[2];

__device__ __forceinline__ void flag(int* status, int code, int64_t idx) {
    if (atomicCAS(status, 0, code) == 0) status[1] = static_cast<int>(idx);
}

// One thread per tet, reading row-major N x 3 coordinate and displacement arrays.
template <int MAT>
__global__ void __launch_bounds__(256) k_tet4_force_aos(int64_t num_elems, const int32_t* __restrict__ conn,
                                                         const double* __restrict__ X, const double* __restrict__ U,
                                                         double lambda, double mu, double* __restrict__ slots,
                                                         int* status) {
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
    if (!(det > 0.0)) flag(status, AM_ENONPOS_J, e);
    double Ji[9];
    am::cof_inv3(J, Ji, det);
    const double w = det / 6.0;
    double H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) H[i * 3 + j] = D[i * 3 + 0] * Ji[0 * 3 + j] + D[i * 3 + 1] * Ji[1 * 3 + j] + D[i * 3 + 2] * Ji[2 * 3 + j];
    double P[9];
    const double Jf = am::stress<double>(MAT, lambda, mu, H, P);
    if (MAT == 1 && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, e);
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

// Sums each node's slots in CSR order. Only slots 0 .. num_slots-1 were written by
// this call, so a CSR range or slot id outside them is flagged and skipped rather
// than read (it would see a previous call's data).
__global__ void __launch_bounds__(256) k_gather_aos(int64_t num_nodes, int64_t num_slots,
                                                     const int32_t* __restrict__ node_ptr,
                                                     const int32_t* __restrict__ node_slots,
                                                     const double* __restrict__ slots, double* __restrict__ f,
                                                     int* status) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= num_nodes) return;
    if (i == num_nodes - 1 && node_ptr[num_nodes] != num_slots) flag(status, AM_EINVAL, num_nodes);
    int64_t beg = node_ptr[i], end = node_ptr[i + 1];
    if (beg < 0 || end > num_slots || beg > end) {
        flag(status, AM_EINVAL, i);
        beg = beg < 0 ? 0 : beg;
        end = end > num_slots ? num_slots : end;
    }
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int64_t p = beg; p < end; ++p) {
        const int64_t s = node_slots[p];
        if (s < 0 || s >= num_slots) {
            flag(status, AM_EINVAL, i);
            continue;
        }
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

// Device addresses of the file-scope arrays, looked up once per device and context.
// In host code the symbol names are only host-side stand-ins, so kernels and copies
// must receive these addresses. The cache is keyed on the current context's unique
// id as well as the device ordinal: after a device reset the module is loaded again
// at possibly another address, and the next call then looks it up again.
struct Scratch {
    unsigned long long ctx_id = 0;
    double* slots = nullptr;
    int* status = nullptr;
};
Scratch g_scratch[kMaxDevices];
std::mutex g_scratch_mutex;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0 when there is none yet), with
// the driver entry points resolved through the runtime (no link against libcuda).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(p);
        resolved = true;
    }
    if (get_current == nullptr || get_id == nullptr) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up with the device current: cudaGetSymbolAddress of both arrays the first time
// this device (in this context) is used; afterwards the cached addresses.
int scratch_addresses(double** slots, int** status) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(AM_ERANGE, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    Scratch& s = g_scratch[dev];
    const unsigned long long id = current_context_id();
    if (s.slots == nullptr || id == 0 || id != s.ctx_id) {
        void* ps = nullptr;
        void* pt = nullptr;
        e = cudaGetSymbolAddress(&ps, g_noalloc_slots);
        if (e != cudaSuccess || ps == nullptr)
            return fail(AM_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        e = cudaGetSymbolAddress(&pt, g_noalloc_status);
        if (e != cudaSuccess || pt == nullptr)
            return fail(AM_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        s.slots = static_cast<double*>(ps);
        s.status = static_cast<int*>(pt);
        // the lookup made the primary context current if no context was yet
        s.ctx_id = id != 0 ? id : current_context_id();
    }
    *slots = s.slots;
    *status = s.status;
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
    int* status = nullptr;
    const int rc = scratch_addresses(&slots, &status);
    if (rc != AM_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e = cudaMemsetAsync(status, 0, 2 * sizeof(int), s);
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("clearing the status word: ") + cudaGetErrorString(e));
    if (num_elems > 0) {
        const unsigned grid = static_cast<unsigned>((num_elems + 255) / 256);
        switch (material) {
            case AM_LINEAR_ELASTIC: k_tet4_force_aos<0><<<grid, 256, 0, s>>>(num_elems, conn, coords, u, lambda, mu, slots, status); break;
            case AM_NEO_HOOKEAN: k_tet4_force_aos<1><<<grid, 256, 0, s>>>(num_elems, conn, coords, u, lambda, mu, slots, status); break;
            default: k_tet4_force_aos<2><<<grid, 256, 0, s>>>(num_elems, conn, coords, u, lambda, mu, slots, status); break;
        }
    }
    k_gather_aos<<<static_cast<unsigned>((num_nodes + 255) / 256), 256, 0, s>>>(num_nodes, 4 * num_elems, node_ptr,
                                                                                 node_slots, slots, f, status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return AM_OK;
}

int am_noalloc_status(void* cuda_stream, int32_t* status, int64_t* index) {
    am::set_free_error("");
    if (status == nullptr) return fail(AM_EINVAL, "null status pointer");
    double* slots = nullptr;
    int* word = nullptr;
    const int rc = scratch_addresses(&slots, &word);
    if (rc != AM_OK) return rc;
    int host[2] = {0, 0};
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e = cudaMemcpyAsync(host, word, sizeof(host), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(AM_ECUDA, std::string("reading the status word: ") + cudaGetErrorString(e));
    *status = host[0];
    if (index != nullptr) *index = host[0] != 0 ? host[1] : -1;
    return AM_OK;
}

}  // extern "C"
