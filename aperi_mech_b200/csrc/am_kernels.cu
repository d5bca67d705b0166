// am_kernels.cu -- sm_100a kernels of the explicit-dynamics hot path.
//
// Force assembly is two kernels per step, with no atomics anywhere:
//   1. an element (or smoothed-cell) kernel writes each element's nodal force
//      contributions to its own "slots" (element e, local node a -> slot);
//   2. a node kernel sums its slots through a node -> slot CSR in ascending
//      slot order (deterministic, the oracle's element order) and, in the time
//      loop, fuses the central-difference update: a = f/m, boundary overwrite,
//      v^{n+1}, and the next step's v^{n+1/2} and u^{n+2}.
// Element math runs in FP64 (T = double) or FP32 (T = float, mixed path). The
// mixed path forms element-local differences (X_a - X_0, u_a - u_0) in FP64
// before casting, evaluates the neo-Hookean det F and log J in FP64, and
// accumulates nodal forces and the state in FP64.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdlib.h>

#include "am_kernels.cuh"
#include "am_math.cuh"

namespace am {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// Programmatic dependent launch (sm_90+ PTX griddepcontrol): a kernel launched with
// programmatic stream serialization may start while its predecessor in the stream is
// still running; it reads only data that no kernel of the step writes (mesh, mass, BC
// words) before pdl_wait(), which returns once the predecessor has completed and its
// writes are visible. pdl_trigger() lets the successor start; both are no-ops for a
// kernel launched without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Load of data the previous kernel in the stream writes (displacements, force slots),
// through the coherent cached path. Under programmatic dependent launch that kernel may
// still be running when this one starts, so such data is not read-only for this
// kernel's lifetime and must not be read through the non-coherent read-only path that
// const __restrict__ pointers allow.
// A double4 is one 32-byte load (sm_100 vector width; the arrays are 32-byte aligned),
// volatile so that it stays after the wait that orders it.
__device__ __forceinline__ double4 ld_dep(const double4* p) {
    double4 r;
    asm volatile("ld.global.ca.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}
__device__ __forceinline__ float4 ld_dep(const float4* p) { return __ldca(p); }
// One 32-byte store (the arrays are 32-byte aligned).
__device__ __forceinline__ void st4(double4* p, const double4& v) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v.x), "d"(v.y), "d"(v.z), "d"(v.w) : "memory");
}
// One 32-byte load through the read-only path, for data that no kernel still running
// writes (kernels launched without programmatic overlap, on arrays finished before).
__device__ __forceinline__ double4 ld_ro4(const double4* p) {
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

__device__ __forceinline__ void flag(int* status, int code, int64_t idx) {
    if (status == nullptr) return;
    if (atomicCAS(status + kStatusCode, 0, code) == 0) status[kStatusIndex] = static_cast<int>(idx);
}

template <typename T>
struct Vec4Of;
template <>
struct Vec4Of<float> {
    using type = float4;
};
template <>
struct Vec4Of<double> {
    using type = double4;
};
template <typename T>
using vec4_t = typename Vec4Of<T>::type;

__device__ __forceinline__ float4 make4(float x, float y, float z) { return make_float4(x, y, z, 0.f); }
__device__ __forceinline__ double4 make4(double x, double y, double z) { return make_double4(x, y, z, 0.0); }

template <typename F>
__device__ __forceinline__ void element_lame(const F& b, int64_t e, double& lambda, double& mu) {
    if (b.mu_field != nullptr || b.kappa_field != nullptr) {
        const double m = b.mu_field ? b.mu_field[e] : b.mu;
        const double k = b.kappa_field ? b.kappa_field[e] : b.lambda + 2.0 * b.mu / 3.0;
        mu = m;
        lambda = k - 2.0 * m / 3.0;
    } else {
        lambda = b.lambda;
        mu = b.mu;
    }
}

// ---------------------------------------------------------------------------
// Hex8 reference-element sign tables (ShapeFunctionsFunctorHex8.h:17-33): node a
// sits at (sx, sy, sz) in {-1,1}^3; the 2x2x2 Gauss point g sits at the same
// signs times 1/sqrt(3) (ElementHexahedron8.h:105-117).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int hex_sign(int a, int j) {
    const int mask = (j == 0) ? 0x66 : (j == 1) ? 0xCC : 0xF0;
    return ((mask >> a) & 1) ? 1 : -1;
}

// ---------------------------------------------------------------------------
// Tet4, 1-point Gauss: one thread per element.
// ---------------------------------------------------------------------------
// Forces of one tet from its node differences relative to node l0: columns of J
// and D are X_l - X_l0 and u_l - u_l0 for l = l1, l2, l3. Writes f[12] (4 nodes x 3)
// and returns det J.
template <typename T, int MAT>
__device__ __forceinline__ T tet4_forces(const T* J, const T* D, double lam, double mu, T* f, int64_t e, int* status) {
    const T det = det3(J);
    if (!(det > T(0))) flag(status, AM_ENONPOS_J, e);
    T Ji[9];
    cof_inv3(J, Ji, det);
    const T w = det / T(6);
    // H = u^T B = D J^-1
    T H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) H[i * 3 + j] = D[i * 3 + 0] * Ji[0 * 3 + j] + D[i * 3 + 1] * Ji[1 * 3 + j] + D[i * 3 + 2] * Ji[2 * 3 + j];
    if (MAT == kNeoHookean) {
        // With P = tau F^-T and F = (J + D) J^-1: w J^-1 P^T = w (J + D)^-1 tau
        // = adj(J + D) tau / (6 det F), det F being the FP64 DetApIm1(H) + 1 the stress uses.
        T tau[9];
        const double Jf = nh_kirchhoff<T>(T(lam), T(mu), H, tau);
        if (!(Jf > 0.0)) flag(status, AM_ENONPOS_J, e);
        T Jc[9], A[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Jc[k] = J[k] + D[k];
        adj3(Jc, A);
        // det F stays FP64; the FP32 path takes its scale from an FP32 reciprocal of
        // 6 det F (on B200 1.7% off the kernel against the FP64 division).
        const T sc = sizeof(T) == 4 ? T(__frcp_rn(static_cast<float>(6.0 * Jf))) : T(1.0 / (6.0 * Jf));
        // the scale folded into tau (six distinct entries)
        T ts[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j) ts[i * 3 + j] = ts[j * 3 + i] = sc * tau[i * 3 + j];
#pragma unroll
        for (int i = 0; i < 3; ++i) f[i] = T(0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T q = A[k * 3 + 0] * ts[0 * 3 + i] + A[k * 3 + 1] * ts[1 * 3 + i] + A[k * 3 + 2] * ts[2 * 3 + i];
                f[(k + 1) * 3 + i] = -q;
                f[i] += q;
            }
        return det;
    }
    T P[9];
    const double Jf = stress<T>(MAT, T(lam), T(mu), H, P);
    if (MAT == kNeoHookean && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, e);
    // Q = w J^-1 P^T ; f_{k+1} = -Q_k ; f_0 = Q_0 + Q_1 + Q_2
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T q = w * (Ji[k * 3 + 0] * P[i * 3 + 0] + Ji[k * 3 + 1] * P[i * 3 + 1] + Ji[k * 3 + 2] * P[i * 3 + 2]);
            f[(k + 1) * 3 + i] = -q;
            f[i] += q;
        }
    return det;
}

template <typename T, int MAT>
__global__ void __launch_bounds__(256) k_tet4_force(GaussBlockDev b, const double4* __restrict__ X4,
                                                     const double4* __restrict__ U4, vec4_t<T>* __restrict__ slots,
                                                     int* status) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    const int4 c = reinterpret_cast<const int4*>(b.conn)[e];
    const double4 x0 = X4[c.x], x1 = X4[c.y], x2 = X4[c.z], x3 = X4[c.w];
    const double4 u0 = U4[c.x], u1 = U4[c.y], u2 = U4[c.z], u3 = U4[c.w];
    // J = X^T dN with dN rows (-1,-1,-1), e1, e2, e3: column j of J is X_{j+1} - X_0.
    const T J[9] = {T(x1.x - x0.x), T(x2.x - x0.x), T(x3.x - x0.x), T(x1.y - x0.y), T(x2.y - x0.y),
                    T(x3.y - x0.y), T(x1.z - x0.z), T(x2.z - x0.z), T(x3.z - x0.z)};
    const T D[9] = {T(u1.x - u0.x), T(u2.x - u0.x), T(u3.x - u0.x), T(u1.y - u0.y), T(u2.y - u0.y),
                    T(u3.y - u0.y), T(u1.z - u0.z), T(u2.z - u0.z), T(u3.z - u0.z)};
    double lam, mu;
    element_lame(b, e, lam, mu);
    T f[12];
    tet4_forces<T, MAT>(J, D, lam, mu, f, e, status);
    const int4 pos = make_int4(b.slot_pos[4 * e], b.slot_pos[4 * e + 1], b.slot_pos[4 * e + 2], b.slot_pos[4 * e + 3]);
    slots[pos.x] = make4(f[0], f[1], f[2]);
    slots[pos.y] = make4(f[3], f[4], f[5]);
    slots[pos.z] = make4(f[6], f[7], f[8]);
    slots[pos.w] = make4(f[9], f[10], f[11]);
}

// ---------------------------------------------------------------------------
// Tet4 one thread per tet with the geometry set up once: J^-1 and w = det J / 6 of the
// reference configuration (constant under the total formulation) are streamed from a
// table in place of four coordinate gathers and a 3x3 inverse per step. H = D J^-1;
// for the neo-Hookean material w J^-1 P^T = w J^-1 adj(F) tau / det F (adj(J + D) =
// adj(F J) = adj(J) adj(F) = 6 w J^-1 adj(F)), otherwise w J^-1 P^T from P.
// ---------------------------------------------------------------------------
template <typename T>
struct Vec2Of;
template <>
struct Vec2Of<float> {
    using type = float2;
};
template <>
struct Vec2Of<double> {
    using type = double2;
};
template <typename T>
__device__ __forceinline__ const T* tet_geo(const GaussBlockDev& b);
template <>
__device__ __forceinline__ const float* tet_geo<float>(const GaussBlockDev& b) { return b.geo32; }
template <>
__device__ __forceinline__ const double* tet_geo<double>(const GaussBlockDev& b) { return b.geo64; }
__device__ __forceinline__ float4 ld_geo4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ld_geo4(const double4* p) { return ld_ro4(p); }

__global__ void __launch_bounds__(256) k_tet4_geometry(const int32_t* __restrict__ conn, int64_t E,
                                                        const double4* __restrict__ X4, float* __restrict__ g32,
                                                        double* __restrict__ g64) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int4 c = reinterpret_cast<const int4*>(conn)[e];
    const double4 x0 = X4[c.x], x1 = X4[c.y], x2 = X4[c.z], x3 = X4[c.w];
    const double J[9] = {x1.x - x0.x, x2.x - x0.x, x3.x - x0.x, x1.y - x0.y, x2.y - x0.y,
                         x3.y - x0.y, x1.z - x0.z, x2.z - x0.z, x3.z - x0.z};
    const double det = det3(J);
    double Ji[9];
    cof_inv3(J, Ji, det);
    const double w = det / 6.0;
    reinterpret_cast<double4*>(g64)[e] = make_double4(Ji[0], Ji[1], Ji[2], Ji[3]);
    reinterpret_cast<double4*>(g64 + 4 * E)[e] = make_double4(Ji[4], Ji[5], Ji[6], Ji[7]);
    reinterpret_cast<double2*>(g64 + 8 * E)[e] = make_double2(Ji[8], w);
    reinterpret_cast<float4*>(g32)[e] = make_float4(float(Ji[0]), float(Ji[1]), float(Ji[2]), float(Ji[3]));
    reinterpret_cast<float4*>(g32 + 4 * E)[e] = make_float4(float(Ji[4]), float(Ji[5]), float(Ji[6]), float(Ji[7]));
    reinterpret_cast<float2*>(g32 + 8 * E)[e] = make_float2(float(Ji[8]), float(w));
}

// A lane's share of a warp chunk (see GaussBlockDev): its K sorted entries (K / 4 words of
// code bytes and of node-rank bytes; rank 0xFF past the chunk's last element) and, for each
// entry that is the last of its node's run, the node's slot.
template <int K>
struct ChunkLane {
    uint32_t cw[K / 4], rw[K / 4];
    int32_t pos[K];
};
__device__ __forceinline__ int chunk_byte(const uint32_t* w, int j) {
    return static_cast<int>((w[j >> 2] >> (8 * (j & 3))) & 0xFFu);
}
// The lane's plan: its words and its run-end slot positions (resolved once by
// k_chunk_positions), independent loads.
template <int K, typename B>
__device__ __forceinline__ ChunkLane<K> chunk_lane(const B& b, int64_t ch, int lane, bool live) {
    constexpr int W = K / 4;
    ChunkLane<K> L;
#pragma unroll
    for (int w = 0; w < W; ++w) L.cw[w] = L.rw[w] = 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < K; ++j) L.pos[j] = -1;
    if (live) {
        const int64_t l = 32 * ch + lane;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            L.cw[w] = b.chunk_code[l * W + w];
            L.rw[w] = b.chunk_rank[l * W + w];
            const int4 p = reinterpret_cast<const int4*>(b.chunk_pos)[l * W + w];
            L.pos[4 * w] = p.x, L.pos[4 * w + 1] = p.y, L.pos[4 * w + 2] = p.z, L.pos[4 * w + 3] = p.w;
        }
    }
    return L;
}

// Set-up, a warp per chunk: the slot position of each lane entry that ends its node's run
// (the next sorted entry, in this lane or the next, has another rank), else -1.
template <int K, typename B>
__global__ void __launch_bounds__(256) k_chunk_positions(B b, int32_t* __restrict__ out) {
    constexpr int W = K / 4;
    const int64_t ch = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x & 31);
    if (32 * ch >= b.chunk_units) return;  // the whole warp
    const int64_t l = 32 * ch + lane;
    uint32_t rw[W];
#pragma unroll
    for (int w = 0; w < W; ++w) rw[w] = b.chunk_rank[l * W + w];
    const int32_t n0 = b.chunk_ptr[ch];
    const uint32_t nw = __shfl_down_sync(kFull, rw[0], 1);
    const int rnext = lane == 31 ? 0x100 : static_cast<int>(nw & 0xFFu);
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int r = chunk_byte(rw, j), after = j < K - 1 ? chunk_byte(rw, j + 1) : rnext;
        out[l * K + j] = (r != after && r != 0xFF) ? b.slot_pos[n0 + r] : -1;
    }
}

// Sums the chunk's entries per node and writes each node's slot once: a lane sums the runs
// of its K sorted entries, a segmented inclusive scan over the lanes (fixed shuffle tree)
// carries a run across lane boundaries, and the lane holding a node's last entry writes it.
// value(q, v) gives entry q's three components. All 32 lanes call it.
template <typename T, int K, typename Value>
__device__ __forceinline__ void chunk_reduce(const ChunkLane<K>& L, int lane, Value value, vec4_t<T>* __restrict__ slots) {
    T run[3] = {T(0), T(0), T(0)}, head[3] = {T(0), T(0), T(0)};
    bool split = false;  // the lane's first run ends inside the lane
    int32_t posh = -1;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int r = chunk_byte(L.rw, j);
        if (j > 0 && r != chunk_byte(L.rw, j - 1)) {
            if (!split) {
                // the first run may continue one from the lanes before: written after the scan
#pragma unroll
                for (int i = 0; i < 3; ++i) head[i] = run[i];
                split = true;
                posh = L.pos[j - 1];
            } else if (chunk_byte(L.rw, j - 1) != 0xFF) {
                slots[L.pos[j - 1]] = make4(run[0], run[1], run[2]);  // a run wholly inside the lane
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) run[i] = T(0);
        }
        if (r != 0xFF) {
            T v[3];
            value(chunk_byte(L.cw, j), v);
#pragma unroll
            for (int i = 0; i < 3; ++i) run[i] += v[i];
        }
    }
    // the last run's sum over the lanes it spans: (value, starts here) scanned with
    // (a, fa) + (b, fb) = (fb ? b : a + b, fa | fb)
    const int r0 = chunk_byte(L.rw, 0);
    const int rprev = __shfl_up_sync(kFull, chunk_byte(L.rw, K - 1), 1);
    bool F = split || lane == 0 || r0 != rprev;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T u[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) u[i] = __shfl_up_sync(kFull, run[i], d);
        const bool fu = __shfl_up_sync(kFull, static_cast<int>(F), d) != 0;
        if (lane >= d) {
            if (!F) {
#pragma unroll
                for (int i = 0; i < 3; ++i) run[i] = u[i] + run[i];
            }
            F = F || fu;
        }
    }
    T carry[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) carry[i] = __shfl_up_sync(kFull, run[i], 1);
    if (split && r0 != 0xFF) {
        const bool cont = lane > 0 && r0 == rprev;
        slots[posh] = make4(cont ? carry[0] + head[0] : head[0], cont ? carry[1] + head[1] : head[1],
                            cont ? carry[2] + head[2] : head[2]);
    }
    if (L.pos[K - 1] >= 0) slots[L.pos[K - 1]] = make4(run[0], run[1], run[2]);
}

// One thread per tet. CHUNKS: the warp's 32 tets (a chunk) stage their corner forces in
// shared memory and sum them per distinct node (about 32 for 128 corners on a Morton-ordered
// tet mesh), a quarter of the slots of four per tet for the node kernel to read.
template <typename T, int MAT, bool CHUNKS>
__global__ void __launch_bounds__(256, CHUNKS && sizeof(T) == 8 ? 3 : 0) k_tet4_force_geo(GaussBlockDev b, const double4* __restrict__ U4,
                                                         vec4_t<T>* __restrict__ slots, int* status) {
    pdl_trigger();
    const int64_t E = b.num_elems;
    const int64_t et = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    // chunked: lanes past the last tet run a copy of it (never summed) to reach the warp sum
    if (!CHUNKS && et >= E) return;
    const int64_t e = et < E ? et : E - 1;
    const int4 c = reinterpret_cast<const int4*>(b.conn)[e];
    const T* geo = tet_geo<T>(b);
    const vec4_t<T> g0 = ld_geo4(reinterpret_cast<const vec4_t<T>*>(geo) + e);
    const vec4_t<T> g1 = ld_geo4(reinterpret_cast<const vec4_t<T>*>(geo + 4 * E) + e);
    const typename Vec2Of<T>::type g2 = __ldg(reinterpret_cast<const typename Vec2Of<T>::type*>(geo + 8 * E) + e);
    int32_t pos[4] = {0, 0, 0, 0};
    const int64_t ch = et >> 5;
    const int lane = static_cast<int>(threadIdx.x & 31);
    const bool live = 32 * ch < E;
    ChunkLane<4> L{};
    if (!CHUNKS) {
#pragma unroll
        for (int a = 0; a < 4; ++a) pos[a] = b.slot_pos[4 * e + a];
    } else {
        L = chunk_lane<4>(b, ch, lane, live);
    }
    double lam, mu;
    element_lame(b, e, lam, mu);
    pdl_wait();
    const double4 u0 = ld_dep(U4 + c.x), u1 = ld_dep(U4 + c.y), u2 = ld_dep(U4 + c.z), u3 = ld_dep(U4 + c.w);
    const T D[9] = {T(u1.x - u0.x), T(u2.x - u0.x), T(u3.x - u0.x), T(u1.y - u0.y), T(u2.y - u0.y),
                    T(u3.y - u0.y), T(u1.z - u0.z), T(u2.z - u0.z), T(u3.z - u0.z)};
    const T Ji[9] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w, g2.x};
    const T w = g2.y;
    if (!(w > T(0))) flag(status, AM_ENONPOS_J, e);
    T H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) H[i * 3 + j] = D[i * 3 + 0] * Ji[0 * 3 + j] + D[i * 3 + 1] * Ji[1 * 3 + j] + D[i * 3 + 2] * Ji[2 * 3 + j];
    T Q[9];
    if (MAT == kNeoHookean) {
        T tau[9];
        const double Jf = nh_kirchhoff<T>(T(lam), T(mu), H, tau);
        if (!(Jf > 0.0)) flag(status, AM_ENONPOS_J, e);
        T F[9], AF[9], K[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = H[k] + ((k % 4 == 0) ? T(1) : T(0));
        adj3(F, AF);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) K[i * 3 + j] = Ji[i * 3 + 0] * AF[0 * 3 + j] + Ji[i * 3 + 1] * AF[1 * 3 + j] + Ji[i * 3 + 2] * AF[2 * 3 + j];
        const T sc = sizeof(T) == 4 ? T(w * __frcp_rn(static_cast<float>(Jf))) : T(w / Jf);
        T ts[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j) ts[i * 3 + j] = ts[j * 3 + i] = sc * tau[i * 3 + j];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                Q[k * 3 + i] = K[k * 3 + 0] * ts[0 * 3 + i] + K[k * 3 + 1] * ts[1 * 3 + i] + K[k * 3 + 2] * ts[2 * 3 + i];
    } else {
        T P[9];
        stress<T>(MAT, T(lam), T(mu), H, P);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                Q[k * 3 + i] = w * (Ji[k * 3 + 0] * P[i * 3 + 0] + Ji[k * 3 + 1] * P[i * 3 + 1] + Ji[k * 3 + 2] * P[i * 3 + 2]);
    }
    // f_{k+1} = -Q_k ; f_0 = Q_0 + Q_1 + Q_2
    T f0[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) f0[i] += Q[k * 3 + i];
    if constexpr (!CHUNKS) {
        slots[pos[0]] = make4(f0[0], f0[1], f0[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) slots[pos[k + 1]] = make4(-Q[k * 3 + 0], -Q[k * 3 + 1], -Q[k * 3 + 2]);
    } else {
        // entry q = 32 a + lane, one component plane per coordinate
        __shared__ T ent[256 / 32][3][128];
        T(&st)[3][128] = ent[threadIdx.x >> 5];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            st[i][lane] = f0[i];
#pragma unroll
            for (int k = 0; k < 3; ++k) st[i][32 * (k + 1) + lane] = -Q[k * 3 + i];
        }
        __syncwarp();
        if (!live) return;  // the whole warp
        chunk_reduce<T, 4>(L, lane, [&](int q, T(&v)[3]) {
            v[0] = st[0][q];
            v[1] = st[1][q];
            v[2] = st[2][q];
        }, slots);
    }
}

// Chunked blocks outside the force (VJP, lumped mass): the per-element (per-patch) kernels
// write corner values to scratch[NN u + a] (unit u, corner a), and a warp per chunk sums
// them per distinct node with the chunk's plan into the block's slots.
template <int NN, typename B>
__global__ void __launch_bounds__(256) k_chunk_sum(B b, const double4* __restrict__ scratch,
                                                    double4* __restrict__ slots) {
    const int64_t ch = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x & 31);
    if (32 * ch >= b.chunk_units) return;  // the whole warp
    const ChunkLane<NN> L = chunk_lane<NN>(b, ch, lane, true);
    chunk_reduce<double, NN>(L, lane, [&](int q, double(&v)[3]) {
        const double4 x = scratch[NN * (32 * ch + (q & 31)) + (q >> 5)];
        v[0] = x.x;
        v[1] = x.y;
        v[2] = x.z;
    }, slots);
}

// ---------------------------------------------------------------------------
// Tet4 element patches (at most 6 tets on at most 8 nodes, e.g. the six tets of a
// split hex): one warp serves 5 patches. The warp first loads the 40 patch nodes
// into shared memory (FP64), then lane 6q+t computes tet t of patch q (30 busy
// lanes), then the 40 (patch, node) pairs sum, in tet order, the contributions of
// the patch's tets to their node and write one slot each.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int local_id(uint32_t packed, int k) { return (packed >> (8 * k)) & 0xFF; }

constexpr int kPatchesPerWarp = 5;
constexpr int kPatchTets = 6;

template <typename T, int MAT>
__global__ void __launch_bounds__(256) k_tet4_patch_force(GaussBlockDev b, const double4* __restrict__ X4,
                                                           const double4* __restrict__ U4,
                                                           vec4_t<T>* __restrict__ slots, int* status) {
    __shared__ double nodes[8][kPatchesPerWarp * 8][6];                  // X, u of the warp's patch nodes
    __shared__ T contrib[8][kPatchesPerWarp * kPatchTets][12];          // per tet: 4 nodes x 3
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int64_t p0 = (static_cast<int64_t>(blockIdx.x) * 8 + w) * kPatchesPerWarp;
    for (int q = lane; q < kPatchesPerWarp * 8; q += 32) {
        const int64_t p = p0 + q / 8;
        const int32_t n = p < b.num_patches ? b.patch_nodes[p * 8 + (q & 7)] : 0;
        const double4 x = X4[n], u = U4[n];
        double* d = nodes[w][q];
        d[0] = x.x;
        d[1] = x.y;
        d[2] = x.z;
        d[3] = u.x;
        d[4] = u.y;
        d[5] = u.z;
    }
    __syncwarp();
    const int pq = lane / kPatchTets, t = lane % kPatchTets;
    const int64_t p = p0 + pq;
    if (pq < kPatchesPerWarp && p < b.num_patches) {
        const int32_t e0 = b.patch_first[p];
        if (t < b.patch_first[p + 1] - e0) {
            const int64_t e = e0 + t;
            const uint32_t loc = b.patch_local[e];
            const double* n0 = nodes[w][pq * 8 + local_id(loc, 0)];
            const double* n1 = nodes[w][pq * 8 + local_id(loc, 1)];
            const double* n2 = nodes[w][pq * 8 + local_id(loc, 2)];
            const double* n3 = nodes[w][pq * 8 + local_id(loc, 3)];
            T J[9], D[9];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                J[i * 3 + 0] = T(n1[i] - n0[i]);
                J[i * 3 + 1] = T(n2[i] - n0[i]);
                J[i * 3 + 2] = T(n3[i] - n0[i]);
                D[i * 3 + 0] = T(n1[3 + i] - n0[3 + i]);
                D[i * 3 + 1] = T(n2[3 + i] - n0[3 + i]);
                D[i * 3 + 2] = T(n3[3 + i] - n0[3 + i]);
            }
            double lam, mu;
            element_lame(b, e, lam, mu);
            T f[12];
            tet4_forces<T, MAT>(J, D, lam, mu, f, e, status);
            T* c = contrib[w][lane];
#pragma unroll
            for (int k = 0; k < 12; ++k) c[k] = f[k];
        }
    }
    __syncwarp();
    for (int q = lane; q < kPatchesPerWarp * 8; q += 32) {
        const int64_t pp = p0 + q / 8;
        if (pp >= b.num_patches) continue;
        const int32_t pos = b.slot_pos[pp * 8 + (q & 7)];
        if (pos < 0) continue;
        const uint32_t gm = b.patch_gather[pp * 8 + (q & 7)];
        T fx = T(0), fy = T(0), fz = T(0);
        for (uint32_t m = gm & 0xFFu; m; m &= m - 1) {  // tets touching the node, ascending
            const int tt = __ffs(m) - 1;
            const T* c = contrib[w][(q / 8) * kPatchTets + tt] + ((gm >> (8 + 2 * tt)) & 3u) * 3;
            fx += c[0];
            fy += c[1];
            fz += c[2];
        }
        slots[pos] = make4(fx, fy, fz);
    }
}

// ---------------------------------------------------------------------------
// Tet4 patches that are split hexes: the six tets around the hex diagonal, which is
// patch-local nodes 0 and 3 in the order the patch builder produces; tet t = (0, a_t, b_t, 3) with
// (a_t, b_t) running round the ring 1-2-4-5-6-7-1. Two threads share a patch:
// thread r takes tets 3r..3r+2, the three around ring nodes R_r = (1, 2, 4, 5) for
// r = 0 and (5, 6, 7, 1) for r = 1, so its tet k is (0, R_r[k], R_r[k+1], 3) and
// both threads run the same code on six of the eight nodes. The pair's sums meet
// with three shuffles: node 0 and node 3 from both threads, and each thread's
// first ring node (1 or 5) from the other thread's last. The reference differences
// X_a - X_0 come from a per-patch table formed at set-up (coalesced loads in place of
// coordinate gathers, and no FP64 subtractions per step). Per thread this halves the
// unrolled code and holds 6 nodes' data and sums instead of 8; that is what fits the
// FP32 kernel in 72 registers at seven 128-thread blocks per SM and the FP64 one in
// 128 at four. On B200, against one thread per patch with gathered coordinates, the
// element kernel ran 55.8 -> 42.4 us (FP32) and 81.9 -> 57.3 us (FP64) per launch.
// ---------------------------------------------------------------------------
template <typename T>
constexpr int hex6_min_blocks() { return sizeof(T) == 4 ? 7 : 4; }
constexpr int kHex6Block = 128;

template <typename T, int MAT, bool CHUNKS>
__global__ void __launch_bounds__(kHex6Block, hex6_min_blocks<T>()) k_tet4_hex6_force(GaussBlockDev b, const double4* __restrict__ X4,
                                                          const double4* __restrict__ U4,
                                                          vec4_t<T>* __restrict__ slots, int* status) {
    const int64_t gt = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t p = gt >> 1;
    const int r = static_cast<int>(gt & 1);
    const bool valid = p < b.num_patches;
    const int64_t pp = valid ? p : 0;
    // Node data relative to patch node 0: X from the set-up table, u gathered in FP64
    // and differenced before the cast to T. The mesh data is read before the wait for
    // the previous kernel (which writes u), and the slot positions, needed only at the
    // end, are sent to L2 now (on B200 that took 2% off the FP32 kernel and 5% off the
    // FP64 one).
    const int4* pn4 = reinterpret_cast<const int4*>(b.patch_nodes + pp * 8);
    const int4 lo = pn4[0], hi = pn4[1];  // patch-local nodes 0-3 and 4-7
    if (CHUNKS) {
        // the lane's chunk plan (warp chunks over the half patches gt)
        const int64_t gu = gt < 2 * b.num_patches ? gt : 0;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.chunk_code + gu));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.chunk_rank + gu));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.chunk_pos + 4 * gu));
    } else {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.slot_pos + pp * 8));
    }
    const int32_t n0 = lo.x, n3 = lo.w;
    int32_t nr[4];
    nr[0] = r ? hi.y : lo.y;
    nr[1] = r ? hi.z : lo.z;
    nr[2] = r ? hi.w : hi.x;
    nr[3] = r ? lo.y : hi.y;
    T dx3[3], dxr[4][3], du3[3], dur[4][3];
    {
        // X_a - X_0, formed in FP64 (and rounded to T) once at set-up
        const T* dxp = (sizeof(T) == 4 ? reinterpret_cast<const T*>(b.patch_dx32)
                                       : reinterpret_cast<const T*>(b.patch_dx64)) + pp;
        const int64_t P = b.num_patches;
        const int ra[4] = {r ? 5 : 1, r ? 6 : 2, r ? 7 : 4, r ? 1 : 5};
#pragma unroll
        for (int i = 0; i < 3; ++i) dx3[i] = dxp[(6 + i) * P];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) dxr[k][i] = dxp[(3 * (ra[k] - 1) + i) * P];
    }
    pdl_trigger();
    pdl_wait();
    const double4 u0 = ld_dep(U4 + n0);
    {
        const double4 u = ld_dep(U4 + n3);
        du3[0] = T(u.x - u0.x);
        du3[1] = T(u.y - u0.y);
        du3[2] = T(u.z - u0.z);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double4 u = ld_dep(U4 + nr[k]);
        dur[k][0] = T(u.x - u0.x);
        dur[k][1] = T(u.y - u0.y);
        dur[k][2] = T(u.z - u0.z);
    }
    T acc0[3] = {T(0), T(0), T(0)}, acc3[3] = {T(0), T(0), T(0)}, accr[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) accr[k][0] = accr[k][1] = accr[k][2] = T(0);
    const int64_t e0 = static_cast<int64_t>(b.patch_first[pp]) + 3 * r;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        // columns of J and D: X_l - X_0 and u_l - u_0 for l = R_r[k], R_r[k+1], 3
        T J[9], D[9];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            J[i * 3 + 0] = dxr[k][i];
            J[i * 3 + 1] = dxr[k + 1][i];
            J[i * 3 + 2] = dx3[i];
            D[i * 3 + 0] = dur[k][i];
            D[i * 3 + 1] = dur[k + 1][i];
            D[i * 3 + 2] = du3[i];
        }
        const int64_t e = e0 + k;
        double lam, mu;
        element_lame(b, e, lam, mu);
        T f[12];
        tet4_forces<T, MAT>(J, D, lam, mu, f, valid ? e : 0, valid ? status : nullptr);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            acc0[i] += f[i];
            accr[k][i] += f[3 + i];
            accr[k + 1][i] += f[6 + i];
            acc3[i] += f[9 + i];
        }
    }
    // Both threads of a pair are in one warp (even lane first) and share `valid`.
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        acc0[i] += __shfl_xor_sync(kFull, acc0[i], 1);
        acc3[i] += __shfl_xor_sync(kFull, acc3[i], 1);
        accr[0][i] += __shfl_xor_sync(kFull, accr[3][i], 1);
    }
    if constexpr (!CHUNKS) {
        if (!valid) return;
        // thread 0 writes nodes 1, 2, 4 and 0; thread 1 nodes 5, 6, 7 and 3
        const int32_t* sp = b.slot_pos + p * 8;
        int32_t pos = sp[r ? 5 : 1];
        if (pos >= 0) slots[pos] = make4(accr[0][0], accr[0][1], accr[0][2]);
        pos = sp[r ? 6 : 2];
        if (pos >= 0) slots[pos] = make4(accr[1][0], accr[1][1], accr[1][2]);
        pos = sp[r ? 7 : 4];
        if (pos >= 0) slots[pos] = make4(accr[2][0], accr[2][1], accr[2][2]);
        pos = sp[r ? 3 : 0];
        if (pos >= 0) slots[pos] = r ? make4(acc3[0], acc3[1], acc3[2]) : make4(acc0[0], acc0[1], acc0[2]);
    } else {
        // the same four node sums as entries 32 a + lane (a: nodes 1, 2, 4, 0 or 5, 6, 7, 3),
        // summed per distinct node over the warp's 16 patches
        __shared__ T ent[kHex6Block / 32][3][128];
        T(&st)[3][128] = ent[threadIdx.x >> 5];
        const int lane = static_cast<int>(threadIdx.x & 31);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            st[i][lane] = accr[0][i];
            st[i][32 + lane] = accr[1][i];
            st[i][64 + lane] = accr[2][i];
            st[i][96 + lane] = r ? acc3[i] : acc0[i];
        }
        __syncwarp();
        const int64_t ch = gt >> 5;
        if (32 * ch >= 2 * b.num_patches) return;  // the whole warp
        const ChunkLane<4> L = chunk_lane<4>(b, ch, lane, true);
        chunk_reduce<T, 4>(L, lane, [&](int q, T(&v)[3]) {
            v[0] = st[0][q];
            v[1] = st[1][q];
            v[2] = st[2][q];
        }, slots);
    }
}

// Set-up for the split-hex kernels: X_a - X_0 in FP64 (and rounded to FP32) for
// patch-local nodes a = 1..7 of every patch (component-major).
__global__ void __launch_bounds__(256) k_hex6_patch_dx(const int32_t* __restrict__ patch_nodes, int64_t num_patches,
                                                       const double4* __restrict__ X4, float* __restrict__ dx32,
                                                       double* __restrict__ dx64) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= num_patches) return;
    const double4 x0 = X4[patch_nodes[p * 8]];
    for (int a = 1; a < 8; ++a) {
        const double4 x = X4[patch_nodes[p * 8 + a]];
        const double d[3] = {x.x - x0.x, x.y - x0.y, x.z - x0.z};
        for (int i = 0; i < 3; ++i) {
            dx64[(3 * (a - 1) + i) * num_patches + p] = d[i];
            dx32[(3 * (a - 1) + i) * num_patches + p] = static_cast<float>(d[i]);
        }
    }
}

// ---------------------------------------------------------------------------
// Hex8, 2x2x2 Gauss in the monomial basis of the trilinear element: one thread
// per element, everything in registers.
//
// Index the nodes by their corner bits (bit j set where xi_j = +1; node numbers
// 0,1,3,2,4,5,7,6 in that order). A nodal field v then reads
//   v(xi) = 1/8 sum_K C_K prod_{j in K} xi_j,   C_K = sum_a S_K(a) v_a,
// with S_K(a) = prod_{j in K} (+-1 by corner bit j of a): three butterfly stages
// give all eight C_K from the eight nodal values (hex_butterfly). The derivative
// d v / d xi_j at a Gauss point xi = c sigma (c = 1/sqrt 3, sigma in {+-1}^3) is
//   1/8 (C_j + c sigma_l C_jl + c sigma_m C_jm + c^2 sigma_l sigma_m C_jlm),
// three additions once the C's carry their powers of c. The nodal forces
//   f_a = -sum_g sum_j dN_a/dxi_j(g) Q_g[j,:],  Q_g = det J_g J_g^-1 P_g^T
// regroup the same way: f_a = -1/8 sum_K S_K(a) R_K with R_K summed over the Gauss
// points from the Q's, and an inverse butterfly turns the R_K into the eight nodal
// forces. The Jacobians are built from 8x the true derivatives (the 1/8 is
// dropped): H = G J^-1 is scale-free, Q = adj(J) P^T grows by 64, and the nodal
// sum applies -1/512 once. Per element this is about half the arithmetic of
// evaluating the 24 shape-function derivatives at every Gauss point.
// ---------------------------------------------------------------------------
// Gauss points unrolled two at a time: full unrolling raises the FP32 kernel to
// 168 registers and spills the FP64 one; two keeps both in registers.
constexpr int kHexGpUnroll = 2;

__host__ __device__ constexpr int hex_node_of_corner(int q) { return q ^ ((q >> 1) & 1); }

// v[K] <- sum_a S_K(a) v[a] (corner-bit order): C_0 in v[0], C_j in v[1 << j].
template <typename T>
__device__ __forceinline__ void hex_butterfly(T* v) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int p = 0; p < 8; ++p)
            if (!((p >> j) & 1)) {
                const int q = p | (1 << j);
                const T sum = v[p] + v[q], dif = v[q] - v[p];
                v[p] = sum;
                v[q] = dif;
            }
}

// F[a] <- sum_K S_K(a) R[K] (the transpose of hex_butterfly).
template <typename T>
__device__ __forceinline__ void hex_butterfly_t(T* v) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int p = 0; p < 8; ++p)
            if (!((p >> j) & 1)) {
                const int q = p | (1 << j);
                const T lo = v[p] - v[q], hi = v[p] + v[q];
                v[p] = lo;
                v[q] = hi;
            }
}

// Scale the butterfly output by the powers of c the Gauss-point formula needs.
template <typename T>
__device__ __forceinline__ void hex_scale_coeffs(T* v) {
    const T c = T(0.57735026918962576451), c2 = T(1.0 / 3.0);
    v[3] *= c;
    v[5] *= c;
    v[6] *= c;
    v[7] *= c2;
}

// 8 d v / d xi_j at the Gauss point of corner bits g (v scaled by hex_scale_coeffs).
template <typename T>
__device__ __forceinline__ T hex_dxi(const T* v, int j, int g) {
    const int l = (j + 1) % 3, m = (j + 2) % 3;
    const T sl = ((g >> l) & 1) ? T(1) : T(-1), sm = ((g >> m) & 1) ? T(1) : T(-1);
    return v[1 << j] + sl * v[(1 << j) | (1 << l)] + sm * (v[(1 << j) | (1 << m)] + sl * v[7]);
}

// R_K += the Gauss point's share (Q row j = d/dxi_j part), before the c powers.
template <typename T>
__device__ __forceinline__ void hex_accumulate_r(T (*R)[8], const T* Q, int g) {
    const T s0 = (g & 1) ? T(1) : T(-1), s1 = (g & 2) ? T(1) : T(-1), s2 = (g & 4) ? T(1) : T(-1);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T q0 = Q[0 * 3 + i], q1 = Q[1 * 3 + i], q2 = Q[2 * 3 + i];
        R[i][1] += q0;
        R[i][2] += q1;
        R[i][4] += q2;
        R[i][3] += s1 * q0 + s0 * q1;
        R[i][5] += s2 * q0 + s0 * q2;
        R[i][6] += s2 * q1 + s1 * q2;
        R[i][7] += s1 * s2 * q0 + s0 * s2 * q1 + s0 * s1 * q2;
    }
}

// Nodal values (corner-bit order) relative to node 0, FP64 difference then T. DEP: the
// values come from the previous kernel (coherent loads, see ld_dep).
template <typename T, bool DEP = false>
__device__ __forceinline__ void hex_load_rel(const double4* __restrict__ A, const int32_t* nd, T (*V)[8]) {
    const double4 a0 = DEP ? ld_dep(A + nd[0]) : ld_ro4(A + nd[0]);
    V[0][0] = V[1][0] = V[2][0] = T(0);
#pragma unroll
    for (int q = 1; q < 8; ++q) {
        const double4 a = DEP ? ld_dep(A + nd[hex_node_of_corner(q)]) : ld_ro4(A + nd[hex_node_of_corner(q)]);
        V[0][q] = T(a.x - a0.x);
        V[1][q] = T(a.y - a0.y);
        V[2][q] = T(a.z - a0.z);
    }
}

__device__ __forceinline__ void hex_conn(const GaussBlockDev& b, int64_t e, int32_t* nd) {
    const int4 c0 = reinterpret_cast<const int4*>(b.conn)[2 * e], c1 = reinterpret_cast<const int4*>(b.conn)[2 * e + 1];
    nd[0] = c0.x, nd[1] = c0.y, nd[2] = c0.z, nd[3] = c0.w, nd[4] = c1.x, nd[5] = c1.y, nd[6] = c1.z, nd[7] = c1.w;
}

// The FP32 kernel is held to 128 registers (four 128-thread blocks per SM); the
// FP64 one keeps its ~250 registers (forcing three blocks per SM spills and was
// slower on B200) and runs in 64-thread blocks.
template <typename T, int MAT>
__global__ void __launch_bounds__(sizeof(T) == 8 ? 64 : 128, sizeof(T) == 8 ? 1 : 4) k_hex8_force(GaussBlockDev b, const double4* __restrict__ X4,
                                                         const double4* __restrict__ U4,
                                                         vec4_t<T>* __restrict__ slots, int* status) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    int32_t nd[8];
    hex_conn(b, e, nd);
    T X[3][8], U[3][8];
    hex_load_rel(X4, nd, X);
    pdl_trigger();
    pdl_wait();
    hex_load_rel<T, true>(U4, nd, U);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        hex_butterfly(X[i]);
        hex_butterfly(U[i]);
        hex_scale_coeffs(X[i]);
        hex_scale_coeffs(U[i]);
    }
    double lam, mu;
    element_lame(b, e, lam, mu);
    T R[3][8];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) R[i][k] = T(0);
    bool bad = false;
#pragma unroll kHexGpUnroll
    for (int g = 0; g < 8; ++g) {
        T J[9], G[9], A[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                J[i * 3 + j] = hex_dxi(X[i], j, g);
                G[i * 3 + j] = hex_dxi(U[i], j, g);
            }
        adj3(J, A);
        const T det = J[0] * A[0] + J[1] * A[3] + J[2] * A[6];
        bad |= !(det > T(0));
        const T id = recip(det);
        T H[9], P[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                H[i * 3 + j] = (G[i * 3 + 0] * A[0 * 3 + j] + G[i * 3 + 1] * A[1 * 3 + j] + G[i * 3 + 2] * A[2 * 3 + j]) * id;
        T Q[9];
        if (MAT == kNeoHookean) {
            // Q = adj(J) P^T with P = tau F^-T and F = (J + G) J^-1 is adj(J + G) tau / det F
            // (the 8x scale of J and G cancels): no F^-1 and no P.
            T tau[9];
            const double Jf = nh_kirchhoff<T>(T(lam), T(mu), H, tau);
            bad |= !(Jf > 0.0);
            T Jc[9], Ac[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) Jc[k] = J[k] + G[k];
            adj3(Jc, Ac);
            const T sc = sizeof(T) == 4 ? T(__frcp_rn(static_cast<float>(Jf))) : T(1.0 / Jf);
            T ts[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = i; j < 3; ++j) ts[i * 3 + j] = ts[j * 3 + i] = sc * tau[i * 3 + j];
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    Q[k * 3 + i] = Ac[k * 3 + 0] * ts[0 * 3 + i] + Ac[k * 3 + 1] * ts[1 * 3 + i] + Ac[k * 3 + 2] * ts[2 * 3 + i];
        } else {
            stress<T>(MAT, T(lam), T(mu), H, P);
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    Q[k * 3 + i] = A[k * 3 + 0] * P[i * 3 + 0] + A[k * 3 + 1] * P[i * 3 + 1] + A[k * 3 + 2] * P[i * 3 + 2];
        }
        hex_accumulate_r(R, Q, g);
    }
    if (bad) flag(status, AM_ENONPOS_J, e);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R[i][0] = T(0);
        hex_scale_coeffs(R[i]);
        hex_butterfly_t(R[i]);
    }
    const T s = T(-1.0 / 512.0);
    const int4 p0 = reinterpret_cast<const int4*>(b.slot_pos)[2 * e], p1 = reinterpret_cast<const int4*>(b.slot_pos)[2 * e + 1];
    const int32_t pos[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
    for (int q = 0; q < 8; ++q) slots[pos[hex_node_of_corner(q)]] = make4(s * R[0][q], s * R[1][q], s * R[2][q]);
}

// ---------------------------------------------------------------------------
// Updated / semi-Lagrangian Gauss elements, FP64 (ComputeInternalForceGaussian.h:57-131 with
// ComputeInternalForceBase.h:158-174): shape-function gradients on the coordinates xc
// (current coordinates at the start of the step, or the semi formulation's reference
// coordinates), dH = inc^T B, H = dH + Href + dH Href, P(H); the force maps back through
// F_ref = I + Href: B F_ref and w / det F_ref. The element keeps one H (for Hex8 the last
// Gauss point's, as the reference's element field), which is also every Gauss point's Href.
// ---------------------------------------------------------------------------
// The element H arrays are component-major (component k of element e at k E + e), so that a
// warp's nine loads and stores are coalesced. They are written by the element kernel of the
// previous step: read after the wait for the predecessor, with coherent loads.
__device__ __forceinline__ void lagr_href(const GaussBlockDev& b, int64_t e, int32_t lagr, int rebase, double* hr) {
    const int64_t E = b.num_elems;
    const double* src = (lagr == 1 || rebase) ? b.hstate : b.href;
#pragma unroll
    for (int k = 0; k < 9; ++k) hr[k] = __ldcg(src + k * E + e);
    if (lagr == 2 && rebase) {
#pragma unroll
        for (int k = 0; k < 9; ++k) b.href[k * E + e] = hr[k];
    }
}
__device__ __forceinline__ void lagr_store_h(const GaussBlockDev& b, int64_t e, const double* H) {
#pragma unroll
    for (int k = 0; k < 9; ++k) b.hstate[k * b.num_elems + e] = H[k];
}

// H = dH + Href + dH Href
__device__ __forceinline__ void lagr_compose(const double* dH, const double* hr, double* H) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            H[i * 3 + j] = dH[i * 3 + j] + hr[i * 3 + j] +
                           (dH[i * 3 + 0] * hr[0 * 3 + j] + dH[i * 3 + 1] * hr[1 * 3 + j] + dH[i * 3 + 2] * hr[2 * 3 + j]);
}

// Pm = P F_ref^T / det F_ref, so that B P'^T w = (B F_ref) P^T (w / det F_ref).
__device__ __forceinline__ void lagr_pull(const double* hr, const double* P, double* Pm) {
    double Fr[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Fr[k] = hr[k] + ((k % 4 == 0) ? 1.0 : 0.0);
    const double idet = 1.0 / det3(Fr);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int m = 0; m < 3; ++m)
            Pm[i * 3 + m] = (P[i * 3 + 0] * Fr[m * 3 + 0] + P[i * 3 + 1] * Fr[m * 3 + 1] + P[i * 3 + 2] * Fr[m * 3 + 2]) * idet;
}

template <int MAT>
__global__ void __launch_bounds__(128) k_tet4_force_lagr(GaussBlockDev b, int32_t lagr, int rebase,
                                                          const double4* __restrict__ XC,
                                                          const double4* __restrict__ INC,
                                                          double4* __restrict__ slots, int* status) {
    pdl_trigger();
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    const int4 c = reinterpret_cast<const int4*>(b.conn)[e];
    const int32_t pos[4] = {b.slot_pos[4 * e], b.slot_pos[4 * e + 1], b.slot_pos[4 * e + 2], b.slot_pos[4 * e + 3]};
    pdl_wait();
    const double4 x0 = ld_dep(XC + c.x), x1 = ld_dep(XC + c.y), x2 = ld_dep(XC + c.z), x3 = ld_dep(XC + c.w);
    const double4 u0 = ld_dep(INC + c.x), u1 = ld_dep(INC + c.y), u2 = ld_dep(INC + c.z), u3 = ld_dep(INC + c.w);
    const double J[9] = {x1.x - x0.x, x2.x - x0.x, x3.x - x0.x, x1.y - x0.y, x2.y - x0.y,
                         x3.y - x0.y, x1.z - x0.z, x2.z - x0.z, x3.z - x0.z};
    const double D[9] = {u1.x - u0.x, u2.x - u0.x, u3.x - u0.x, u1.y - u0.y, u2.y - u0.y,
                         u3.y - u0.y, u1.z - u0.z, u2.z - u0.z, u3.z - u0.z};
    const double det = det3(J);
    if (!(det > 0.0)) flag(status, AM_ENONPOS_J, e);
    double Ji[9];
    cof_inv3(J, Ji, det);
    const double w = det / 6.0;
    double dH[9], hr[9], H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dH[i * 3 + j] = D[i * 3 + 0] * Ji[0 * 3 + j] + D[i * 3 + 1] * Ji[1 * 3 + j] + D[i * 3 + 2] * Ji[2 * 3 + j];
    lagr_href(b, e, lagr, rebase, hr);
    lagr_compose(dH, hr, H);
    lagr_store_h(b, e, H);
    double lam, mu;
    element_lame(b, e, lam, mu);
    double P[9], Pm[9];
    const double Jf = stress<double>(MAT, lam, mu, H, P);
    if (MAT == kNeoHookean && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, e);
    lagr_pull(hr, P, Pm);
    double f[12];
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double q = w * (Ji[k * 3 + 0] * Pm[i * 3 + 0] + Ji[k * 3 + 1] * Pm[i * 3 + 1] + Ji[k * 3 + 2] * Pm[i * 3 + 2]);
            f[(k + 1) * 3 + i] = -q;
            f[i] += q;
        }
    slots[pos[0]] = make4(f[0], f[1], f[2]);
    slots[pos[1]] = make4(f[3], f[4], f[5]);
    slots[pos[2]] = make4(f[6], f[7], f[8]);
    slots[pos[3]] = make4(f[9], f[10], f[11]);
}

template <int MAT>
__global__ void __launch_bounds__(64) k_hex8_force_lagr(GaussBlockDev b, int32_t lagr, int rebase,
                                                         const double4* __restrict__ XC,
                                                         const double4* __restrict__ INC,
                                                         double4* __restrict__ slots, int* status) {
    pdl_trigger();
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    int32_t nd[8];
    hex_conn(b, e, nd);
    double X[3][8], U[3][8];
    pdl_wait();
    hex_load_rel<double, true>(XC, nd, X);
    hex_load_rel<double, true>(INC, nd, U);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        hex_butterfly(X[i]);
        hex_butterfly(U[i]);
        hex_scale_coeffs(X[i]);
        hex_scale_coeffs(U[i]);
    }
    double lam, mu;
    element_lame(b, e, lam, mu);
    double hr[9];
    lagr_href(b, e, lagr, rebase, hr);
    double R[3][8];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) R[i][k] = 0.0;
    bool bad = false;
    for (int g = 0; g < 8; ++g) {
        double J[9], G[9], A[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                J[i * 3 + j] = hex_dxi(X[i], j, g);
                G[i * 3 + j] = hex_dxi(U[i], j, g);
            }
        adj3(J, A);
        const double det = J[0] * A[0] + J[1] * A[3] + J[2] * A[6];
        bad |= !(det > 0.0);
        const double id = 1.0 / det;
        double dH[9], H[9], P[9], Pm[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                dH[i * 3 + j] = (G[i * 3 + 0] * A[0 * 3 + j] + G[i * 3 + 1] * A[1 * 3 + j] + G[i * 3 + 2] * A[2 * 3 + j]) * id;
        lagr_compose(dH, hr, H);
        // The reference's last Gauss point (its node 7 sign pattern) is corner 6 here.
        if (g == 6) lagr_store_h(b, e, H);
        const double Jf = stress<double>(MAT, lam, mu, H, P);
        if (MAT == kNeoHookean) bad |= !(Jf > 0.0);
        lagr_pull(hr, P, Pm);
        double Q[9];
#pragma unroll
        for (int kk = 0; kk < 3; ++kk)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                Q[kk * 3 + i] = A[kk * 3 + 0] * Pm[i * 3 + 0] + A[kk * 3 + 1] * Pm[i * 3 + 1] + A[kk * 3 + 2] * Pm[i * 3 + 2];
        hex_accumulate_r(R, Q, g);
    }
    if (bad) flag(status, AM_ENONPOS_J, e);
    int32_t pos[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) pos[a] = b.slot_pos[8 * e + a];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R[i][0] = 0.0;
        hex_scale_coeffs(R[i]);
        hex_butterfly_t(R[i]);
    }
    const double sc = -1.0 / 512.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) slots[pos[hex_node_of_corner(q)]] = make4(sc * R[0][q], sc * R[1][q], sc * R[2][q]);
}

// ---------------------------------------------------------------------------
// Smoothed / RKPM cells (ComputeInternalForceSmoothedCell.h:416-442, no F-bar):
// H = sum_k u_k (x) b_k ; P(H) ; f_k = -V b_k P^T written to the cell's slots.
// The mixed path subtracts the first entry's displacement (partition of nullity
// makes H invariant) before casting to FP32.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ const T* cell_grads(const CellBlockDev& b);
template <>
__device__ __forceinline__ const double* cell_grads<double>(const CellBlockDev& b) { return b.grads64; }
template <>
__device__ __forceinline__ const float* cell_grads<float>(const CellBlockDev& b) { return b.grads32; }

template <typename T, int MAT>
__global__ void __launch_bounds__(256) k_cell_force_thread(CellBlockDev b, const double4* __restrict__ U4,
                                                            vec4_t<T>* __restrict__ slots, int* status) {
    pdl_trigger();
    pdl_wait();
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= b.num_cells) return;
    const int32_t s0 = b.ptr[c], s1 = b.ptr[c + 1];
    if (s1 <= s0) return;
    const T* gr = cell_grads<T>(b);
    const bool diff = sizeof(T) == 4;
    const double4 ur = ld_dep(U4 + b.nodes[s0]);
    T H[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) H[k] = T(0);
    for (int32_t s = s0; s < s1; ++s) {
        const double4 u = ld_dep(U4 + b.nodes[s]);
        const T du[3] = {T(diff ? u.x - ur.x : u.x), T(diff ? u.y - ur.y : u.y), T(diff ? u.z - ur.z : u.z)};
        const T gg[3] = {gr[3 * s], gr[3 * s + 1], gr[3 * s + 2]};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) H[i * 3 + j] += du[i] * gg[j];
    }
    double lam, mu;
    element_lame(b, c, lam, mu);
    T P[9];
    const double Jf = stress<T>(MAT, T(lam), T(mu), H, P);
    if (MAT == kNeoHookean && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, c);
    const T V = T(b.volumes[c]);
    for (int32_t s = s0; s < s1; ++s) {
        const T gg[3] = {gr[3 * s], gr[3 * s + 1], gr[3 * s + 2]};
        T f[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) f[i] = (gg[0] * P[i * 3 + 0] + gg[1] * P[i * 3 + 1] + gg[2] * P[i * 3 + 2]) * -V;
        slots[b.slot_pos[s]] = make4(f[0], f[1], f[2]);
    }
}

// LPC lanes per cell (a power of two up to 32): the group strides over the cell's
// entries, combines its partial H by a butterfly over the group (every lane then
// holds the same H and P), and each lane writes the forces of its own entries.
// Narrow groups keep the lanes busy on cells of a few tens of entries and repeat
// the stress update on fewer lanes.
template <typename T, int MAT, int LPC>
__global__ void __launch_bounds__(256) k_cell_force_group(CellBlockDev b, const double4* __restrict__ U4,
                                                          vec4_t<T>* __restrict__ slots, int* status) {
    pdl_trigger();
    pdl_wait();
    const int64_t gt = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t c = gt / LPC;
    const int r = static_cast<int>(threadIdx.x % LPC);
    const unsigned gmask = LPC == 32 ? kFull : (((1u << LPC) - 1u) << ((threadIdx.x & 31) & ~(LPC - 1)));
    const bool valid = c < b.num_cells;
    const int32_t s0 = valid ? b.ptr[c] : 0, s1 = valid ? b.ptr[c + 1] : 0;
    const T* gr = cell_grads<T>(b);
    const bool diff = sizeof(T) == 4;
    const double4 ur = s1 > s0 ? ld_dep(U4 + b.nodes[s0]) : make_double4(0.0, 0.0, 0.0, 0.0);
    T H[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) H[k] = T(0);
    for (int32_t s = s0 + r; s < s1; s += LPC) {
        const double4 u = ld_dep(U4 + b.nodes[s]);
        const T du[3] = {T(diff ? u.x - ur.x : u.x), T(diff ? u.y - ur.y : u.y), T(diff ? u.z - ur.z : u.z)};
        const T gg[3] = {gr[3 * s], gr[3 * s + 1], gr[3 * s + 2]};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) H[i * 3 + j] += du[i] * gg[j];
    }
    // Butterfly over the group: fixed pairing, identical result on every lane.
#pragma unroll
    for (int off = LPC / 2; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 9; ++k) H[k] += __shfl_xor_sync(gmask, H[k], off);
    if (!valid || s1 <= s0) return;
    double lam, mu;
    element_lame(b, c, lam, mu);
    T P[9];
    const double Jf = stress<T>(MAT, T(lam), T(mu), H, P);
    if (r == 0 && MAT == kNeoHookean && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, c);
    const T V = T(b.volumes[c]);
    for (int32_t s = s0 + r; s < s1; s += LPC) {
        const T gg[3] = {gr[3 * s], gr[3 * s + 1], gr[3 * s + 2]};
        T f[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) f[i] = (gg[0] * P[i * 3 + 0] + gg[1] * P[i * 3 + 1] + gg[2] * P[i * 3 + 2]) * -V;
        slots[b.slot_pos[s]] = make4(f[0], f[1], f[2]);
    }
}

__device__ __forceinline__ void warp_sum2(double& x, double& y) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        x += __shfl_xor_sync(kFull, x, off);
        y += __shfl_xor_sync(kFull, y, off);
    }
}

// ---------------------------------------------------------------------------
// Cell-stress form of the generic cell path (ComputeInternalForceSmoothedCell.h:416-442
// with the scatter turned into a gather). The cell kernel writes per cell the nine values
// M_c = -V_c P_c; the gather kernel then forms, for every node the block touches,
// f_n = sum over its entries (c, b) of M_c b, in a fixed order, into the node's one slot.
//
// Both kernels run a warp per octet of eight consecutive items (cells, or nodes): lane
// 8k + j takes item j of the octet and rows k, k + 4, ... of the octet's row list, so a
// quarter-warp (the eight lanes the load unit serves together) reads one row of all eight
// items. Set-up aligns the rows by offset (partner index minus item index) where that
// pads little, so that on a locality-numbered mesh a quarter-warp's eight gathers hit
// eight consecutive nodes or cells; rows hold packed records (gradient in x, y, z; the
// partner index in w, -1 for padding), one 16-byte (FP32) or 32-byte (FP64) load each.
// Per entry this reads a record twice (32 B mixed) instead of a record, a slot position
// and a slot written and read back (52 B), and the per-node sums need no slot per entry.
// M is stored as three component arrays (values 0-3, 4-7 and 8 of every cell), so that
// the eight lanes of a quarter-warp read contiguous pieces.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t rec_index(const float4& r) { return __float_as_int(r.w); }
__device__ __forceinline__ int32_t rec_index(const double4& r) { return static_cast<int32_t>(__double_as_longlong(r.w)); }
// Records are written once at set-up: the read-only path.
__device__ __forceinline__ float4 ld_rec(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ld_rec(const double4* p) { return ld_ro4(p); }
template <typename T>
__device__ __forceinline__ vec4_t<T> pad_rec() {
    vec4_t<T> z;
    z.x = z.y = z.z = T(0);
    if constexpr (sizeof(T) == 4) {
        z.w = __int_as_float(-1);
    } else {
        z.w = __longlong_as_double(-1LL);
    }
    return z;
}
template <typename T>
__device__ __forceinline__ const vec4_t<T>* cell_recs(const CellBlockDev& b);
template <>
__device__ __forceinline__ const float4* cell_recs<float>(const CellBlockDev& b) { return b.orec32; }
template <>
__device__ __forceinline__ const double4* cell_recs<double>(const CellBlockDev& b) { return b.orec64; }
template <typename T>
__device__ __forceinline__ const vec4_t<T>* node_recs(const CellBlockDev& b);
template <>
__device__ __forceinline__ const float4* node_recs<float>(const CellBlockDev& b) { return b.nrec32; }
template <>
__device__ __forceinline__ const double4* node_recs<double>(const CellBlockDev& b) { return b.nrec64; }

// Part k (0, 1, 2) of M_c in the component arrays of a block of E cells.
template <typename T>
__device__ __forceinline__ void store_cell_matrix(T* M, int64_t E, int64_t c, int k, const T (&m)[9]) {
    if (k == 0) {
        vec4_t<T> v;
        v.x = m[0], v.y = m[1], v.z = m[2], v.w = m[3];
        reinterpret_cast<vec4_t<T>*>(M)[c] = v;
    } else if (k == 1) {
        vec4_t<T> v;
        v.x = m[4], v.y = m[5], v.z = m[6], v.w = m[7];
        reinterpret_cast<vec4_t<T>*>(M + 4 * E)[c] = v;
    } else if (k == 2) {
        M[8 * E + c] = m[8];
    }
}
template <typename T>
__device__ __forceinline__ void load_cell_matrix(const T* M, int64_t E, int32_t c, T (&m)[9]) {
    const vec4_t<T> a = ld_dep(reinterpret_cast<const vec4_t<T>*>(M) + c);
    const vec4_t<T> b = ld_dep(reinterpret_cast<const vec4_t<T>*>(M + 4 * E) + c);
    m[0] = a.x, m[1] = a.y, m[2] = a.z, m[3] = a.w, m[4] = b.x, m[5] = b.y, m[6] = b.z, m[7] = b.w;
    m[8] = __ldca(M + 8 * E + c);
}

// Cell octets: H over the rows (UNR rows per lane in flight: the batch's displacement
// gathers issued together, the next batch's records loaded while they are in flight),
// combined over the four lanes of a cell, P(H), and M_c written by lanes k = 0, 1, 2.
template <typename T, int MAT, int UNR, bool FBAR, int G>
__global__ void __launch_bounds__(256) k_cell_stress(CellBlockDev b, const double4* __restrict__ U4, T* __restrict__ M,
                                                     int* status) {
    constexpr int L = 32 / G;  // lanes per cell
    pdl_trigger();
    const int64_t o = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x & 31), j = lane % G, k = lane / G;
    const int64_t c = G * o + j;
    const bool valid = c < b.num_cells;
    const bool live = o < b.num_octets;
    const int32_t r0 = live ? b.o_ptr[o] : 0, rows = live ? b.o_ptr[o + 1] - r0 : 0;
    const vec4_t<T>* rec = cell_recs<T>(b) + G * static_cast<int64_t>(r0) + j;
    const int32_t ref = valid ? b.c_ref[c] : -1;
    const bool diff = sizeof(T) == 4;
    vec4_t<T> rr[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) rr[u] = k + L * u < rows ? ld_rec(rec + G * (k + L * u)) : pad_rec<T>();
    pdl_wait();
    const double4 ur = ref >= 0 ? ld_dep(U4 + ref) : make_double4(0.0, 0.0, 0.0, 0.0);
    T H[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) H[q] = T(0);
#pragma unroll 1
    for (int32_t r = k; r < rows; r += L * UNR) {
        double4 uu[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int32_t n = rec_index(rr[u]);
            uu[u] = n >= 0 ? ld_dep(U4 + n) : ur;
        }
        vec4_t<T> nx[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int32_t rn = r + L * (UNR + u);
            nx[u] = rn < rows ? ld_rec(rec + G * rn) : pad_rec<T>();
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const T du[3] = {T(diff ? uu[u].x - ur.x : uu[u].x), T(diff ? uu[u].y - ur.y : uu[u].y),
                             T(diff ? uu[u].z - ur.z : uu[u].z)};
            const T gg[3] = {rr[u].x, rr[u].y, rr[u].z};
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) H[a * 3 + d] += du[a] * gg[d];
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) rr[u] = nx[u];
    }
    // the L lanes of a cell (j, j + G, ...): fixed pairing, same H on each
#pragma unroll
    for (int off = G; off < 32; off <<= 1)
#pragma unroll
        for (int q = 0; q < 9; ++q) H[q] += __shfl_xor_sync(kFull, H[q], off);
    if (!valid) return;
    if constexpr (FBAR) {
        // F-bar subcells: H goes to the matrix array (zero for a subcell without entries);
        // the per-vertex kernel forms M from it
        store_cell_matrix<T>(M, b.num_cells, c, k, H);
        return;
    }
    if (ref < 0) return;
    double lam, mu;
    element_lame(b, c, lam, mu);
    T P[9];
    const double Jf = stress<T>(MAT, T(lam), T(mu), H, P);
    if (k == 0 && MAT == kNeoHookean && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, c);
    const T V = T(b.volumes[c]);
    T m[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = -V * P[q];
    store_cell_matrix<T>(M, b.num_cells, c, k, m);
}

// F-bar in the cell-stress form (ComputeInternalForceSmoothedCell.h:354-413): a warp per
// cell (group of at most 32 subcells), a lane per subcell. H of each subcell comes from the
// octet kernel; J-bar = sum J V / sum V over the cell, the subcell's F-bar stress and the
// dual pressure as in k_fbar_fused, and M = -V P replaces H in the matrix array for the
// node-major gather.
template <typename T, int MAT>
__global__ void __launch_bounds__(256) k_fbar_cell_stress(CellBlockDev b, T* __restrict__ M, int* status) {
    pdl_trigger();
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const bool gvalid = g < b.num_groups;
    const int64_t s0 = gvalid ? b.group_ptr[g] : 0;
    const int ns = gvalid ? static_cast<int>(b.group_ptr[g + 1] - s0) : 0;
    const bool own = lane < ns;
    const int64_t s = s0 + lane;
    const double V = own ? b.volumes[s] : 0.0;
    double lam = 0.0, mu = 0.0;
    if (own) element_lame(b, s, lam, mu);
    pdl_wait();
    T H[9];
    double J = 1.0;
    if (own) {
        load_cell_matrix(M, b.num_cells, static_cast<int32_t>(s), H);
        J = det_ap_im1(H) + 1.0;
        if (!(J > 0.0)) flag(status, AM_ENONPOS_J, s);
    }
    double jv = own ? J * V : 0.0, vol = own ? V : 0.0;
    warp_sum2(jv, vol);
    const double Jbar = ns > 0 ? jv / vol : 1.0;
    double js = 1.0, pd = 0.0, unused = 0.0;
    T Pb[9];
    if (own) {
        const double ratio = Jbar / J;
        js = cbrt(ratio);
        T Hb[9];
        if (fabs(ratio - 1.0) < 3.0 * 2.2204460492503131e-16) {
#pragma unroll
            for (int m = 0; m < 9; ++m) Hb[m] = H[m];
        } else {
#pragma unroll
            for (int m = 0; m < 9; ++m) Hb[m] = H[m] * T(js);
            Hb[0] += T(js - 1.0);
            Hb[4] += T(js - 1.0);
            Hb[8] += T(js - 1.0);
        }
        const double Jb = stress<T>(MAT, T(lam), T(mu), Hb, Pb);
        if (MAT == kNeoHookean && !(Jb > 0.0)) flag(status, AM_ENONPOS_J, s);
        double pf = static_cast<double>(Pb[0] + Pb[4] + Pb[8]);
#pragma unroll
        for (int m = 0; m < 9; ++m) pf += static_cast<double>(Pb[m] * H[m]);
        pd = js / (3.0 * Jbar) * V * pf;
    }
    warp_sum2(pd, unused);
    if (!own) return;
    pd /= vol;
    T F[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) F[m] = H[m];
    F[0] += T(1);
    F[4] += T(1);
    F[8] += T(1);
    double pf = 0.0;
#pragma unroll
    for (int m = 0; m < 9; ++m) pf += static_cast<double>(Pb[m] * F[m]);
    const T scal = T(pd - js / (3.0 * J) * pf);
    T A[9];
    adj3(F, A);
    const T Vt = T(V);
    T m[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) m[i * 3 + j] = -Vt * (Pb[i * 3 + j] * T(js) + scal * A[j * 3 + i]);
#pragma unroll
    for (int k = 0; k < 3; ++k) store_cell_matrix<T>(M, b.num_cells, s, k, m);
}

// Node octets: f = sum of M_c b over the rows in FP64 (products in the slot precision),
// combined over the node's four lanes, written to the node's slot by lane k = 0.
template <typename T, int UNR, int G>
__global__ void __launch_bounds__(256) k_cell_gather(CellBlockDev b, const T* __restrict__ M, vec4_t<T>* __restrict__ slots) {
    constexpr int L = 32 / G;  // lanes per node
    pdl_trigger();
    const int64_t o = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x & 31), j = lane % G, k = lane / G;
    const int64_t i = G * o + j;
    const bool valid = i < b.t_count;
    const bool live = o < b.num_node_octets;
    const int32_t r0 = live ? b.n_ptr[o] : 0, rows = live ? b.n_ptr[o + 1] - r0 : 0;
    const int32_t pos = valid && k == 0 ? b.slot_pos[i] : 0;
    const vec4_t<T>* rec = node_recs<T>(b) + G * static_cast<int64_t>(r0) + j;
    vec4_t<T> rr[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) rr[u] = k + L * u < rows ? ld_rec(rec + G * (k + L * u)) : pad_rec<T>();
    pdl_wait();
    double f[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
    for (int32_t r = k; r < rows; r += L * UNR) {
        T mm[UNR][9];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int32_t c = rec_index(rr[u]);
            if (c >= 0) {
                load_cell_matrix(M, b.num_cells, c, mm[u]);
            } else {
#pragma unroll
                for (int q = 0; q < 9; ++q) mm[u][q] = T(0);
            }
        }
        vec4_t<T> nx[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int32_t rn = r + L * (UNR + u);
            nx[u] = rn < rows ? ld_rec(rec + G * rn) : pad_rec<T>();
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
                f[a] += static_cast<double>(mm[u][3 * a] * rr[u].x + mm[u][3 * a + 1] * rr[u].y + mm[u][3 * a + 2] * rr[u].z);
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) rr[u] = nx[u];
    }
#pragma unroll
    for (int off = G; off < 32; off <<= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) f[a] += __shfl_xor_sync(kFull, f[a], off);
    if (valid && k == 0) slots[pos] = make4(T(f[0]), T(f[1]), T(f[2]));
}

// ---------------------------------------------------------------------------
// Four-entry cells grouped as split hexes (a tet mesh's element smoothing cells):
// the split-hex Tet4 kernel's pair split, with each cell's stored gradients b_e and
// volume V in place of the tet's own geometry. Entry e of the patch's tet t sits on
// local node (0, a_t, b_t, 3)[e]; H = sum_e (u_e - u_0) (x) b_e, P(H), and the entry
// forces -V b_e P^T are summed per patch node and written to its slot.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void load_cell12(const T* p, T* g);
template <>
__device__ __forceinline__ void load_cell12<float>(const float* p, float* g) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 v = __ldg(q + k);
        g[4 * k] = v.x;
        g[4 * k + 1] = v.y;
        g[4 * k + 2] = v.z;
        g[4 * k + 3] = v.w;
    }
}
template <>
__device__ __forceinline__ void load_cell12<double>(const double* p, double* g) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double2 v = __ldg(q + k);
        g[2 * k] = v.x;
        g[2 * k + 1] = v.y;
    }
}

template <typename T, int MAT, bool CHUNKS>
__global__ void __launch_bounds__(kHex6Block, hex6_min_blocks<T>()) k_cell_hex6_force(CellBlockDev b, const double4* U4,
                                                                                    vec4_t<T>* slots, int* status) {
    const int64_t gt = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t p = gt >> 1;
    const int r = static_cast<int>(gt & 1);
    const bool valid = p < b.num_patches;
    const int64_t pp = valid ? p : 0;
    const int4* pn4 = reinterpret_cast<const int4*>(b.patch_nodes + pp * 8);
    const int4 lo = pn4[0], hi = pn4[1];
    if (CHUNKS) {
        // the lane's chunk plan (warp chunks over the half patches gt)
        const int64_t gu = gt < 2 * b.num_patches ? gt : 0;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.chunk_code + gu));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.chunk_rank + gu));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.chunk_pos + 4 * gu));
    } else {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(b.slot_pos + pp * 8));
    }
    const int32_t n0 = lo.x, n3 = lo.w;
    int32_t nr[4];
    nr[0] = r ? hi.y : lo.y;
    nr[1] = r ? hi.z : lo.z;
    nr[2] = r ? hi.w : hi.x;
    nr[3] = r ? lo.y : hi.y;
    const int64_t c0 = static_cast<int64_t>(b.patch_first[pp]) + 3 * r;
    pdl_trigger();
    pdl_wait();
    T du3[3], dur[4][3];
    const double4 u0 = ld_dep(U4 + n0);
    {
        const double4 u = ld_dep(U4 + n3);
        du3[0] = T(u.x - u0.x);
        du3[1] = T(u.y - u0.y);
        du3[2] = T(u.z - u0.z);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double4 u = ld_dep(U4 + nr[k]);
        dur[k][0] = T(u.x - u0.x);
        dur[k][1] = T(u.y - u0.y);
        dur[k][2] = T(u.z - u0.z);
    }
    T acc0[3] = {T(0), T(0), T(0)}, acc3[3] = {T(0), T(0), T(0)}, accr[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) accr[k][0] = accr[k][1] = accr[k][2] = T(0);
    const T* gr = cell_grads<T>(b);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int64_t c = c0 + k;
        T g[12];  // b_e for the entries on local nodes 0, R_r[k], R_r[k+1], 3
        load_cell12<T>(gr + 12 * c, g);
        T H[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) H[i * 3 + j] = dur[k][i] * g[3 + j] + dur[k + 1][i] * g[6 + j] + du3[i] * g[9 + j];
        double lam, mu;
        element_lame(b, c, lam, mu);
        T P[9];
        const double Jf = stress<T>(MAT, T(lam), T(mu), H, P);
        if (valid && MAT == kNeoHookean && !(Jf > 0.0)) flag(status, AM_ENONPOS_J, c);
        const T V = T(b.volumes[c]);
        T f[4][3];
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                f[e][i] = (g[3 * e] * P[i * 3 + 0] + g[3 * e + 1] * P[i * 3 + 1] + g[3 * e + 2] * P[i * 3 + 2]) * -V;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            acc0[i] += f[0][i];
            accr[k][i] += f[1][i];
            accr[k + 1][i] += f[2][i];
            acc3[i] += f[3][i];
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        acc0[i] += __shfl_xor_sync(kFull, acc0[i], 1);
        acc3[i] += __shfl_xor_sync(kFull, acc3[i], 1);
        accr[0][i] += __shfl_xor_sync(kFull, accr[3][i], 1);
    }
    if constexpr (!CHUNKS) {
        if (!valid) return;
        const int32_t* sp = b.slot_pos + p * 8;
        int32_t pos = sp[r ? 5 : 1];
        if (pos >= 0) slots[pos] = make4(accr[0][0], accr[0][1], accr[0][2]);
        pos = sp[r ? 6 : 2];
        if (pos >= 0) slots[pos] = make4(accr[1][0], accr[1][1], accr[1][2]);
        pos = sp[r ? 7 : 4];
        if (pos >= 0) slots[pos] = make4(accr[2][0], accr[2][1], accr[2][2]);
        pos = sp[r ? 3 : 0];
        if (pos >= 0) slots[pos] = r ? make4(acc3[0], acc3[1], acc3[2]) : make4(acc0[0], acc0[1], acc0[2]);
    } else {
        // as in k_tet4_hex6_force: the four node sums summed per distinct node over the warp
        __shared__ T ent[kHex6Block / 32][3][128];
        T(&st)[3][128] = ent[threadIdx.x >> 5];
        const int lane = static_cast<int>(threadIdx.x & 31);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            st[i][lane] = accr[0][i];
            st[i][32 + lane] = accr[1][i];
            st[i][64 + lane] = accr[2][i];
            st[i][96 + lane] = r ? acc3[i] : acc0[i];
        }
        __syncwarp();
        const int64_t ch = gt >> 5;
        if (32 * ch >= 2 * b.num_patches) return;  // the whole warp
        const ChunkLane<4> L = chunk_lane<4>(b, ch, lane, true);
        chunk_reduce<T, 4>(L, lane, [&](int q, T(&v)[3]) {
            v[0] = st[0][q];
            v[1] = st[1][q];
            v[2] = st[2][q];
        }, slots);
    }
}

// ---------------------------------------------------------------------------
// F-bar smoothed cells (ForEachCellComputeForceFbar, ComputeInternalForceSmoothedCell.h:
// 354-413) in three passes over the scratch fb (kFbarStride values per subcell):
//   k_fbar_h     per subcell: H_s = sum_k u_k (x) b_k, J_s = DetApIm1(H_s) + 1 -> fb[0..9]
//   k_fbar_cell  per cell (kFbarLanes lanes striding over its subcells):
//                Jbar = sum J_s V_s / sum V_s; Hbar_s = js H_s + (js - 1) I with
//                js = cbrt(Jbar / J_s) (H_s itself when Jbar / J_s is within 3 eps of 1);
//                Pbar_s = P(Hbar_s); the dual pressure p = sum js / (3 Jbar) V_s Pbar_s : F_s
//                / sum V_s; P_s = js Pbar_s + (p - js / (3 J_s) Pbar_s : F_s) cof(F_s) -> fb[10..18]
//   k_fbar_force per subcell: f_k = -V_s b_k P_s^T into the subcell's slots.
// Lane sums combine by fixed butterflies, so the result does not depend on scheduling.
// The scalar chain (Jbar, js, p) is FP64 in both precisions.
// ---------------------------------------------------------------------------
constexpr int kFbarLanes = 8;

template <typename T, int LPC>
__global__ void __launch_bounds__(256) k_fbar_h(CellBlockDev b, const double4* __restrict__ U4, int* status) {
    const int64_t c = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPC;
    const int r = static_cast<int>(threadIdx.x % LPC);
    const unsigned gmask = LPC == 32 ? kFull : (((1u << LPC) - 1u) << ((threadIdx.x & 31) & ~(LPC - 1)));
    const bool valid = c < b.num_cells;
    const int32_t s0 = valid ? b.ptr[c] : 0, s1 = valid ? b.ptr[c + 1] : 0;
    const T* gr = cell_grads<T>(b);
    const bool diff = sizeof(T) == 4;
    const double4 ur = s1 > s0 ? ld_dep(U4 + b.nodes[s0]) : make_double4(0.0, 0.0, 0.0, 0.0);
    T H[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) H[k] = T(0);
    for (int32_t s = s0 + r; s < s1; s += LPC) {
        const double4 u = ld_dep(U4 + b.nodes[s]);
        const T du[3] = {T(diff ? u.x - ur.x : u.x), T(diff ? u.y - ur.y : u.y), T(diff ? u.z - ur.z : u.z)};
        const T gg[3] = {gr[3 * s], gr[3 * s + 1], gr[3 * s + 2]};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) H[i * 3 + j] += du[i] * gg[j];
    }
#pragma unroll
    for (int off = LPC / 2; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 9; ++k) H[k] += __shfl_xor_sync(gmask, H[k], off);
    if (!valid || r != 0) return;
    const double J = det_ap_im1(H) + 1.0;
    if (!(J > 0.0)) flag(status, AM_ENONPOS_J, c);
    T* o = static_cast<T*>(b.fbar) + kFbarStride * c;
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = H[k];
    o[9] = T(J);
}

__device__ __forceinline__ void fbar_combine(double& x, double& y) {
#pragma unroll
    for (int off = kFbarLanes / 2; off > 0; off >>= 1) {
        x += __shfl_xor_sync(kFull, x, off);
        y += __shfl_xor_sync(kFull, y, off);
    }
}

template <typename T, int MAT>
__global__ void __launch_bounds__(256) k_fbar_cell(CellBlockDev b, int* status) {
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kFbarLanes;
    const int r = static_cast<int>(threadIdx.x % kFbarLanes);
    const bool valid = g < b.num_groups;
    const int64_t s0 = valid ? b.group_ptr[g] : 0, s1 = valid ? b.group_ptr[g + 1] : 0;
    T* fb = static_cast<T*>(b.fbar);
    double jv = 0.0, vol = 0.0;
    for (int64_t s = s0 + r; s < s1; s += kFbarLanes) {
        jv += static_cast<double>(fb[kFbarStride * s + 9]) * b.volumes[s];
        vol += b.volumes[s];
    }
    fbar_combine(jv, vol);
    const double Jbar = s1 > s0 ? jv / vol : 1.0;
    double pd = 0.0, unused = 0.0;
    for (int64_t s = s0 + r; s < s1; s += kFbarLanes) {
        T* o = fb + kFbarStride * s;
        T H[9], Hb[9], Pb[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) H[k] = o[k];
        const double ratio = Jbar / static_cast<double>(o[9]);
        const double js = cbrt(ratio);
        if (fabs(ratio - 1.0) < 3.0 * 2.2204460492503131e-16) {
#pragma unroll
            for (int k = 0; k < 9; ++k) Hb[k] = H[k];
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k) Hb[k] = H[k] * T(js);
            Hb[0] += T(js - 1.0);
            Hb[4] += T(js - 1.0);
            Hb[8] += T(js - 1.0);
        }
        double lam, mu;
        element_lame(b, s, lam, mu);
        const double Jb = stress<T>(MAT, T(lam), T(mu), Hb, Pb);
        if (MAT == kNeoHookean && !(Jb > 0.0)) flag(status, AM_ENONPOS_J, s);
        double pf = static_cast<double>(Pb[0] + Pb[4] + Pb[8]);
#pragma unroll
        for (int k = 0; k < 9; ++k) pf += static_cast<double>(Pb[k] * H[k]);
        pd += js / (3.0 * Jbar) * b.volumes[s] * pf;
#pragma unroll
        for (int k = 0; k < 9; ++k) o[10 + k] = Pb[k];
    }
    fbar_combine(pd, unused);
    if (s1 <= s0) return;
    pd /= vol;
    for (int64_t s = s0 + r; s < s1; s += kFbarLanes) {
        T* o = fb + kFbarStride * s;
        T F[9], Pb[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            F[k] = o[k];
            Pb[k] = o[10 + k];
        }
        F[0] += T(1);
        F[4] += T(1);
        F[8] += T(1);
        const double J = static_cast<double>(o[9]);
        const double js = cbrt(Jbar / J);
        double pf = 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) pf += static_cast<double>(Pb[k] * F[k]);
        // (p - js / (3 J) Pbar : F) J F^-T = (p - js / (3 J) Pbar : F) cof(F)
        const T scal = T(pd - js / (3.0 * J) * pf);
        T A[9];
        adj3(F, A);  // cof(F) = adj(F)^T
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) o[10 + i * 3 + j] = Pb[i * 3 + j] * T(js) + scal * A[j * 3 + i];
    }
}

template <typename T, int LPC>
__global__ void __launch_bounds__(256) k_fbar_force(CellBlockDev b, vec4_t<T>* __restrict__ slots) {
    const int64_t c = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPC;
    const int r = static_cast<int>(threadIdx.x % LPC);
    if (c >= b.num_cells) return;
    const int32_t s0 = b.ptr[c], s1 = b.ptr[c + 1];
    if (s1 <= s0) return;
    const T* gr = cell_grads<T>(b);
    const T* o = static_cast<const T*>(b.fbar) + kFbarStride * c + 10;
    T P[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) P[k] = o[k];
    const T V = T(b.volumes[c]);
    for (int32_t s = s0 + r; s < s1; s += LPC) {
        const T gg[3] = {gr[3 * s], gr[3 * s + 1], gr[3 * s + 2]};
        T f[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) f[i] = (gg[0] * P[i * 3 + 0] + gg[1] * P[i * 3 + 1] + gg[2] * P[i * 3 + 2]) * -V;
        slots[b.slot_pos[s]] = make4(f[0], f[1], f[2]);
    }
}

// F-bar in one pass for cells of at most 32 subcells: one warp per cell. Eight lanes
// take one subcell's entries together (coalesced, four subcells at a time) and combine
// its H by a butterfly; the subcell's H and J go to shared memory. Then one lane per
// subcell forms J-bar and the dual pressure over the warp (fixed butterflies), the
// barred and un-barred stresses, back into shared memory; and eight lanes per subcell
// write its forces. Same formulas as k_fbar_h / k_fbar_cell / k_fbar_force, no global
// scratch and one launch.
constexpr int kFbarMaxSub = 32;
constexpr int kFbarWarps = 4;


template <typename T, int MAT>
__global__ void __launch_bounds__(32 * kFbarWarps) k_fbar_fused(CellBlockDev b, const double4* __restrict__ U4,
                                                                 vec4_t<T>* __restrict__ slots, int* status) {
    __shared__ T sh_t[kFbarWarps][kFbarMaxSub][18];  // H, then the subcell stress
    __shared__ double sh_j[kFbarWarps][kFbarMaxSub];
    pdl_trigger();
    pdl_wait();
    const int w = static_cast<int>(threadIdx.x >> 5);
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int q = lane >> 3, r8 = lane & 7;
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const bool gvalid = g < b.num_groups;
    const int64_t s0 = gvalid ? b.group_ptr[g] : 0;
    const int ns = gvalid ? static_cast<int>(b.group_ptr[g + 1] - s0) : 0;
    const T* gr = cell_grads<T>(b);
    const bool diff = sizeof(T) == 4;
    // H of every subcell, four at a time.
    for (int base = 0; base < ns; base += 4) {
        const int k = base + q;
        const bool has = k < ns;
        const int64_t s = s0 + k;
        const int32_t e0 = has ? b.ptr[s] : 0, e1 = has ? b.ptr[s + 1] : 0;
        const double4 ur = e1 > e0 ? ld_dep(U4 + b.nodes[e0]) : make_double4(0.0, 0.0, 0.0, 0.0);
        T H[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) H[m] = T(0);
        for (int32_t e = e0 + r8; e < e1; e += 8) {
            const double4 u = ld_dep(U4 + b.nodes[e]);
            const T du[3] = {T(diff ? u.x - ur.x : u.x), T(diff ? u.y - ur.y : u.y), T(diff ? u.z - ur.z : u.z)};
            const T gg[3] = {gr[3 * e], gr[3 * e + 1], gr[3 * e + 2]};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) H[i * 3 + j] += du[i] * gg[j];
        }
#pragma unroll
        for (int off = 4; off > 0; off >>= 1)
#pragma unroll
            for (int m = 0; m < 9; ++m) H[m] += __shfl_xor_sync(kFull, H[m], off);
        if (has && r8 == 0) {
#pragma unroll
            for (int m = 0; m < 9; ++m) sh_t[w][k][m] = H[m];
            const double J = det_ap_im1(H) + 1.0;
            sh_j[w][k] = J;
            if (!(J > 0.0)) flag(status, AM_ENONPOS_J, s);
        }
    }
    __syncwarp();
    // J-bar, stresses and the dual pressure: one lane per subcell.
    const bool own = lane < ns;
    const int64_t s = s0 + lane;
    T H[9], Pb[9];
    double V = 0.0, J = 1.0;
    if (own) {
#pragma unroll
        for (int m = 0; m < 9; ++m) H[m] = sh_t[w][lane][m];
        J = sh_j[w][lane];
        V = b.volumes[s];
    }
    double jv = own ? J * V : 0.0, vol = own ? V : 0.0;
    warp_sum2(jv, vol);
    const double Jbar = ns > 0 ? jv / vol : 1.0;
    double js = 1.0, pd = 0.0, unused = 0.0;
    if (own) {
        const double ratio = Jbar / J;
        js = cbrt(ratio);
        T Hb[9];
        if (fabs(ratio - 1.0) < 3.0 * 2.2204460492503131e-16) {
#pragma unroll
            for (int m = 0; m < 9; ++m) Hb[m] = H[m];
        } else {
#pragma unroll
            for (int m = 0; m < 9; ++m) Hb[m] = H[m] * T(js);
            Hb[0] += T(js - 1.0);
            Hb[4] += T(js - 1.0);
            Hb[8] += T(js - 1.0);
        }
        double lam, mu;
        element_lame(b, s, lam, mu);
        const double Jb = stress<T>(MAT, T(lam), T(mu), Hb, Pb);
        if (MAT == kNeoHookean && !(Jb > 0.0)) flag(status, AM_ENONPOS_J, s);
        double pf = static_cast<double>(Pb[0] + Pb[4] + Pb[8]);
#pragma unroll
        for (int m = 0; m < 9; ++m) pf += static_cast<double>(Pb[m] * H[m]);
        pd = js / (3.0 * Jbar) * V * pf;
    }
    warp_sum2(pd, unused);
    if (own) {
        pd /= vol;
        T F[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) F[m] = H[m];
        F[0] += T(1);
        F[4] += T(1);
        F[8] += T(1);
        double pf = 0.0;
#pragma unroll
        for (int m = 0; m < 9; ++m) pf += static_cast<double>(Pb[m] * F[m]);
        const T scal = T(pd - js / (3.0 * J) * pf);
        T A[9];
        adj3(F, A);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) sh_t[w][lane][9 + i * 3 + j] = Pb[i * 3 + j] * T(js) + scal * A[j * 3 + i];
    }
    __syncwarp();
    // Forces, eight lanes per subcell.
    for (int base = 0; base < ns; base += 4) {
        const int k = base + q;
        if (k >= ns) continue;
        const int64_t sk = s0 + k;
        const int32_t e0 = b.ptr[sk], e1 = b.ptr[sk + 1];
        T P[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) P[m] = sh_t[w][k][9 + m];
        const T Vt = T(b.volumes[sk]);
        for (int32_t e = e0 + r8; e < e1; e += 8) {
            const T gg[3] = {gr[3 * e], gr[3 * e + 1], gr[3 * e + 2]};
            T f[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) f[i] = (gg[0] * P[i * 3 + 0] + gg[1] * P[i * 3 + 1] + gg[2] * P[i * 3 + 2]) * -Vt;
            slots[b.slot_pos[e]] = make4(f[0], f[1], f[2]);
        }
    }
}

// ---------------------------------------------------------------------------
// VJP kernels (FP64): slots receive (dF/du)^T lam per element node; gmu/gkappa
// receive lam^T dF/dmu_e and lam^T dF/dkappa_e (lambda_e = kappa_e - 2/3 mu_e).
// Lambda = sum_a lam_a (x) B_a ; lam . f_e = -sum_gp w Lambda : P.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_theta(double* gmu, double* gk, int64_t e, double w_ldmu_ldlam,
                                            double w_ldlam, int accumulate) {
    if (gmu) gmu[e] = accumulate ? gmu[e] + w_ldmu_ldlam : w_ldmu_ldlam;
    if (gk) gk[e] = accumulate ? gk[e] + w_ldlam : w_ldlam;
}

// VJP of one tet: J, D, DL hold X, u and lam differences (columns l1-l0, l2-l0,
// l3-l0). Writes g[12] and the element's (dF/dmu)^T lam, (dF/dkappa)^T lam.
template <int MAT>
__device__ __forceinline__ void tet4_vjp(const double* J, const double* D, const double* DL, double lam, double mu,
                                         double* g, double& tm, double& tk) {
    const double det = det3(J);
    double Ji[9];
    cof_inv3(J, Ji, det);
    const double w = det / 6.0;
    double H[9], L[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            H[i * 3 + j] = D[i * 3 + 0] * Ji[0 * 3 + j] + D[i * 3 + 1] * Ji[1 * 3 + j] + D[i * 3 + 2] * Ji[2 * 3 + j];
            L[i * 3 + j] = DL[i * 3 + 0] * Ji[0 * 3 + j] + DL[i * 3 + 1] * Ji[1 * 3 + j] + DL[i * 3 + 2] * Ji[2 * 3 + j];
        }
    double dP[9], ldl, ldm;
    stress_vjp(MAT, lam, mu, H, L, dP, &ldl, &ldm);
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double q = w * (Ji[k * 3 + 0] * dP[i * 3 + 0] + Ji[k * 3 + 1] * dP[i * 3 + 1] + Ji[k * 3 + 2] * dP[i * 3 + 2]);
            g[(k + 1) * 3 + i] = -q;
            g[i] += q;
        }
    tm = -w * (ldm - 2.0 / 3.0 * ldl);
    tk = -w * ldl;
}

template <int MAT>
__global__ void __launch_bounds__(256) k_tet4_vjp(GaussBlockDev b, const double4* __restrict__ X4,
                                                   const double4* __restrict__ U4, const double4* __restrict__ L4,
                                                   double4* __restrict__ slots, double* gmu, double* gk,
                                                   int accumulate) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    const int4 c = reinterpret_cast<const int4*>(b.conn)[e];
    const double4 x0 = X4[c.x], x1 = X4[c.y], x2 = X4[c.z], x3 = X4[c.w];
    const double4 u0 = U4[c.x], u1 = U4[c.y], u2 = U4[c.z], u3 = U4[c.w];
    const double4 l0 = L4[c.x], l1 = L4[c.y], l2 = L4[c.z], l3 = L4[c.w];
    const double J[9] = {x1.x - x0.x, x2.x - x0.x, x3.x - x0.x, x1.y - x0.y, x2.y - x0.y,
                         x3.y - x0.y, x1.z - x0.z, x2.z - x0.z, x3.z - x0.z};
    const double D[9] = {u1.x - u0.x, u2.x - u0.x, u3.x - u0.x, u1.y - u0.y, u2.y - u0.y,
                         u3.y - u0.y, u1.z - u0.z, u2.z - u0.z, u3.z - u0.z};
    const double DL[9] = {l1.x - l0.x, l2.x - l0.x, l3.x - l0.x, l1.y - l0.y, l2.y - l0.y,
                          l3.y - l0.y, l1.z - l0.z, l2.z - l0.z, l3.z - l0.z};
    double lam, mu;
    element_lame(b, e, lam, mu);
    double g[12], tm, tk;
    tet4_vjp<MAT>(J, D, DL, lam, mu, g, tm, tk);
    for (int a = 0; a < 4; ++a) slots[b.slot_pos[4 * e + a]] = make4(g[3 * a], g[3 * a + 1], g[3 * a + 2]);
    store_theta(gmu, gk, e, tm, tk, accumulate);
}

template <int MAT>
__global__ void __launch_bounds__(256) k_tet4_patch_vjp(GaussBlockDev b, const double4* __restrict__ X4,
                                                         const double4* __restrict__ U4,
                                                         const double4* __restrict__ L4, double4* __restrict__ slots,
                                                         double* gmu, double* gk, int accumulate) {
    __shared__ double sh[32][168];  // [0, 72): node dX, du, dlam ; [72, 168): 8 tets x 4 nodes x 3
    const int lane = threadIdx.x & 31;
    const int g = lane & 7;
    const int pl = threadIdx.x >> 3;
    const int64_t p = static_cast<int64_t>(blockIdx.x) * 32 + pl;
    const bool valid = p < b.num_patches;
    const int32_t n = valid ? b.patch_nodes[p * 8 + g] : 0;
    const double4 x = X4[n], u = U4[n], l = L4[n];
    const int src = lane & ~7;
    double* s = sh[pl];
    s[g * 9 + 0] = x.x - __shfl_sync(kFull, x.x, src);
    s[g * 9 + 1] = x.y - __shfl_sync(kFull, x.y, src);
    s[g * 9 + 2] = x.z - __shfl_sync(kFull, x.z, src);
    s[g * 9 + 3] = u.x - __shfl_sync(kFull, u.x, src);
    s[g * 9 + 4] = u.y - __shfl_sync(kFull, u.y, src);
    s[g * 9 + 5] = u.z - __shfl_sync(kFull, u.z, src);
    s[g * 9 + 6] = l.x - __shfl_sync(kFull, l.x, src);
    s[g * 9 + 7] = l.y - __shfl_sync(kFull, l.y, src);
    s[g * 9 + 8] = l.z - __shfl_sync(kFull, l.z, src);
    int32_t e0 = 0, cnt = 0;
    if (valid) {
        e0 = b.patch_first[p];
        cnt = b.patch_first[p + 1] - e0;
    }
    const uint32_t loc = (g < cnt) ? b.patch_local[e0 + g] : 0u;
    __syncwarp();
    if (g < cnt) {
        const int64_t e = e0 + g;
        const double* n0 = s + local_id(loc, 0) * 9;
        const double* n1 = s + local_id(loc, 1) * 9;
        const double* n2 = s + local_id(loc, 2) * 9;
        const double* n3 = s + local_id(loc, 3) * 9;
        double J[9], D[9], DL[9];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            J[i * 3 + 0] = n1[i] - n0[i];
            J[i * 3 + 1] = n2[i] - n0[i];
            J[i * 3 + 2] = n3[i] - n0[i];
            D[i * 3 + 0] = n1[3 + i] - n0[3 + i];
            D[i * 3 + 1] = n2[3 + i] - n0[3 + i];
            D[i * 3 + 2] = n3[3 + i] - n0[3 + i];
            DL[i * 3 + 0] = n1[6 + i] - n0[6 + i];
            DL[i * 3 + 1] = n2[6 + i] - n0[6 + i];
            DL[i * 3 + 2] = n3[6 + i] - n0[6 + i];
        }
        double lam, mu;
        element_lame(b, e, lam, mu);
        double gv[12], tm, tk;
        tet4_vjp<MAT>(J, D, DL, lam, mu, gv, tm, tk);
        double* c = s + 72 + g * 12;
#pragma unroll
        for (int k = 0; k < 12; ++k) c[k] = gv[k];
        store_theta(gmu, gk, e, tm, tk, accumulate);
    }
    __syncwarp();
    double fx = 0.0, fy = 0.0, fz = 0.0;
    const uint32_t gm = valid ? b.patch_gather[p * 8 + g] : 0u;
    for (uint32_t m = gm & 0xFFu; m; m &= m - 1) {
        const int t = __ffs(m) - 1;
        const double* c = s + 72 + t * 12 + ((gm >> (8 + 2 * t)) & 3u) * 3;
        fx += c[0];
        fy += c[1];
        fz += c[2];
    }
    if (valid) {
        const int32_t pos = b.slot_pos[p * 8 + g];
        if (pos >= 0) slots[pos] = make4(fx, fy, fz);
    }
}

// VJP of the Hex8 forces in the monomial basis (see k_hex8_force): the
// Gauss point's dP[grad lam] takes the place of P in the same regrouped nodal
// sum, and the material-field contractions are summed over the Gauss points in
// order. One thread per element, FP64.
template <int MAT>
__global__ void __launch_bounds__(64) k_hex8_vjp(GaussBlockDev b, const double4* __restrict__ X4,
                                                       const double4* __restrict__ U4, const double4* __restrict__ L4,
                                                       double4* __restrict__ slots, double* gmu, double* gk,
                                                       int accumulate) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    int32_t nd[8];
    hex_conn(b, e, nd);
    double X[3][8], U[3][8], W[3][8];
    hex_load_rel(X4, nd, X);
    hex_load_rel(U4, nd, U);
    hex_load_rel(L4, nd, W);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        hex_butterfly(X[i]);
        hex_butterfly(U[i]);
        hex_butterfly(W[i]);
        hex_scale_coeffs(X[i]);
        hex_scale_coeffs(U[i]);
        hex_scale_coeffs(W[i]);
    }
    double lam, mu;
    element_lame(b, e, lam, mu);
    double R[3][8];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) R[i][k] = 0.0;
    double tm = 0.0, tk = 0.0;
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
        double J[9], A[9], H[9], L[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) J[i * 3 + j] = hex_dxi(X[i], j, g);
        adj3(J, A);
        const double det = J[0] * A[0] + J[1] * A[3] + J[2] * A[6];
        const double id = 1.0 / det;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double g0 = hex_dxi(U[i], 0, g), g1 = hex_dxi(U[i], 1, g), g2 = hex_dxi(U[i], 2, g);
            const double l0 = hex_dxi(W[i], 0, g), l1 = hex_dxi(W[i], 1, g), l2 = hex_dxi(W[i], 2, g);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                H[i * 3 + j] = (g0 * A[0 * 3 + j] + g1 * A[1 * 3 + j] + g2 * A[2 * 3 + j]) * id;
                L[i * 3 + j] = (l0 * A[0 * 3 + j] + l1 * A[1 * 3 + j] + l2 * A[2 * 3 + j]) * id;
            }
        }
        double dP[9], ldl, ldm;
        stress_vjp(MAT, lam, mu, H, L, dP, &ldl, &ldm);
        const double w = det * (1.0 / 512.0);
        tm -= w * (ldm - 2.0 / 3.0 * ldl);
        tk -= w * ldl;
        double Q[9];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                Q[k * 3 + i] = A[k * 3 + 0] * dP[i * 3 + 0] + A[k * 3 + 1] * dP[i * 3 + 1] + A[k * 3 + 2] * dP[i * 3 + 2];
        hex_accumulate_r(R, Q, g);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R[i][0] = 0.0;
        hex_scale_coeffs(R[i]);
        hex_butterfly_t(R[i]);
    }
    const double s = -1.0 / 512.0;
    const int4 p0 = reinterpret_cast<const int4*>(b.slot_pos)[2 * e], p1 = reinterpret_cast<const int4*>(b.slot_pos)[2 * e + 1];
    const int32_t pos[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
    for (int q = 0; q < 8; ++q) slots[pos[hex_node_of_corner(q)]] = make4(s * R[0][q], s * R[1][q], s * R[2][q]);
    store_theta(gmu, gk, e, tm, tk, accumulate);
}

template <int MAT>
__global__ void __launch_bounds__(256) k_cell_vjp(CellBlockDev b, const double4* __restrict__ U4,
                                                   const double4* __restrict__ L4, double4* __restrict__ slots,
                                                   double* gmu, double* gk, int accumulate) {
    const int lane = threadIdx.x & 31;
    const int64_t c = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (c >= b.num_cells) return;
    const int32_t s0 = b.ptr[c], s1 = b.ptr[c + 1];
    double H[9], L[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) H[k] = L[k] = 0.0;
    for (int32_t s = s0 + lane; s < s1; s += 32) {
        const int32_t n = b.nodes[s];
        const double4 u = U4[n], l = L4[n];
        const double gg[3] = {b.grads64[3 * s], b.grads64[3 * s + 1], b.grads64[3 * s + 2]};
        const double uu[3] = {u.x, u.y, u.z}, ll[3] = {l.x, l.y, l.z};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                H[i * 3 + j] += uu[i] * gg[j];
                L[i * 3 + j] += ll[i] * gg[j];
            }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            H[k] += __shfl_xor_sync(kFull, H[k], off);
            L[k] += __shfl_xor_sync(kFull, L[k], off);
        }
    double lam, mu;
    element_lame(b, c, lam, mu);
    double dP[9], ldl, ldm;
    stress_vjp(MAT, lam, mu, H, L, dP, &ldl, &ldm);
    const double V = b.volumes[c];
    if (b.gather) {
        // cell-stress form: -V dP per cell, summed per node by the gather kernel
        double m[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) m[k] = -V * dP[k];
        store_cell_matrix<double>(static_cast<double*>(b.cmat), b.num_cells, c, lane, m);
    } else {
        for (int32_t s = s0 + lane; s < s1; s += 32) {
            const double gg[3] = {b.grads64[3 * s], b.grads64[3 * s + 1], b.grads64[3 * s + 2]};
            double f[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) f[i] = (gg[0] * dP[i * 3 + 0] + gg[1] * dP[i * 3 + 1] + gg[2] * dP[i * 3 + 2]) * -V;
            slots[b.slot_pos[s]] = make4(f[0], f[1], f[2]);
        }
    }
    if (lane == 0) store_theta(gmu, gk, c, -V * (ldm - 2.0 / 3.0 * ldl), -V * ldl, accumulate);
}

// VJP of F-bar cells in the cell-stress form (a warp per cell of at most 32 subcells, a lane
// per subcell; FP64). The F-bar force is f = -dW/du of W = sum_s V_s psi(Fbar_s), so its VJP
// with lam is the derivative along L_s = sum_k lam_k (x) b_k (W's Hessian is symmetric):
//   dJ_s = cof(F_s) : L_s, dJbar = sum V_s dJ_s / V, djs = js / 3 (dJbar / Jbar - dJ_s / J_s),
//   dFbar = djs F + js L, dPbar = dP/dF(Hbar)[dFbar], pf = Pbar : F, dpf = dPbar : F + Pbar : L,
//   dP = djs Pbar + js dPbar + dscal cof(F) + scal dcof(F)[L]
// with scal = p - js pf / (3 J) and its derivative dscal. H_s (in M) and L_s (in Lm) come
// from the octet kernel; M = -V_s dP_s replaces H_s for the node-major gather. The moduli of
// subcell s enter lam^T f = -sum_s V_s Pbar_s : dFbar_s only through Pbar_s.
template <int MAT>
__global__ void __launch_bounds__(256) k_fbar_cell_vjp(CellBlockDev b, double* __restrict__ M,
                                                        const double* __restrict__ Lm, double* gmu, double* gk,
                                                        int accumulate) {
    pdl_trigger();
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const bool gvalid = g < b.num_groups;
    const int64_t s0 = gvalid ? b.group_ptr[g] : 0;
    const int ns = gvalid ? static_cast<int>(b.group_ptr[g + 1] - s0) : 0;
    if (ns == 0) return;  // the whole warp
    const bool own = lane < ns;
    const int64_t s = s0 + lane;
    const double V = own ? b.volumes[s] : 0.0;
    double lam = 0.0, mu = 0.0;
    if (own) element_lame(b, s, lam, mu);
    pdl_wait();
    double H[9], L[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) H[q] = L[q] = 0.0;
    if (own) {
        load_cell_matrix(M, b.num_cells, static_cast<int32_t>(s), H);
        load_cell_matrix(Lm, b.num_cells, static_cast<int32_t>(s), L);
    }
    double F[9], A[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = H[q];
    F[0] += 1.0;
    F[4] += 1.0;
    F[8] += 1.0;
    adj3(F, A);  // cof(F)_ij = A_ji
    const double J = det_ap_im1(H) + 1.0;
    double dJ = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dJ += A[j * 3 + i] * L[i * 3 + j];
    double jv = own ? J * V : 0.0, vol = V, djv = own ? dJ * V : 0.0, unused = 0.0;
    warp_sum2(jv, vol);
    warp_sum2(djv, unused);
    const double Jbar = jv / vol, dJbar = djv / vol;
    const double ratio = Jbar / J;
    const double js = cbrt(ratio);
    const double djs = js / 3.0 * (dJbar / Jbar - dJ / J);
    double Hb[9], dFb[9];
    if (fabs(ratio - 1.0) < 3.0 * 2.2204460492503131e-16) {
#pragma unroll
        for (int q = 0; q < 9; ++q) Hb[q] = H[q];
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q) Hb[q] = H[q] * js;
        Hb[0] += js - 1.0;
        Hb[4] += js - 1.0;
        Hb[8] += js - 1.0;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) dFb[q] = djs * F[q] + js * L[q];
    double Pb[9], dPb[9], ldl = 0.0, ldm = 0.0;
    stress<double>(MAT, lam, mu, Hb, Pb);
    stress_vjp(MAT, lam, mu, Hb, dFb, dPb, &ldl, &ldm);
    double pf = 0.0, dpf = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        pf += Pb[q] * F[q];
        dpf += dPb[q] * F[q] + Pb[q] * L[q];
    }
    double pd = own ? V * js * pf / (3.0 * Jbar) : 0.0;
    double dpd = own ? V * (djs * pf + js * dpf - js * pf * dJbar / Jbar) / (3.0 * Jbar) : 0.0;
    warp_sum2(pd, dpd);
    if (!own) return;
    pd /= vol;
    dpd /= vol;
    const double scal = pd - js * pf / (3.0 * J);
    const double dscal = dpd - (djs * pf + js * dpf) / (3.0 * J) + js * pf * dJ / (3.0 * J * J);
    double m[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        // row r of cof(F) is F_a x F_c (rows a = r + 1, c = r + 2): its derivative along L
        const int a = (r + 1) % 3, c = (r + 2) % 3;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            const double dG = L[a * 3 + i1] * F[c * 3 + i2] - L[a * 3 + i2] * F[c * 3 + i1] + F[a * 3 + i1] * L[c * 3 + i2] -
                              F[a * 3 + i2] * L[c * 3 + i1];
            const int q = r * 3 + i;
            m[q] = -V * (djs * Pb[q] + js * dPb[q] + dscal * A[i * 3 + r] + scal * dG);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) store_cell_matrix<double>(M, b.num_cells, s, k, m);
    store_theta(gmu, gk, s, -V * (ldm - 2.0 / 3.0 * ldl), -V * ldl, accumulate);
}

// VJP of the split-hex-grouped cells (FP64, one thread per patch): the cell VJP above
// for the patch's six cells, summed per patch node.
template <int MAT>
__global__ void __launch_bounds__(64) k_cell_hex6_vjp(CellBlockDev b, const double4* __restrict__ U4,
                                                       const double4* __restrict__ L4, double4* __restrict__ slots,
                                                       double* gmu, double* gk, int accumulate) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= b.num_patches) return;
    constexpr int kRing[7] = {1, 2, 4, 5, 6, 7, 1};
    double acc[8][3];
#pragma unroll
    for (int a = 0; a < 8; ++a) acc[a][0] = acc[a][1] = acc[a][2] = 0.0;
    const int64_t c0 = b.patch_first[p];
#pragma unroll 1
    for (int t = 0; t < 6; ++t) {
        const int64_t c = c0 + t;
        const int ln[4] = {0, kRing[t], kRing[t + 1], 3};
        double g[12];
        load_cell12<double>(b.grads64 + 12 * c, g);
        double H[9], L[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) H[k] = L[k] = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int32_t n = b.patch_nodes[p * 8 + ln[e]];
            const double4 u = U4[n], l = L4[n];
            const double uu[3] = {u.x, u.y, u.z}, ll[3] = {l.x, l.y, l.z};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    H[i * 3 + j] += uu[i] * g[3 * e + j];
                    L[i * 3 + j] += ll[i] * g[3 * e + j];
                }
        }
        double lam, mu;
        element_lame(b, c, lam, mu);
        double dP[9], ldl, ldm;
        stress_vjp(MAT, lam, mu, H, L, dP, &ldl, &ldm);
        const double V = b.volumes[c];
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                acc[ln[e]][i] += (g[3 * e] * dP[i * 3 + 0] + g[3 * e + 1] * dP[i * 3 + 1] + g[3 * e + 2] * dP[i * 3 + 2]) * -V;
        store_theta(gmu, gk, c, -V * (ldm - 2.0 / 3.0 * ldl), -V * ldl, accumulate);
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int32_t pos = b.slot_pos[p * 8 + a];
        if (pos >= 0) slots[pos] = make4(acc[a][0], acc[a][1], acc[a][2]);
    }
}

// ---------------------------------------------------------------------------
// Lumped mass slots (src/MassUtils.cpp:17-46): slot (e, a) = rho V_e / n_en with
// V_e = sum_gp w_gp (ComputeElementVolumeFunctor.h:20-79).
// ---------------------------------------------------------------------------
__device__ double element_volume(int nn, const double* X) {
    double V = 0.0;
    const int ngp = nn == 8 ? 8 : 1;
    for (int gp = 0; gp < ngp; ++gp) {
        double dN[24];
        if (nn == 8) {
            const double loc = 1.0 / sqrt(3.0);
            const double xi[3] = {hex_sign(gp, 0) * loc, hex_sign(gp, 1) * loc, hex_sign(gp, 2) * loc};
            for (int a = 0; a < 8; ++a) {
                const double p0 = hex_sign(a, 0), p1 = hex_sign(a, 1), p2 = hex_sign(a, 2);
                dN[a * 3 + 0] = 0.125 * p0 * (1.0 + p1 * xi[1]) * (1.0 + p2 * xi[2]);
                dN[a * 3 + 1] = 0.125 * p1 * (1.0 + p0 * xi[0]) * (1.0 + p2 * xi[2]);
                dN[a * 3 + 2] = 0.125 * p2 * (1.0 + p0 * xi[0]) * (1.0 + p1 * xi[1]);
            }
        } else {
            const double t[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
            for (int k = 0; k < 12; ++k) dN[k] = t[k];
        }
        double J[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double acc = 0.0;
                for (int a = 0; a < nn; ++a) acc += X[a * 3 + i] * dN[a * 3 + j];
                J[i * 3 + j] = acc;
            }
        V += (nn == 8 ? 1.0 : 1.0 / 6.0) * det3(J);
    }
    return V;
}

// Patched Tet4 blocks: per patch node, the sum over the patch's tets (set-up only).
__global__ void k_tet4_patch_volume_slots(GaussBlockDev b, double density, const double4* __restrict__ X4,
                                          double4* __restrict__ slots) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= b.num_patches) return;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int32_t e = b.patch_first[p]; e < b.patch_first[p + 1]; ++e) {
        double X[12];
        for (int a = 0; a < 4; ++a) {
            const double4 x = X4[b.conn[4 * static_cast<int64_t>(e) + a]];
            X[a * 3 + 0] = x.x;
            X[a * 3 + 1] = x.y;
            X[a * 3 + 2] = x.z;
        }
        const double me = element_volume(4, X) * density / 4;
        const uint32_t loc = b.patch_local[e];
        for (int k = 0; k < 4; ++k) acc[local_id(loc, k)] += me;
    }
    for (int a = 0; a < 8; ++a) {
        const int32_t pos = b.slot_pos[p * 8 + a];
        if (pos >= 0) slots[pos] = make_double4(acc[a], 0.0, 0.0, 0.0);
    }
}

__global__ void k_gauss_volume_slots(GaussBlockDev b, double density, const double4* __restrict__ X4,
                                     double4* __restrict__ slots) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= b.num_elems) return;
    const int nn = b.kind == AM_HEX8_GAUSS ? 8 : 4;
    double X[24];
    for (int a = 0; a < nn; ++a) {
        const double4 x = X4[b.conn[e * nn + a]];
        X[a * 3 + 0] = x.x;
        X[a * 3 + 1] = x.y;
        X[a * 3 + 2] = x.z;
    }
    const double me = element_volume(nn, X) * density / nn;
    for (int a = 0; a < nn; ++a) slots[b.slot_pos[e * nn + a]] = make_double4(me, 0.0, 0.0, 0.0);
}

// ---------------------------------------------------------------------------
// Node kernels.
// ---------------------------------------------------------------------------
// Sum of node i's slots: a contiguous node-major range, summed in ascending
// logical-slot order (FP64 accumulation for both slot types).
constexpr int kNodeBlock = 128;  // 7-8% faster node kernels than 256-thread blocks on B200

// Node-centric gather of a node's force slots (node-major, contiguous), summed in
// FP64 in slot order. BATCH loads are issued before the first add. A node of a hex
// mesh, or of the split-hex tet patches, has at most eight slots, so BATCH = 8
// takes every slot in one round; that wins when the slot array sits in L2 (the
// loads are latency-bound), while BATCH = 4 keeps more warps resident, which wins
// when the slots stream from HBM (see gather_batch8).
// The run-invariant part of a node's gather: its slot range and interface row, which
// a kernel can read before it waits for the kernels that write the slots.
struct NodeSlots {
    int32_t p0, p1, row;
};
__device__ __forceinline__ NodeSlots node_slots(const NodeDev& nd, int64_t i, bool own) {
    NodeSlots q{0, 0, -1};
    if (own) {
        q.row = nd.iface_row != nullptr ? nd.iface_row[i] : -1;
        if (nd.f_given == nullptr && q.row < 0) {
            q.p0 = nd.node_ptr[i];
            q.p1 = nd.node_ptr[i + 1];
        }
    }
    return q;
}

template <typename S, int BATCH, int LPN>
__device__ __forceinline__ void gather(const NodeDev& nd, const vec4_t<S>* __restrict__ slots, int64_t i, bool own,
                                       const NodeSlots& q, double& fx, double& fy, double& fz) {
    // LPN lanes per node: lane r takes every LPN-th slot from r (the group reads the
    // node's contiguous range with coalesced loads), then the partial sums combine by
    // a fixed butterfly, so every lane holds the same total and the order is fixed.
    const int r = LPN == 1 ? 0 : static_cast<int>(threadIdx.x % LPN);
    fx = fy = fz = 0.0;
    const int32_t row = q.row;
    if (own && nd.f_given != nullptr) {
        // Two-pass coupling: the node's generalized force, already summed.
        if (r == 0) {
            fx = nd.f_given[3 * i];
            fy = nd.f_given[3 * i + 1];
            fz = nd.f_given[3 * i + 2];
        }
    } else if (row >= 0) {
        // Interface node: the summed force of all ranks (one lane contributes it).
        if (r == 0) {
            fx = nd.iface_f[3 * static_cast<int64_t>(row)];
            fy = nd.iface_f[3 * static_cast<int64_t>(row) + 1];
            fz = nd.iface_f[3 * static_cast<int64_t>(row) + 2];
        }
    } else if (own) {
        const int32_t p1 = q.p1;
        for (int32_t p = q.p0 + r; p < p1; p += BATCH * LPN) {
            vec4_t<S> v[BATCH];
#pragma unroll
            for (int k = 0; k < BATCH; ++k)
                if (p + k * LPN < p1) v[k] = ld_dep(slots + p + k * LPN);
#pragma unroll
            for (int k = 0; k < BATCH; ++k)
                if (p + k * LPN < p1) {
                    fx += static_cast<double>(v[k].x);
                    fy += static_cast<double>(v[k].y);
                    fz += static_cast<double>(v[k].z);
                }
        }
    }
    if (LPN > 1) {
        const unsigned gmask = LPN == 32 ? kFull : (((1u << LPN) - 1u) << ((threadIdx.x & 31) & ~(LPN - 1)));
#pragma unroll
        for (int off = LPN / 2; off > 0; off >>= 1) {
            fx += __shfl_xor_sync(gmask, fx, off);
            fy += __shfl_xor_sync(gmask, fy, off);
            fz += __shfl_xor_sync(gmask, fz, off);
        }
    }
}

template <typename S, int BATCH, int LPN>
__device__ __forceinline__ void gather(const NodeDev& nd, const vec4_t<S>* __restrict__ slots, int64_t i, bool own,
                                       double& fx, double& fy, double& fz) {
    gather<S, BATCH, LPN>(nd, slots, i, own, node_slots(nd, i, own), fx, fy, fz);
}

// BoundaryCondition::ApplyVelocity / ApplyAcceleration: for each component the
// last active BC in list order that prescribes it overwrites the value.
__device__ __forceinline__ void apply_bc(uint32_t word, uint32_t active, const double* __restrict__ scale,
                                         const double* __restrict__ values, double& x, double& y, double& z) {
    uint32_t m = word & 0x3FFu & active;
    if (m) {
        const int k = 31 - __clz(m);
        x = values[k * 3 + 0] * scale[k];
    }
    m = (word >> 10) & 0x3FFu & active;
    if (m) {
        const int k = 31 - __clz(m);
        y = values[k * 3 + 1] * scale[k];
    }
    m = (word >> 20) & 0x3FFu & active;
    if (m) {
        const int k = 31 - __clz(m);
        z = values[k * 3 + 2] * scale[k];
    }
}

__device__ __forceinline__ void free_mask(uint32_t word, uint32_t active, double& mx, double& my, double& mz) {
    mx = (word & 0x3FFu & active) ? 0.0 : 1.0;
    my = ((word >> 10) & 0x3FFu & active) ? 0.0 : 1.0;
    mz = ((word >> 20) & 0x3FFu & active) ? 0.0 : 1.0;
}

template <typename S, int BATCH, int LPN>
__global__ void __launch_bounds__(kNodeBlock) k_gather_force(NodeDev nd, const vec4_t<S>* __restrict__ slots,
                                                              double* __restrict__ f, int accumulate) {
    const int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPN;
    const bool own = i < nd.num_nodes;
    if (LPN == 1 && !own) return;
    double fx, fy, fz;
    gather<S, BATCH, LPN>(nd, slots, i, own, fx, fy, fz);
    if (!own || threadIdx.x % LPN != 0) return;
    if (accumulate) {
        f[3 * i + 0] += fx;
        f[3 * i + 1] += fy;
        f[3 * i + 2] += fz;
    } else {
        f[3 * i + 0] = fx;
        f[3 * i + 1] = fy;
        f[3 * i + 2] = fz;
    }
}

// The node-summed force as one double4 per node (for the transposed coupling's
// 32-byte gathers).
template <typename S, int BATCH, int LPN>
__global__ void __launch_bounds__(kNodeBlock) k_gather_force4(NodeDev nd, const vec4_t<S>* __restrict__ slots,
                                                               double4* __restrict__ f) {
    const int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPN;
    const bool own = i < nd.num_nodes;
    if (LPN == 1 && !own) return;
    double fx, fy, fz;
    gather<S, BATCH, LPN>(nd, slots, i, own, fx, fy, fz);
    if (!own || threadIdx.x % LPN != 0) return;
    f[i] = make_double4(fx, fy, fz, 0.0);
}

// One thread per local interface node: its own slots summed (no interface override).
template <typename S, int LPN>
__global__ void __launch_bounds__(kNodeBlock) k_iface_gather(NodeDev nd, const vec4_t<S>* __restrict__ slots,
                                                              int64_t num_local, const int32_t* __restrict__ local_nodes,
                                                              const int32_t* __restrict__ rows, double* __restrict__ buf) {
    // LPN lanes per node, as the node kernels take them: the same summation order, so a
    // decomposed step on one rank reproduces the plain step bit for bit.
    const int64_t k = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPN;
    const bool own = k < num_local;
    if (LPN == 1 && !own) return;
    nd.iface_row = nullptr;
    double fx, fy, fz;
    gather<S, 4, LPN>(nd, slots, own ? local_nodes[k] : 0, own, fx, fy, fz);
    if (!own || threadIdx.x % LPN != 0) return;
    const int64_t r = rows[k];
    buf[3 * r] = fx;
    buf[3 * r + 1] = fy;
    buf[3 * r + 2] = fz;
}

template <typename S, int BATCH, int LPN>
__global__ void __launch_bounds__(kNodeBlock) k_init_accel(NodeDev nd, const vec4_t<S>* __restrict__ slots,
                                                            double4* __restrict__ A4, int* status) {
    const int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPN;
    const bool own = i < nd.num_nodes;
    if (LPN == 1 && !own) return;
    double fx, fy, fz;
    gather<S, BATCH, LPN>(nd, slots, i, own, fx, fy, fz);
    if (!own || threadIdx.x % LPN != 0) return;
    const double m = nd.mass[i];
    if (nd.has_g) {
        fx += nd.g[0] * m;
        fy += nd.g[1] * m;
        fz += nd.g[2] * m;
    }
    const double ax = fx / m, ay = fy / m, az = fz / m;
    if (!isfinite(ax) || !isfinite(ay) || !isfinite(az)) flag(status, AM_ENAN, i);
    A4[i] = make_double4(ax, ay, az, 0.0);
}

// Displacement update d^{n+1} = d^n + dt v^{n+1/2}. Under the updated / semi formulations
// (UpdateDisplacementsUpdatedFunctor, ExplicitTimeIntegrator.h:141-244) the increment
// dt v (rounded once) also feeds inc: the updated formulation first moves xc by the last
// step's increment (the current coordinates advance every step) and replaces inc; the
// semi formulation accumulates inc, after moving xc by it and clearing it when the
// reference configuration was just updated (rebase).
__device__ __forceinline__ void displace(const NodeDev& nd, int64_t i, int rebase, double dt, double vx, double vy,
                                         double vz, double4& u) {
    if (nd.lagr == 0) {
        u.x = u.x + dt * vx;
        u.y = u.y + dt * vy;
        u.z = u.z + dt * vz;
        return;
    }
    const double dx = __dmul_rn(dt, vx), dy = __dmul_rn(dt, vy), dz = __dmul_rn(dt, vz);
    u.x = __dadd_rn(u.x, dx);
    u.y = __dadd_rn(u.y, dy);
    u.z = __dadd_rn(u.z, dz);
    double4 q = nd.inc[i];
    if (nd.lagr == 1 || rebase) {
        double4 x = nd.xc[i];
        x.x = __dadd_rn(x.x, q.x);
        x.y = __dadd_rn(x.y, q.y);
        x.z = __dadd_rn(x.z, q.z);
        nd.xc[i] = x;
        q = make_double4(0.0, 0.0, 0.0, 0.0);
    }
    nd.inc[i] = make_double4(__dadd_rn(q.x, dx), __dadd_rn(q.y, dy), __dadd_rn(q.z, dz), 0.0);
}

__global__ void __launch_bounds__(256) k_prologue(NodeDev nd, const StepParams* __restrict__ table,
                                                   double4* __restrict__ U4, double4* __restrict__ V4,
                                                   const double4* __restrict__ A4, double4* __restrict__ u_copy,
                                                   int rebase) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nd.num_nodes) return;
    const StepParams& P = table[0];
    const double4 v = V4[i], a = A4[i];
    double vx = v.x + P.half * a.x, vy = v.y + P.half * a.y, vz = v.z + P.half * a.z;
    const uint32_t w = nd.bcword[i];
    if (w) apply_bc(w, P.vact, P.vscale, nd.bcvalues, vx, vy, vz);
    double4 u = U4[i];
    displace(nd, i, rebase, P.dt, vx, vy, vz, u);
    U4[i] = u;
    V4[i] = make_double4(vx, vy, vz, 0.0);
    if (u_copy) u_copy[i] = u;
}

template <typename S, int BATCH, int LPN>
__global__ void __launch_bounds__(kNodeBlock) k_node_step(NodeDev nd, const vec4_t<S>* __restrict__ slots,
                                                           const StepParams* __restrict__ table, int64_t step,
                                                           int advance, double4* __restrict__ U4,
                                                           double4* __restrict__ V4, double4* __restrict__ A4,
                                                           double4* __restrict__ u_copy, int* status, int rebase) {
    const int64_t t = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / LPN;
    bool own;
    int64_t i;
    if (nd.subset_nodes != nullptr) {
        own = t < nd.subset_count;
        i = own ? nd.subset_nodes[t] : 0;
    } else {
        i = t;
        own = t < nd.num_nodes && !(nd.skip_iface && nd.iface_row[t] >= 0);
    }
    // The node's own data is independent of the gather: issue its loads first (mass,
    // BC word and slot range before the wait for the element kernels, v and u after it).
    const int64_t j = own ? i : 0;
    const double m = nd.mass[j];
    const uint32_t w = nd.bcword[j];
    const NodeSlots q = node_slots(nd, i, own);
    pdl_trigger();
    pdl_wait();
    const double4 vh = ld_dep(V4 + j);
    const double4 u0 = advance ? ld_dep(U4 + j) : make_double4(0.0, 0.0, 0.0, 0.0);
    double fx, fy, fz;
    gather<S, BATCH, LPN>(nd, slots, i, own, q, fx, fy, fz);
    if (!own || threadIdx.x % LPN != 0) return;
    if (nd.has_g) {
        fx += nd.g[0] * m;
        fy += nd.g[1] * m;
        fz += nd.g[2] * m;
    }
    // a^{n+1} = f / m (ExplicitTimeIntegrator.h:247-283), then the acceleration BC at t^{n+1}.
    double ax = fx / m, ay = fy / m, az = fz / m;
    const StepParams& P = table[step];
    if (w) apply_bc(w, P.aact, P.ascale, nd.bcvalues, ax, ay, az);
    if (!isfinite(ax) || !isfinite(ay) || !isfinite(az)) flag(status, AM_ENAN, i);
    // v^{n+1} = v^{n+1/2} + dt/2 a^{n+1} (:329-364)
    const double vx = vh.x + P.half * ax, vy = vh.y + P.half * ay, vz = vh.z + P.half * az;
    if (advance) {
        // Next step: v^{n+3/2} = v^{n+1} + dt'/2 a^{n+1} (:286-326), velocity BC at t_mid',
        // u^{n+2} = u^{n+1} + dt' v^{n+3/2} (:97-134).
        const StepParams& Q = table[step + 1];
        double wx = vx + Q.half * ax, wy = vy + Q.half * ay, wz = vz + Q.half * az;
        if (w) apply_bc(w, Q.vact, Q.vscale, nd.bcvalues, wx, wy, wz);
        double4 u = u0;
        displace(nd, i, rebase, Q.dt, wx, wy, wz, u);
        st4(U4 + i, u);
        st4(V4 + i, make_double4(wx, wy, wz, 0.0));
        if (u_copy) st4(u_copy + i, u);
    } else {
        st4(V4 + i, make_double4(vx, vy, vz, 0.0));
        st4(A4 + i, make_double4(ax, ay, az, 0.0));
    }
}

// Reverse of the acceleration step: lam = Ma (abar + h vbar) / m, the cotangent
// of the internal force at step `step`.
__global__ void k_adj_prep(NodeDev nd, const StepParams* __restrict__ table, int64_t step,
                           const double4* __restrict__ VB, const double4* __restrict__ AB, double4* __restrict__ L4) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nd.num_nodes) return;
    const StepParams& P = table[step];
    const double m = nd.mass[i];
    double mx, my, mz;
    free_mask(nd.bcword[i], P.aact, mx, my, mz);
    const double4 vb = VB[i], ab = AB[i];
    L4[i] = make_double4(mx * (ab.x + P.half * vb.x) / m, my * (ab.y + P.half * vb.y) / m,
                         mz * (ab.z + P.half * vb.z) / m, 0.0);
}

// Reverse of the rest of step `step` given g = (dF/du)^T lam in the slots; then
// prepares lam for step-1 (or for the initial acceleration when step == 0).
__global__ void __launch_bounds__(kNodeBlock) k_adj_update(NodeDev nd, const double4* __restrict__ slots,
                                                            const StepParams* __restrict__ table, int64_t step,
                                                            double4* __restrict__ UB, double4* __restrict__ VB,
                                                            double4* __restrict__ AB, double4* __restrict__ L4) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nd.num_nodes) return;
    double gx, gy, gz;
    gather<double, 4, 1>(nd, slots, i, true, gx, gy, gz);
    const StepParams& P = table[step];
    double4 ub = UB[i];
    const double4 vb = VB[i];
    ub.x += gx;
    ub.y += gy;
    ub.z += gz;
    const uint32_t w = nd.bcword[i];
    double mx, my, mz;
    free_mask(w, P.vact, mx, my, mz);
    const double wx = mx * (vb.x + P.dt * ub.x), wy = my * (vb.y + P.dt * ub.y), wz = mz * (vb.z + P.dt * ub.z);
    const double ax = P.half * wx, ay = P.half * wy, az = P.half * wz;
    UB[i] = ub;
    VB[i] = make_double4(wx, wy, wz, 0.0);
    AB[i] = make_double4(ax, ay, az, 0.0);
    const double m = nd.mass[i];
    if (step > 0) {
        const StepParams& Q = table[step - 1];
        free_mask(w, Q.aact, mx, my, mz);
        L4[i] = make_double4(mx * (ax + Q.half * wx) / m, my * (ay + Q.half * wy) / m, mz * (az + Q.half * wz) / m, 0.0);
    } else {
        L4[i] = make_double4(ax / m, ay / m, az / m, 0.0);
    }
}

// Loss L = sum_s |u_s|^2 over the sensor list and its seed dL/du = 2 u_s added to UB
// (UB is zero on entry). One block: each thread takes a strided share of the list,
// the loss is summed by a fixed tree, so it is the same on every run. A node listed
// twice receives 2u twice; sums of equal addends starting from zero do not depend
// on their order, so the atomic adds are deterministic too.
__global__ void __launch_bounds__(256) k_sensor_seed(const double4* __restrict__ U4, int32_t num_sensors,
                                                     const int32_t* __restrict__ sensors, double4* __restrict__ UB,
                                                     double* loss) {
    __shared__ double part[256];
    double L = 0.0;
    for (int32_t k = threadIdx.x; k < num_sensors; k += blockDim.x) {
        const int32_t n = sensors[k];
        const double4 u = U4[n];
        L += u.x * u.x + u.y * u.y + u.z * u.z;
        atomicAdd(&UB[n].x, 2.0 * u.x);
        atomicAdd(&UB[n].y, 2.0 * u.y);
        atomicAdd(&UB[n].z, 2.0 * u.z);
    }
    part[threadIdx.x] = L;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = part[0];
}

// ---- power method (stable time increment) ----
// A dof is prescribed when any boundary condition of the list names its component.
__device__ __forceinline__ void prescribed(uint32_t w, bool& px, bool& py, bool& pz) {
    px = (w & 0x3FFu) != 0;
    py = ((w >> 10) & 0x3FFu) != 0;
    pz = ((w >> 20) & 0x3FFu) != 0;
}

__global__ void __launch_bounds__(256) k_pm_perturb(NodeDev nd, const double4* __restrict__ U4,
                                                    const double4* __restrict__ V4, const double* __restrict__ l,
                                                    double eps, double4* __restrict__ W4) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nd.num_nodes) return;
    bool px, py, pz;
    prescribed(nd.bcword[i], px, py, pz);
    const double4 u = U4[i], v = V4[i];
    const double le = l[i] * eps;
    W4[i] = make_double4(px ? u.x : u.x + v.x * le, py ? u.y : u.y + v.y * le, pz ? u.z : u.z + v.z * le, 0.0);
}

__global__ void __launch_bounds__(256) k_pm_next(NodeDev nd, const double* __restrict__ fe,
                                                 const double* __restrict__ fu, const double* __restrict__ l, double eps,
                                                 double4* __restrict__ V4, double* __restrict__ partial) {
    __shared__ double sq[256];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (i < nd.num_nodes) {
        bool px, py, pz;
        prescribed(nd.bcword[i], px, py, pz);
        const double d = l[i] * eps * nd.mass[i];
        const double vx = px ? 0.0 : (fe[3 * i] - fu[3 * i]) / d;
        const double vy = py ? 0.0 : (fe[3 * i + 1] - fu[3 * i + 1]) / d;
        const double vz = pz ? 0.0 : (fe[3 * i + 2] - fu[3 * i + 2]) / d;
        V4[i] = make_double4(vx, vy, vz, 0.0);
        acc = vx * vx + vy * vy + vz * vz;
    }
    sq[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sq[threadIdx.x] += sq[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sq[0];
}

__global__ void k_pm_scale(int64_t n, double4* __restrict__ V4, double scale) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 v = V4[i];
    V4[i] = make_double4(v.x * scale, v.y * scale, v.z * scale, 0.0);
}

// Two-pass coupling. kRkLanes lanes share a row (or column): lane r takes every
// kRkLanes-th entry, so the group reads the row's contiguous entries together, and the
// partial sums combine by a fixed butterfly (a fixed order for every run).
constexpr int kRkLanes = 8;

__device__ __forceinline__ void rk_combine(double& x, double& y, double& z) {
#pragma unroll
    for (int off = kRkLanes / 2; off > 0; off >>= 1) {
        x += __shfl_xor_sync(kFull, x, off);
        y += __shfl_xor_sync(kFull, y, off);
        z += __shfl_xor_sync(kFull, z, off);
    }
}

// Physical displacement P = Psi U (ComputeValues: neighbours taken from the last; a
// row without neighbours copies the coefficient).
__global__ void __launch_bounds__(128) k_rk_rows4(int64_t n, int64_t num_nodes, const int64_t* __restrict__ ptr,
                                                 const int32_t* __restrict__ nbr, const double* __restrict__ val,
                                                 const double4* __restrict__ U4, double4* __restrict__ P4) {
    const int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kRkLanes;
    const int r = static_cast<int>(threadIdx.x % kRkLanes);
    const bool own = i < n;
    double x = 0.0, y = 0.0, z = 0.0;
    int64_t b = 0, e = 0;
    if (own) {
        b = ptr[i];
        e = ptr[i + 1];
        for (int64_t k = e - 1 - r; k >= b; k -= kRkLanes) {
            const double4 u = ld_ro4(U4 + nbr[k]);
            const double w = val[k];
            x += w * u.x;
            y += w * u.y;
            z += w * u.z;
        }
    }
    rk_combine(x, y, z);
    if (!own || r != 0) return;
    // A row without neighbours copies its node's coefficient; a refinement point past the
    // nodes has none and stays at zero.
    P4[i] = b != e ? make_double4(x, y, z, 0.0) : i < num_nodes ? U4[i] : make_double4(0.0, 0.0, 0.0, 0.0);
}

// Generalized force f = Psi^T f_local (ScatterValues as a gather over the transposed
// functions, no atomics).
__global__ void __launch_bounds__(128) k_rk_cols3(int64_t n, const int64_t* __restrict__ tptr,
                                                 const int32_t* __restrict__ tsrc, const double* __restrict__ tval,
                                                 const double4* __restrict__ fl, double* __restrict__ f) {
    const int64_t j = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kRkLanes;
    const int r = static_cast<int>(threadIdx.x % kRkLanes);
    const bool own = j < n;
    double x = 0.0, y = 0.0, z = 0.0;
    if (own) {
        const int64_t e = tptr[j + 1];
        for (int64_t k = tptr[j] + r; k < e; k += kRkLanes) {
            const double4 g = ld_ro4(fl + tsrc[k]);
            const double w = tval[k];
            x += w * g.x;
            y += w * g.y;
            z += w * g.z;
        }
    }
    rk_combine(x, y, z);
    if (!own || r != 0) return;
    f[3 * j] = x;
    f[3 * j + 1] = y;
    f[3 * j + 2] = z;
}

// The coupling in warp octets (the row layout of the cell-stress form): item i (a point for
// the rows of Psi, a node for its columns) sums w * in[idx] over its rows, lane 8k + j taking
// item j of the octet and rows k, k + 4, ...; records are (w, idx) pairs in one 16-byte load,
// idx -1 for padding. Rows are aligned by offset where that pads little, so a quarter-warp's
// eight gathers read consecutive nodes or points. Rows of Psi without neighbours copy the
// node's coefficient (out4 set, row_ptr the original offsets); columns write out3.
template <int UNR>
__global__ void __launch_bounds__(256) k_rk_octets(int64_t count, int64_t num_octets, const int32_t* __restrict__ optr,
                                                   const double2* __restrict__ rec, const double4* __restrict__ in,
                                                   const int64_t* __restrict__ row_ptr, int64_t num_nodes,
                                                   double4* __restrict__ out4, double* __restrict__ out3) {
    const int64_t o = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x & 31), j = lane & 7, k = lane >> 3;
    const int64_t i = 8 * o + j;
    const bool valid = i < count;
    const bool live = o < num_octets;
    const int32_t r0 = live ? optr[o] : 0, rows = live ? optr[o + 1] - r0 : 0;
    const double2* rp = rec + 8 * static_cast<int64_t>(r0) + j;
    const double2 pad = make_double2(0.0, __longlong_as_double(-1LL));
    double2 rr[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) rr[u] = k + 4 * u < rows ? __ldg(rp + 8 * (k + 4 * u)) : pad;
    double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll 1
    for (int32_t r = k; r < rows; r += 4 * UNR) {
        double4 g[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int32_t idx = static_cast<int32_t>(__double_as_longlong(rr[u].y));
            g[u] = idx >= 0 ? ld_ro4(in + idx) : make_double4(0.0, 0.0, 0.0, 0.0);
        }
        double2 nx[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int32_t rn = r + 4 * (UNR + u);
            nx[u] = rn < rows ? __ldg(rp + 8 * rn) : pad;
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            x += rr[u].x * g[u].x;
            y += rr[u].x * g[u].y;
            z += rr[u].x * g[u].z;
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) rr[u] = nx[u];
    }
#pragma unroll
    for (int off = 8; off < 32; off <<= 1) {
        x += __shfl_xor_sync(kFull, x, off);
        y += __shfl_xor_sync(kFull, y, off);
        z += __shfl_xor_sync(kFull, z, off);
    }
    if (!valid || k != 0) return;
    if (out4 != nullptr) {
        out4[i] = row_ptr[i + 1] != row_ptr[i] ? make_double4(x, y, z, 0.0)
                  : i < num_nodes              ? in[i]
                                               : make_double4(0.0, 0.0, 0.0, 0.0);
    } else {
        out3[3 * i] = x;
        out3[3 * i + 1] = y;
        out3[3 * i + 2] = z;
    }
}

__global__ void k_pack4(const double* __restrict__ in, double4* __restrict__ out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_double4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.0);
}
__global__ void k_unpack4(const double4* __restrict__ in, double* __restrict__ out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = in[i];
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
}
__global__ void k_scatter_elems(const int32_t* __restrict__ order, int64_t n, const double* __restrict__ src,
                                double* __restrict__ dst) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) dst[order[k]] = src[k];
}

__global__ void k_iface_pack(int64_t n, const int32_t* __restrict__ rows, const double* __restrict__ own,
                             double* __restrict__ send) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t r = rows[k];
    send[3 * k] = own[3 * r];
    send[3 * k + 1] = own[3 * r + 1];
    send[3 * k + 2] = own[3 * r + 2];
}

__global__ void k_iface_combine(int64_t rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                int64_t num_own, const double* __restrict__ own, const double* __restrict__ recv,
                                double* __restrict__ out) {
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double x = 0.0, y = 0.0, z = 0.0;
    for (int32_t e = ptr[r]; e < ptr[r + 1]; ++e) {
        const int64_t j = idx[e];
        const double* src = j < num_own ? own + 3 * j : recv + 3 * (j - num_own);
        x += src[0];
        y += src[1];
        z += src[2];
    }
    out[3 * r] = x;
    out[3 * r + 1] = y;
    out[3 * r + 2] = z;
}

__global__ void k_zero4(double4* __restrict__ out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_double4(0.0, 0.0, 0.0, 0.0);
}

__global__ void k_stress_batch(int32_t mat, double lambda, double mu, int64_t n, const double* __restrict__ H,
                               double* __restrict__ P) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double h[9], p[9];
    for (int k = 0; k < 9; ++k) h[k] = H[9 * i + k];
    stress<double>(mat, lambda, mu, h, p);
    for (int k = 0; k < 9; ++k) P[9 * i + k] = p[k];
}

// Quadrature point kernel: Gauss B and w (QuadratureGaussian.h:17-39) or the
// smoothed face-normal quadrature (QuadratureSmoothed.h:32-142).
__global__ void k_quadrature_batch(int32_t kind, int32_t smoothed, int64_t n, const double* __restrict__ Xall,
                                   double* __restrict__ Ball, double* __restrict__ wall) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int nn = kind == AM_HEX8_GAUSS ? 8 : 4;
    const double* X = Xall + e * nn * 3;
    if (smoothed) {
        double B[24];
        for (int k = 0; k < nn * 3; ++k) B[k] = 0.0;
        double vol = 0.0;
        if (nn == 4) {
            const int faces[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
            for (int j = 0; j < 4; ++j) {
                const double* p0 = X + 3 * faces[j][0];
                const double* p1 = X + 3 * faces[j][1];
                const double* p2 = X + 3 * faces[j][2];
                const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
                const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
                const double nr[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                                      (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
                vol += p0[0] * nr[0] + p0[1] * nr[1] + p0[2] * nr[2];
                for (int l = 0; l < 3; ++l)
                    for (int i = 0; i < 3; ++i) B[faces[j][l] * 3 + i] += nr[i] / 3.0;
            }
        } else {
            const int faces[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
            for (int j = 0; j < 6; ++j) {
                double mid[3] = {0.0, 0.0, 0.0};
                for (int k = 0; k < 4; ++k)
                    for (int i = 0; i < 3; ++i) mid[i] += X[faces[j][k] * 3 + i];
                for (int i = 0; i < 3; ++i) mid[i] /= 4.0;
                int km1 = 3;
                for (int k = 0; k < 4; ++k) {
                    double e1[3], e2[3];
                    for (int i = 0; i < 3; ++i) {
                        e1[i] = X[faces[j][km1] * 3 + i] - mid[i];
                        e2[i] = X[faces[j][k] * 3 + i] - mid[i];
                    }
                    const double nr[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                                          (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
                    vol += mid[0] * nr[0] + mid[1] * nr[1] + mid[2] * nr[2];
                    for (int l = 0; l < 4; ++l) {
                        const double wgt = (l == k || l == km1) ? 5.0 / 12.0 : 1.0 / 12.0;
                        for (int i = 0; i < 3; ++i) B[faces[j][l] * 3 + i] += nr[i] * wgt;
                    }
                    km1 = k;
                }
            }
        }
        vol /= 3.0;
        for (int k = 0; k < nn * 3; ++k) Ball[e * nn * 3 + k] = B[k] / vol;
        wall[e] = vol;
        return;
    }
    const int ngp = nn == 8 ? 8 : 1;
    for (int gp = 0; gp < ngp; ++gp) {
        double dN[24];
        if (nn == 8) {
            const double loc = 1.0 / sqrt(3.0);
            const double xi[3] = {hex_sign(gp, 0) * loc, hex_sign(gp, 1) * loc, hex_sign(gp, 2) * loc};
            for (int a = 0; a < 8; ++a) {
                const double p0 = hex_sign(a, 0), p1 = hex_sign(a, 1), p2 = hex_sign(a, 2);
                dN[a * 3 + 0] = 0.125 * p0 * (1.0 + p1 * xi[1]) * (1.0 + p2 * xi[2]);
                dN[a * 3 + 1] = 0.125 * p1 * (1.0 + p0 * xi[0]) * (1.0 + p2 * xi[2]);
                dN[a * 3 + 2] = 0.125 * p2 * (1.0 + p0 * xi[0]) * (1.0 + p1 * xi[1]);
            }
        } else {
            const double t[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
            for (int k = 0; k < 12; ++k) dN[k] = t[k];
        }
        double J[9], Ji[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double acc = 0.0;
                for (int a = 0; a < nn; ++a) acc += X[a * 3 + i] * dN[a * 3 + j];
                J[i * 3 + j] = acc;
            }
        const double det = det3(J);
        cof_inv3(J, Ji, det);
        double* B = Ball + (e * ngp + gp) * nn * 3;
        for (int a = 0; a < nn; ++a)
            for (int j = 0; j < 3; ++j)
                B[a * 3 + j] = dN[a * 3 + 0] * Ji[0 * 3 + j] + dN[a * 3 + 1] * Ji[1 * 3 + j] + dN[a * 3 + 2] * Ji[2 * 3 + j];
        wall[e * ngp + gp] = (nn == 8 ? 1.0 : 1.0 / 6.0) * det;
    }
}

inline unsigned grid_for(int64_t n, int per_block) { return static_cast<unsigned>((n + per_block - 1) / per_block); }

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
// Launch with programmatic stream serialization (the kernel calls pdl_wait before it
// reads anything its predecessor writes).
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...) != cudaSuccess) {
        // Clear the error and launch in the ordinary way (the kernel's wait is then a no-op);
        // a failure of that launch is what the caller's error check reports.
        (void)cudaGetLastError();
        kernel<<<grid, block, 0, s>>>(static_cast<KArgs>(args)...);
    }
}

#define AM_DISPATCH_MAT(MATVAR, CALL)                    \
    switch (MATVAR) {                                    \
        case kLinearElastic: { constexpr int M = 0; CALL; break; } \
        case kNeoHookean: { constexpr int M = 1; CALL; break; }    \
        default: { constexpr int M = 2; CALL; break; }             \
    }

void launch_gauss_force(const GaussBlockDev& b, int mixed, const double4* X4, const double4* U4, void* slots,
                        int* status, cudaStream_t s) {
    if (b.num_elems == 0) return;
    if (b.kind == AM_TET4_GAUSS && b.patched == 2 && b.patch_dx32 != nullptr && b.patch_dx64 != nullptr) {
        const unsigned grid = grid_for(2 * b.num_patches, kHex6Block);
        if (b.chunk_ptr != nullptr) {
            if (mixed) {
                AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_hex6_force<float, M, true>, grid, kHex6Block, s, b, X4, U4, static_cast<float4*>(slots), status)));
            } else {
                AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_hex6_force<double, M, true>, grid, kHex6Block, s, b, X4, U4, static_cast<double4*>(slots), status)));
            }
        } else if (mixed) {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_hex6_force<float, M, false>, grid, kHex6Block, s, b, X4, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_hex6_force<double, M, false>, grid, kHex6Block, s, b, X4, U4, static_cast<double4*>(slots), status)));
        }
    } else if (b.kind == AM_TET4_GAUSS && b.patched) {
        const unsigned grid = grid_for(b.num_patches, 8 * kPatchesPerWarp);
        if (mixed) {
            AM_DISPATCH_MAT(b.material, (k_tet4_patch_force<float, M><<<grid, 256, 0, s>>>(b, X4, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (k_tet4_patch_force<double, M><<<grid, 256, 0, s>>>(b, X4, U4, static_cast<double4*>(slots), status)));
        }
    } else if (b.kind == AM_TET4_GAUSS && b.geo64 != nullptr) {
        const unsigned grid = grid_for(b.num_elems, 256);
        if (b.chunk_ptr != nullptr) {
            if (mixed) {
                AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_force_geo<float, M, true>, grid, 256, s, b, U4, static_cast<float4*>(slots), status)));
            } else {
                AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_force_geo<double, M, true>, grid, 256, s, b, U4, static_cast<double4*>(slots), status)));
            }
        } else if (mixed) {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_force_geo<float, M, false>, grid, 256, s, b, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_force_geo<double, M, false>, grid, 256, s, b, U4, static_cast<double4*>(slots), status)));
        }
    } else if (b.kind == AM_TET4_GAUSS) {
        const unsigned grid = grid_for(b.num_elems, 256);
        if (mixed) {
            AM_DISPATCH_MAT(b.material, (k_tet4_force<float, M><<<grid, 256, 0, s>>>(b, X4, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (k_tet4_force<double, M><<<grid, 256, 0, s>>>(b, X4, U4, static_cast<double4*>(slots), status)));
        }
    } else {
        const unsigned grid = grid_for(b.num_elems, 128);
        if (mixed) {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_hex8_force<float, M>, grid, 128, s, b, X4, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_hex8_force<double, M>, grid_for(b.num_elems, 64), 64, s, b, X4, U4, static_cast<double4*>(slots), status)));
        }
    }
}

// Lanes per cell from the block's mean entries per cell: on B200, eight lanes for the
// RKPM nodal cells (about 66 entries) ran the kernel 1.55x faster than a full warp.
inline int lanes_per_cell(const CellBlockDev& b) {
    const double mean = static_cast<double>(b.num_entries) / static_cast<double>(b.num_cells);
    return mean <= 16.0 ? 4 : mean <= 96.0 ? 8 : mean <= 192.0 ? 16 : 32;
}

#define AM_CELL_GROUP(T, LPC)                                                                         \
    AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_force_group<T, M, LPC>, grid_for(b.num_cells * LPC, 256), 256, s, \
                                            b, U4, static_cast<vec4_t<T>*>(slots), status)))

template <typename T, int LPC>
void launch_fbar_lpc(const CellBlockDev& b, const double4* U4, void* slots, int* status, cudaStream_t s) {
    const unsigned gs = grid_for(b.num_cells * LPC, 256);
    k_fbar_h<T, LPC><<<gs, 256, 0, s>>>(b, U4, status);
    AM_DISPATCH_MAT(b.material, (k_fbar_cell<T, M><<<grid_for(b.num_groups * kFbarLanes, 256), 256, 0, s>>>(b, status)));
    k_fbar_force<T, LPC><<<gs, 256, 0, s>>>(b, static_cast<vec4_t<T>*>(slots));
}

template <typename T>
void launch_fbar(const CellBlockDev& b, const double4* U4, void* slots, int* status, cudaStream_t s) {
    const int lpc = lanes_per_cell(b);
    if (lpc == 4) {
        launch_fbar_lpc<T, 4>(b, U4, slots, status, s);
    } else if (lpc == 8) {
        launch_fbar_lpc<T, 8>(b, U4, slots, status, s);
    } else if (lpc == 16) {
        launch_fbar_lpc<T, 16>(b, U4, slots, status, s);
    } else {
        launch_fbar_lpc<T, 32>(b, U4, slots, status, s);
    }
}

template <typename T, int UNR, int G>
void launch_cell_stress_g(const CellBlockDev& b, const double4* U4, int* status, cudaStream_t s) {
    if (b.group_ptr != nullptr) {
        // F-bar: H per subcell, then M per cell of subcells
        launch_pdl(k_cell_stress<T, kLinearElastic, UNR, true, G>, grid_for(b.num_octets * 32, 256), 256, s, b, U4,
                   static_cast<T*>(b.cmat), status);
        AM_DISPATCH_MAT(b.material, (launch_pdl(k_fbar_cell_stress<T, M>, grid_for(b.num_groups * 32, 256), 256, s, b,
                                                static_cast<T*>(b.cmat), status)));
        return;
    }
    AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_stress<T, M, UNR, false, G>, grid_for(b.num_octets * 32, 256), 256, s, b,
                                            U4, static_cast<T*>(b.cmat), status)));
}
template <typename T, int UNR>
void launch_cell_stress_unr(const CellBlockDev& b, const double4* U4, int* status, cudaStream_t s) {
    if (b.group_items[0] == 1)
        launch_cell_stress_g<T, UNR, 1>(b, U4, status, s);
    else
        launch_cell_stress_g<T, UNR, 8>(b, U4, status, s);
}
template <typename T, int UNR>
void launch_cell_gather_unr(const CellBlockDev& b, void* slots, cudaStream_t s) {
    if (b.group_items[1] == 1)
        launch_pdl(k_cell_gather<T, UNR, 1>, grid_for(b.num_node_octets * 32, 256), 256, s, b, static_cast<const T*>(b.cmat),
                   static_cast<vec4_t<T>*>(slots));
    else
        launch_pdl(k_cell_gather<T, UNR, 8>, grid_for(b.num_node_octets * 32, 256), 256, s, b, static_cast<const T*>(b.cmat),
                   static_cast<vec4_t<T>*>(slots));
}
// Rows in flight per lane: unroll[0] (cell kernel) and unroll[1] (gather kernel), 1, 2 or 4.
template <typename T>
void launch_cell_gather_form(const CellBlockDev& b, const double4* U4, void* slots, int* status, cudaStream_t s) {
    if (b.unroll[0] == 1) {
        launch_cell_stress_unr<T, 1>(b, U4, status, s);
    } else if (b.unroll[0] == 2) {
        launch_cell_stress_unr<T, 2>(b, U4, status, s);
    } else {
        launch_cell_stress_unr<T, 4>(b, U4, status, s);
    }
    if (b.unroll[1] == 1) {
        launch_cell_gather_unr<T, 1>(b, slots, s);
    } else if (b.unroll[1] == 2) {
        launch_cell_gather_unr<T, 2>(b, slots, s);
    } else {
        launch_cell_gather_unr<T, 4>(b, slots, s);
    }
}

int launch_cell_force(const CellBlockDev& b, int mixed, const double4* U4, void* slots, int* status, cudaStream_t s) {
    if (b.num_cells == 0) return 0;
    if (b.gather) {
        if (mixed)
            launch_cell_gather_form<float>(b, U4, slots, status, s);
        else
            launch_cell_gather_form<double>(b, U4, slots, status, s);
        return b.group_ptr != nullptr ? 3 : 2;
    }
    if (b.patched == 2) {
        const unsigned grid = grid_for(2 * b.num_patches, kHex6Block);
        if (b.chunk_ptr != nullptr) {
            if (mixed) {
                AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_hex6_force<float, M, true>, grid, kHex6Block, s, b, U4, static_cast<float4*>(slots), status)));
            } else {
                AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_hex6_force<double, M, true>, grid, kHex6Block, s, b, U4, static_cast<double4*>(slots), status)));
            }
        } else if (mixed) {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_hex6_force<float, M, false>, grid, kHex6Block, s, b, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_hex6_force<double, M, false>, grid, kHex6Block, s, b, U4, static_cast<double4*>(slots), status)));
        }
        return 1;
    }
    if (b.group_ptr != nullptr && b.fused) {
        const unsigned grid = grid_for(b.num_groups * 32, 32 * kFbarWarps);
        if (mixed) {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_fbar_fused<float, M>, grid, 32 * kFbarWarps, s, b, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_fbar_fused<double, M>, grid, 32 * kFbarWarps, s, b, U4, static_cast<double4*>(slots), status)));
        }
        return 1;
    }
    if (b.fbar != nullptr) {
        if (mixed)
            launch_fbar<float>(b, U4, slots, status, s);
        else
            launch_fbar<double>(b, U4, slots, status, s);
        return 3;
    }
    if (b.max_entries <= 8) {
        const unsigned grid = grid_for(b.num_cells, 256);
        if (mixed) {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_force_thread<float, M>, grid, 256, s, b, U4, static_cast<float4*>(slots), status)));
        } else {
            AM_DISPATCH_MAT(b.material, (launch_pdl(k_cell_force_thread<double, M>, grid, 256, s, b, U4, static_cast<double4*>(slots), status)));
        }
        return 1;
    }
    const int lpc = lanes_per_cell(b);
    if (mixed) {
        if (lpc == 4) {
            AM_CELL_GROUP(float, 4);
        } else if (lpc == 8) {
            AM_CELL_GROUP(float, 8);
        } else if (lpc == 16) {
            AM_CELL_GROUP(float, 16);
        } else {
            AM_CELL_GROUP(float, 32);
        }
    } else {
        if (lpc == 4) {
            AM_CELL_GROUP(double, 4);
        } else if (lpc == 8) {
            AM_CELL_GROUP(double, 8);
        } else if (lpc == 16) {
            AM_CELL_GROUP(double, 16);
        } else {
            AM_CELL_GROUP(double, 32);
        }
    }
    return 1;
}

void launch_gauss_vjp(const GaussBlockDev& b, const double4* X4, const double4* U4, const double4* L4, double4* slots,
                      double* gmu, double* gkappa, int accumulate, cudaStream_t s) {
    if (b.num_elems == 0) return;
    if (b.kind == AM_TET4_GAUSS && b.patched) {
        const unsigned grid = grid_for(b.num_patches, 32);
        AM_DISPATCH_MAT(b.material, (k_tet4_patch_vjp<M><<<grid, 256, 0, s>>>(b, X4, U4, L4, slots, gmu, gkappa, accumulate)));
    } else if (b.kind == AM_TET4_GAUSS) {
        const unsigned grid = grid_for(b.num_elems, 256);
        AM_DISPATCH_MAT(b.material, (k_tet4_vjp<M><<<grid, 256, 0, s>>>(b, X4, U4, L4, slots, gmu, gkappa, accumulate)));
    } else {
        const unsigned grid = grid_for(b.num_elems, 128);
        AM_DISPATCH_MAT(b.material, (k_hex8_vjp<M><<<grid_for(b.num_elems, 64), 64, 0, s>>>(b, X4, U4, L4, slots, gmu, gkappa, accumulate)));
    }
}

// F-bar cells in the cell-stress form: H_s on u into M, L_s on lam into Lm (the octet
// kernel of the force, FP64), the per-cell VJP writing M = -V_s dP_s, then the gather.
template <int UNR, int G>
void launch_fbar_vjp_g(const CellBlockDev& b, const double4* U4, const double4* L4, double* Lm, double* gmu,
                       double* gkappa, int accumulate, cudaStream_t s) {
    const unsigned grid = grid_for(b.num_octets * 32, 256);
    double* Hm = static_cast<double*>(b.cmat);
    // the H-only instance returns before any status flag
    launch_pdl(k_cell_stress<double, kLinearElastic, UNR, true, G>, grid, 256, s, b, U4, Hm, static_cast<int*>(nullptr));
    launch_pdl(k_cell_stress<double, kLinearElastic, UNR, true, G>, grid, 256, s, b, L4, Lm, static_cast<int*>(nullptr));
    AM_DISPATCH_MAT(b.material, (launch_pdl(k_fbar_cell_vjp<M>, grid_for(b.num_groups * 32, 256), 256, s, b, Hm,
                                            static_cast<const double*>(Lm), gmu, gkappa, accumulate)));
}
template <int UNR>
void launch_fbar_vjp_unr(const CellBlockDev& b, const double4* U4, const double4* L4, double* Lm, double* gmu,
                         double* gkappa, int accumulate, cudaStream_t s) {
    if (b.group_items[0] == 1)
        launch_fbar_vjp_g<UNR, 1>(b, U4, L4, Lm, gmu, gkappa, accumulate, s);
    else
        launch_fbar_vjp_g<UNR, 8>(b, U4, L4, Lm, gmu, gkappa, accumulate, s);
}

int launch_cell_vjp(const CellBlockDev& b, const double4* U4, const double4* L4, double* Lm, double4* slots,
                    double* gmu, double* gkappa, int accumulate, cudaStream_t s) {
    if (b.num_cells == 0) return 0;
    int count = 2;
    if (b.group_ptr != nullptr) {
        if (b.unroll[0] == 1)
            launch_fbar_vjp_unr<1>(b, U4, L4, Lm, gmu, gkappa, accumulate, s);
        else if (b.unroll[0] == 2)
            launch_fbar_vjp_unr<2>(b, U4, L4, Lm, gmu, gkappa, accumulate, s);
        else
            launch_fbar_vjp_unr<4>(b, U4, L4, Lm, gmu, gkappa, accumulate, s);
        count = 4;
    } else if (b.patched == 2) {
        AM_DISPATCH_MAT(b.material, (k_cell_hex6_vjp<M><<<grid_for(b.num_patches, 64), 64, 0, s>>>(b, U4, L4, slots, gmu, gkappa, accumulate)));
        return 1;
    } else {
        const unsigned grid = grid_for(b.num_cells * 32, 256);
        AM_DISPATCH_MAT(b.material, (k_cell_vjp<M><<<grid, 256, 0, s>>>(b, U4, L4, slots, gmu, gkappa, accumulate)));
        if (!b.gather) return 1;
    }
    if (b.unroll[1] == 1) {
        launch_cell_gather_unr<double, 1>(b, slots, s);
    } else if (b.unroll[1] == 2) {
        launch_cell_gather_unr<double, 2>(b, slots, s);
    } else {
        launch_cell_gather_unr<double, 4>(b, slots, s);
    }
    return count;
}

void launch_tet4_geometry(const int32_t* conn, int64_t num_elems, const double4* X4, float* geo32, double* geo64,
                          cudaStream_t s) {
    if (num_elems == 0) return;
    k_tet4_geometry<<<grid_for(num_elems, 256), 256, 0, s>>>(conn, num_elems, X4, geo32, geo64);
}

void launch_hex6_patch_dx(const int32_t* patch_nodes, int64_t num_patches, const double4* X4, float* dx32,
                          double* dx64, cudaStream_t stream) {
    if (num_patches <= 0) return;
    k_hex6_patch_dx<<<grid_for(num_patches, 256), 256, 0, stream>>>(patch_nodes, num_patches, X4, dx32, dx64);
}

void launch_chunk_positions(const GaussBlockDev& b, int32_t* out, cudaStream_t s) {
    if (b.chunk_units == 0) return;
    k_chunk_positions<4, GaussBlockDev><<<grid_for(b.chunk_units, 256), 256, 0, s>>>(b, out);
}
void launch_chunk_positions(const CellBlockDev& b, int32_t* out, cudaStream_t s) {
    if (b.chunk_units == 0) return;
    k_chunk_positions<4, CellBlockDev><<<grid_for(b.chunk_units, 256), 256, 0, s>>>(b, out);
}

void launch_chunk_sum(const GaussBlockDev& b, const double4* scratch, double4* slots, cudaStream_t s) {
    if (b.chunk_units == 0) return;
    k_chunk_sum<4, GaussBlockDev><<<grid_for(b.chunk_units, 256), 256, 0, s>>>(b, scratch, slots);
}
void launch_chunk_sum(const CellBlockDev& b, const double4* scratch, double4* slots, cudaStream_t s) {
    if (b.chunk_units == 0) return;
    k_chunk_sum<4, CellBlockDev><<<grid_for(b.chunk_units, 256), 256, 0, s>>>(b, scratch, slots);
}

void launch_gauss_volume_slots(const GaussBlockDev& b, double density, const double4* X4, double4* slots,
                               cudaStream_t s) {
    if (b.num_elems == 0) return;
    if (b.kind == AM_TET4_GAUSS && b.patched)
        k_tet4_patch_volume_slots<<<grid_for(b.num_patches, 128), 128, 0, s>>>(b, density, X4, slots);
    else
        k_gauss_volume_slots<<<grid_for(b.num_elems, 128), 128, 0, s>>>(b, density, X4, slots);
}

// Per node the slots are summed by LPN lanes: one lane for meshes of Gauss elements
// (at most eight slots per node), four or eight for cell blocks with tens of
// entries per node. With one lane, BATCH = 8 when the slot array fits comfortably
// in L2 (126 MB on B200), else 4: on B200 the eight-deep batch was ~10% faster for
// the 70^3 Tet4 mesh's 44 MB of FP32 slots and ~5-10% slower for the 128^3 Hex8
// mesh's 268 MB.
// Lanes per node. Up to six slots per node (the warp-chunked tet meshes: 3.4 per node on
// the split-hex 70^3 mesh, 5.7 with one thread per tet; one per node and block for cells in
// the cell-stress form) take one lane: on B200 the 70^3 split-hex node kernel ran 14.6
// against 18.9 us (mixed) and 19.4 against 21.0 us (FP64) with two. Meshes of Gauss
// elements with up to a dozen slots per node take two lanes (each reads every other slot
// of the node's contiguous range, so a warp's loads cover whole lines, and a butterfly adds
// the halves) for FP64 slots, and for FP32 slots when the slot array sits in L2; FP32 slots
// streaming from HBM keep one lane per node. On B200, before the warp chunks: 70^3 Tet4 node
// kernel 23.1 -> 21.3 us mixed and 32.0 -> 28.8 us FP64, 128^3 Hex8 153.9 -> 133.8 us
// FP64, but 95.2 -> 103.5 us mixed. Cell meshes with tens of slots per node take four or
// eight lanes.
inline int node_lanes(const NodeDev& nd, int mixed) {
    if (nd.lanes == 1 || nd.lanes == 2 || nd.lanes == 4 || nd.lanes == 8) return nd.lanes;
    const double per_node = static_cast<double>(nd.num_slots) / static_cast<double>(nd.num_nodes);
    if (per_node <= 6.0) return 1;
    if (per_node <= 12.0) return (!mixed || nd.num_slots * 16 <= (int64_t{64} << 20)) ? 2 : 1;
    // one thread per tet on a tet mesh (about 23 slots per node): 2 lanes ran the node
    // kernel in 40.9 us against 49.8 (1), 47.6 (4) and 60.2 (8) on the renumbered 70^3 mesh
    if (per_node <= 32.0) return 2;
    return per_node <= 40.0 ? 4 : 8;
}
inline bool gather_batch8(const NodeDev& nd, int mixed) {
    const int64_t bytes = nd.num_slots * (mixed ? 16 : 32);
    return bytes <= (int64_t{64} << 20);
}

#define AM_NODE_DISPATCH_PDL(KERNEL, ...)                                                             \
    do {                                                                                              \
        const int lpn = node_lanes(nd, mixed);                                                               \
        const unsigned grid = grid_for((nd.subset_nodes ? nd.subset_count : nd.num_nodes) * lpn, kNodeBlock); \
        const bool b8 = gather_batch8(nd, mixed);                                                     \
        if (mixed) {                                                                                  \
            const float4* sl = static_cast<const float4*>(slots);                                     \
            if (lpn == 8) launch_pdl(KERNEL<float, 4, 8>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__);   \
            else if (lpn == 4) launch_pdl(KERNEL<float, 2, 4>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__); \
            else if (lpn == 2) launch_pdl(KERNEL<float, 4, 2>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__); \
            else if (b8) launch_pdl(KERNEL<float, 8, 1>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__);    \
            else launch_pdl(KERNEL<float, 4, 1>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__);            \
        } else {                                                                                      \
            const double4* sl = static_cast<const double4*>(slots);                                   \
            if (lpn == 8) launch_pdl(KERNEL<double, 4, 8>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__);  \
            else if (lpn == 4) launch_pdl(KERNEL<double, 2, 4>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__); \
            else if (lpn == 2) launch_pdl(KERNEL<double, 4, 2>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__); \
            else if (b8) launch_pdl(KERNEL<double, 8, 1>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__);   \
            else launch_pdl(KERNEL<double, 4, 1>, grid, kNodeBlock, s, nd, sl, __VA_ARGS__);           \
        }                                                                                             \
    } while (0)

#define AM_NODE_DISPATCH(KERNEL, ...)                                                                 \
    do {                                                                                              \
        const int lpn = node_lanes(nd, mixed);                                                               \
        const unsigned grid = grid_for(nd.num_nodes * lpn, kNodeBlock);                               \
        const bool b8 = gather_batch8(nd, mixed);                                                     \
        if (mixed) {                                                                                  \
            const float4* sl = static_cast<const float4*>(slots);                                     \
            if (lpn == 8) KERNEL<float, 4, 8><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);        \
            else if (lpn == 4) KERNEL<float, 2, 4><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);   \
            else if (lpn == 2) KERNEL<float, 4, 2><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);   \
            else if (b8) KERNEL<float, 8, 1><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);         \
            else KERNEL<float, 4, 1><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);                 \
        } else {                                                                                      \
            const double4* sl = static_cast<const double4*>(slots);                                   \
            if (lpn == 8) KERNEL<double, 4, 8><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);       \
            else if (lpn == 4) KERNEL<double, 2, 4><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);  \
            else if (lpn == 2) KERNEL<double, 4, 2><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);  \
            else if (b8) KERNEL<double, 8, 1><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);        \
            else KERNEL<double, 4, 1><<<grid, kNodeBlock, 0, s>>>(nd, sl, __VA_ARGS__);                \
        }                                                                                             \
    } while (0)

void launch_gather_force(const NodeDev& nd, int mixed, const void* slots, double* f, int accumulate, cudaStream_t s) {
    AM_NODE_DISPATCH(k_gather_force, f, accumulate);
}
void launch_gather_force4(const NodeDev& nd, int mixed, const void* slots, double4* f, cudaStream_t s) {
    AM_NODE_DISPATCH(k_gather_force4, f);
}

void launch_iface_gather(const NodeDev& nd, int mixed, const void* slots, int64_t num_local,
                         const int32_t* local_nodes, const int32_t* rows, double* buf, cudaStream_t s) {
    if (num_local == 0) return;
    const int lpn = node_lanes(nd, mixed);
    const unsigned grid = grid_for(num_local * lpn, kNodeBlock);
#define AM_IFACE(S, V, L) k_iface_gather<S, L><<<grid, kNodeBlock, 0, s>>>(nd, static_cast<const V*>(slots), num_local, local_nodes, rows, buf)
    if (mixed) {
        if (lpn == 8) AM_IFACE(float, float4, 8);
        else if (lpn == 4) AM_IFACE(float, float4, 4);
        else if (lpn == 2) AM_IFACE(float, float4, 2);
        else AM_IFACE(float, float4, 1);
    } else {
        if (lpn == 8) AM_IFACE(double, double4, 8);
        else if (lpn == 4) AM_IFACE(double, double4, 4);
        else if (lpn == 2) AM_IFACE(double, double4, 2);
        else AM_IFACE(double, double4, 1);
    }
#undef AM_IFACE
}

void launch_init_accel(const NodeDev& nd, int mixed, const void* slots, double4* A4, int* status, cudaStream_t s) {
    AM_NODE_DISPATCH(k_init_accel, A4, status);
}

void launch_prologue(const NodeDev& nd, const StepParams* table, double4* U4, double4* V4, const double4* A4,
                     double4* u_copy, int rebase, cudaStream_t s) {
    k_prologue<<<grid_for(nd.num_nodes, 256), 256, 0, s>>>(nd, table, U4, V4, A4, u_copy, rebase);
}

void launch_node_step(const NodeDev& nd, int mixed, const void* slots, const StepParams* table, int64_t step,
                      int advance, double4* U4, double4* V4, double4* A4, double4* u_copy, int* status,
                      cudaStream_t s, int rebase) {
    AM_NODE_DISPATCH_PDL(k_node_step, table, step, advance, U4, V4, A4, u_copy, status, rebase);
}

void launch_adj_prep(const NodeDev& nd, const StepParams* table, int64_t step, const double4* VB, const double4* AB,
                     double4* L4, cudaStream_t s) {
    k_adj_prep<<<grid_for(nd.num_nodes, 256), 256, 0, s>>>(nd, table, step, VB, AB, L4);
}

void launch_adj_update(const NodeDev& nd, const double4* slots, const StepParams* table, int64_t step, double4* UB,
                       double4* VB, double4* AB, double4* L4, cudaStream_t s) {
    k_adj_update<<<grid_for(nd.num_nodes, kNodeBlock), kNodeBlock, 0, s>>>(nd, slots, table, step, UB, VB, AB, L4);
}

void launch_sensor_seed(const double4* U4, int32_t num_sensors, const int32_t* sensors, double4* UB, double* loss,
                        cudaStream_t s) {
    k_sensor_seed<<<1, 256, 0, s>>>(U4, num_sensors, sensors, UB, loss);
}

void launch_pm_perturb(const NodeDev& nd, const double4* U4, const double4* V4, const double* l, double eps,
                       double4* W4, cudaStream_t s) {
    k_pm_perturb<<<grid_for(nd.num_nodes, 256), 256, 0, s>>>(nd, U4, V4, l, eps, W4);
}
int64_t launch_pm_next(const NodeDev& nd, const double* f_eps, const double* f_u, const double* l, double eps,
                       double4* V4, double* partial, cudaStream_t s) {
    const unsigned grid = grid_for(nd.num_nodes, 256);
    k_pm_next<<<grid, 256, 0, s>>>(nd, f_eps, f_u, l, eps, V4, partial);
    return grid;
}
void launch_pm_scale(int64_t n, double4* V4, double scale, cudaStream_t s) {
    if (n > 0) k_pm_scale<<<grid_for(n, 256), 256, 0, s>>>(n, V4, scale);
}

void launch_gauss_force_lagr(const GaussBlockDev& b, int32_t lagr, int rebase, const double4* XC, const double4* INC,
                             void* slots, int* status, cudaStream_t s) {
    if (b.num_elems == 0) return;
    double4* sl = static_cast<double4*>(slots);
    if (b.kind == AM_HEX8_GAUSS) {
        AM_DISPATCH_MAT(b.material, (launch_pdl(k_hex8_force_lagr<M>, grid_for(b.num_elems, 64), 64, s, b, lagr, rebase, XC, INC, sl, status)));
    } else {
        AM_DISPATCH_MAT(b.material, (launch_pdl(k_tet4_force_lagr<M>, grid_for(b.num_elems, 128), 128, s, b, lagr, rebase, XC, INC, sl, status)));
    }
}

void launch_rk_rows4(int64_t n, int64_t num_nodes, const int64_t* ptr, const int32_t* nbr, const double* val,
                     const double4* U4, double4* P4, cudaStream_t s) {
    if (n > 0) k_rk_rows4<<<grid_for(n * kRkLanes, 128), 128, 0, s>>>(n, num_nodes, ptr, nbr, val, U4, P4);
}
void launch_rk_cols3(int64_t n, const int64_t* tptr, const int32_t* tsrc, const double* tval, const double4* f_local,
                     double* f, cudaStream_t s) {
    if (n > 0) k_rk_cols3<<<grid_for(n * kRkLanes, 128), 128, 0, s>>>(n, tptr, tsrc, tval, f_local, f);
}

void launch_rk_octets(int64_t count, int64_t num_octets, const int32_t* optr, const double2* rec, const double4* in,
                      const int64_t* row_ptr, int64_t num_nodes, double4* out4, double* out3, cudaStream_t s) {
    if (count > 0) k_rk_octets<4><<<grid_for(num_octets * 32, 256), 256, 0, s>>>(count, num_octets, optr, rec, in, row_ptr,
                                                                                num_nodes, out4, out3);
}

void launch_pack4(const double* aos3, double4* out, int64_t n, cudaStream_t s) {
    if (n > 0) k_pack4<<<grid_for(n, 256), 256, 0, s>>>(aos3, out, n);
}
void launch_unpack4(const double4* in, double* aos3, int64_t n, cudaStream_t s) {
    if (n > 0) k_unpack4<<<grid_for(n, 256), 256, 0, s>>>(in, aos3, n);
}
void launch_zero4(double4* out, int64_t n, cudaStream_t s) {
    if (n > 0) k_zero4<<<grid_for(n, 256), 256, 0, s>>>(out, n);
}

void launch_stress_batch(int32_t mat, double lambda, double mu, int64_t n, const double* H, double* P,
                         cudaStream_t s) {
    if (n > 0) k_stress_batch<<<grid_for(n, 128), 128, 0, s>>>(mat, lambda, mu, n, H, P);
}

void launch_quadrature_batch(int32_t kind, int32_t smoothed, int64_t n, const double* X, double* B, double* w,
                             cudaStream_t s) {
    if (n > 0) k_quadrature_batch<<<grid_for(n, 64), 64, 0, s>>>(kind, smoothed, n, X, B, w);
}

void launch_iface_pack(int64_t n, const int32_t* rows, const double* own, double* send, cudaStream_t s) {
    if (n > 0) k_iface_pack<<<grid_for(n, 256), 256, 0, s>>>(n, rows, own, send);
}

void launch_iface_combine(int64_t rows, const int32_t* ptr, const int32_t* idx, int64_t num_own, const double* own,
                          const double* recv, double* out, cudaStream_t s) {
    if (rows > 0) k_iface_combine<<<grid_for(rows, 256), 256, 0, s>>>(rows, ptr, idx, num_own, own, recv, out);
}

void launch_scatter_elems(const int32_t* order, int64_t n, const double* src, double* dst, cudaStream_t s) {
    if (n > 0) k_scatter_elems<<<grid_for(n, 256), 256, 0, s>>>(order, n, src, dst);
}

}  // namespace am
