// am_rkpm.cu -- set-up of RKPM one-pass smoothing cells (the smoothed-cell data
// consumed by the cell force kernels): nodal cells on the thex corner hexes, and
// element cells (one per tet, functions at the vertices).
//
// The nodal smoothing domain of a tet-mesh vertex is the union of the hexes that
// the thex refinement puts at that vertex in each of its tets (corners, edge
// midpoints, face centroids, centroid; MeshLabelerProcessor.h:228-282 labels only
// the original vertices active). Per vertex v (aperi-mech references):
//   neighbours of every refinement point: ball search with the neighbour's kernel
//     radius, sorted by the tweaked squared distance, truncated to max_neighbors
//     (NeighborSearchProcessor.h:224-263, src/NeighborSearchProcessor.cpp:186-245,
//     NeighborSelectorFunctor.h:60-101);
//   reproducing-kernel function values with a linear basis and the cubic B-spline
//     kernel of the neighbour's radius, moment matrix solved in FP64 on the GPU
//     (FunctionCreationProcessor.h:85-130, ShapeFunctionsFunctorReproducingKernel.h:189-257);
//   one-pass smoothed gradients b_{v,j} = sum_hex sum_k B_hex,k V_hex psi_k(j) / V_v
//     (SmoothedCellDataProcessor.h:541-675, QuadratureSmoothed.h:97-142);
//   lumped mass: rho V_hex / 8 to the hex points, scattered through the functions
//     (src/MassUtils.cpp:17-112, FunctionEvaluationProcessor.h:130-176).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/aperi_b200.h"

namespace am {
void set_free_error(const std::string& msg);  // am_context.cu
}

struct am_cells {
    int64_t num_nodes = 0;
    std::vector<double> points;      // P x 3
    std::vector<int64_t> nbr_ptr;    // P + 1
    std::vector<int32_t> nbr;
    std::vector<double> psi;
    std::vector<int64_t> cell_ptr;   // N + 1
    std::vector<int32_t> cell_nodes;
    std::vector<double> cell_grads;  // x 3
    std::vector<double> cell_volumes;
    std::vector<double> mass;
    std::vector<int64_t> group_ptr;  // subcells of each cell, when the cells hold subcells
};

namespace {

struct Fail {
    int code;
    std::string msg;
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Fail{e == cudaErrorMemoryAllocation ? AM_ENOMEM : AM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <typename F>
void parallel_for(int64_t n, F&& fn) {
    const int nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::atomic<int64_t> next(0);
    const int64_t chunk = 256;
    auto work = [&] {
        for (;;) {
            const int64_t b = next.fetch_add(chunk);
            if (b >= n) return;
            const int64_t e = std::min(n, b + chunk);
            for (int64_t i = b; i < e; ++i) fn(i);
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

// ---- reproducing-kernel function values (FP64, one thread per point) ----
__device__ double rk_kernel(double dx, double dy, double dz, double R) {
    const double r = sqrt(dx * dx + dy * dy + dz * dz) / R;
    if (r < 0.5) return 1.0 + 6.0 * r * r * (-1.0 + r);
    if (r < 1.0) return 2.0 * (1.0 + r * (-3.0 + 3.0 * r - 1.0 * r * r));
    return 0.0;
}

// 4x4 inverse by Gauss-Jordan elimination with partial pivoting; false if singular.
__device__ bool gj_inverse4(const double* M, double* R) {
    double A[4][8];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            A[i][j] = M[i * 4 + j];
            A[i][j + 4] = (i == j) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r)
            if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
        if (A[piv][c] == 0.0) return false;
        if (piv != c)
            for (int j = 0; j < 8; ++j) {
                const double t = A[c][j];
                A[c][j] = A[piv][j];
                A[piv][j] = t;
            }
        const double d = 1.0 / A[c][c];
        for (int j = 0; j < 8; ++j) A[c][j] *= d;
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double f = A[r][c];
            if (f == 0.0) continue;
            for (int j = 0; j < 8; ++j) A[r][j] -= f * A[c][j];
        }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) R[i * 4 + j] = A[i][j + 4];
    return true;
}

__global__ void k_rk_values(int64_t P, const double* __restrict__ pts, const double* __restrict__ X,
                            const double* __restrict__ R, const int64_t* __restrict__ ptr,
                            const int32_t* __restrict__ nbr, double* __restrict__ psi) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int64_t s0 = ptr[p], s1 = ptr[p + 1];
    if (s1 == s0) return;
    if (s1 - s0 == 1) {
        psi[s0] = 1.0;
        return;
    }
    const double px = pts[3 * p], py = pts[3 * p + 1], pz = pts[3 * p + 2];
    double M[16];
    for (int k = 0; k < 16; ++k) M[k] = 0.0;
    double ksum = 0.0;
    for (int64_t s = s0; s < s1; ++s) {
        const int32_t j = nbr[s];
        const double h[4] = {1.0, px - X[3 * j], py - X[3 * j + 1], pz - X[3 * j + 2]};
        const double phi = rk_kernel(h[1], h[2], h[3], R[j]);
        if (phi == 0.0) continue;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) M[r * 4 + c] += phi * h[r] * h[c];
        ksum += phi;
    }
    double Mi[16];
    const bool ok = gj_inverse4(M, Mi);
    double nrm = 0.0;
    for (int k = 0; k < 16; ++k) nrm += Mi[k] * Mi[k];
    const bool shepard = !ok || sqrt(nrm) < 1e-15;
    for (int64_t s = s0; s < s1; ++s) {
        const int32_t j = nbr[s];
        const double h[4] = {1.0, px - X[3 * j], py - X[3 * j + 1], pz - X[3 * j + 2]};
        const double phi = rk_kernel(h[1], h[2], h[3], R[j]);
        if (shepard) {
            psi[s] = phi / ksum;
        } else {
            psi[s] = phi == 0.0 ? 0.0 : (Mi[0] * h[0] + Mi[1] * h[1] + Mi[2] * h[2] + Mi[3] * h[3]) * phi;
        }
    }
}

// ---- thex refinement points ----
struct Thex {
    int64_t n_vert = 0;
    std::vector<std::array<int32_t, 2>> edges;
    std::vector<std::array<int32_t, 3>> faces;
    int64_t edge_id(int32_t a, int32_t b) const {
        const std::array<int32_t, 2> k = {std::min(a, b), std::max(a, b)};
        return n_vert + (std::lower_bound(edges.begin(), edges.end(), k) - edges.begin());
    }
    int64_t face_id(int32_t a, int32_t b, int32_t c) const {
        std::array<int32_t, 3> k = {a, b, c};
        std::sort(k.begin(), k.end());
        return n_vert + static_cast<int64_t>(edges.size()) + (std::lower_bound(faces.begin(), faces.end(), k) - faces.begin());
    }
    int64_t centroid_id(int64_t t) const { return n_vert + static_cast<int64_t>(edges.size() + faces.size()) + t; }
};

// Hex8 smoothed quadrature of the corner hex (faces split into 4 triangles about their mid points).
void hex_smoothed(const double* X, double* B, double* vol) {
    static const int faces[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
    for (int k = 0; k < 24; ++k) B[k] = 0.0;
    double V = 0.0;
    for (int f = 0; f < 6; ++f) {
        double mid[3] = {0, 0, 0};
        for (int k = 0; k < 4; ++k)
            for (int i = 0; i < 3; ++i) mid[i] += X[faces[f][k] * 3 + i];
        for (int i = 0; i < 3; ++i) mid[i] /= 4.0;
        int km1 = 3;
        for (int k = 0; k < 4; ++k) {
            double e1[3], e2[3];
            for (int i = 0; i < 3; ++i) {
                e1[i] = X[faces[f][km1] * 3 + i] - mid[i];
                e2[i] = X[faces[f][k] * 3 + i] - mid[i];
            }
            const double n[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                                 (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
            V += mid[0] * n[0] + mid[1] * n[1] + mid[2] * n[2];
            for (int l = 0; l < 4; ++l) {
                const double w = (l == k || l == km1) ? 5.0 / 12.0 : 1.0 / 12.0;
                for (int i = 0; i < 3; ++i) B[faces[f][l] * 3 + i] += n[i] * w;
            }
            km1 = k;
        }
    }
    V /= 3.0;
    for (int k = 0; k < 24; ++k) B[k] /= V;
    *vol = V;
}

// Tet4 smoothed quadrature (QuadratureSmoothed.h:32-63): the four faces' area normals,
// each shared equally by its three nodes, over the volume from the divergence theorem.
// For a tet these are the exact gradients of the linear shape functions.
void tet_smoothed(const double* X, double* B, double* vol) {
    static const int faces[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
    for (int k = 0; k < 12; ++k) B[k] = 0.0;
    double V = 0.0;
    for (int f = 0; f < 4; ++f) {
        const double* p0 = X + 3 * faces[f][0];
        const double* p1 = X + 3 * faces[f][1];
        const double* p2 = X + 3 * faces[f][2];
        const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
        const double n[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                             (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
        V += p0[0] * n[0] + p0[1] * n[1] + p0[2] * n[2];
        for (int l = 0; l < 3; ++l)
            for (int i = 0; i < 3; ++i) B[faces[f][l] * 3 + i] += n[i] / 3.0;
    }
    V /= 3.0;
    for (int k = 0; k < 12; ++k) B[k] /= V;
    *vol = V;
}

// Neighbours of every point of c->points (ball search with the neighbour's kernel
// radius on a uniform grid of cell size rmax, sorted by the tweaked squared distance,
// truncated to max_neighbors) and the reproducing-kernel function values there (FP64,
// on the GPU): fills c->nbr_ptr, c->nbr, c->psi.
void rk_functions(am_cells* c, int64_t N, const double* X, const double* R, double rmax, int32_t max_neighbors) {
    const std::vector<double>& pts = c->points;
    const int64_t P = static_cast<int64_t>(pts.size() / 3);
    // Uniform grid over the active nodes, cell size = largest kernel radius.
    double lo[3] = {X[0], X[1], X[2]}, hi[3] = {X[0], X[1], X[2]};
    for (int64_t j = 0; j < N; ++j)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], X[3 * j + k]);
            hi[k] = std::max(hi[k], X[3 * j + k]);
        }
    int64_t dim[3];
    for (int k = 0; k < 3; ++k) dim[k] = std::max<int64_t>(1, static_cast<int64_t>((hi[k] - lo[k]) / rmax) + 1);
    auto cell_of = [&](const double* x, int k) {
        return std::min<int64_t>(dim[k] - 1, std::max<int64_t>(0, static_cast<int64_t>((x[k] - lo[k]) / rmax)));
    };
    const int64_t ncell = dim[0] * dim[1] * dim[2];
    std::vector<int64_t> gptr(ncell + 1, 0);
    std::vector<int32_t> gnode(N);
    for (int64_t j = 0; j < N; ++j)
        ++gptr[1 + cell_of(X + 3 * j, 0) + dim[0] * (cell_of(X + 3 * j, 1) + dim[1] * cell_of(X + 3 * j, 2))];
    for (int64_t g = 0; g < ncell; ++g) gptr[g + 1] += gptr[g];
    {
        std::vector<int64_t> fill(gptr.begin(), gptr.end() - 1);
        for (int64_t j = 0; j < N; ++j)
            gnode[fill[cell_of(X + 3 * j, 0) + dim[0] * (cell_of(X + 3 * j, 1) + dim[1] * cell_of(X + 3 * j, 2))]++] =
                static_cast<int32_t>(j);
    }
    // Neighbours of every point.
    std::vector<std::vector<int32_t>> nb(P);
    parallel_for(P, [&](int64_t q) {
        const double* x = &pts[q * 3];
        std::vector<std::pair<double, int32_t>> cand;
        const int64_t cx = cell_of(x, 0), cy = cell_of(x, 1), cz = cell_of(x, 2);
        for (int64_t gz = std::max<int64_t>(0, cz - 1); gz <= std::min(dim[2] - 1, cz + 1); ++gz)
            for (int64_t gy = std::max<int64_t>(0, cy - 1); gy <= std::min(dim[1] - 1, cy + 1); ++gy)
                for (int64_t gx = std::max<int64_t>(0, cx - 1); gx <= std::min(dim[0] - 1, cx + 1); ++gx) {
                    const int64_t g = gx + dim[0] * (gy + dim[1] * gz);
                    for (int64_t s = gptr[g]; s < gptr[g + 1]; ++s) {
                        const int32_t j = gnode[s];
                        const double dx = x[0] - X[j * 3], dy = x[1] - X[j * 3 + 1], dz = x[2] - X[j * 3 + 2];
                        if (dx * dx + dy * dy + dz * dz > R[j] * R[j]) continue;
                        const double ex = X[j * 3] * (1 + 1.0e-6) - x[0], ey = X[j * 3 + 1] * (1 + 1.0e-7) - x[1],
                                     ez = X[j * 3 + 2] * (1 + 1.0e-8) - x[2];
                        cand.push_back({ex * ex + ey * ey + ez * ez, j});
                    }
                }
        std::sort(cand.begin(), cand.end());
        if (static_cast<int64_t>(cand.size()) > max_neighbors) cand.resize(max_neighbors);
        nb[q].reserve(cand.size());
        for (const auto& cd : cand) nb[q].push_back(cd.second);
    });
    c->nbr_ptr.assign(P + 1, 0);
    for (int64_t q = 0; q < P; ++q) c->nbr_ptr[q + 1] = c->nbr_ptr[q] + static_cast<int64_t>(nb[q].size());
    const int64_t S = c->nbr_ptr[P];
    c->nbr.resize(S);
    parallel_for(P, [&](int64_t q) { std::copy(nb[q].begin(), nb[q].end(), c->nbr.begin() + c->nbr_ptr[q]); });
    std::vector<std::vector<int32_t>>().swap(nb);
    // Function values on the GPU in FP64.
    c->psi.assign(S, 0.0);
    {
        double *dp = nullptr, *dx = nullptr, *dr = nullptr, *dv = nullptr;
        int64_t* dptr = nullptr;
        int32_t* dn = nullptr;
        auto cleanup = [&] {
            cudaFree(dp);
            cudaFree(dx);
            cudaFree(dr);
            cudaFree(dv);
            cudaFree(dptr);
            cudaFree(dn);
        };
        try {
            ck(cudaMalloc(&dp, P * 3 * sizeof(double)), "rk points");
            ck(cudaMalloc(&dx, N * 3 * sizeof(double)), "rk coords");
            ck(cudaMalloc(&dr, N * sizeof(double)), "rk radii");
            ck(cudaMalloc(&dv, std::max<int64_t>(S, 1) * sizeof(double)), "rk values");
            ck(cudaMalloc(&dptr, (P + 1) * sizeof(int64_t)), "rk ptr");
            ck(cudaMalloc(&dn, std::max<int64_t>(S, 1) * sizeof(int32_t)), "rk nbr");
            ck(cudaMemcpy(dp, pts.data(), P * 3 * sizeof(double), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemcpy(dx, X, N * 3 * sizeof(double), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemcpy(dr, R, N * sizeof(double), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemcpy(dptr, c->nbr_ptr.data(), (P + 1) * sizeof(int64_t), cudaMemcpyHostToDevice), "upload");
            if (S > 0) ck(cudaMemcpy(dn, c->nbr.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemset(dv, 0, std::max<int64_t>(S, 1) * sizeof(double)), "memset");
            k_rk_values<<<static_cast<unsigned>((P + 127) / 128), 128>>>(P, dp, dx, dr, dptr, dn, dv);
            ck(cudaGetLastError(), "rk kernel");
            if (S > 0) ck(cudaMemcpy(c->psi.data(), dv, S * sizeof(double), cudaMemcpyDeviceToHost), "download");
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
    }
}

// Nodal cells on the thex corner hexes; with subcells every corner hex is its own
// subcell and group_ptr collects the hexes of each vertex.
// mode: kOnePass (vertex cells, one-pass gradients), kSubcells (one subcell per corner hex),
// kTwoPass (vertex cells whose entries are the corner-hex points themselves, with the
// hexes' smoothed gradients b_p = sum_hex B_hex,k(p) V_hex / V_cell; the functions
// couple the points to the vertices at run time).
enum NodalMode { kOnePass = 0, kSubcells = 1, kTwoPass = 2 };

int nodal_cells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R, int32_t max_neighbors,
                double density, int mode, am_cells** out) {
    const bool subcells = mode == kSubcells;
    am::set_free_error("");
    if (!out) return AM_EINVAL;
    *out = nullptr;
    try {
        if (N <= 0 || T <= 0 || !X || !tets || !R) throw Fail{AM_EINVAL, "empty mesh or null array"};
        if (max_neighbors <= 0) throw Fail{AM_EINVAL, "max_neighbors must be positive"};
        if (!(density > 0.0)) throw Fail{AM_EINVAL, "density must be positive"};
        for (int64_t i = 0; i < 4 * T; ++i)
            if (tets[i] < 0 || tets[i] >= N) throw Fail{AM_EINVAL, "tet node index out of range"};
        double rmax = 0.0;
        for (int64_t j = 0; j < N; ++j) {
            if (!(R[j] > 0.0)) throw Fail{AM_EINVAL, "kernel radii must be positive"};
            rmax = std::max(rmax, R[j]);
        }
        auto c = new am_cells();
        std::unique_ptr<am_cells> hold(c);
        c->num_nodes = N;
        // Refinement points: vertices, edge midpoints, face centroids, tet centroids.
        Thex tx;
        tx.n_vert = N;
        tx.edges.reserve(6 * T);
        tx.faces.reserve(4 * T);
        for (int64_t t = 0; t < T; ++t) {
            const int32_t* v = tets + 4 * t;
            for (int i = 0; i < 4; ++i)
                for (int j = i + 1; j < 4; ++j) tx.edges.push_back({std::min(v[i], v[j]), std::max(v[i], v[j])});
            for (int i = 0; i < 4; ++i) {
                std::array<int32_t, 3> f;
                int k = 0;
                for (int j = 0; j < 4; ++j)
                    if (j != i) f[k++] = v[j];
                std::sort(f.begin(), f.end());
                tx.faces.push_back(f);
            }
        }
        std::sort(tx.edges.begin(), tx.edges.end());
        tx.edges.erase(std::unique(tx.edges.begin(), tx.edges.end()), tx.edges.end());
        std::sort(tx.faces.begin(), tx.faces.end());
        tx.faces.erase(std::unique(tx.faces.begin(), tx.faces.end()), tx.faces.end());
        const int64_t P = N + static_cast<int64_t>(tx.edges.size() + tx.faces.size()) + T;
        std::vector<double>& pts = c->points;
        pts.resize(P * 3);
        std::copy(X, X + 3 * N, pts.begin());
        int64_t p = N;
        for (const auto& e : tx.edges) {
            for (int k = 0; k < 3; ++k) pts[p * 3 + k] = (X[e[0] * 3 + k] + X[e[1] * 3 + k]) * 0.5;
            ++p;
        }
        for (const auto& f : tx.faces) {
            for (int k = 0; k < 3; ++k) pts[p * 3 + k] = ((X[f[0] * 3 + k] + X[f[1] * 3 + k]) + X[f[2] * 3 + k]) / 3.0;
            ++p;
        }
        for (int64_t t = 0; t < T; ++t) {
            std::array<int32_t, 4> s = {tets[4 * t], tets[4 * t + 1], tets[4 * t + 2], tets[4 * t + 3]};
            std::sort(s.begin(), s.end());
            for (int k = 0; k < 3; ++k)
                pts[p * 3 + k] = (((X[s[0] * 3 + k] + X[s[1] * 3 + k]) + X[s[2] * 3 + k]) + X[s[3] * 3 + k]) * 0.25;
            ++p;
        }
        rk_functions(c, N, X, R, rmax, max_neighbors);
        // Corner hexes of each vertex (tet order) -> one-pass cell gradients.
        std::vector<int64_t> vptr(N + 1, 0);
        for (int64_t i = 0; i < 4 * T; ++i) ++vptr[tets[i] + 1];
        for (int64_t j = 0; j < N; ++j) vptr[j + 1] += vptr[j];
        std::vector<int64_t> vcorner(4 * T);
        {
            std::vector<int64_t> fill(vptr.begin(), vptr.end() - 1);
            for (int64_t i = 0; i < 4 * T; ++i) vcorner[fill[tets[i]]++] = i;  // i = 4 t + corner
        }
        std::vector<std::vector<int32_t>> cn(N);
        std::vector<std::vector<double>> cg(N);
        c->cell_volumes.assign(N, 0.0);
        std::vector<double> hexvol(4 * T);
        std::vector<std::array<int64_t, 8>> hexpts(4 * T);
        parallel_for(T, [&](int64_t t) {
            const int32_t* v = tets + 4 * t;
            for (int i = 0; i < 4; ++i) {
                int32_t o[3];
                int k = 0;
                for (int j = 0; j < 4; ++j)
                    if (j != i) o[k++] = v[j];
                double d[3][3];
                for (int a = 0; a < 3; ++a)
                    for (int q = 0; q < 3; ++q) d[a][q] = X[o[a] * 3 + q] - X[v[i] * 3 + q];
                const double det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) -
                                   d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                                   d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
                if (det < 0) std::swap(o[1], o[2]);
                auto& hp = hexpts[4 * t + i];
                hp = {v[i], tx.edge_id(v[i], o[0]), tx.face_id(v[i], o[0], o[1]), tx.edge_id(v[i], o[1]),
                      tx.edge_id(v[i], o[2]), tx.face_id(v[i], o[0], o[2]), tx.centroid_id(t), tx.face_id(v[i], o[1], o[2])};
            }
        });
        std::atomic<int> bad(0);
        if (subcells) {
            // One subcell per corner hex, in vertex order then tet order; entries are the
            // union of the hex points' neighbours (first appearance), b = sum_k B_k V psi / V.
            const int64_t S = 4 * T;
            std::vector<std::vector<int32_t>> sn(S);
            std::vector<std::vector<double>> sg(S);
            c->cell_volumes.assign(S, 0.0);
            parallel_for(S, [&](int64_t q) {
                thread_local std::vector<int32_t> where;
                if (static_cast<int64_t>(where.size()) < N) where.assign(N, -1);
                const int64_t h = vcorner[q];
                const auto& hp = hexpts[h];
                double hx[24], B[24], V;
                for (int k = 0; k < 8; ++k)
                    for (int d = 0; d < 3; ++d) hx[k * 3 + d] = pts[hp[k] * 3 + d];
                hex_smoothed(hx, B, &V);
                if (!(V > 0.0)) bad = 1;
                hexvol[h] = V;
                c->cell_volumes[q] = V;
                for (int k = 0; k < 8; ++k)
                    for (int64_t e = c->nbr_ptr[hp[k]]; e < c->nbr_ptr[hp[k] + 1]; ++e) {
                        const int32_t j = c->nbr[e];
                        int32_t idx = where[j];
                        if (idx < 0) {
                            idx = static_cast<int32_t>(sn[q].size());
                            where[j] = idx;
                            sn[q].push_back(j);
                            sg[q].insert(sg[q].end(), {0.0, 0.0, 0.0});
                        }
                        for (int d = 0; d < 3; ++d) sg[q][idx * 3 + d] += B[k * 3 + d] * V * c->psi[e];
                    }
                for (double& g : sg[q]) g /= V;
                for (int32_t j : sn[q]) where[j] = -1;
            });
            if (bad) throw Fail{AM_ENONPOS_J, "a corner hex of the thex refinement has non-positive volume"};
            c->cell_ptr.assign(S + 1, 0);
            for (int64_t q = 0; q < S; ++q) c->cell_ptr[q + 1] = c->cell_ptr[q] + static_cast<int64_t>(sn[q].size());
            const int64_t K = c->cell_ptr[S];
            if (K >= (int64_t(1) << 31)) throw Fail{AM_ERANGE, "cell entry count beyond int32 indexing"};
            c->cell_nodes.resize(K);
            c->cell_grads.resize(K * 3);
            parallel_for(S, [&](int64_t q) {
                std::copy(sn[q].begin(), sn[q].end(), c->cell_nodes.begin() + c->cell_ptr[q]);
                std::copy(sg[q].begin(), sg[q].end(), c->cell_grads.begin() + 3 * c->cell_ptr[q]);
            });
            c->group_ptr = vptr;
        } else {
        const bool two_pass = mode == kTwoPass;
        const int64_t W = two_pass ? P : N;  // entry ids: points (two-pass) or nodes
        parallel_for(N, [&](int64_t vtx) {
            thread_local std::vector<int32_t> where;  // node (point) -> entry of the current cell, -1 if none
            if (static_cast<int64_t>(where.size()) < W) where.assign(W, -1);
            double Vc = 0.0;
            for (int64_t s = vptr[vtx]; s < vptr[vtx + 1]; ++s) {
                const int64_t h = vcorner[s];
                const auto& hp = hexpts[h];
                double hx[24], B[24], V;
                for (int k = 0; k < 8; ++k)
                    for (int q = 0; q < 3; ++q) hx[k * 3 + q] = pts[hp[k] * 3 + q];
                hex_smoothed(hx, B, &V);
                if (!(V > 0.0)) bad = 1;
                hexvol[h] = V;
                Vc += V;
                if (two_pass) {
                    for (int k = 0; k < 8; ++k) {
                        const int32_t q8 = static_cast<int32_t>(hp[k]);
                        int32_t idx = where[q8];
                        if (idx < 0) {
                            idx = static_cast<int32_t>(cn[vtx].size());
                            where[q8] = idx;
                            cn[vtx].push_back(q8);
                            cg[vtx].insert(cg[vtx].end(), {0.0, 0.0, 0.0});
                        }
                        for (int q = 0; q < 3; ++q) cg[vtx][idx * 3 + q] += B[k * 3 + q] * V;
                    }
                    continue;
                }
                for (int k = 0; k < 8; ++k)
                    for (int64_t e = c->nbr_ptr[hp[k]]; e < c->nbr_ptr[hp[k] + 1]; ++e) {
                        const int32_t j = c->nbr[e];
                        int32_t idx = where[j];
                        if (idx < 0) {
                            idx = static_cast<int32_t>(cn[vtx].size());
                            where[j] = idx;
                            cn[vtx].push_back(j);
                            cg[vtx].insert(cg[vtx].end(), {0.0, 0.0, 0.0});
                        }
                        for (int q = 0; q < 3; ++q) cg[vtx][idx * 3 + q] += B[k * 3 + q] * V * c->psi[e];
                    }
            }
            for (double& g : cg[vtx]) g /= Vc;
            for (int32_t j : cn[vtx]) where[j] = -1;
            c->cell_volumes[vtx] = Vc;
        });
        if (bad) throw Fail{AM_ENONPOS_J, "a corner hex of the thex refinement has non-positive volume"};
        c->cell_ptr.assign(N + 1, 0);
        for (int64_t j = 0; j < N; ++j) c->cell_ptr[j + 1] = c->cell_ptr[j] + static_cast<int64_t>(cn[j].size());
        const int64_t K = c->cell_ptr[N];
        if (K >= (int64_t(1) << 31)) throw Fail{AM_ERANGE, "cell entry count beyond int32 indexing"};
        c->cell_nodes.resize(K);
        c->cell_grads.resize(K * 3);
        parallel_for(N, [&](int64_t j) {
            std::copy(cn[j].begin(), cn[j].end(), c->cell_nodes.begin() + c->cell_ptr[j]);
            std::copy(cg[j].begin(), cg[j].end(), c->cell_grads.begin() + 3 * c->cell_ptr[j]);
        });
        }
        // Lumped mass: rho V_hex / 8 to each hex point, scattered to the neighbours.
        std::vector<double> mfe(P, 0.0);
        for (int64_t h = 0; h < 4 * T; ++h)
            for (int k = 0; k < 8; ++k) mfe[hexpts[h][k]] += hexvol[h] * density / 8;
        c->mass.assign(N, 0.0);
        for (int64_t q = 0; q < P; ++q)
            for (int64_t e = c->nbr_ptr[q]; e < c->nbr_ptr[q + 1]; ++e) c->mass[c->nbr[e]] += mfe[q] * c->psi[e];
        *out = hold.release();
        return AM_OK;
    } catch (const Fail& f) {
        am::set_free_error(f.msg);
        return f.code;
    } catch (const std::bad_alloc&) {
        am::set_free_error("host allocation failed");
        return AM_ENOMEM;
    } catch (const std::exception& e) {
        am::set_free_error(e.what());
        return AM_EINVAL;
    }
}

}  // namespace

extern "C" {

int am_rkpm_nodal_cells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                        int32_t max_neighbors, double density, am_cells** out) {
    return nodal_cells(N, X, T, tets, R, max_neighbors, density, kOnePass, out);
}

int am_rkpm_nodal_subcells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                           int32_t max_neighbors, double density, am_cells** out) {
    return nodal_cells(N, X, T, tets, R, max_neighbors, density, kSubcells, out);
}

int am_rkpm_nodal_cells_two_pass(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                                 int32_t max_neighbors, double density, am_cells** out) {
    return nodal_cells(N, X, T, tets, R, max_neighbors, density, kTwoPass, out);
}

}  // extern "C"

namespace {

// Element cells of Tet4 (nn = 4) or Hex8 (nn = 8) elements.
int element_cells(int nn, int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                  int32_t max_neighbors, double density, am_cells** out) {
    am::set_free_error("");
    if (!out) return AM_EINVAL;
    *out = nullptr;
    try {
        if (N <= 0 || T <= 0 || !X || !tets || !R) throw Fail{AM_EINVAL, "empty mesh or null array"};
        if (max_neighbors <= 0) throw Fail{AM_EINVAL, "max_neighbors must be positive"};
        if (!(density > 0.0)) throw Fail{AM_EINVAL, "density must be positive"};
        for (int64_t i = 0; i < nn * T; ++i)
            if (tets[i] < 0 || tets[i] >= N) throw Fail{AM_EINVAL, "element node index out of range"};
        double rmax = 0.0;
        for (int64_t j = 0; j < N; ++j) {
            if (!(R[j] > 0.0)) throw Fail{AM_EINVAL, "kernel radii must be positive"};
            rmax = std::max(rmax, R[j]);
        }
        auto c = new am_cells();
        std::unique_ptr<am_cells> hold(c);
        c->num_nodes = N;
        // The functions are needed at the vertices only.
        c->points.assign(X, X + 3 * N);
        rk_functions(c, N, X, R, rmax, max_neighbors);
        // One cell per element: entries = union of the vertices' neighbours (vertex order,
        // then neighbour order); b_{t,j} = sum_k B_{t,k} V_t psi_k(j) / V_t, B the smoothed
        // gradients (for a tet the exact linear ones; for a hex QuadratureSmoothed.h:97-142).
        std::vector<std::vector<int32_t>> cn(T);
        std::vector<std::vector<double>> cg(T);
        c->cell_volumes.assign(T, 0.0);
        std::atomic<int> bad(0);
        parallel_for(T, [&](int64_t t) {
            const int32_t* v = tets + nn * t;
            double B[24], V;
            if (nn == 8) {
                double hx[24];
                for (int k = 0; k < 8; ++k)
                    for (int d = 0; d < 3; ++d) hx[k * 3 + d] = X[v[k] * 3 + d];
                hex_smoothed(hx, B, &V);
                if (!(V > 0.0)) {
                    bad = 1;
                    return;
                }
            } else {
            double J[9];  // J[i][a] = x_{a+1,i} - x_{0,i}
            for (int i = 0; i < 3; ++i)
                for (int a = 0; a < 3; ++a) J[i * 3 + a] = X[v[a + 1] * 3 + i] - X[v[0] * 3 + i];
            const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                               J[2] * (J[3] * J[7] - J[4] * J[6]);
            if (!(det > 0.0)) {
                bad = 1;
                return;
            }
            const double id = 1.0 / det;
            // Rows of J^-1 are the gradients of the barycentric coordinates 1..3.
            const double Ji[9] = {(J[4] * J[8] - J[5] * J[7]) * id, (J[2] * J[7] - J[1] * J[8]) * id,
                                  (J[1] * J[5] - J[2] * J[4]) * id, (J[5] * J[6] - J[3] * J[8]) * id,
                                  (J[0] * J[8] - J[2] * J[6]) * id, (J[2] * J[3] - J[0] * J[5]) * id,
                                  (J[3] * J[7] - J[4] * J[6]) * id, (J[1] * J[6] - J[0] * J[7]) * id,
                                  (J[0] * J[4] - J[1] * J[3]) * id};
            for (int i = 0; i < 3; ++i) {
                B[3 + i] = Ji[0 * 3 + i];
                B[6 + i] = Ji[1 * 3 + i];
                B[9 + i] = Ji[2 * 3 + i];
                B[i] = -(B[3 + i] + B[6 + i] + B[9 + i]);
            }
            V = det / 6.0;
            }
            c->cell_volumes[t] = V;
            for (int k = 0; k < nn; ++k)
                for (int64_t e = c->nbr_ptr[v[k]]; e < c->nbr_ptr[v[k] + 1]; ++e) {
                    const int32_t j = c->nbr[e];
                    size_t idx = std::find(cn[t].begin(), cn[t].end(), j) - cn[t].begin();
                    if (idx == cn[t].size()) {
                        cn[t].push_back(j);
                        cg[t].insert(cg[t].end(), {0.0, 0.0, 0.0});
                    }
                    for (int q = 0; q < 3; ++q) cg[t][idx * 3 + q] += B[k * 3 + q] * V * c->psi[e];
                }
            for (double& g : cg[t]) g /= V;
        });
        if (bad) throw Fail{AM_ENONPOS_J, "an element has non-positive volume"};
        c->cell_ptr.assign(T + 1, 0);
        for (int64_t t = 0; t < T; ++t) c->cell_ptr[t + 1] = c->cell_ptr[t] + static_cast<int64_t>(cn[t].size());
        const int64_t K = c->cell_ptr[T];
        if (K >= (int64_t(1) << 31)) throw Fail{AM_ERANGE, "cell entry count beyond int32 indexing"};
        c->cell_nodes.resize(K);
        c->cell_grads.resize(K * 3);
        parallel_for(T, [&](int64_t t) {
            std::copy(cn[t].begin(), cn[t].end(), c->cell_nodes.begin() + c->cell_ptr[t]);
            std::copy(cg[t].begin(), cg[t].end(), c->cell_grads.begin() + 3 * c->cell_ptr[t]);
        });
        // Lumped mass: rho V_t / nn to the vertices, scattered through the functions.
        std::vector<double> mfe(N, 0.0);
        for (int64_t t = 0; t < T; ++t)
            for (int k = 0; k < nn; ++k) mfe[tets[nn * t + k]] += density * c->cell_volumes[t] / nn;
        c->mass.assign(N, 0.0);
        for (int64_t q = 0; q < N; ++q)
            for (int64_t e = c->nbr_ptr[q]; e < c->nbr_ptr[q + 1]; ++e) c->mass[c->nbr[e]] += mfe[q] * c->psi[e];
        *out = hold.release();
        return AM_OK;
    } catch (const Fail& f) {
        am::set_free_error(f.msg);
        return f.code;
    } catch (const std::bad_alloc&) {
        am::set_free_error("host allocation failed");
        return AM_ENOMEM;
    } catch (const std::exception& e) {
        am::set_free_error(e.what());
        return AM_EINVAL;
    }
}

}  // namespace

extern "C" {

int am_rkpm_element_cells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                          int32_t max_neighbors, double density, am_cells** out) {
    return element_cells(4, N, X, T, tets, R, max_neighbors, density, out);
}

int am_rkpm_hex8_element_cells(int64_t N, const double* X, int64_t E, const int32_t* hexes, const double* R,
                               int32_t max_neighbors, double density, am_cells** out) {
    return element_cells(8, N, X, E, hexes, R, max_neighbors, density, out);
}

int am_smoothed_element_cells(int64_t N, const double* X, int64_t E, int32_t nodes_per_elem, const int32_t* conn,
                              double density, am_cells** out) {
    am::set_free_error("");
    if (!out) return AM_EINVAL;
    *out = nullptr;
    const int nn = nodes_per_elem;
    if (N <= 0 || !X || E < 0 || (nn != 4 && nn != 8) || (E > 0 && !conn) || !(density > 0.0)) {
        am::set_free_error("am_smoothed_element_cells: bad arguments");
        return AM_EINVAL;
    }
    if (E * nn >= (int64_t(1) << 31)) {
        am::set_free_error("cell entry count beyond int32 indexing");
        return AM_ERANGE;
    }
    try {
        for (int64_t k = 0; k < E * nn; ++k)
            if (conn[k] < 0 || conn[k] >= N) throw Fail{AM_EINVAL, "connectivity index out of range"};
        std::unique_ptr<am_cells> hold(new am_cells());
        am_cells* c = hold.get();
        c->num_nodes = N;
        c->cell_ptr.resize(E + 1);
        for (int64_t e = 0; e <= E; ++e) c->cell_ptr[e] = nn * e;
        c->cell_nodes.assign(conn, conn + nn * E);
        c->cell_grads.assign(3 * nn * E, 0.0);
        c->cell_volumes.assign(E, 0.0);
        std::atomic<int> bad(0);
        parallel_for(E, [&](int64_t e) {
            double x[24], B[24], V = 0.0;
            for (int k = 0; k < nn; ++k)
                for (int i = 0; i < 3; ++i) x[3 * k + i] = X[3 * static_cast<int64_t>(conn[nn * e + k]) + i];
            if (nn == 8)
                hex_smoothed(x, B, &V);
            else
                tet_smoothed(x, B, &V);
            if (!(V > 0.0)) {
                bad = 1;
                return;
            }
            std::copy(B, B + 3 * nn, c->cell_grads.begin() + 3 * nn * e);
            c->cell_volumes[e] = V;
        });
        if (bad) throw Fail{AM_ENONPOS_J, "an element has non-positive volume"};
        // Lumped mass rho V / nn to each vertex, in element order (src/MassUtils.cpp:17-46).
        c->mass.assign(N, 0.0);
        for (int64_t e = 0; e < E; ++e)
            for (int k = 0; k < nn; ++k) c->mass[conn[nn * e + k]] += c->cell_volumes[e] * density / nn;
        *out = hold.release();
        return AM_OK;
    } catch (const Fail& f) {
        am::set_free_error(f.msg);
        return f.code;
    } catch (const std::bad_alloc&) {
        am::set_free_error("host allocation failed");
        return AM_ENOMEM;
    }
}

int am_cells_sizes(const am_cells* c, int64_t* num_cells, int64_t* num_entries, int64_t* num_points,
                   int64_t* num_nbr_entries) {
    if (!c) return AM_EINVAL;
    if (num_cells) *num_cells = c->cell_ptr.empty() ? 0 : static_cast<int64_t>(c->cell_ptr.size()) - 1;
    if (num_entries) *num_entries = static_cast<int64_t>(c->cell_nodes.size());
    if (num_points) *num_points = static_cast<int64_t>(c->points.size() / 3);
    if (num_nbr_entries) *num_nbr_entries = static_cast<int64_t>(c->nbr.size());
    return AM_OK;
}

int am_cells_groups(const am_cells* c, int64_t* num_groups, int64_t* group_ptr) {
    if (!c) return AM_EINVAL;
    if (num_groups) *num_groups = c->group_ptr.empty() ? 0 : static_cast<int64_t>(c->group_ptr.size()) - 1;
    if (group_ptr) std::copy(c->group_ptr.begin(), c->group_ptr.end(), group_ptr);
    return AM_OK;
}

int am_cells_get(const am_cells* c, int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads, double* cell_volumes,
                 double* mass) {
    if (!c) return AM_EINVAL;
    if (cell_ptr) std::copy(c->cell_ptr.begin(), c->cell_ptr.end(), cell_ptr);
    if (cell_nodes) std::copy(c->cell_nodes.begin(), c->cell_nodes.end(), cell_nodes);
    if (cell_grads) std::copy(c->cell_grads.begin(), c->cell_grads.end(), cell_grads);
    if (cell_volumes) std::copy(c->cell_volumes.begin(), c->cell_volumes.end(), cell_volumes);
    if (mass) std::copy(c->mass.begin(), c->mass.end(), mass);
    return AM_OK;
}

int am_cells_get_points(const am_cells* c, double* points, int64_t* nbr_ptr, int32_t* nbr, double* values) {
    if (!c) return AM_EINVAL;
    if (points) std::copy(c->points.begin(), c->points.end(), points);
    if (nbr_ptr) std::copy(c->nbr_ptr.begin(), c->nbr_ptr.end(), nbr_ptr);
    if (nbr) std::copy(c->nbr.begin(), c->nbr.end(), nbr);
    if (values) std::copy(c->psi.begin(), c->psi.end(), values);
    return AM_OK;
}

void am_cells_destroy(am_cells* c) { delete c; }

}  // extern "C"
