// consumer.cpp -- a C++ host of libaperi_b200.so without Python: it builds one Tet4 part
// through the element shim (B200Element, an aperi::ElementBase) inside an
// aperi::InternalForceContribution, evaluates the internal force the way the
// reference's solver does (zeroed force field, contribution accumulates), then runs the
// central-difference loop through the C ABI and writes the force and the final state.
//
//   consumer <input.bin> <output.bin>
//
// Input (little-endian): int64 N, E, nsteps, cells (0: Gauss Tet4, 1: finite-element
// element smoothing cells built by am_smoothed_element_cells), material, num_fixed;
// double lambda, mu, density, dt; double coords[N*3]; int32 conn[E*4]; double u[N*3];
// double v0[N*3]; int32 fixed[num_fixed] (nodes with all components held at zero).
// Output: double f[N*3], u[N*3], v[N*3], a[N*3].
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200_element.h"

namespace {

void check(int rc, am_ctx* ctx, const char* what) {
    if (rc != AM_OK) throw std::runtime_error(std::string(what) + ": " + am_last_error(ctx));
}

void cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
void read(FILE* f, T* p, size_t n) {
    if (n && std::fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short input file");
}

template <typename T>
void write(FILE* f, const T* p, size_t n) {
    if (n && std::fwrite(p, sizeof(T), n, f) != n) throw std::runtime_error("short write");
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    am_ctx* ctx = nullptr;
    double* du = nullptr;
    double* df = nullptr;
    try {
        FILE* in = std::fopen(argv[1], "rb");
        if (!in) throw std::runtime_error("cannot open input");
        int64_t hdr[6];
        double par[4];
        read(in, hdr, 6);
        read(in, par, 4);
        const int64_t N = hdr[0], E = hdr[1], nsteps = hdr[2], cells = hdr[3], nfixed = hdr[5];
        const int32_t material = static_cast<int32_t>(hdr[4]);
        std::vector<double> X(3 * N), u(3 * N), v0(3 * N);
        std::vector<int32_t> conn(4 * E), fixed(nfixed);
        read(in, X.data(), X.size());
        read(in, conn.data(), conn.size());
        read(in, u.data(), u.size());
        read(in, v0.data(), v0.size());
        read(in, fixed.data(), fixed.size());
        std::fclose(in);

        check(am_create(N, X.data(), &ctx), nullptr, "am_create");
        cuda(cudaMalloc(&du, 3 * N * sizeof(double)), "cudaMalloc");
        cuda(cudaMalloc(&df, 3 * N * sizeof(double)), "cudaMalloc");
        aperi::Field<aperi::Real> u_field(du, N), f_field(df, N);

        am_block_desc d{};
        d.material = material;
        d.lambda = par[0];
        d.mu = par[1];
        d.density = par[2];
        d.num_elems = E;
        std::vector<double> mass;
        am_cells* cell_data = nullptr;
        std::vector<int64_t> cptr;
        std::vector<int32_t> cnodes;
        std::vector<double> cgrads, cvols;
        if (cells) {
            // element smoothing cells from the library's host set-up: no Python involved
            check(am_smoothed_element_cells(N, X.data(), E, 4, conn.data(), par[2], &cell_data), nullptr,
                  "am_smoothed_element_cells");
            int64_t nc = 0, ne = 0;
            check(am_cells_sizes(cell_data, &nc, &ne, nullptr, nullptr), nullptr, "am_cells_sizes");
            cptr.resize(nc + 1);
            cnodes.resize(ne);
            cgrads.resize(3 * ne);
            cvols.resize(nc);
            mass.resize(N);
            check(am_cells_get(cell_data, cptr.data(), cnodes.data(), cgrads.data(), cvols.data(), mass.data()), nullptr,
                  "am_cells_get");
            am_cells_destroy(cell_data);
            d.kind = AM_SMOOTHED_CELLS;
            d.cell_ptr = cptr.data();
            d.cell_nodes = cnodes.data();
            d.cell_grads = cgrads.data();
            d.cell_volumes = cvols.data();
        } else {
            d.kind = AM_TET4_GAUSS;
            d.conn = conn.data();
        }
        auto element = std::make_shared<B200Element>(ctx, d, static_cast<size_t>(N), u_field, f_field);
        aperi::InternalForceContribution contribution(element);
        if (nfixed > 0) {
            am_bc_desc bc{};
            bc.num_nodes = nfixed;
            bc.nodes = fixed.data();
            bc.component_mask = 7;
            bc.kind = AM_BC_DISPLACEMENT;
            bc.time_function = AM_TF_RAMP;
            const double ab[2] = {0.0, 1.0}, ord[2] = {0.0, 1.0};
            bc.num_points = 2;
            bc.abscissa = ab;
            bc.ordinate = ord;
            bc.active_start = 0.0;
            bc.active_end = 1.7976931348623157e308;  // always active
            check(am_set_boundary_conditions(ctx, 1, &bc), ctx, "am_set_boundary_conditions");
        }
        if (!mass.empty()) check(am_set_mass(ctx, mass.data()), ctx, "am_set_mass");
        check(am_finalize(ctx), ctx, "am_finalize");

        // ExplicitSolver::ComputeForce: zero the force field, then each contribution adds.
        cuda(cudaMemcpy(du, u.data(), 3 * N * sizeof(double), cudaMemcpyHostToDevice), "H2D");
        cuda(cudaMemset(df, 0, 3 * N * sizeof(double)), "memset");
        contribution.ComputeForce(f_field, 0.0, par[3]);
        std::vector<double> f(3 * N), uo(3 * N), vo(3 * N), ao(3 * N);
        cuda(cudaDeviceSynchronize(), "synchronize");
        cuda(cudaMemcpy(f.data(), df, 3 * N * sizeof(double), cudaMemcpyDeviceToHost), "D2H");

        // The time loop through the ABI: state from rest with v0, pre-loop acceleration, steps.
        std::vector<double> zero(3 * N, 0.0);
        check(am_set_state(ctx, AM_HOST, zero.data(), v0.data(), nullptr), ctx, "am_set_state");
        check(am_init_acceleration(ctx, AM_FP64), ctx, "am_init_acceleration");
        check(am_run(ctx, AM_FP64, nsteps, par[3], 0.0), ctx, "am_run");
        check(am_get_state(ctx, AM_HOST, uo.data(), vo.data(), ao.data()), ctx, "am_get_state");

        FILE* out = std::fopen(argv[2], "wb");
        if (!out) throw std::runtime_error("cannot open output");
        write(out, f.data(), f.size());
        write(out, uo.data(), uo.size());
        write(out, vo.data(), vo.size());
        write(out, ao.data(), ao.size());
        std::fclose(out);
        cudaFree(du);
        cudaFree(df);
        am_destroy(ctx);
        std::printf("consumer ok: %lld nodes, %lld elements, %lld steps\n", static_cast<long long>(N),
                    static_cast<long long>(E), static_cast<long long>(nsteps));
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "consumer failed: %s\n", e.what());
        if (du) cudaFree(du);
        if (df) cudaFree(df);
        if (ctx) am_destroy(ctx);
        return 1;
    }
}
