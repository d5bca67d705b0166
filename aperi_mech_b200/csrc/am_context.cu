// am_context.cu -- the C ABI (include/aperi_b200.h): context set-up, layout
// building, the stream-ordered time loop and the checkpointed adjoint.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/aperi_b200.h"
#include "am_host.hpp"
#include "am_order.hpp"
#include "am_chunks.hpp"
#include "am_kernels.cuh"

namespace {

struct AmError {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw AmError{code, msg}; }

void ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(AM_ENOMEM, std::string(what) + ": " + cudaGetErrorString(e));
    }
    fail(AM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
T* dalloc(size_t count, const char* what) {
    void* p = nullptr;
    if (count == 0) return nullptr;
    ck(cudaMalloc(&p, count * sizeof(T)), what);
    return static_cast<T*>(p);
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// NCCL, opened at run time (libnccl.so.2: the copy a host framework already loaded, or
// the system one), so the library carries no link-time dependency on it and a
// process that never decomposes a mesh never loads it.
struct NcclApi {
    void* handle = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
};

const NcclApi& nccl() {
    static NcclApi api = [] {
        NcclApi a;
        a.handle = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        if (!a.handle) return a;
        a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(dlsym(a.handle, "ncclGetUniqueId"));
        a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(dlsym(a.handle, "ncclCommInitRank"));
        a.all_reduce = reinterpret_cast<decltype(a.all_reduce)>(dlsym(a.handle, "ncclAllReduce"));
        a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(dlsym(a.handle, "ncclCommDestroy"));
        a.error_string = reinterpret_cast<decltype(a.error_string)>(dlsym(a.handle, "ncclGetErrorString"));
        a.group_start = reinterpret_cast<decltype(a.group_start)>(dlsym(a.handle, "ncclGroupStart"));
        a.group_end = reinterpret_cast<decltype(a.group_end)>(dlsym(a.handle, "ncclGroupEnd"));
        a.send = reinterpret_cast<decltype(a.send)>(dlsym(a.handle, "ncclSend"));
        a.recv = reinterpret_cast<decltype(a.recv)>(dlsym(a.handle, "ncclRecv"));
        return a;
    }();
    if (!api.handle || !api.get_unique_id || !api.comm_init_rank || !api.all_reduce || !api.comm_destroy)
        fail(AM_ESTATE, "libnccl.so.2 could not be opened");
    return api;
}

void nccl_check(ncclResult_t r, const char* what) {
    if (r != ncclSuccess) {
        const char* msg = nccl().error_string ? nccl().error_string(r) : "";
        fail(AM_ECUDA, std::string(what) + ": " + msg);
    }
}

// Octet rows of the cell-stress form: items 8o .. 8o + 7 (cells, or nodes), item j with
// entries ptr[j] .. ptr[j+1] whose partners (node, or cell) ascend. Rows are aligned by
// offset (partner minus item, or their anchors': on a locality-numbered mesh consecutive
// items see the same offsets, so a row's eight partners are consecutive) when that pads by
// at most 35% over the octet's entries; otherwise each item's entries fill rows from the
// first. src holds, per (row, item) at 8 row + item, the entry or -1 (padding).
struct OctetRows {
    std::vector<int32_t> ptr;
    std::vector<int32_t> src;
};

OctetRows octet_rows(int64_t count, const std::vector<int32_t>& ptr, const std::vector<int32_t>& partner,
                     const int32_t* item_anchor = nullptr, const int32_t* partner_anchor = nullptr, int items = 8) {
    if (items == 1) {
        // a warp per item: its rows are its entries
        OctetRows o;
        o.ptr.assign(ptr.begin(), ptr.begin() + count + 1);
        o.src.resize(static_cast<size_t>(ptr[count]));
        for (size_t e = 0; e < o.src.size(); ++e) o.src[e] = static_cast<int32_t>(e);
        return o;
    }
    // the alignment key of an entry: its partner's anchor minus its item's (anchors default to
    // the indices themselves; F-bar subcells are anchored at their vertex)
    auto key = [&](int64_t item, int32_t e) {
        const int64_t pa = partner_anchor ? partner_anchor[partner[e]] : partner[e];
        return pa - (item_anchor ? item_anchor[item] : item);
    };
    OctetRows o;
    const int64_t O = (count + 7) / 8;
    o.ptr.reserve(O + 1);
    o.ptr.push_back(0);
    std::vector<int32_t> rowsrc;
    for (int64_t q = 0; q < O; ++q) {
        int32_t at[8], end[8];
        int64_t total = 0, longest = 0;
        for (int j = 0; j < 8; ++j) {
            const int64_t item = 8 * q + j;
            at[j] = item < count ? ptr[item] : 0;
            end[j] = item < count ? ptr[item + 1] : 0;
            total += end[j] - at[j];
            longest = std::max<int64_t>(longest, end[j] - at[j]);
        }
        // aligned rows: merge the offset lists, a row per offset (times its largest multiplicity)
        rowsrc.clear();
        int32_t p[8];
        std::copy(at, at + 8, p);
        while (true) {
            int64_t off = INT64_MAX;
            for (int j = 0; j < 8; ++j)
                if (p[j] < end[j]) off = std::min<int64_t>(off, key(8 * q + j, p[j]));
            if (off == INT64_MAX) break;
            int32_t run[8], mult = 0;
            for (int j = 0; j < 8; ++j) {
                run[j] = 0;
                while (p[j] + run[j] < end[j] && key(8 * q + j, p[j] + run[j]) == off) ++run[j];
                mult = std::max(mult, run[j]);
            }
            for (int32_t t = 0; t < mult; ++t)
                for (int j = 0; j < 8; ++j) rowsrc.push_back(t < run[j] ? p[j] + t : -1);
            for (int j = 0; j < 8; ++j) p[j] += run[j];
        }
        const int64_t aligned = static_cast<int64_t>(rowsrc.size()) / 8;
        if (8 * aligned * 100 <= 135 * total) {
            o.src.insert(o.src.end(), rowsrc.begin(), rowsrc.end());
            o.ptr.push_back(o.ptr.back() + static_cast<int32_t>(aligned));
        } else {
            for (int64_t r = 0; r < longest; ++r)
                for (int j = 0; j < 8; ++j) o.src.push_back(at[j] + r < end[j] ? static_cast<int32_t>(at[j] + r) : -1);
            o.ptr.push_back(o.ptr.back() + static_cast<int32_t>(longest));
        }
        if (static_cast<int64_t>(o.src.size()) >= (int64_t(1) << 31)) fail(AM_ERANGE, "octet rows beyond int32 indexing");
    }
    return o;
}

float bits32(int32_t v) {
    float f;
    std::memcpy(&f, &v, sizeof f);
    return f;
}
double bits64(int32_t v) {
    const int64_t w = v;
    double d;
    std::memcpy(&d, &w, sizeof d);
    return d;
}

struct Block {
    int32_t kind = 0;
    int32_t material = 0;
    double lambda = 0, mu = 0, density = 0;
    int64_t num_elems = 0;
    int64_t num_entries = 0;  // slots of this block
    int64_t slot_base = 0;
    int64_t slot_count = -1;  // logical slots when they differ from num_entries (patched cells)
    int32_t* conn = nullptr;
    double* mu_field = nullptr;
    double* kappa_field = nullptr;
    int32_t* cell_ptr = nullptr;
    int32_t* cell_nodes = nullptr;
    double* grads64 = nullptr;
    float* grads32 = nullptr;
    double* volumes = nullptr;
    int32_t max_entries = 0;
    // Updated / semi-Lagrangian state (am_set_formulation): H of the last force evaluation
    // and the semi formulation's reference H, 9 per element.
    double* hstate = nullptr;
    double* href = nullptr;
    // F-bar cells (am_set_cell_groups): the cells are subcells grouped by group_ptr.
    int64_t num_groups = 0;
    int64_t* group_ptr = nullptr;
    int32_t max_group = 0;
    bool fbar_fused = true;
    double* fbar64 = nullptr;  // kFbarStride per subcell, allocated on first use
    float* fbar32 = nullptr;
    // Tet4 element patches (see GaussBlockDev)
    int32_t patched = 0;
    int64_t num_patches = 0;
    int32_t* patch_first = nullptr;
    int32_t* patch_nodes = nullptr;
    uint32_t* patch_local = nullptr;
    uint32_t* patch_gather = nullptr;
    float* patch_dx32 = nullptr;
    double* patch_dx64 = nullptr;
    float* geo32 = nullptr;  // per-tet J^-1 and w (see GaussBlockDev)
    double* geo64 = nullptr;
    int32_t* chunk_ptr = nullptr;  // warp chunks of such a block (see GaussBlockDev)
    uint32_t* chunk_code = nullptr;
    uint32_t* chunk_rank = nullptr;
    int32_t* chunk_pos = nullptr;
    int64_t chunk_units = 0;             // tets, or split-hex half patches (see GaussBlockDev)
    int32_t* chunk_ident = nullptr;      // 0 .. nn E - 1: per-corner positions into chunk_scratch
    double4* chunk_scratch = nullptr;    // nn E per-corner values (VJP, lumped mass), on first use
    // Cell-stress form of a generic cell block (no patches, cells of more than eight entries,
    // no F-bar groups or groups of at most 32 subcells): octet row records of the cells and of the nodes the block
    // touches (one logical slot each), a node of each cell, and the per-cell matrices
    // M = -V P of each precision.
    bool gather = false;
    int32_t unroll[2][2] = {{4, 2}, {4, 4}};  // [FP64, mixed][cell kernel, gather kernel]
    int32_t group_items[2] = {8, 8};          // items per warp: cell side, node side
    int64_t num_octets = 0, num_node_octets = 0, t_count = 0;
    int32_t* o_ptr = nullptr;
    int32_t* n_ptr = nullptr;
    int32_t* c_ref = nullptr;
    float4* orec32 = nullptr;
    double4* orec64 = nullptr;
    float4* nrec32 = nullptr;
    double4* nrec64 = nullptr;
    float* cmat32 = nullptr;
    double* cmat64 = nullptr;
    double* vjp_lmat = nullptr;  // F-bar VJP: L_s per subcell (component arrays), allocated on first use
    std::vector<int32_t> host_cell_ptr;  // until am_finalize: the CSR and gradients the records
    std::vector<double> host_grads;      // are built from, and the F-bar groups
    std::vector<int64_t> host_group_ptr;
    const int32_t* slot_pos = nullptr;  // block-local view into the context's position array
    std::vector<int32_t> host_nodes;    // node of each logical slot (-1: unused), for the node CSR
    // Processing order of a Gauss block's elements: order[k] is the caller's index of the
    // block's k-th element as stored and run here (empty: the caller's order). Per-element
    // inputs are permuted into it and per-element outputs back out of it.
    std::vector<int32_t> order;
    int32_t* order_dev = nullptr;

    // A per-element array given in the caller's order, in the processing order.
    std::vector<double> to_order(const double* v) const {
        if (order.empty()) return std::vector<double>(v, v + num_elems);
        std::vector<double> out(num_elems);
        for (int64_t k = 0; k < num_elems; ++k) out[k] = v[order[k]];
        return out;
    }
    // A per-element host array in the processing order, back into the caller's order.
    void from_order(double* v) const {
        if (order.empty()) return;
        std::vector<double> tmp(v, v + num_elems);
        for (int64_t k = 0; k < num_elems; ++k) v[order[k]] = tmp[k];
    }

    am::GaussBlockDev gauss() const {
        am::GaussBlockDev g{};
        g.kind = kind;
        g.material = material;
        g.lambda = lambda;
        g.mu = mu;
        g.num_elems = num_elems;
        g.conn = conn;
        g.mu_field = mu_field;
        g.kappa_field = kappa_field;
        g.slot_pos = slot_pos;
        g.patched = patched;
        g.num_patches = num_patches;
        g.patch_first = patch_first;
        g.patch_nodes = patch_nodes;
        g.patch_local = patch_local;
        g.patch_gather = patch_gather;
        g.patch_dx32 = patch_dx32;
        g.patch_dx64 = patch_dx64;
        g.geo32 = geo32;
        g.geo64 = geo64;
        g.chunk_ptr = chunk_ptr;
        g.chunk_code = chunk_code;
        g.chunk_rank = chunk_rank;
        g.chunk_pos = chunk_pos;
        g.chunk_units = chunk_units;
        g.hstate = hstate;
        g.href = href;
        return g;
    }
    // A chunked block's per-corner view for the kernels that write one value per element (or
    // patch) node: positions into the scratch array (allocated on first use) at 4 u + a, unit
    // u and corner a. Per tet the identity; a split-hex patch p's node k (tets or cells) is
    // corner a of half patch 2p + r (thread r writes nodes 1, 2, 4, 0 or 5, 6, 7, 3).
    void ensure_corners() {
        const size_t n = static_cast<size_t>(4 * std::max<int64_t>(chunk_units, 1));
        if (!chunk_ident) {
            std::vector<int32_t> id(n);
            if (patched == 2) {
                constexpr int kR[8] = {0, 0, 0, 1, 0, 1, 1, 1}, kA[8] = {3, 0, 1, 3, 2, 0, 1, 2};
                for (int64_t p = 0; p < num_patches; ++p)
                    for (int k = 0; k < 8; ++k) id[8 * p + k] = static_cast<int32_t>(4 * (2 * p + kR[k]) + kA[k]);
            } else {
                for (size_t k = 0; k < n; ++k) id[k] = static_cast<int32_t>(k);
            }
            chunk_ident = dalloc<int32_t>(n, "chunk corner positions");
            ck(cudaMemcpy(chunk_ident, id.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        }
        if (!chunk_scratch) chunk_scratch = dalloc<double4>(n, "chunk corner values");
    }
    am::GaussBlockDev gauss_corners() {
        ensure_corners();
        am::GaussBlockDev g = gauss();
        g.slot_pos = chunk_ident;
        return g;
    }
    am::CellBlockDev cells() const {
        am::CellBlockDev c{};
        c.material = material;
        c.lambda = lambda;
        c.mu = mu;
        c.num_cells = num_elems;
        c.ptr = cell_ptr;
        c.nodes = cell_nodes;
        c.grads64 = grads64;
        c.grads32 = grads32;
        c.volumes = volumes;
        c.mu_field = mu_field;
        c.kappa_field = kappa_field;
        c.slot_pos = slot_pos;
        c.num_entries = num_entries;
        c.max_entries = max_entries;
        c.patched = patched;
        c.num_patches = num_patches;
        c.patch_first = patch_first;
        c.patch_nodes = patch_nodes;
        c.num_groups = num_groups;
        c.group_ptr = group_ptr;
        c.max_group = max_group;
        c.fused = fbar_fused && max_group <= 32 ? 1 : 0;  // kFbarMaxSub
        c.gather = gather ? 1 : 0;
        c.num_octets = num_octets;
        c.o_ptr = o_ptr;
        c.orec32 = orec32;
        c.orec64 = orec64;
        c.c_ref = c_ref;
        c.t_count = t_count;
        c.num_node_octets = num_node_octets;
        c.group_items[0] = group_items[0];
        c.group_items[1] = group_items[1];
        c.n_ptr = n_ptr;
        c.nrec32 = nrec32;
        c.nrec64 = nrec64;
        c.cmat = cmat64;
        c.unroll[0] = unroll[0][0];
        c.unroll[1] = unroll[0][1];
        c.chunk_ptr = chunk_ptr;
        c.chunk_code = chunk_code;
        c.chunk_rank = chunk_rank;
        c.chunk_pos = chunk_pos;
        c.chunk_units = chunk_units;
        return c;
    }
    // The device view for a force evaluation at the given precision (F-bar scratch attached).
    am::CellBlockDev cells_for(int mixed) {
        am::CellBlockDev c = cells();
        if (gather) {
            c.cmat = mixed ? static_cast<void*>(cmat32) : static_cast<void*>(cmat64);
            c.unroll[0] = unroll[mixed ? 1 : 0][0];
            c.unroll[1] = unroll[mixed ? 1 : 0][1];
        }
        if (group_ptr && !c.fused) {
            const size_t n = static_cast<size_t>(std::max<int64_t>(num_elems, 1)) * am::kFbarStride;
            if (mixed) {
                if (!fbar32) fbar32 = dalloc<float>(n, "F-bar scratch (FP32)");
                c.fbar = fbar32;
            } else {
                if (!fbar64) fbar64 = dalloc<double>(n, "F-bar scratch");
                c.fbar = fbar64;
            }
        }
        return c;
    }
    void release() {
        dfree(conn);
        dfree(mu_field);
        dfree(kappa_field);
        dfree(cell_ptr);
        dfree(cell_nodes);
        dfree(grads64);
        dfree(grads32);
        dfree(volumes);
        dfree(patch_first);
        dfree(patch_nodes);
        dfree(patch_local);
        dfree(patch_gather);
        dfree(patch_dx32);
        dfree(patch_dx64);
        dfree(geo32);
        dfree(geo64);
        dfree(chunk_ptr);
        dfree(chunk_code);
        dfree(chunk_rank);
        dfree(chunk_pos);
        dfree(chunk_ident);
        dfree(chunk_scratch);
        dfree(order_dev);
        dfree(hstate);
        dfree(href);
        dfree(group_ptr);
        dfree(fbar64);
        dfree(fbar32);
        dfree(o_ptr);
        dfree(n_ptr);
        dfree(c_ref);
        dfree(orec32);
        dfree(orec64);
        dfree(nrec32);
        dfree(nrec64);
        dfree(cmat32);
        dfree(cmat64);
        dfree(vjp_lmat);
    }

    // The cell-stress form's records (see above), built at am_finalize once the block is
    // known to take no F-bar groups. A cell's entries run in ascending node, a node's in
    // ascending cell; the block's logical slots become its nodes in ascending order.
    void build_gather(int64_t num_points) {
        const int64_t E = num_elems, K = num_entries;
        std::vector<int32_t> cnt(num_points + 1, 0);
        for (int64_t s = 0; s < K; ++s) ++cnt[host_nodes[s] + 1];
        std::vector<int32_t> local(num_points, -1), nodes;
        for (int64_t n = 0; n < num_points; ++n)
            if (cnt[n + 1] > 0) {
                local[n] = static_cast<int32_t>(nodes.size());
                nodes.push_back(static_cast<int32_t>(n));
            }
        const int64_t T = static_cast<int64_t>(nodes.size());
        // cell-major entries sorted by node (cperm: original entry of each sorted position)
        std::vector<int32_t> cperm(K), cpart(K);
        for (int64_t c = 0; c < E; ++c) {
            const int32_t a = host_cell_ptr[c], z = host_cell_ptr[c + 1];
            for (int32_t q = a; q < z; ++q) cperm[q] = q;
            std::stable_sort(cperm.begin() + a, cperm.begin() + z,
                             [&](int32_t x, int32_t y) { return host_nodes[x] < host_nodes[y]; });
            for (int32_t q = a; q < z; ++q) cpart[q] = host_nodes[cperm[q]];
        }
        // node-major entries in ascending cell (tperm: original entry; tpart: cell)
        std::vector<int32_t> tptr(T + 1, 0);
        for (int64_t i = 0; i < T; ++i) tptr[i + 1] = tptr[i] + cnt[nodes[i] + 1];
        std::vector<int32_t> fill(tptr.begin(), tptr.end() - 1), tperm(K), tpart(K);
        for (int64_t c = 0; c < E; ++c)
            for (int32_t s = host_cell_ptr[c]; s < host_cell_ptr[c + 1]; ++s) {
                const int32_t k = fill[local[host_nodes[s]]]++;
                tperm[k] = s;
                tpart[k] = static_cast<int32_t>(c);
            }
        // F-bar subcells are anchored at their group (the vertex of a nodal cell), so that the
        // subcells of a vertex line up on the nodes they share
        std::vector<int32_t> canc;
        if (!host_group_ptr.empty()) {
            canc.resize(E);
            for (size_t g = 0; g + 1 < host_group_ptr.size(); ++g)
                for (int64_t c = host_group_ptr[g]; c < host_group_ptr[g + 1]; ++c) canc[c] = static_cast<int32_t>(g);
        }
        const int32_t* anc = canc.empty() ? nullptr : canc.data();
        // Items of many entries (more than 160 on average: the nodes of F-bar subcells, about
        // 840 each on the h = 1/32 box) take a warp each; 32 lanes then read consecutive rows.
        group_items[0] = E > 0 && K > 160 * E ? 1 : 8;
        group_items[1] = T > 0 && K > 160 * T ? 1 : 8;
        const OctetRows co = octet_rows(E, host_cell_ptr, cpart, anc, nullptr, group_items[0]);
        const OctetRows no = octet_rows(T, tptr, tpart, nullptr, anc, group_items[1]);
        auto records = [&](const OctetRows& o, const std::vector<int32_t>& perm, const std::vector<int32_t>& part,
                           float4*& r32, double4*& r64, const char* what) {
            const size_t R = o.src.size();
            std::vector<float4> h32(R);
            std::vector<double4> h64(R);
            for (size_t q = 0; q < R; ++q) {
                const int32_t e = o.src[q];
                if (e < 0) {
                    h32[q] = make_float4(0.f, 0.f, 0.f, bits32(-1));
                    h64[q] = make_double4(0.0, 0.0, 0.0, bits64(-1));
                    continue;
                }
                const double* g = host_grads.data() + 3 * static_cast<int64_t>(perm[e]);
                h32[q] = make_float4(static_cast<float>(g[0]), static_cast<float>(g[1]), static_cast<float>(g[2]), bits32(part[e]));
                h64[q] = make_double4(g[0], g[1], g[2], bits64(part[e]));
            }
            r32 = dalloc<float4>(std::max<size_t>(R, 1), what);
            r64 = dalloc<double4>(std::max<size_t>(R, 1), what);
            ck(cudaMemcpy(r32, h32.data(), R * sizeof(float4), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemcpy(r64, h64.data(), R * sizeof(double4), cudaMemcpyHostToDevice), "upload");
        };
        records(co, cperm, cpart, orec32, orec64, "cell octet records");
        records(no, tperm, tpart, nrec32, nrec64, "node octet records");
        // The mixed path's differences are taken against the cell's first entry as given
        // (for nodal cells a node next to the cell's own), which keeps them small.
        std::vector<int32_t> ref(E, -1);
        for (int64_t c = 0; c < E; ++c)
            if (host_cell_ptr[c + 1] > host_cell_ptr[c]) ref[c] = host_nodes[host_cell_ptr[c]];
        num_octets = static_cast<int64_t>(co.ptr.size()) - 1;
        num_node_octets = static_cast<int64_t>(no.ptr.size()) - 1;
        o_ptr = dalloc<int32_t>(co.ptr.size(), "cell octet rows");
        n_ptr = dalloc<int32_t>(no.ptr.size(), "node octet rows");
        c_ref = dalloc<int32_t>(std::max<int64_t>(E, 1), "cell reference nodes");
        cmat32 = dalloc<float>(std::max<int64_t>(9 * E, 1), "cell matrices (FP32)");
        cmat64 = dalloc<double>(std::max<int64_t>(9 * E, 1), "cell matrices");
        ck(cudaMemcpy(o_ptr, co.ptr.data(), co.ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(n_ptr, no.ptr.data(), no.ptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(c_ref, ref.data(), E * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        t_count = T;
        host_nodes = std::move(nodes);
        gather = true;
    }
};

using am::WarpChunks;
using am::build_warp_chunks;

// The plan's device arrays; the block's logical slots become the chunks' distinct nodes.
void upload_warp_chunks(Block& b, WarpChunks& wc, int64_t units) {
    const int64_t C = static_cast<int64_t>(wc.ptr.size()) - 1;
    const size_t words = wc.code.size();
    b.chunk_ptr = dalloc<int32_t>(C + 1, "chunk offsets");
    b.chunk_code = dalloc<uint32_t>(words, "chunk entry codes");
    b.chunk_rank = dalloc<uint32_t>(words, "chunk entry ranks");
    ck(cudaMemcpy(b.chunk_ptr, wc.ptr.data(), (C + 1) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(b.chunk_code, wc.code.data(), words * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(b.chunk_rank, wc.rank.data(), words * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload");
    b.slot_count = static_cast<int64_t>(wc.nodes.size());
    b.host_nodes = std::move(wc.nodes);
    b.chunk_units = units;
}

// Greedy element patches: consecutive tets are grouped while the patch has at most
// 6 tets on at most 8 distinct nodes (the six tets of a split hex form one patch).
struct TetPatches {
    std::vector<int32_t> first;   // P + 1
    std::vector<int32_t> nodes;   // P x 8, unused entries repeat entry 0
    std::vector<int32_t> used;    // distinct nodes per patch
    std::vector<uint32_t> local;  // per element: packed local ids
    std::vector<uint32_t> gather; // P x 8: tets touching each patch node and its slot in each
};

TetPatches build_tet_patches(const int32_t* conn, int64_t E) {
    TetPatches tp;
    tp.local.resize(E);
    tp.first.push_back(0);
    int32_t cur[8];
    int nn = 0, nt = 0;
    auto close = [&](int64_t next_first) {
        for (int a = 0; a < 8; ++a) tp.nodes.push_back(a < nn ? cur[a] : cur[0]);
        tp.used.push_back(nn);
        tp.first.push_back(static_cast<int32_t>(next_first));
        nn = 0;
        nt = 0;
    };
    for (int64_t e = 0; e < E; ++e) {
        const int32_t* c = conn + 4 * e;
        int fresh = 0;
        for (int k = 0; k < 4; ++k) {
            bool seen = false;
            for (int a = 0; a < nn; ++a) seen |= cur[a] == c[k];
            for (int j = 0; j < k; ++j) seen |= c[j] == c[k];
            fresh += !seen;
        }
        if (nt > 0 && (nt == 6 || nn + fresh > 8)) close(e);
        uint32_t packed = 0;
        for (int k = 0; k < 4; ++k) {
            int id = -1;
            for (int a = 0; a < nn; ++a)
                if (cur[a] == c[k]) id = a;
            if (id < 0) {
                id = nn;
                cur[nn++] = c[k];
            }
            packed |= static_cast<uint32_t>(id) << (8 * k);
        }
        tp.local[e] = packed;
        ++nt;
    }
    if (nt > 0) close(E);
    const int64_t P = static_cast<int64_t>(tp.used.size());
    tp.gather.assign(8 * P, 0u);
    for (int64_t q = 0; q < P; ++q)
        for (int32_t e = tp.first[q]; e < tp.first[q + 1]; ++e) {
            const uint32_t t = static_cast<uint32_t>(e - tp.first[q]);
            for (int k = 0; k < 4; ++k) {
                const uint32_t a = (tp.local[e] >> (8 * k)) & 0xFFu;
                tp.gather[8 * q + a] |= (1u << t) | (static_cast<uint32_t>(k) << (8 + 2 * t));
            }
        }
    return tp;
}

// True when every patch is exactly one hex's six-tet split in the canonical local
// order (tet t on local nodes 0, a_t, b_t, 3 with a = 1,2,4,5,6,7 and b = 2,4,5,6,7,1).
bool hex6_patches(const TetPatches& tp) {
    static const uint32_t kHex6[6] = {0x03020100u, 0x03040200u, 0x03050400u, 0x03060500u, 0x03070600u, 0x03010700u};
    const int64_t P = static_cast<int64_t>(tp.used.size());
    for (int64_t q = 0; q < P; ++q) {
        if (tp.first[q + 1] - tp.first[q] != 6 || tp.used[q] != 8) return false;
        for (int t = 0; t < 6; ++t)
            if (tp.local[tp.first[q] + t] != kHex6[t]) return false;
    }
    return true;
}

}  // namespace

struct am_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int64_t N = 0;
    double4* X4 = nullptr;
    double4* U4 = nullptr;
    double4* V4 = nullptr;
    double4* A4 = nullptr;
    double4* W4 = nullptr;  // scratch nodal vector (external u)
    double4* L4 = nullptr;  // cotangent / external lambda
    double* mass = nullptr;
    uint32_t* bcword = nullptr;
    double* bcvalues = nullptr;
    int* status = nullptr;
    double* f_scratch = nullptr;   // N x 3
    double* io_scratch = nullptr;  // N x 3 host<->device staging
    int32_t* node_ptr = nullptr;
    int32_t* slot_pos = nullptr;   // logical slot -> node-major position (-1: unused)
    double4* slots64 = nullptr;    // node-major force slots (FP64 path)
    float4* slots32 = nullptr;     // node-major force slots (mixed path)
    int64_t num_slots = 0;         // logical slots
    int64_t num_used_slots = 0;    // slots referenced by a node
    std::vector<double4*> adj_bufs;  // cached adjoint checkpoint / segment buffers
    int64_t adj_key[3] = {0, 0, 0};
    // Tet4 element patches: 2 (default) split-hex patches where every tet lies on a
    // six-tet ring, else generic patches; APERI_B200_TET4_PATCHES=1 generic patches only,
    // =0 one thread per tet.
    int32_t tet4_patches = 2;
    // Element processing order of Gauss blocks: the locality order chosen from the mesh
    // (element_order, the default) or, with APERI_B200_ELEMENT_ORDER=input, the caller's.
    bool locality_order = true;
    // Generic cell blocks in the cell-stress form (per-cell M, node-major gather; the
    // default) or, with APERI_B200_CELL_GATHER=0, with one force slot per entry.
    // APERI_B200_CELL_UNROLL: rows per lane in flight in its kernels (see am_create).
    // Tet4 blocks run one thread per tet stream their reference J^-1 and weight from a
    // table built at am_add_block (the default) or, with APERI_B200_TET4_GEOMETRY=0,
    // gather the coordinates and invert J every step.
    bool tet_geometry = true;
    // One-thread-per-tet blocks (total formulation, geometry table) and split-hex patches
    // write one slot per distinct node of each warp's 32 tets (16 patches) (the default) or,
    // with APERI_B200_WARP_CHUNKS=0, one per tet or patch node.
    bool warp_chunks = true;
    int32_t node_lanes = 0;  // APERI_B200_NODE_LANES (1, 2, 4, 8): lanes per node; 0 chosen per mesh
    bool cell_gather = true;
    // The defaults measured fastest on the RKPM nodal cells of the h = 1/46 box: FP64 4 and
    // 2 (the FP64 gather at 4 holds 128 registers), mixed 4 and 4.
    int32_t cell_unroll[2][2] = {{4, 2}, {4, 4}};
    std::vector<double> host_X;  // coordinates (N x 3), for the element order at am_add_block
    am::StepParams* table = nullptr;
    int64_t table_cap = 0;
    // CUDA graphs of the step loop: kGraphSteps steps (element and node kernels, with their
    // programmatic launch edges) captured once per precision and replayed for every full
    // chunk of a run, the chunk's rows of the step table first copied to a fixed chunk table
    // that the graph reads. Captured at the end of a precision's first run, after it made any
    // lazily allocated buffers. APERI_B200_GRAPHS=0 launches every kernel on the stream.
    static constexpr int64_t kGraphSteps = 32;
    bool use_graphs = true;
    am::StepParams* chunk_table = nullptr;
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
    am::StepParams* table_host = nullptr;  // pinned staging
    cudaEvent_t table_copied = nullptr;    // the last upload out of table_host has executed
    std::vector<Block> blocks;
    std::vector<am::host::BoundaryCondition> bcs;
    double g[3] = {0, 0, 0};
    bool finalized = false;
    bool mass_set = false;
    std::string err;
    int64_t launches = 0;
    bool profiling = false;
    double prof_ms[5] = {0, 0, 0, 0, 0};
    int64_t prof_launches[5] = {0, 0, 0, 0, 0};
    bool mass_from_caller = false;
    // Domain decomposition (am_set_interface / am_set_nccl).
    int64_t iface_local = 0;          // this rank's interface nodes
    int64_t iface_global = 0;         // rows of the exchange buffer (all ranks' interface nodes)
    int32_t* iface_nodes = nullptr;   // local node ids
    int32_t* iface_rows = nullptr;    // their rows
    int32_t* iface_row_of = nullptr;  // per local node: row or -1
    double* iface_buf = nullptr;      // iface_global x 3
    ncclComm_t comm = nullptr;
    // Neighbour exchange (am_set_neighbors), in place of the all-rank sum of every row:
    // the rows are this rank's interface nodes; each neighbour gets the partial forces of
    // the nodes it shares, and every row sums its holders' partials in ascending rank.
    int32_t my_rank = -1;
    std::vector<int32_t> nbr_ranks;
    std::vector<int64_t> nbr_off;     // per neighbour: offset of its entries (num_nbr + 1)
    int32_t* nbr_send_rows = nullptr; // per shared entry: its row
    double* nbr_own = nullptr;        // rows x 3: this rank's partial forces
    double* nbr_send = nullptr;       // shared entries x 3
    double* nbr_recv = nullptr;       // shared entries x 3
    int32_t* comb_ptr = nullptr;      // rows + 1
    int32_t* comb_idx = nullptr;      // sources in ascending holder rank (row, or rows + entry)
    // Overlap of the exchange with the interior nodes' update (APERI_B200_EXCHANGE_OVERLAP=0
    // keeps exchange and update in sequence): a second stream carries the exchange.
    bool overlap = true;
    cudaStream_t xstream = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_done = nullptr;
    // Power method for the stable time increment (am_set_power_method).
    std::vector<double> pm_start;     // N x 3 start vector, scaled by eps l on first use
    double* pm_l = nullptr;           // N: max edge length per node
    double4* pm_v = nullptr;          // the eigenvector estimate
    double* pm_fu = nullptr;          // N x 3: F(u)
    double* pm_fe = nullptr;          // N x 3: F(u + v l eps)
    double* pm_partial = nullptr;     // per-block sums of squares
    bool pm_initialized = false;
    // Updated / semi-Lagrangian formulation (am_set_formulation).
    int32_t lagr = 0;                 // 0 total, 1 updated, 2 semi
    int32_t lagr_interval = 1;        // semi: steps between reference updates
    int64_t lagr_steps = 0;           // steps completed since the state was set
    bool lagr_rebased = false;        // the element H of step lagr_steps is already the reference
    double4* xc = nullptr;            // current (updated) or reference (semi) coordinates
    double4* lagr_inc = nullptr;      // displacement increment
    // Points the cell entries index (am_set_rk_points): the nodes, then the refinement
    // points of two-pass nodal cells. 0: the nodes alone.
    int64_t num_points = 0;
    int64_t points() const { return num_points > N ? num_points : N; }
    // Two-pass reproducing-kernel coupling (am_set_rk_functions).
    int64_t* rk_ptr = nullptr;        // points + 1: rows of Psi
    int32_t* rk_nbr = nullptr;
    double* rk_val = nullptr;
    int64_t* rkt_ptr = nullptr;       // N + 1: columns of Psi (transposed CSR)
    int32_t* rkt_src = nullptr;
    double* rkt_val = nullptr;
    // The same rows and columns in warp octets (APERI_B200_RK_OCTETS=0 keeps the CSR kernels):
    // octet row offsets and (value, index) records.
    bool rk_octets = true;
    int64_t rko_count = 0, rkto_count = 0;
    int32_t* rko_ptr = nullptr;
    int32_t* rkto_ptr = nullptr;
    double2* rko_rec = nullptr;
    double2* rkto_rec = nullptr;
    double4* rk_u = nullptr;          // physical displacement Psi U
    double4* rk_f_local = nullptr;
    double4* rk_l = nullptr;  // the cotangent at the points (VJP with the two-pass coupling)    // element forces at the nodes
    double* rk_f = nullptr;           // N x 3: generalized force Psi^T f_local
    std::vector<cudaEvent_t> events;
    std::vector<std::pair<int, int64_t>> mark_slot;
    size_t n_marks = 0;

    am::NodeDev node_dev() const {
        am::NodeDev nd{};
        nd.num_nodes = N;
        nd.node_ptr = node_ptr;
        nd.mass = mass;
        nd.bcword = bcword;
        nd.bcvalues = bcvalues;
        nd.g[0] = g[0];
        nd.g[1] = g[1];
        nd.g[2] = g[2];
        nd.has_g = (g[0] != 0.0 || g[1] != 0.0 || g[2] != 0.0) ? 1 : 0;
        nd.num_slots = num_used_slots;
        if (iface_row_of) {
            nd.iface_row = iface_row_of;
            nd.iface_f = iface_buf;
        }
        nd.f_given = rk_f;
        nd.lagr = lagr;
        nd.xc = xc;
        nd.inc = lagr_inc;
        nd.lanes = node_lanes;
        return nd;
    }

    int64_t total_elems() const {
        int64_t t = 0;
        for (const auto& b : blocks) t += b.num_elems;
        return t;
    }

    void* slots(int mixed) {
        if (mixed) {
            if (!slots32) slots32 = dalloc<float4>(static_cast<size_t>(num_used_slots), "slot buffer (FP32)");
            return slots32;
        }
        return slots64;
    }

    void check_launch(const char* what) {
        ck(cudaGetLastError(), what);
    }

    // Element/cell force kernels of every block into the slot buffer. With the two-pass
    // coupling (ExplicitSolver::ComputeForce, src/Solvers/Explicit.cpp:146-186) the blocks
    // see the physical displacement Psi U, their forces are gathered per node and scattered
    // to the generalized force Psi^T f, which the node kernels then read (f_given).
    // The two-pass functions: Psi in (nodes) -> out (points); Psi^T in (points) -> out (nodes, N x 3).
    void rk_rows(const double4* in, double4* out) {
        if (rko_rec)
            am::launch_rk_octets(points(), rko_count, rko_ptr, rko_rec, in, rk_ptr, N, out, nullptr, stream);
        else
            am::launch_rk_rows4(points(), N, rk_ptr, rk_nbr, rk_val, in, out, stream);
        ++launches;
    }
    void rk_cols(const double4* in, double* out) {
        if (rkto_rec)
            am::launch_rk_octets(N, rkto_count, rkto_ptr, rkto_rec, in, nullptr, N, nullptr, out, stream);
        else
            am::launch_rk_cols3(N, rkt_ptr, rkt_src, rkt_val, in, out, stream);
        ++launches;
    }

    void element_forces(int mixed, const double4* U) {
        void* s = slots(mixed);
        if (lagr) {
            // The semi formulation's reference configuration moved after the last step
            // (StepScheduler at update_interval, src/Application.cpp:301-308): the element
            // kernels take the stored H as the reference gradient first.
            const int rebase = (lagr == 2 && lagr_steps > 0 && lagr_steps % lagr_interval == 0 && !lagr_rebased) ? 1 : 0;
            for (auto& b : blocks) {
                am::launch_gauss_force_lagr(b.gauss(), lagr, rebase, xc, lagr_inc, s, status, stream);
                ++launches;
            }
            if (rebase) lagr_rebased = true;
            check_launch("element force kernel");
            return;
        }
        if (num_points > N && !rk_ptr) fail(AM_ESTATE, "cells on refinement points run after am_set_rk_functions");
        if (rk_ptr) {
            rk_rows(U, rk_u);
            U = rk_u;
        }
        for (auto& b : blocks) {
            if (b.kind == AM_SMOOTHED_CELLS) {
                if (mixed && !b.grads32) fail(AM_ESTATE, "mixed precision needs FP32 cell gradients");
                launches += am::launch_cell_force(b.cells_for(mixed), mixed, U, s, status, stream);
            } else {
                am::launch_gauss_force(b.gauss(), mixed, X4, U, s, status, stream);
                ++launches;
            }
        }
        if (rk_ptr) {
            am::NodeDev nd = node_dev();
            nd.f_given = nullptr;
            nd.num_nodes = points();  // the local force lives on the points
            am::launch_gather_force4(nd, mixed, s, rk_f_local, stream);
            ++launches;
            rk_cols(rk_f_local, rk_f);
        }
        check_launch("element force kernel");
    }

    // Interface exchange between the element kernels and the node kernel: each rank's
    // partial interface forces into their rows, the rows summed over ranks.
    void exchange(int mixed) {
        if (!iface_row_of) return;
        if (!nbr_ranks.empty()) {
            exchange_send(mixed);
            exchange_finish(stream);
            return;
        }
        ck(cudaMemsetAsync(iface_buf, 0, static_cast<size_t>(iface_global) * 3 * sizeof(double), stream), "memset");
        am::NodeDev nd = node_dev();
        am::launch_iface_gather(nd, mixed, slots(mixed), iface_local, iface_nodes, iface_rows, iface_buf, stream);
        ++launches;
        check_launch("interface gather kernel");
        if (comm)
            nccl_check(nccl().all_reduce(iface_buf, iface_buf, static_cast<size_t>(iface_global) * 3, ncclDouble, ncclSum,
                                         comm, stream),
                       "interface all-reduce");
    }

    // Neighbour exchange, first half (context stream): this rank's partial forces of its
    // interface nodes into their rows, then into the per-neighbour send buffer.
    void exchange_send(int mixed) {
        am::NodeDev nd = node_dev();
        am::launch_iface_gather(nd, mixed, slots(mixed), iface_local, iface_nodes, iface_rows, nbr_own, stream);
        am::launch_iface_pack(nbr_off.back(), nbr_send_rows, nbr_own, nbr_send, stream);
        launches += 2;
        check_launch("interface gather kernels");
    }
    // Second half, on stream s: the grouped sends and receives with each neighbour, then
    // every row's sum in ascending holder rank into the rows the node kernels read.
    void exchange_finish(cudaStream_t s) {
        if (!comm) fail(AM_ESTATE, "the neighbour exchange needs am_set_nccl");
        const NcclApi& a = nccl();
        nccl_check(a.group_start(), "ncclGroupStart");
        for (size_t j = 0; j < nbr_ranks.size(); ++j) {
            const size_t n = static_cast<size_t>(nbr_off[j + 1] - nbr_off[j]) * 3;
            nccl_check(a.send(nbr_send + 3 * nbr_off[j], n, ncclDouble, nbr_ranks[j], comm, s), "ncclSend");
            nccl_check(a.recv(nbr_recv + 3 * nbr_off[j], n, ncclDouble, nbr_ranks[j], comm, s), "ncclRecv");
        }
        nccl_check(a.group_end(), "ncclGroupEnd");
        am::launch_iface_combine(iface_local, comb_ptr, comb_idx, iface_local, nbr_own, nbr_recv, iface_buf, s);
        ++launches;
        check_launch("interface combine kernel");
    }

    // PowerMethodProcessor::ComputeStableTimeIncrement (include/PowerMethodProcessor.h:331-480)
    // at the current displacement, FP64: the increment 2 / sqrt(lambda) of the largest
    // eigenvalue of M^-1 K estimated by power iteration on finite differences of the
    // internal force, with the reference's stopping rules (relative change below
    // tolerance, or the variance of the last five estimates below variation_tolerance
    // times their mean) and its choice of result (the last estimate when converged, else
    // the smallest of the last five).
    double stable_time_increment(double previous, int32_t num_iterations, double eps, double tol, double vartol,
                                 int32_t* iterations, int32_t* converged_out) {
        if (!pm_l) fail(AM_ESTATE, "am_set_power_method first");
        if (iface_row_of) fail(AM_ESTATE, "the power method is not available on a decomposed mesh");
        if (lagr) fail(AM_ESTATE, "the power method is built for the total formulation");
        if (num_iterations < 1 || !(eps > 0.0) || !(tol > 0.0)) fail(AM_EINVAL, "bad power-method parameters");
        if (!pm_initialized) {
            // InitializeEigenvector: the start vector scaled by eps times the node's edge length.
            std::vector<double> l(N);
            ck(cudaMemcpy(l.data(), pm_l, N * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
            std::vector<double4> v(N);
            for (int64_t i = 0; i < N; ++i) {
                const double sc = eps * l[i];
                v[i] = make_double4(pm_start[3 * i] * sc, pm_start[3 * i + 1] * sc, pm_start[3 * i + 2] * sc, 0.0);
            }
            ck(cudaMemcpy(pm_v, v.data(), N * sizeof(double4), cudaMemcpyHostToDevice), "upload");
            pm_initialized = true;
        }
        const am::NodeDev nd = node_dev();
        element_forces(0, U4);
        am::launch_gather_force(nd, 0, slots64, pm_fu, 0, stream);
        ++launches;
        double stable_np1 = previous == 0.0 ? 1.0e-16 : previous;
        constexpr int kWindow = 5;
        double recent[kWindow] = {0, 0, 0, 0, 0};
        bool converged = false, oscillating = false;
        int32_t used = num_iterations;
        const int64_t nblocks = (N + 255) / 256;
        std::vector<double> part(static_cast<size_t>(nblocks));
        for (int32_t k = 0; k < num_iterations; ++k) {
            const double stable_n = stable_np1;
            am::launch_pm_perturb(nd, U4, pm_v, pm_l, eps, W4, stream);
            element_forces(0, W4);
            am::launch_gather_force(nd, 0, slots64, pm_fe, 0, stream);
            am::launch_pm_next(nd, pm_fe, pm_fu, pm_l, eps, pm_v, pm_partial, stream);
            launches += 3;
            check_launch("power-method kernels");
            ck(cudaMemcpyAsync(part.data(), pm_partial, nblocks * sizeof(double), cudaMemcpyDeviceToHost, stream), "D2H");
            ck(cudaStreamSynchronize(stream), "synchronize");
            double sum = 0.0;
            for (double x : part) sum += x;
            const double lambda = std::sqrt(sum);
            if (!(lambda > 0.0) || !std::isfinite(lambda)) fail(AM_ENAN, "power method: zero or non-finite estimate");
            am::launch_pm_scale(N, pm_v, 1.0 / lambda, stream);
            ++launches;
            stable_np1 = 2.0 / std::sqrt(lambda);
            recent[k % kWindow] = stable_np1;
            if (std::abs(stable_np1 - stable_n) < tol * stable_np1) {
                converged = true;
                used = k + 1;
                break;
            }
            if (k >= kWindow) {
                double mean = 0.0;
                for (double r : recent) mean += r;
                mean /= kWindow;
                double var = 0.0;
                for (double r : recent) var += (r - mean) * (r - mean);
                var /= (kWindow - 1);
                if (k > kWindow + 1) {
                    // The reference's alternation test over the window (its first pass
                    // always ends the scan, so it never reports an oscillation).
                    double alt = 0.0;
                    for (int i = 0; i < kWindow - 1; ++i) {
                        const double diff = recent[i + 1] - recent[i];
                        if (i > 0 && diff * alt < 0) {
                            oscillating = true;
                        } else {
                            oscillating = false;
                            break;
                        }
                        alt = diff;
                    }
                }
                if (var < vartol * mean || (oscillating && var < vartol * mean * 2.0)) {
                    converged = true;
                    used = k + 1;
                    break;
                }
            }
        }
        double result = stable_np1;
        if (!converged || oscillating) result = *std::min_element(recent, recent + kWindow);
        if (iterations) *iterations = used;
        if (converged_out) *converged_out = converged ? 1 : 0;
        return result;
    }

    // With the two-pass coupling (f = Psi^T F(Psi u)) the VJP runs at (Psi u, Psi lam) and its
    // point values are gathered and mapped back by Psi^T into rk_f, the node kernels' force.
    void vjp(const double4* U, const double4* L, double* gmu, double* gkappa, int accumulate) {
        if (rk_ptr) {
            rk_rows(U, rk_u);
            rk_rows(L, rk_l);
            U = rk_u;
            L = rk_l;
        }
        int64_t off = 0;
        for (const auto& b : blocks) {
            double* gm = gmu ? gmu + off : nullptr;
            double* gk = gkappa ? gkappa + off : nullptr;
            if (b.kind == AM_SMOOTHED_CELLS && b.chunk_ptr) {
                // per-corner values, then the chunk sums (scratch allocated by prepare_vjp)
                am::CellBlockDev c = b.cells();
                c.slot_pos = b.chunk_ident;
                launches += am::launch_cell_vjp(c, U, L, b.vjp_lmat, b.chunk_scratch, gm, gk, accumulate, stream);
                am::launch_chunk_sum(b.cells(), b.chunk_scratch, slots64, stream);
                ++launches;
            } else if (b.kind == AM_SMOOTHED_CELLS) {
                launches += am::launch_cell_vjp(b.cells(), U, L, b.vjp_lmat, slots64, gm, gk, accumulate, stream);
            } else if (b.chunk_ptr) {
                // per-corner values, then the chunk sums (scratch allocated by prepare_vjp)
                am::GaussBlockDev g = b.gauss();
                g.slot_pos = b.chunk_ident;
                am::launch_gauss_vjp(g, X4, U, L, b.chunk_scratch, gm, gk, accumulate, stream);
                am::launch_chunk_sum(b.gauss(), b.chunk_scratch, slots64, stream);
                launches += 2;
            } else {
                am::launch_gauss_vjp(b.gauss(), X4, U, L, slots64, gm, gk, accumulate, stream);
                ++launches;
            }
            off += b.num_elems;
        }
        if (rk_ptr) {
            am::NodeDev nd = node_dev();
            nd.f_given = nullptr;
            nd.num_nodes = points();
            am::launch_gather_force4(nd, 0, slots64, rk_f_local, stream);
            ++launches;
            rk_cols(rk_f_local, rk_f);
        }
        check_launch("vjp kernel");
    }

    // The VJP's refusals and scratch: F-bar cells only in the cell-stress form (cells of at
    // most 32 subcells), which keeps L_s per subcell beside H_s.
    void prepare_vjp(const char* what) {
        for (auto& b : blocks) {
            if (b.chunk_ptr) b.ensure_corners();
            if (!b.group_ptr) continue;
            if (!b.gather) fail(AM_ESTATE, std::string(what) + " on F-bar cells needs the cell-stress form (cells of at most 32 subcells)");
            if (!b.vjp_lmat) b.vjp_lmat = dalloc<double>(std::max<int64_t>(9 * b.num_elems, 1), "F-bar VJP scratch");
        }
    }

    // Per-element arrays over all blocks (block after block), from the processing order
    // back into the caller's: on the host in place, on the device through a scratch copy.
    void elems_to_caller_host(double* v) const {
        if (!v) return;
        int64_t off = 0;
        for (const auto& b : blocks) {
            b.from_order(v + off);
            off += b.num_elems;
        }
    }
    void elems_to_caller_device(double* v) {
        if (!v) return;
        int64_t off = 0;
        for (const auto& b : blocks) {
            if (b.order_dev) {
                double* tmp = dalloc<double>(b.num_elems, "element scratch");
                std::unique_ptr<double, void (*)(double*)> hold(tmp, [](double* p) { cudaFree(p); });
                ck(cudaMemcpyAsync(tmp, v + off, b.num_elems * sizeof(double), cudaMemcpyDeviceToDevice, stream), "copy");
                am::launch_scatter_elems(b.order_dev, b.num_elems, tmp, v + off, stream);
                ++launches;
                ck(cudaStreamSynchronize(stream), "synchronize");
            }
            off += b.num_elems;
        }
    }

    void reset_status() { ck(cudaMemsetAsync(status, 0, 2 * sizeof(int), stream), "reset status"); }

    void check_status() {
        int h[2] = {0, 0};
        ck(cudaMemcpyAsync(h, status, sizeof(h), cudaMemcpyDeviceToHost, stream), "read status");
        ck(cudaStreamSynchronize(stream), "synchronize");
        if (h[0] == AM_ENONPOS_J) {
            // Gauss elements are counted in the processing order; with one block it maps back.
            int64_t idx = h[1];
            if (blocks.size() == 1 && !blocks[0].order.empty() && idx >= 0 && idx < blocks[0].num_elems)
                idx = blocks[0].order[idx];
            fail(AM_ENONPOS_J, "non-positive Jacobian determinant at element/cell " + std::to_string(idx));
        }
        if (h[0] == AM_ENAN) fail(AM_ENAN, "non-finite acceleration at node " + std::to_string(h[1]));
        if (h[0] != 0) fail(h[0], "device status " + std::to_string(h[0]));
    }

    // Profiling marks: each mark closes the interval since the previous mark and
    // books it to a slot (-1: not booked). Elapsed times are read lazily by
    // am_profile_read, so marks add no host synchronization to the timed work.
    // Creates events up to `count` pending marks. Called before work is enqueued (at
    // am_profile_enable and at the start of each run), so event creation never sits
    // between the kernels being timed.
    void reserve_marks(size_t count) {
        while (events.size() < count) {
            cudaEvent_t e;
            ck(cudaEventCreate(&e), "event create");
            events.push_back(e);
        }
    }

    void mark(int slot, int64_t nlaunch) {
        if (!profiling) return;
        if (n_marks >= events.size()) reserve_marks(std::max<size_t>(2 * events.size(), 64));
        ck(cudaEventRecord(events[n_marks], stream), "event record");
        mark_slot.resize(n_marks + 1);
        mark_slot[n_marks] = {slot, nlaunch};
        ++n_marks;
    }

    void collect_marks() {
        if (n_marks == 0) return;
        ck(cudaStreamSynchronize(stream), "synchronize (profiling)");
        for (size_t k = 1; k < n_marks; ++k) {
            const int slot = mark_slot[k].first;
            if (slot < 0) continue;
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, events[k - 1], events[k]), "elapsed");
            prof_ms[slot] += ms;
            prof_launches[slot] += mark_slot[k].second;
        }
        n_marks = 0;
    }

    // Host time-function evaluation for steps [0, dts.size()) from t0 into the device table.
    void upload_table(const std::vector<double>& dts, double t0) {
        const int64_t n = static_cast<int64_t>(dts.size());
        if (n + 1 > table_cap) {
            dfree(table);
            if (table_host) cudaFreeHost(table_host);
            table_host = nullptr;
            table_cap = std::max<int64_t>({n + 1, 2 * table_cap, 1024});
            table = dalloc<am::StepParams>(table_cap, "step table");
            ck(cudaMallocHost(&table_host, table_cap * sizeof(am::StepParams)), "pinned step table");
        }
        // The staging buffer is reused once the previous upload out of it has executed;
        // kernels still reading the device table are ordered before the new copy.
        if (!table_copied) ck(cudaEventCreateWithFlags(&table_copied, cudaEventDisableTiming), "event create");
        ck(cudaEventSynchronize(table_copied), "wait for the previous table upload");
        double time = t0;
        for (int64_t k = 0; k < n; ++k) {
            am::StepParams& P = table_host[k];
            std::memset(&P, 0, sizeof(P));
            P.dt = dts[k];
            P.half = 0.5 * dts[k];
            const double t_mid = time + 0.5 * dts[k];
            const double t_next = time + dts[k];
            for (size_t b = 0; b < bcs.size(); ++b) {
                if (bcs[b].Active(t_mid)) {
                    P.vact |= 1u << b;
                    P.vscale[b] = bcs[b].VelocityScale(t_mid);
                }
                if (bcs[b].Active(t_next)) {
                    P.aact |= 1u << b;
                    P.ascale[b] = bcs[b].AccelerationScale(t_next);
                }
            }
            time += dts[k];
        }
        ck(cudaMemcpyAsync(table, table_host, n * sizeof(am::StepParams), cudaMemcpyHostToDevice, stream), "table upload");
        ck(cudaEventRecord(table_copied, stream), "event record");
    }

    // A setter that changes what the step kernels are given (conditions, fields, mass, body
    // acceleration, functions, exchange) drops the captured graphs; the next run captures anew.
    // An executable graph still in flight is freed once it completes.
    void drop_graphs() {
        for (auto& g : step_graph) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
    }

    // Captures kGraphSteps advancing steps (element kernels, node kernel) reading the chunk
    // table, on the context stream.
    int64_t graph_step_launches = 0;
    void capture_step_graph(int mixed) {
        if (!chunk_table) chunk_table = dalloc<am::StepParams>(kGraphSteps + 1, "chunk step table");
        const am::NodeDev nd = node_dev();
        void* s = slots(mixed);
        const int64_t before = launches;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaGraph_t g = nullptr;
        try {
            for (int64_t k = 0; k < kGraphSteps; ++k) {
                element_forces(mixed, U4);
                am::launch_node_step(nd, mixed, s, chunk_table, k, 1, U4, V4, A4, nullptr, status, stream, 0);
                ++launches;
            }
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            launches = before;
            throw;
        }
        ck(cudaStreamEndCapture(stream, &g), "end capture");
        graph_step_launches = (launches - before) / kGraphSteps;
        launches = before;
        const cudaError_t e = cudaGraphInstantiate(&step_graph[mixed], g, 0);
        cudaGraphDestroy(g);
        ck(e, "graph instantiate");
    }

    // Steps [n0, n1) of the uploaded table, from a consistent (U4, V4, A4). u_hist[k]
    // (optional) receives the displacement the element kernels use at step n0+k.
    void run_range(int mixed, int64_t n0, int64_t n1, double4* const* u_hist) {
        if (n1 <= n0) return;
        if (profiling) reserve_marks(n_marks + static_cast<size_t>(3 * (n1 - n0) + 2));
        const am::NodeDev nd = node_dev();
        void* s = slots(mixed);
        mark(-1, 0);
        // Semi formulation: a reference update due at the end of the previous run moves the
        // coordinates in this run's first displacement update.
        const auto due = [&](int64_t done) { return lagr == 2 && done > 0 && done % lagr_interval == 0; };
        am::launch_prologue(nd, table + n0, U4, V4, A4, u_hist ? u_hist[0] : nullptr, due(lagr_steps) ? 1 : 0, stream);
        ++launches;
        check_launch("prologue kernel");
        mark(1, 1);
        const bool split = !nbr_ranks.empty() && overlap && comm && xstream;
        int64_t n = n0;
        // Full chunks by graph replay (forward runs on a single domain, total formulation, no
        // per-kernel marks). The run's last step (which does not advance) stays on the stream.
        const bool graphs = use_graphs && !u_hist && !lagr && !iface_row_of && !profiling;
        if (graphs && step_graph[mixed] && n1 - n0 - 1 >= kGraphSteps) {
            for (; n1 - n - 1 >= kGraphSteps; n += kGraphSteps) {
                ck(cudaMemcpyAsync(chunk_table, table + n, (kGraphSteps + 1) * sizeof(am::StepParams),
                                   cudaMemcpyDeviceToDevice, stream), "chunk table");
                ck(cudaGraphLaunch(step_graph[mixed], stream), "graph launch");
                launches += kGraphSteps * graph_step_launches;
            }
        }
        for (; n < n1; ++n) {
            element_forces(mixed, U4);
            mark(0, static_cast<int64_t>(blocks.size()));
            const int advance = (n + 1 < n1) ? 1 : 0;
            double4* uc = (u_hist && advance) ? u_hist[n + 1 - n0] : nullptr;
            if (lagr) {
                ++lagr_steps;
                lagr_rebased = false;
            }
            if (split) {
                // The exchange runs on the second stream while the interior nodes update on
                // the context stream; the interface nodes update once it has landed.
                exchange_send(mixed);
                ck(cudaEventRecord(ev_ready, stream), "event record");
                ck(cudaStreamWaitEvent(xstream, ev_ready, 0), "stream wait");
                exchange_finish(xstream);
                ck(cudaEventRecord(ev_done, xstream), "event record");
                am::NodeDev interior = nd;
                interior.skip_iface = 1;
                am::launch_node_step(interior, mixed, s, table, n, advance, U4, V4, A4, uc, status, stream, 0);
                ck(cudaStreamWaitEvent(stream, ev_done, 0), "stream wait");
                am::NodeDev rim = nd;
                rim.subset_nodes = iface_nodes;
                rim.subset_count = iface_local;
                am::launch_node_step(rim, mixed, s, table, n, advance, U4, V4, A4, uc, status, stream, 0);
                launches += 2;
                check_launch("node step kernels");
                mark(1, 2);
                continue;
            }
            if (iface_row_of) {
                exchange(mixed);
                mark(4, 1);
            }
            am::launch_node_step(nd, mixed, s, table, n, advance, U4, V4, A4, uc, status, stream,
                                 due(lagr_steps) ? 1 : 0);
            ++launches;
            check_launch("node step kernel");
            mark(1, 1);
        }
        // The graph is captured at the end of a precision's first run (after that run made any
        // lazily allocated buffers), so that later runs replay it without a capture of their own.
        if (graphs && !step_graph[mixed]) capture_step_graph(mixed);
    }

    void init_acceleration(int mixed) {
        if (lagr && mixed) fail(AM_EINVAL, "the updated/semi formulations run in FP64");
        element_forces(mixed, U4);
        exchange(mixed);
        am::launch_init_accel(node_dev(), mixed, slots(mixed), A4, status, stream);
        ++launches;
        check_launch("init acceleration kernel");
    }

    // Updated / semi state at the undeformed start: coordinates X, no increment, H = 0.
    void reset_lagrangian() {
        ck(cudaMemcpyAsync(xc, X4, N * sizeof(double4), cudaMemcpyDeviceToDevice, stream), "copy");
        ck(cudaMemsetAsync(lagr_inc, 0, N * sizeof(double4), stream), "memset");
        for (auto& b : blocks) {
            ck(cudaMemsetAsync(b.hstate, 0, static_cast<size_t>(b.num_elems) * 9 * sizeof(double), stream), "memset");
            if (b.href) ck(cudaMemsetAsync(b.href, 0, static_cast<size_t>(b.num_elems) * 9 * sizeof(double), stream), "memset");
        }
        lagr_steps = 0;
        lagr_rebased = false;
    }

    void require_finalized() const {
        if (!finalized) fail(AM_ESTATE, "am_finalize has not been called");
    }

    void release() {
        for (auto& b : blocks) b.release();
        dfree(X4);
        dfree(U4);
        dfree(V4);
        dfree(A4);
        dfree(W4);
        dfree(L4);
        dfree(mass);
        dfree(bcword);
        dfree(bcvalues);
        dfree(status);
        dfree(f_scratch);
        dfree(io_scratch);
        dfree(node_ptr);
        dfree(slot_pos);
        dfree(slots64);
        dfree(slots32);
        dfree(pm_l);
        dfree(pm_v);
        dfree(pm_fu);
        dfree(pm_fe);
        dfree(pm_partial);
        dfree(xc);
        dfree(lagr_inc);
        dfree(rk_ptr);
        dfree(rk_nbr);
        dfree(rk_val);
        dfree(rkt_ptr);
        dfree(rkt_src);
        dfree(rkt_val);
        dfree(rko_ptr);
        dfree(rkto_ptr);
        dfree(rko_rec);
        dfree(rkto_rec);
        dfree(rk_u);
        dfree(rk_f_local);
        dfree(rk_l);
        dfree(rk_f);
        dfree(iface_nodes);
        dfree(iface_rows);
        dfree(iface_row_of);
        dfree(iface_buf);
        dfree(nbr_send_rows);
        dfree(nbr_own);
        dfree(nbr_send);
        dfree(nbr_recv);
        dfree(comb_ptr);
        dfree(comb_idx);
        for (auto& g : step_graph)
            if (g) cudaGraphExecDestroy(g);
        dfree(chunk_table);
        if (ev_ready) cudaEventDestroy(ev_ready);
        if (ev_done) cudaEventDestroy(ev_done);
        if (xstream) cudaStreamDestroy(xstream);
        if (comm) nccl().comm_destroy(comm);
        comm = nullptr;
        for (auto& pbuf : adj_bufs) dfree(pbuf);
        adj_bufs.clear();
        dfree(table);
        if (table_host) cudaFreeHost(table_host);
        table_host = nullptr;
        for (auto e : events) cudaEventDestroy(e);
        events.clear();
        if (table_copied) cudaEventDestroy(table_copied);
        table_copied = nullptr;
        if (own_stream && stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }
};

namespace {

template <typename F>
int guarded(am_ctx* ctx, F&& fn) {
    try {
        fn();
        if (ctx) ctx->err.clear();
        return AM_OK;
    } catch (const AmError& e) {
        if (ctx) ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->err = "host allocation failed";
        return AM_ENOMEM;
    } catch (const std::exception& e) {
        if (ctx) ctx->err = e.what();
        return AM_EINVAL;
    }
}

thread_local std::string g_free_error;

// Copies an N x 3 nodal array (host or device) into a double4 device buffer.
void load_nodal(am_ctx* c, am_memory where, const double* src, double4* dst) {
    if (src == nullptr) {
        am::launch_zero4(dst, c->N, c->stream);
    } else if (where == AM_HOST) {
        ck(cudaMemcpyAsync(c->io_scratch, src, c->N * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "H2D");
        am::launch_pack4(c->io_scratch, dst, c->N, c->stream);
    } else {
        am::launch_pack4(src, dst, c->N, c->stream);
    }
    c->launches += 1;
    ck(cudaGetLastError(), "pack kernel");
}

void store_nodal(am_ctx* c, am_memory where, const double4* src, double* dst) {
    if (dst == nullptr) return;
    if (where == AM_HOST) {
        am::launch_unpack4(src, c->io_scratch, c->N, c->stream);
        ck(cudaMemcpyAsync(dst, c->io_scratch, c->N * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "synchronize");
    } else {
        am::launch_unpack4(src, dst, c->N, c->stream);
    }
    c->launches += 1;
    ck(cudaGetLastError(), "unpack kernel");
}

void run_schedule(am_ctx* c, int prec, const std::vector<double>& dts, double t0) {
    c->require_finalized();
    if (prec != AM_FP64 && prec != AM_MIXED) fail(AM_EINVAL, "unknown precision");
    if (c->lagr && prec != AM_FP64) fail(AM_EINVAL, "the updated/semi formulations run in FP64");
    for (double d : dts)
        if (!(d >= 0.0) || !std::isfinite(d)) fail(AM_EINVAL, "time increments must be finite and non-negative");
    if (dts.empty()) return;
    c->upload_table(dts, t0);
    c->reset_status();
    c->run_range(prec == AM_MIXED, 0, static_cast<int64_t>(dts.size()), nullptr);
    c->check_status();
}

}  // namespace

namespace am {
void set_free_error(const std::string& msg) { g_free_error = msg; }
}  // namespace am

extern "C" {

const char* am_status_string(int status) {
    switch (status) {
        case AM_OK: return "ok";
        case AM_EINVAL: return "invalid argument";
        case AM_ENOMEM: return "out of device memory";
        case AM_ECUDA: return "CUDA error";
        case AM_ENONPOS_J: return "non-positive Jacobian determinant";
        case AM_ENAN: return "non-finite value";
        case AM_ESTATE: return "call out of order";
        case AM_ERANGE: return "size beyond limit";
        default: return "unknown status";
    }
}

const char* am_last_error(const am_ctx* ctx) {
    if (ctx == nullptr) return g_free_error.c_str();
    return ctx->err.c_str();
}

int am_create(int64_t num_nodes, const double* coords, am_ctx** out) {
    if (out == nullptr) return AM_EINVAL;
    *out = nullptr;
    auto c = std::make_unique<am_ctx>();
    const int rc = guarded(c.get(), [&] {
        if (num_nodes <= 0 || coords == nullptr) fail(AM_EINVAL, "num_nodes must be positive and coords non-null");
        if (num_nodes >= (int64_t(1) << 31)) fail(AM_ERANGE, "node count beyond int32 indexing");
        for (int64_t k = 0; k < num_nodes * 3; ++k)
            if (!std::isfinite(coords[k])) fail(AM_EINVAL, "non-finite coordinate");
        ck(cudaGetDevice(&c->device), "cudaGetDevice");
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream create");
        c->own_stream = true;
        const char* patches = std::getenv("APERI_B200_TET4_PATCHES");
        c->tet4_patches = patches && patches[0] == '0' ? 0 : patches && patches[0] == '1' ? 1 : 2;
        c->N = num_nodes;
        const size_t N = static_cast<size_t>(num_nodes);
        c->X4 = dalloc<double4>(N, "coordinates");
        c->U4 = dalloc<double4>(N, "displacement");
        c->V4 = dalloc<double4>(N, "velocity");
        c->A4 = dalloc<double4>(N, "acceleration");
        c->W4 = dalloc<double4>(N, "scratch");
        c->L4 = dalloc<double4>(N, "cotangent");
        c->mass = dalloc<double>(N, "mass");
        c->bcword = dalloc<uint32_t>(N, "bc word");
        c->bcvalues = dalloc<double>(AM_MAX_BCS * 3, "bc values");
        c->status = dalloc<int>(2, "status");
        c->f_scratch = dalloc<double>(N * 3, "force scratch");
        c->io_scratch = dalloc<double>(N * 3, "io scratch");
        const char* graphs = std::getenv("APERI_B200_GRAPHS");
        c->use_graphs = !(graphs && graphs[0] == '0');
        const char* nl = std::getenv("APERI_B200_NODE_LANES");
        c->node_lanes = nl ? std::atoi(nl) : 0;
        const char* ro = std::getenv("APERI_B200_RK_OCTETS");
        c->rk_octets = !(ro && ro[0] == '0');
        const char* tg = std::getenv("APERI_B200_TET4_GEOMETRY");
        c->tet_geometry = !(tg && tg[0] == '0');
        const char* wch = std::getenv("APERI_B200_WARP_CHUNKS");
        c->warp_chunks = !(wch && wch[0] == '0');
        const char* cg = std::getenv("APERI_B200_CELL_GATHER");
        c->cell_gather = !(cg && cg[0] == '0');
        // four digits: FP64 cell, FP64 gather, mixed cell, mixed gather kernel (1, 2 or 4)
        const char* cu = std::getenv("APERI_B200_CELL_UNROLL");
        for (int q = 0; cu && q < 4 && cu[q]; ++q)
            c->cell_unroll[q / 2][q % 2] = cu[q] == '1' ? 1 : cu[q] == '2' ? 2 : 4;
        const char* order = std::getenv("APERI_B200_ELEMENT_ORDER");
        c->locality_order = !(order && std::strcmp(order, "input") == 0);
        c->host_X.assign(coords, coords + 3 * N);
        std::vector<double4> x(N);
        for (size_t i = 0; i < N; ++i) x[i] = make_double4(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], 0.0);
        ck(cudaMemcpy(c->X4, x.data(), N * sizeof(double4), cudaMemcpyHostToDevice), "coords upload");
        ck(cudaMemset(c->U4, 0, N * sizeof(double4)), "memset");
        ck(cudaMemset(c->V4, 0, N * sizeof(double4)), "memset");
        ck(cudaMemset(c->A4, 0, N * sizeof(double4)), "memset");
        ck(cudaMemset(c->W4, 0, N * sizeof(double4)), "memset");
        ck(cudaMemset(c->L4, 0, N * sizeof(double4)), "memset");
        ck(cudaMemset(c->mass, 0, N * sizeof(double)), "memset");
        ck(cudaMemset(c->bcword, 0, N * sizeof(uint32_t)), "memset");
        ck(cudaMemset(c->bcvalues, 0, AM_MAX_BCS * 3 * sizeof(double)), "memset");
        ck(cudaMemset(c->status, 0, 2 * sizeof(int)), "memset");
    });
    if (rc != AM_OK) {
        g_free_error = c->err;
        c->release();
        return rc;
    }
    *out = c.release();
    return AM_OK;
}

void am_destroy(am_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->release();
    delete ctx;
}

int am_set_stream(am_ctx* ctx, void* stream) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        if (stream == nullptr) {
            ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream create");
            ctx->own_stream = true;
        } else {
            ctx->stream = static_cast<cudaStream_t>(stream);
            ctx->own_stream = false;
        }
    });
}

int am_add_block(am_ctx* ctx, const am_block_desc* d, int32_t* block_id) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        if (ctx->finalized) fail(AM_ESTATE, "am_add_block after am_finalize");
        if (!d) fail(AM_EINVAL, "null block descriptor");
        if (d->kind < AM_TET4_GAUSS || d->kind > AM_SMOOTHED_CELLS) fail(AM_EINVAL, "unknown block kind");
        if (d->material < AM_LINEAR_ELASTIC || d->material > AM_ELASTIC_SVK) fail(AM_EINVAL, "unknown material");
        if (d->num_elems < 0) fail(AM_EINVAL, "negative element count");
        if (!(d->density > 0.0)) fail(AM_EINVAL, "density must be positive");
        if (!std::isfinite(d->lambda) || !std::isfinite(d->mu)) fail(AM_EINVAL, "non-finite Lame parameters");
        Block b;
        b.kind = d->kind;
        b.material = d->material;
        b.lambda = d->lambda;
        b.mu = d->mu;
        b.density = d->density;
        b.num_elems = d->num_elems;
        b.slot_base = ctx->num_slots;
        const int64_t E = d->num_elems;
        try {
            if (d->kind == AM_SMOOTHED_CELLS) {
                if (ctx->lagr) fail(AM_EINVAL, "the updated/semi formulations are built for Gauss elements");
                if (E > 0 && (!d->cell_ptr || !d->cell_nodes || !d->cell_grads || !d->cell_volumes))
                    fail(AM_EINVAL, "cell block needs cell_ptr, cell_nodes, cell_grads and cell_volumes");
                const int64_t K = E > 0 ? d->cell_ptr[E] : 0;
                if (E > 0 && d->cell_ptr[0] != 0) fail(AM_EINVAL, "cell_ptr[0] must be 0");
                if (K >= (int64_t(1) << 31)) fail(AM_ERANGE, "entry count beyond int32 indexing");
                std::vector<int32_t> ptr(E + 1);
                int32_t maxlen = 0;
                for (int64_t c = 0; c <= E; ++c) {
                    if (c > 0 && d->cell_ptr[c] < d->cell_ptr[c - 1]) fail(AM_EINVAL, "cell_ptr must be non-decreasing");
                    ptr[c] = static_cast<int32_t>(d->cell_ptr[c]);
                    if (c > 0) maxlen = std::max<int32_t>(maxlen, ptr[c] - ptr[c - 1]);
                }
                for (int64_t s = 0; s < K; ++s)
                    if (d->cell_nodes[s] < 0 || d->cell_nodes[s] >= ctx->points()) fail(AM_EINVAL, "cell node index out of range");
                std::vector<float> g32(K * 3);
                for (int64_t s = 0; s < K * 3; ++s) {
                    if (!std::isfinite(d->cell_grads[s])) fail(AM_EINVAL, "non-finite cell gradient");
                    g32[s] = static_cast<float>(d->cell_grads[s]);
                }
                for (int64_t c = 0; c < E; ++c)
                    if (!(d->cell_volumes[c] > 0.0)) fail(AM_EINVAL, "cell volumes must be positive");
                b.num_entries = K;
                b.max_entries = maxlen;
                b.cell_ptr = dalloc<int32_t>(E + 1, "cell ptr");
                ck(cudaMemcpy(b.cell_ptr, ptr.data(), (E + 1) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                if (K > 0) {
                    b.cell_nodes = dalloc<int32_t>(K, "cell nodes");
                    b.grads64 = dalloc<double>(K * 3, "cell grads");
                    b.grads32 = dalloc<float>(K * 3, "cell grads fp32");
                    ck(cudaMemcpy(b.cell_nodes, d->cell_nodes, K * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                    ck(cudaMemcpy(b.grads64, d->cell_grads, K * 3 * sizeof(double), cudaMemcpyHostToDevice), "upload");
                    ck(cudaMemcpy(b.grads32, g32.data(), K * 3 * sizeof(float), cudaMemcpyHostToDevice), "upload");
                }
                if (E > 0) {
                    b.volumes = dalloc<double>(E, "cell volumes");
                    ck(cudaMemcpy(b.volumes, d->cell_volumes, E * sizeof(double), cudaMemcpyHostToDevice), "upload");
                }
                b.host_nodes.assign(d->cell_nodes, d->cell_nodes + K);
                if (maxlen > 8 && ctx->cell_gather) {
                    b.host_cell_ptr = ptr;
                    b.host_grads.assign(d->cell_grads, d->cell_grads + 3 * K);
                }
                // Cells of four entries that group into split hexes (a tet mesh's element
                // cells) run as patches like the Gauss tets: one slot per patch node.
                bool four = E > 0 && ctx->tet4_patches == 2;
                for (int64_t c = 0; c < E && four; ++c) four = ptr[c + 1] - ptr[c] == 4;
                if (four) {
                    TetPatches tp = build_tet_patches(d->cell_nodes, E);
                    const int64_t P = static_cast<int64_t>(tp.used.size());
                    if (static_cast<double>(E) >= 2.5 * static_cast<double>(P) && hex6_patches(tp)) {
                        b.patched = 2;
                        b.num_patches = P;
                        b.slot_count = 8 * P;
                        b.patch_first = dalloc<int32_t>(P + 1, "patch offsets");
                        b.patch_nodes = dalloc<int32_t>(8 * P, "patch nodes");
                        ck(cudaMemcpy(b.patch_first, tp.first.data(), (P + 1) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                        ck(cudaMemcpy(b.patch_nodes, tp.nodes.data(), 8 * P * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                        b.host_nodes.assign(tp.nodes.begin(), tp.nodes.begin() + 8 * P);
                        if (ctx->warp_chunks && ctx->lagr == 0) {
                            // warp chunks over the half patches, as for the split-hex tets
                            constexpr int kNode[2][4] = {{1, 2, 4, 0}, {5, 6, 7, 3}};
                            std::vector<int32_t> half(8 * P);
                            for (int64_t q = 0; q < P; ++q)
                                for (int r = 0; r < 2; ++r)
                                    for (int a = 0; a < 4; ++a) half[4 * (2 * q + r) + a] = tp.nodes[8 * q + kNode[r][a]];
                            WarpChunks wc;
                            if (build_warp_chunks(half.data(), 2 * P, 4, wc)) upload_warp_chunks(b, wc, 2 * P);
                        }
                    }
                }
            } else {
                const int nn = d->kind == AM_HEX8_GAUSS ? 8 : 4;
                if (E > 0 && !d->conn) fail(AM_EINVAL, "null connectivity");
                const int64_t S = E * nn;
                if (ctx->num_slots + S >= (int64_t(1) << 31)) fail(AM_ERANGE, "slot count beyond int32 indexing");
                for (int64_t s = 0; s < S; ++s)
                    if (d->conn[s] < 0 || d->conn[s] >= ctx->N) fail(AM_EINVAL, "connectivity index out of range");
                b.num_entries = S;
                // The elements run in the locality order (element_order); the block keeps
                // that order's connectivity, and per-element data are permuted through it.
                const int32_t* conn = d->conn;
                std::vector<int32_t> conn_ordered;
                if (ctx->locality_order && E > 1) {
                    am::ElementOrder eo = am::element_order(d->conn, E, nn, ctx->host_X,
                                                    d->kind == AM_TET4_GAUSS && ctx->tet4_patches == 2 && ctx->lagr == 0);
                    conn_ordered.resize(S);
                    for (int64_t k = 0; k < E; ++k)
                        std::copy(d->conn + nn * static_cast<int64_t>(eo.order[k]), d->conn + nn * static_cast<int64_t>(eo.order[k]) + nn,
                                  conn_ordered.begin() + nn * k);
                    conn = conn_ordered.data();
                    b.order = std::move(eo.order);
                    b.order_dev = dalloc<int32_t>(E, "element order");
                    ck(cudaMemcpy(b.order_dev, b.order.data(), E * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                }
                if (S > 0) {
                    b.conn = dalloc<int32_t>(S, "connectivity");
                    ck(cudaMemcpy(b.conn, conn, S * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                }
                b.host_nodes.assign(conn, conn + S);
                if (d->kind == AM_TET4_GAUSS && E > 0 && ctx->tet4_patches && ctx->lagr == 0) {
                    // Patch the tets when patches hold 2.5 tets or more on average; fewer
                    // would leave most of the eight lanes per patch idle.
                    TetPatches tp = build_tet_patches(conn, E);
                    const int64_t P = static_cast<int64_t>(tp.used.size());
                    // Split-hex patches (six tets in the canonical local order) get the
                    // register-resident kernel. Other tets run one thread per tet unless
                    // generic patches are asked for (APERI_B200_TET4_PATCHES=1): on a
                    // renumbered 70^3 mesh in Morton order (3.9 tets per patch) the generic
                    // patch kernel took 170 us against 82 us for one thread per tet (mixed).
                    const bool hex6 = ctx->tet4_patches == 2 && hex6_patches(tp);
                    if ((hex6 || ctx->tet4_patches == 1) && static_cast<double>(E) >= 2.5 * static_cast<double>(P)) {
                        b.patched = hex6 ? 2 : 1;
                        b.num_patches = P;
                        b.num_entries = 8 * P;
                        b.patch_first = dalloc<int32_t>(P + 1, "patch offsets");
                        b.patch_nodes = dalloc<int32_t>(8 * P, "patch nodes");
                        b.patch_local = dalloc<uint32_t>(E, "patch local ids");
                        b.patch_gather = dalloc<uint32_t>(8 * P, "patch gather masks");
                        ck(cudaMemcpy(b.patch_gather, tp.gather.data(), 8 * P * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload");
                        ck(cudaMemcpy(b.patch_first, tp.first.data(), (P + 1) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                        ck(cudaMemcpy(b.patch_nodes, tp.nodes.data(), 8 * P * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
                        ck(cudaMemcpy(b.patch_local, tp.local.data(), E * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload");
                        if (hex6) {
                            b.patch_dx32 = dalloc<float>(21 * P, "patch coordinate differences");
                            b.patch_dx64 = dalloc<double>(21 * P, "patch coordinate differences");
                            am::launch_hex6_patch_dx(b.patch_nodes, P, ctx->X4, b.patch_dx32, b.patch_dx64, ctx->stream);
                            ck(cudaGetLastError(), "patch coordinate differences");
                        }
                        b.host_nodes.assign(8 * P, -1);
                        for (int64_t q = 0; q < P; ++q)
                            for (int a = 0; a < tp.used[q]; ++a) b.host_nodes[8 * q + a] = tp.nodes[8 * q + a];
                        if (hex6 && ctx->warp_chunks) {
                            // warp chunks over the half patches: thread r of patch p writes
                            // patch nodes 1, 2, 4, 0 (r = 0) or 5, 6, 7, 3 (r = 1)
                            constexpr int kNode[2][4] = {{1, 2, 4, 0}, {5, 6, 7, 3}};
                            std::vector<int32_t> half(8 * P);
                            for (int64_t q = 0; q < P; ++q)
                                for (int r = 0; r < 2; ++r)
                                    for (int a = 0; a < 4; ++a) half[4 * (2 * q + r) + a] = tp.nodes[8 * q + kNode[r][a]];
                            WarpChunks wc;
                            if (build_warp_chunks(half.data(), 2 * P, 4, wc)) upload_warp_chunks(b, wc, 2 * P);
                        }
                    }
                }
                if (d->kind == AM_TET4_GAUSS && E > 0 && b.patched == 0 && ctx->lagr == 0 && ctx->tet_geometry) {
                    // one thread per tet: the reference geometry is set up once
                    b.geo32 = dalloc<float>(10 * E, "tet geometry (FP32)");
                    b.geo64 = dalloc<double>(10 * E, "tet geometry");
                    am::launch_tet4_geometry(b.conn, E, ctx->X4, b.geo32, b.geo64, ctx->stream);
                    ck(cudaGetLastError(), "tet geometry");
                }
                // Warp chunks for the one-thread-per-tet kernel (Hex8 measured no gain: its
                // issue-bound element kernel paid for the warp sums what its node kernel saved).
                WarpChunks wc;
                if (ctx->warp_chunks && E > 0 && d->kind == AM_TET4_GAUSS && b.geo64 && build_warp_chunks(conn, E, nn, wc))
                    upload_warp_chunks(b, wc, E);
            }
            if (ctx->num_slots + b.num_entries >= (int64_t(1) << 31)) fail(AM_ERANGE, "slot count beyond int32 indexing");
            if (d->mu_field && E > 0) {
                for (int64_t e = 0; e < E; ++e)
                    if (!(d->mu_field[e] > 0.0)) fail(AM_EINVAL, "shear modulus field must be positive");
                b.mu_field = dalloc<double>(E, "mu field");
                const std::vector<double> v = b.to_order(d->mu_field);
                ck(cudaMemcpy(b.mu_field, v.data(), E * sizeof(double), cudaMemcpyHostToDevice), "upload");
            }
            if (d->kappa_field && E > 0) {
                for (int64_t e = 0; e < E; ++e)
                    if (!(d->kappa_field[e] > 0.0)) fail(AM_EINVAL, "bulk modulus field must be positive");
                b.kappa_field = dalloc<double>(E, "kappa field");
                const std::vector<double> v = b.to_order(d->kappa_field);
                ck(cudaMemcpy(b.kappa_field, v.data(), E * sizeof(double), cudaMemcpyHostToDevice), "upload");
            }
        } catch (...) {
            b.release();
            throw;
        }
        ctx->num_slots += b.slot_count >= 0 ? b.slot_count : b.num_entries;
        ctx->blocks.push_back(std::move(b));
        if (block_id) *block_id = static_cast<int32_t>(ctx->blocks.size() - 1);
    });
}

int am_set_boundary_conditions(am_ctx* ctx, int32_t num_bcs, const am_bc_desc* bcs) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        if (num_bcs < 0 || num_bcs > AM_MAX_BCS) fail(AM_ERANGE, "at most AM_MAX_BCS boundary conditions");
        if (num_bcs > 0 && !bcs) fail(AM_EINVAL, "null boundary-condition array");
        std::vector<am::host::BoundaryCondition> list;
        std::vector<uint32_t> word(ctx->N, 0u);
        std::vector<double> values(AM_MAX_BCS * 3, 0.0);
        for (int32_t k = 0; k < num_bcs; ++k) {
            const am_bc_desc& d = bcs[k];
            am::host::BoundaryCondition bc;
            if (d.kind != AM_BC_DISPLACEMENT && d.kind != AM_BC_VELOCITY)
                fail(AM_EINVAL, "Boundary condition type must be 'velocity' or 'displacement'.");
            if (d.time_function != AM_TF_RAMP && d.time_function != AM_TF_SMOOTH_STEP) fail(AM_EINVAL, "unknown time function");
            if (d.num_points <= 0 || !d.abscissa || !d.ordinate) fail(AM_EINVAL, "time function needs at least one point");
            if (d.num_nodes < 0 || (d.num_nodes > 0 && !d.nodes)) fail(AM_EINVAL, "bad node list");
            bc.kind = d.kind;
            bc.time_function = d.time_function;
            bc.component_mask = d.component_mask & 7;
            for (int c = 0; c < 3; ++c) bc.values[c] = d.values[c];
            bc.abscissa.assign(d.abscissa, d.abscissa + d.num_points);
            bc.ordinate.assign(d.ordinate, d.ordinate + d.num_points);
            bc.active_start = d.active_start;
            bc.active_end = d.active_end;
            bc.Finish();
            for (int64_t i = 0; i < d.num_nodes; ++i) {
                const int32_t n = d.nodes[i];
                if (n < 0 || n >= ctx->N) fail(AM_EINVAL, "boundary-condition node out of range");
                for (int c = 0; c < 3; ++c)
                    if (bc.component_mask & (1 << c)) word[n] |= 1u << (10 * c + k);
            }
            for (int c = 0; c < 3; ++c) values[k * 3 + c] = d.values[c];
            bc.nodes.assign(d.nodes, d.nodes + d.num_nodes);
            list.push_back(std::move(bc));
        }
        ck(cudaMemcpy(ctx->bcword, word.data(), ctx->N * sizeof(uint32_t), cudaMemcpyHostToDevice), "bc upload");
        ck(cudaMemcpy(ctx->bcvalues, values.data(), values.size() * sizeof(double), cudaMemcpyHostToDevice), "bc upload");
        ctx->bcs = std::move(list);
    });
}

int am_set_block_fields(am_ctx* ctx, int32_t block_id, const double* mu_field, const double* kappa_field) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        if (block_id < 0 || block_id >= static_cast<int32_t>(ctx->blocks.size())) fail(AM_EINVAL, "no such block");
        Block& b = ctx->blocks[block_id];
        const int64_t E = b.num_elems;
        auto upload = [&](const double* src, double*& dst, const char* what) {
            if (!src || E == 0) return;
            for (int64_t e = 0; e < E; ++e)
                if (!(src[e] > 0.0)) fail(AM_EINVAL, std::string(what) + " field must be positive");
            if (!dst) dst = dalloc<double>(E, what);
            const std::vector<double> v = b.to_order(src);
            ck(cudaMemcpyAsync(dst, v.data(), E * sizeof(double), cudaMemcpyHostToDevice, ctx->stream), "field upload");
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
        };
        upload(mu_field, b.mu_field, "shear modulus");
        upload(kappa_field, b.kappa_field, "bulk modulus");
    });
}

int am_set_cell_groups(am_ctx* ctx, int32_t block_id, int64_t num_cells, const int64_t* group_ptr) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        if (ctx->finalized) fail(AM_ESTATE, "am_set_cell_groups after am_finalize");
        if (block_id < 0 || block_id >= static_cast<int32_t>(ctx->blocks.size())) fail(AM_EINVAL, "bad block id");
        Block& b = ctx->blocks[block_id];
        if (b.kind != AM_SMOOTHED_CELLS) fail(AM_EINVAL, "cell groups need a smoothed-cell block");
        if (b.group_ptr) fail(AM_ESTATE, "cell groups already set");
        if (b.patched)
            fail(AM_ESTATE, "cell groups on four-entry cells grouped as split hexes (APERI_B200_TET4_PATCHES=0 keeps them ungrouped)");
        if (num_cells < 0 || !group_ptr) fail(AM_EINVAL, "null cell groups");
        if (group_ptr[0] != 0 || group_ptr[num_cells] != b.num_elems)
            fail(AM_EINVAL, "group_ptr must run from 0 to the block's subcell count");
        for (int64_t g = 0; g < num_cells; ++g)
            if (group_ptr[g + 1] < group_ptr[g]) fail(AM_EINVAL, "group_ptr must be non-decreasing");
        // As the reference, F-bar applies only when the cells hold more than one subcell
        // in total (ForEachCellComputeForce_Impl: num_subcells != num_cells).
        if (num_cells == b.num_elems) return;
        b.num_groups = num_cells;
        for (int64_t g = 0; g < num_cells; ++g)
            b.max_group = std::max<int32_t>(b.max_group, static_cast<int32_t>(group_ptr[g + 1] - group_ptr[g]));
        // APERI_B200_FBAR_PASSES=3 keeps the three-pass form for every cell size.
        const char* passes = std::getenv("APERI_B200_FBAR_PASSES");
        b.fbar_fused = !(passes && passes[0] == '3');
        b.group_ptr = dalloc<int64_t>(num_cells + 1, "cell groups");
        ck(cudaMemcpy(b.group_ptr, group_ptr, (num_cells + 1) * sizeof(int64_t), cudaMemcpyHostToDevice), "upload");
        if (!b.host_grads.empty()) b.host_group_ptr.assign(group_ptr, group_ptr + num_cells + 1);
    });
}

int am_set_body_acceleration(am_ctx* ctx, const double g[3]) {
    if (!ctx || !g) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        for (int i = 0; i < 3; ++i) {
            if (!std::isfinite(g[i])) fail(AM_EINVAL, "non-finite body acceleration");
            ctx->g[i] = g[i];
        }
    });
}

int am_set_mass(am_ctx* ctx, const double* mass) {
    if (!ctx || !mass) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        for (int64_t i = 0; i < ctx->N; ++i)
            if (!(mass[i] > 0.0)) fail(AM_EINVAL, "nodal masses must be positive");
        ck(cudaMemcpy(ctx->mass, mass, ctx->N * sizeof(double), cudaMemcpyHostToDevice), "mass upload");
        ctx->mass_set = true;
        ctx->mass_from_caller = true;
    });
}

int am_finalize(am_ctx* ctx) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        if (ctx->finalized) fail(AM_ESTATE, "am_finalize called twice");
        if (ctx->blocks.empty()) fail(AM_EINVAL, "no blocks");
        const int64_t N = ctx->N, NP = ctx->points();
        if (NP > N && !ctx->mass_set) fail(AM_ESTATE, "cells on refinement points need the generalized mass (am_set_mass)");
        // Generic cell blocks (without F-bar groups, or with groups of at most 32 subcells)
        // take the cell-stress form: one logical slot per node they touch instead of one per
        // entry.
        int64_t base = 0;
        for (auto& b : ctx->blocks) {
            if (!b.host_grads.empty() && b.patched == 0 && (!b.group_ptr || b.cells().fused)) {
                std::memcpy(b.unroll, ctx->cell_unroll, sizeof b.unroll);
                b.build_gather(NP);
            }
            std::vector<double>().swap(b.host_grads);
            std::vector<int32_t>().swap(b.host_cell_ptr);
            std::vector<int64_t>().swap(b.host_group_ptr);
            b.slot_base = base;
            base += static_cast<int64_t>(b.host_nodes.size());
        }
        ctx->num_slots = base;
        const int64_t S = ctx->num_slots;
        // Node-major slot layout: node (or point) i owns positions [ptr[i], ptr[i+1]); within
        // a node the positions follow ascending logical slot (block order, then element order).
        std::vector<int32_t> ptr(NP + 1, 0), pos(S, -1);
        for (const auto& b : ctx->blocks)
            for (int32_t n : b.host_nodes)
                if (n >= 0) ++ptr[n + 1];
        for (int64_t i = 0; i < NP; ++i) ptr[i + 1] += ptr[i];
        std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
        for (const auto& b : ctx->blocks)
            for (int64_t k = 0; k < static_cast<int64_t>(b.host_nodes.size()); ++k)
                if (b.host_nodes[k] >= 0) pos[b.slot_base + k] = fill[b.host_nodes[k]]++;
        ctx->num_used_slots = ptr[NP];
        ctx->node_ptr = dalloc<int32_t>(NP + 1, "node ptr");
        ck(cudaMemcpy(ctx->node_ptr, ptr.data(), (NP + 1) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        if (S > 0) {
            ctx->slot_pos = dalloc<int32_t>(S, "slot positions");
            ck(cudaMemcpy(ctx->slot_pos, pos.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
            ctx->slots64 = dalloc<double4>(static_cast<size_t>(std::max<int64_t>(ctx->num_used_slots, 1)), "slot buffer");
        }
        for (auto& b : ctx->blocks) {
            b.slot_pos = ctx->slot_pos + b.slot_base;
            std::vector<int32_t>().swap(b.host_nodes);
            if (b.chunk_ptr) {
                b.chunk_pos = dalloc<int32_t>(static_cast<size_t>(128 * ((b.chunk_units + 31) / 32)), "chunk positions");
                if (b.kind == AM_SMOOTHED_CELLS)
                    am::launch_chunk_positions(b.cells(), b.chunk_pos, ctx->stream);
                else
                    am::launch_chunk_positions(b.gauss(), b.chunk_pos, ctx->stream);
                ++ctx->launches;
                ck(cudaGetLastError(), "chunk positions");
            }
        }
        bool has_cells = false;
        for (const auto& b : ctx->blocks) has_cells |= b.kind == AM_SMOOTHED_CELLS;
        if (!ctx->mass_set) {
            if (has_cells) fail(AM_EINVAL, "smoothed-cell blocks need an explicit lumped mass (am_set_mass)");
            // Lumped mass (src/MassUtils.cpp:17-112) on the device, summed in element order.
            for (auto& b : ctx->blocks) {
                if (b.chunk_ptr) {
                    // allocates the scratch first: it is an argument of the launch below
                    const am::GaussBlockDev corners = b.gauss_corners();
                    am::launch_gauss_volume_slots(corners, b.density, ctx->X4, b.chunk_scratch, ctx->stream);
                    am::launch_chunk_sum(b.gauss(), b.chunk_scratch, ctx->slots64, ctx->stream);
                    ctx->launches += 2;
                } else {
                    am::launch_gauss_volume_slots(b.gauss(), b.density, ctx->X4, ctx->slots64, ctx->stream);
                    ++ctx->launches;
                }
            }
            am::launch_gather_force(ctx->node_dev(), 0, ctx->slots64, ctx->f_scratch, 0, ctx->stream);
            ++ctx->launches;
            ck(cudaGetLastError(), "mass kernels");
            std::vector<double> f(N * 3), m(N);
            ck(cudaMemcpyAsync(f.data(), ctx->f_scratch, N * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
            for (auto& b : ctx->blocks) {
                // the per-corner scratch of the chunked mass comes back on first use (VJP)
                dfree(b.chunk_ident);
                dfree(b.chunk_scratch);
            }
            for (int64_t i = 0; i < N; ++i) {
                m[i] = f[3 * i];
                if (!(m[i] > 0.0)) fail(AM_EINVAL, "node " + std::to_string(i) + " has no mass (not connected to an element)");
            }
            ck(cudaMemcpy(ctx->mass, m.data(), N * sizeof(double), cudaMemcpyHostToDevice), "mass upload");
            ctx->mass_set = true;
        }
        if (ctx->lagr) {
            ctx->xc = dalloc<double4>(N, "current coordinates");
            ctx->lagr_inc = dalloc<double4>(N, "displacement increment");
            for (auto& b : ctx->blocks) {
                const size_t n9 = static_cast<size_t>(std::max<int64_t>(b.num_elems, 1)) * 9;
                b.hstate = dalloc<double>(n9, "element H");
                if (ctx->lagr == 2) b.href = dalloc<double>(n9, "reference H");
            }
            ctx->reset_lagrangian();
        }
        ctx->finalized = true;
    });
}

int am_get_mass(am_ctx* ctx, double* mass) {
    if (!ctx || !mass) return AM_EINVAL;
    return guarded(ctx, [&] {
        ck(cudaMemcpyAsync(mass, ctx->mass, ctx->N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
    });
}

int am_set_state(am_ctx* ctx, am_memory where, const double* u, const double* v, const double* a) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        load_nodal(ctx, where, u, ctx->U4);
        load_nodal(ctx, where, v, ctx->V4);
        load_nodal(ctx, where, a, ctx->A4);
        // The displacement is always set (null: zero), so the updated / semi state restarts
        // from the undeformed configuration with it.
        if (ctx->lagr) ctx->reset_lagrangian();
        if (where == AM_HOST) ck(cudaStreamSynchronize(ctx->stream), "synchronize");
    });
}

int am_get_state(am_ctx* ctx, am_memory where, double* u, double* v, double* a) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        store_nodal(ctx, where, ctx->U4, u);
        store_nodal(ctx, where, ctx->V4, v);
        store_nodal(ctx, where, ctx->A4, a);
    });
}

int am_internal_force(am_ctx* ctx, am_precision prec, am_memory where, const double* u, double* f, int accumulate) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        if (!u || !f) fail(AM_EINVAL, "null u or f");
        if (ctx->lagr) fail(AM_ESTATE, "am_internal_force evaluates the total formulation");
        const int mixed = prec == AM_MIXED;
        load_nodal(ctx, where, u, ctx->W4);
        ctx->reset_status();
        ctx->element_forces(mixed, ctx->W4);
        ctx->exchange(mixed);
        double* out = ctx->f_scratch;
        if (where == AM_DEVICE) out = f;
        else if (accumulate) ck(cudaMemcpyAsync(out, f, ctx->N * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream), "H2D");
        am::launch_gather_force(ctx->node_dev(), mixed, ctx->slots(mixed), out, accumulate, ctx->stream);
        ++ctx->launches;
        ck(cudaGetLastError(), "gather kernel");
        if (where == AM_HOST)
            ck(cudaMemcpyAsync(f, out, ctx->N * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ctx->check_status();
    });
}

int am_init_acceleration(am_ctx* ctx, am_precision prec) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        ctx->reset_status();
        ctx->init_acceleration(prec == AM_MIXED);
        ctx->check_status();
    });
}

int am_run(am_ctx* ctx, am_precision prec, int64_t nsteps, double dt, double t0) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        if (nsteps < 0) fail(AM_EINVAL, "negative step count");
        run_schedule(ctx, prec, std::vector<double>(static_cast<size_t>(nsteps), dt), t0);
    });
}

int am_run_schedule(am_ctx* ctx, am_precision prec, int64_t nsteps, const double* dts, double t0) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        if (nsteps < 0 || (nsteps > 0 && !dts)) fail(AM_EINVAL, "bad schedule");
        run_schedule(ctx, prec, std::vector<double>(dts, dts + nsteps), t0);
    });
}

int am_solve(am_ctx* ctx, am_precision prec, double dt, double t_end, int64_t max_steps, int64_t* steps_done) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        if (!(dt > 0.0) || !std::isfinite(t_end)) fail(AM_EINVAL, "dt must be positive and t_end finite");
        ctx->reset_status();
        ctx->init_acceleration(prec == AM_MIXED);
        ctx->check_status();
        const std::vector<double> dts = am::host::DirectTimeSchedule(dt, t_end, max_steps);
        run_schedule(ctx, prec, dts, 0.0);
        if (steps_done) *steps_done = static_cast<int64_t>(dts.size());
    });
}

int am_set_power_method(am_ctx* ctx, const double* start, const double* max_edge_length) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        ctx->require_finalized();
        if (!start || !max_edge_length) fail(AM_EINVAL, "null start vector or edge lengths");
        for (int64_t i = 0; i < ctx->N; ++i)
            if (!(max_edge_length[i] > 0.0)) fail(AM_EINVAL, "edge lengths must be positive");
        ctx->pm_start.assign(start, start + 3 * ctx->N);
        if (!ctx->pm_l) {
            ctx->pm_l = dalloc<double>(ctx->N, "edge lengths");
            ctx->pm_v = dalloc<double4>(ctx->N, "eigenvector");
            ctx->pm_fu = dalloc<double>(3 * ctx->N, "force");
            ctx->pm_fe = dalloc<double>(3 * ctx->N, "force");
            ctx->pm_partial = dalloc<double>((ctx->N + 255) / 256, "partial sums");
        }
        ck(cudaMemcpy(ctx->pm_l, max_edge_length, ctx->N * sizeof(double), cudaMemcpyHostToDevice), "upload");
        ctx->pm_initialized = false;
    });
}

int am_stable_time_increment(am_ctx* ctx, double previous, int32_t num_iterations, double epsilon, double tolerance,
                             double variation_tolerance, double* dt, int32_t* iterations, int32_t* converged) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        ctx->reset_status();
        const double r = ctx->stable_time_increment(previous, num_iterations, epsilon, tolerance, variation_tolerance,
                                                    iterations, converged);
        ctx->check_status();
        if (dt) *dt = r;
    });
}

int am_solve_power_method(am_ctx* ctx, am_precision prec, double scale_factor, int64_t update_interval, double t_end,
                          int64_t max_steps, int64_t* steps_done, double* last_increment) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        if (!(scale_factor > 0.0) || update_interval < 1 || !std::isfinite(t_end))
            fail(AM_EINVAL, "scale_factor and update_interval must be positive, t_end finite");
        ctx->reset_status();
        ctx->init_acceleration(prec == AM_MIXED);
        ctx->check_status();
        // ExplicitSolver::Solve with PowerMethodTimeStepper (include/TimeStepper.h:138-221):
        // at increments 0, k, 2k, ... the stable increment is recomputed at the current
        // state (seeded with the previous one) and scaled; the last step ends at t_end.
        double time = 0.0, inc_dt = 0.0;
        int64_t n = 0;
        while (!(time >= t_end) && n < max_steps) {
            const double full = ctx->stable_time_increment(inc_dt / scale_factor, 50, 1.0e-5, 1.0e-3, 1.0e-7, nullptr,
                                                           nullptr);
            inc_dt = full * scale_factor;
            std::vector<double> dts;
            const double t_chunk = time;
            for (int64_t k = 0; k < update_interval && !(time >= t_end) && n < max_steps; ++k, ++n) {
                const double d = time + inc_dt <= t_end ? inc_dt : (time > t_end ? 0.0 : t_end - time);
                dts.push_back(d);
                time += d;
            }
            run_schedule(ctx, prec, dts, t_chunk);
        }
        if (steps_done) *steps_done = n;
        if (last_increment) *last_increment = inc_dt;
    });
}

int am_vjp_force(am_ctx* ctx, am_memory where, const double* u, const double* lam, double* gu, double* gmu,
                 double* gkappa) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        if (ctx->iface_row_of) fail(AM_ESTATE, "the VJP is not available on a decomposed mesh");
        if (ctx->lagr) fail(AM_ESTATE, "the VJP is built for the total formulation");
        ctx->prepare_vjp("the VJP");
        if (!u || !lam || !gu) fail(AM_EINVAL, "null u, lam or gu");
        load_nodal(ctx, where, u, ctx->W4);
        load_nodal(ctx, where, lam, ctx->L4);
        const int64_t E = ctx->total_elems();
        double* gm = nullptr;
        double* gk = nullptr;
        std::unique_ptr<double, void (*)(double*)> hold_m(nullptr, [](double* p) { if (p) cudaFree(p); });
        std::unique_ptr<double, void (*)(double*)> hold_k(nullptr, [](double* p) { if (p) cudaFree(p); });
        if (gmu) {
            gm = (where == AM_DEVICE) ? gmu : dalloc<double>(E, "gmu");
            if (where != AM_DEVICE) hold_m.reset(gm);
        }
        if (gkappa) {
            gk = (where == AM_DEVICE) ? gkappa : dalloc<double>(E, "gkappa");
            if (where != AM_DEVICE) hold_k.reset(gk);
        }
        ctx->vjp(ctx->W4, ctx->L4, gm, gk, 0);
        double* out = where == AM_DEVICE ? gu : ctx->f_scratch;
        if (ctx->rk_ptr) {
            ck(cudaMemcpyAsync(out, ctx->rk_f, ctx->N * 3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        } else {
            am::launch_gather_force(ctx->node_dev(), 0, ctx->slots64, out, 0, ctx->stream);
            ++ctx->launches;
        }
        ck(cudaGetLastError(), "gather kernel");
        if (where == AM_HOST) {
            ck(cudaMemcpyAsync(gu, out, ctx->N * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            if (gmu) ck(cudaMemcpyAsync(gmu, gm, E * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            if (gkappa) ck(cudaMemcpyAsync(gkappa, gk, E * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
            ctx->elems_to_caller_host(gmu);
            ctx->elems_to_caller_host(gkappa);
        } else {
            ctx->elems_to_caller_device(gm);
            ctx->elems_to_caller_device(gk);
        }
        ck(cudaStreamSynchronize(ctx->stream), "synchronize");
    });
}

int am_adjoint(am_ctx* ctx, int64_t nsteps, double dt, int32_t ckpt_every, int32_t num_sensors, const int32_t* sensors,
               double* loss, double* gmu, double* gkappa) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->require_finalized();
        if (ctx->iface_row_of) fail(AM_ESTATE, "the adjoint is not available on a decomposed mesh");
        if (ctx->lagr) fail(AM_ESTATE, "the adjoint is built for the total formulation");
        ctx->prepare_vjp("the adjoint");
        if (nsteps <= 0 || !(dt > 0.0)) fail(AM_EINVAL, "nsteps and dt must be positive");
        if (ckpt_every <= 0) fail(AM_EINVAL, "ckpt_every must be positive");
        if (num_sensors < 0 || (num_sensors > 0 && !sensors)) fail(AM_EINVAL, "bad sensor list");
        for (int32_t s = 0; s < num_sensors; ++s)
            if (sensors[s] < 0 || sensors[s] >= ctx->N) fail(AM_EINVAL, "sensor node out of range");
        const size_t N = static_cast<size_t>(ctx->N);
        const int64_t E = ctx->total_elems();
        const int64_t nseg = (nsteps + ckpt_every - 1) / ckpt_every;
        // Buffers (nodal double4 vectors) are cached on the context and reused while the
        // checkpoint layout and the sizes stay the same.
        const int64_t n_vec = 3 * nseg + ckpt_every + 6;
        const int64_t n_aux = 2 * ((E + 3) / 4) + (num_sensors + 7) / 8 + 2;
        if (ctx->adj_key[0] != n_vec || ctx->adj_key[1] != n_aux || ctx->adj_key[2] != ctx->N) {
            ck(cudaStreamSynchronize(ctx->stream), "synchronize");
            for (auto& pbuf : ctx->adj_bufs) dfree(pbuf);
            ctx->adj_bufs.clear();
            ctx->adj_key[0] = ctx->adj_key[1] = ctx->adj_key[2] = 0;
            for (int64_t k = 0; k < n_vec; ++k) ctx->adj_bufs.push_back(dalloc<double4>(N, "adjoint buffer"));
            ctx->adj_bufs.push_back(dalloc<double4>(n_aux, "adjoint buffer"));
            ctx->adj_key[0] = n_vec;
            ctx->adj_key[1] = n_aux;
            ctx->adj_key[2] = ctx->N;
        }
        std::vector<double4*>& B = ctx->adj_bufs;
        std::vector<double4*> ck_u(nseg), ck_v(nseg), ck_a(nseg), seg(ckpt_every);
        for (int64_t s = 0; s < nseg; ++s) {
            ck_u[s] = B[3 * s];
            ck_v[s] = B[3 * s + 1];
            ck_a[s] = B[3 * s + 2];
        }
        for (int32_t k = 0; k < ckpt_every; ++k) seg[k] = B[3 * nseg + k];
        double4* UB = B[3 * nseg + ckpt_every + 0];
        double4* VB = B[3 * nseg + ckpt_every + 1];
        double4* AB = B[3 * nseg + ckpt_every + 2];
        double4* fin_u = B[3 * nseg + ckpt_every + 3];
        double4* fin_v = B[3 * nseg + ckpt_every + 4];
        double4* fin_a = B[3 * nseg + ckpt_every + 5];
        double* gm = reinterpret_cast<double*>(B[n_vec]);
        double* gk = gm + 4 * ((E + 3) / 4);
        int32_t* dsens = reinterpret_cast<int32_t*>(gk + 4 * ((E + 3) / 4));
        double* dloss = reinterpret_cast<double*>(B[n_vec] + (n_aux - 1));
        cudaStream_t st = ctx->stream;
        const size_t bytes = N * sizeof(double4);
        ck(cudaMemsetAsync(gm, 0, E * sizeof(double), st), "memset");
        ck(cudaMemsetAsync(gk, 0, E * sizeof(double), st), "memset");
        if (num_sensors > 0)
            ck(cudaMemcpyAsync(dsens, sensors, num_sensors * sizeof(int32_t), cudaMemcpyHostToDevice, st), "H2D");
        // Forward pass (FP64) with checkpoints of (u, v, a) at the start of each segment;
        // the last segment records its displacements directly, so it needs no recompute.
        ctx->reset_status();
        ctx->init_acceleration(0);
        ctx->upload_table(std::vector<double>(static_cast<size_t>(nsteps), dt), 0.0);
        for (int64_t s = 0; s < nseg; ++s) {
            ck(cudaMemcpyAsync(ck_u[s], ctx->U4, bytes, cudaMemcpyDeviceToDevice, st), "checkpoint");
            ck(cudaMemcpyAsync(ck_v[s], ctx->V4, bytes, cudaMemcpyDeviceToDevice, st), "checkpoint");
            ck(cudaMemcpyAsync(ck_a[s], ctx->A4, bytes, cudaMemcpyDeviceToDevice, st), "checkpoint");
            ctx->run_range(0, s * ckpt_every, std::min<int64_t>(nsteps, (s + 1) * ckpt_every),
                           s == nseg - 1 ? seg.data() : nullptr);
        }
        ctx->check_status();
        ck(cudaMemcpyAsync(fin_u, ctx->U4, bytes, cudaMemcpyDeviceToDevice, st), "save");
        ck(cudaMemcpyAsync(fin_v, ctx->V4, bytes, cudaMemcpyDeviceToDevice, st), "save");
        ck(cudaMemcpyAsync(fin_a, ctx->A4, bytes, cudaMemcpyDeviceToDevice, st), "save");
        // Cotangent of the loss.
        am::launch_zero4(UB, ctx->N, st);
        am::launch_zero4(VB, ctx->N, st);
        am::launch_zero4(AB, ctx->N, st);
        am::launch_sensor_seed(ctx->U4, num_sensors, dsens, UB, dloss, st);
        ctx->launches += 4;
        const am::NodeDev nd = ctx->node_dev();
        am::launch_adj_prep(nd, ctx->table, nsteps - 1, VB, AB, ctx->L4, st);
        ++ctx->launches;
        // Reverse pass, one segment at a time: recompute the segment's displacements
        // from its checkpoint, then transpose its steps in reverse order.
        for (int64_t s = nseg - 1; s >= 0; --s) {
            const int64_t n0 = s * ckpt_every, n1 = std::min<int64_t>(nsteps, (s + 1) * ckpt_every);
            if (s != nseg - 1) {
                ck(cudaMemcpyAsync(ctx->U4, ck_u[s], bytes, cudaMemcpyDeviceToDevice, st), "restore");
                ck(cudaMemcpyAsync(ctx->V4, ck_v[s], bytes, cudaMemcpyDeviceToDevice, st), "restore");
                ck(cudaMemcpyAsync(ctx->A4, ck_a[s], bytes, cudaMemcpyDeviceToDevice, st), "restore");
                ctx->run_range(0, n0, n1, seg.data());
            }
            if (ctx->profiling) ctx->reserve_marks(ctx->n_marks + static_cast<size_t>(2 * (n1 - n0) + 1));
            ctx->mark(-1, 0);
            for (int64_t n = n1 - 1; n >= n0; --n) {
                ctx->vjp(seg[n - n0], ctx->L4, gm, gk, 1);
                ctx->mark(2, static_cast<int64_t>(ctx->blocks.size()));
                am::launch_adj_update(nd, ctx->slots64, ctx->table, n, UB, VB, AB, ctx->L4, st);
                ++ctx->launches;
                ctx->mark(3, 1);
            }
            ck(cudaGetLastError(), "adjoint kernels");
        }
        // Initial acceleration a^0 = F(u^0)/m: only the material-field cotangent remains.
        ctx->vjp(ck_u[0], ctx->L4, gm, gk, 1);
        ck(cudaMemcpyAsync(ctx->U4, fin_u, bytes, cudaMemcpyDeviceToDevice, st), "restore");
        ck(cudaMemcpyAsync(ctx->V4, fin_v, bytes, cudaMemcpyDeviceToDevice, st), "restore");
        ck(cudaMemcpyAsync(ctx->A4, fin_a, bytes, cudaMemcpyDeviceToDevice, st), "restore");
        if (loss) ck(cudaMemcpyAsync(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        if (gmu) ck(cudaMemcpyAsync(gmu, gm, E * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        if (gkappa) ck(cudaMemcpyAsync(gkappa, gk, E * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        ctx->check_status();
        ctx->elems_to_caller_host(gmu);
        ctx->elems_to_caller_host(gkappa);
    });
}

int am_stress(int32_t material, double lambda, double mu, int64_t n, am_memory where, const double* H, double* P) {
    am_ctx* none = nullptr;
    const int rc = guarded(none, [&] {
        if (material < AM_LINEAR_ELASTIC || material > AM_ELASTIC_SVK) fail(AM_EINVAL, "unknown material");
        if (n < 0 || (n > 0 && (!H || !P))) fail(AM_EINVAL, "bad arrays");
        if (n == 0) return;
        const double* dH = H;
        double* dP = P;
        std::unique_ptr<double, void (*)(double*)> h1(nullptr, [](double* p) { if (p) cudaFree(p); });
        std::unique_ptr<double, void (*)(double*)> h2(nullptr, [](double* p) { if (p) cudaFree(p); });
        if (where == AM_HOST) {
            double* a = dalloc<double>(n * 9, "H");
            h1.reset(a);
            double* b = dalloc<double>(n * 9, "P");
            h2.reset(b);
            ck(cudaMemcpy(a, H, n * 9 * sizeof(double), cudaMemcpyHostToDevice), "H2D");
            dH = a;
            dP = b;
        }
        am::launch_stress_batch(material, lambda, mu, n, dH, dP, 0);
        ck(cudaGetLastError(), "stress kernel");
        if (where == AM_HOST) ck(cudaMemcpy(P, dP, n * 9 * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        ck(cudaDeviceSynchronize(), "synchronize");
    });
    if (rc != AM_OK) {
        // message kept for am_last_error(NULL)
    }
    return rc;
}

int am_quadrature(int32_t kind, int32_t smoothed, int64_t n, am_memory where, const double* X, double* B, double* w) {
    am_ctx* none = nullptr;
    return guarded(none, [&] {
        if (kind != AM_TET4_GAUSS && kind != AM_HEX8_GAUSS) fail(AM_EINVAL, "quadrature kind must be Tet4 or Hex8");
        if (n < 0 || (n > 0 && (!X || !B || !w))) fail(AM_EINVAL, "bad arrays");
        if (n == 0) return;
        const int nn = kind == AM_HEX8_GAUSS ? 8 : 4;
        const int np = smoothed ? 1 : (kind == AM_HEX8_GAUSS ? 8 : 1);
        const size_t nx = n * nn * 3, nb = n * np * nn * 3, nw = n * np;
        const double* dX = X;
        double* dB = B;
        double* dw = w;
        std::vector<std::unique_ptr<double, void (*)(double*)>> hold;
        if (where == AM_HOST) {
            double* a = dalloc<double>(nx, "X");
            hold.emplace_back(a, [](double* p) { cudaFree(p); });
            double* b = dalloc<double>(nb, "B");
            hold.emplace_back(b, [](double* p) { cudaFree(p); });
            double* c = dalloc<double>(nw, "w");
            hold.emplace_back(c, [](double* p) { cudaFree(p); });
            ck(cudaMemcpy(a, X, nx * sizeof(double), cudaMemcpyHostToDevice), "H2D");
            dX = a;
            dB = b;
            dw = c;
        }
        am::launch_quadrature_batch(kind, smoothed, n, dX, dB, dw, 0);
        ck(cudaGetLastError(), "quadrature kernel");
        if (where == AM_HOST) {
            ck(cudaMemcpy(B, dB, nb * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
            ck(cudaMemcpy(w, dw, nw * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        }
        ck(cudaDeviceSynchronize(), "synchronize");
    });
}

int am_complete_properties(double props[5], char* msg, int msg_len) {
    if (!props) return AM_EINVAL;
    try {
        am::host::LinearElasticProperties p;
        p.youngs_modulus = props[0];
        p.poisson_ratio = props[1];
        p.shear_modulus = props[2];
        p.lambda = props[3];
        p.bulk_modulus = props[4];
        p.CompleteProperties();
        props[0] = p.youngs_modulus;
        props[1] = p.poisson_ratio;
        props[2] = p.shear_modulus;
        props[3] = p.lambda;
        props[4] = p.bulk_modulus;
        return AM_OK;
    } catch (const std::exception& e) {
        if (msg && msg_len > 0) std::snprintf(msg, static_cast<size_t>(msg_len), "%s", e.what());
        return AM_EINVAL;
    }
}

int am_element_order(int64_t num_nodes, const double* coords, int64_t num_elems, int32_t nodes_per_elem,
                     const int32_t* conn, int32_t try_rings, int32_t* order, int32_t* rings) {
    am::set_free_error("");
    if (num_nodes <= 0 || !coords || num_elems < 0 || (nodes_per_elem != 4 && nodes_per_elem != 8) ||
        (num_elems > 0 && (!conn || !order))) {
        am::set_free_error("am_element_order: bad arguments");
        return AM_EINVAL;
    }
    try {
        for (int64_t s = 0; s < num_elems * nodes_per_elem; ++s)
            if (conn[s] < 0 || conn[s] >= num_nodes) {
                am::set_free_error("am_element_order: connectivity index out of range");
                return AM_EINVAL;
            }
        const std::vector<double> X(coords, coords + 3 * num_nodes);
        am::ElementOrder eo = am::element_order(conn, num_elems, nodes_per_elem, X, try_rings != 0);
        std::copy(eo.order.begin(), eo.order.end(), order);
        if (rings) *rings = eo.rings ? 1 : 0;
        return AM_OK;
    } catch (const std::bad_alloc&) {
        am::set_free_error("am_element_order: host allocation failed");
        return AM_ENOMEM;
    }
}

int64_t am_launch_count(const am_ctx* ctx) { return ctx ? ctx->launches : 0; }

int am_get_layout(const am_ctx* ctx, int64_t* used_slots, int32_t* patched_tet4_blocks) {
    if (!ctx) return AM_EINVAL;
    if (used_slots) *used_slots = ctx->num_used_slots;
    if (patched_tet4_blocks) {
        int32_t n = 0;
        for (const auto& b : ctx->blocks) n += b.patched ? 1 : 0;
        *patched_tet4_blocks = n;
    }
    return AM_OK;
}

int am_set_interface(am_ctx* ctx, int64_t num_local, const int32_t* local_nodes, const int32_t* rows,
                     int64_t num_global) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        ctx->require_finalized();
        if (!ctx->mass_from_caller)
            fail(AM_ESTATE, "a decomposed mesh needs the global lumped mass from am_set_mass before am_finalize");
        if (ctx->iface_row_of) fail(AM_ESTATE, "interface already set");
        if (ctx->rk_ptr) fail(AM_ESTATE, "a decomposed mesh with the two-pass coupling is not built");
        if (ctx->lagr) fail(AM_ESTATE, "a decomposed mesh runs the total formulation");
        if (num_local < 0 || num_global < num_local || (num_local > 0 && (!local_nodes || !rows)))
            fail(AM_EINVAL, "bad interface arrays");
        if (num_global >= (int64_t(1) << 31)) fail(AM_ERANGE, "interface beyond int32 indexing");
        std::vector<int32_t> row_of(ctx->N, -1);
        std::vector<char> row_used(static_cast<size_t>(num_global), 0);
        for (int64_t k = 0; k < num_local; ++k) {
            if (local_nodes[k] < 0 || local_nodes[k] >= ctx->N) fail(AM_EINVAL, "interface node out of range");
            if (rows[k] < 0 || rows[k] >= num_global) fail(AM_EINVAL, "interface row out of range");
            if (row_of[local_nodes[k]] >= 0 || row_used[rows[k]]) fail(AM_EINVAL, "interface node or row repeated");
            row_of[local_nodes[k]] = rows[k];
            row_used[rows[k]] = 1;
        }
        ctx->iface_local = num_local;
        ctx->iface_global = num_global;
        ctx->iface_row_of = dalloc<int32_t>(ctx->N, "interface rows");
        ck(cudaMemcpy(ctx->iface_row_of, row_of.data(), ctx->N * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        ctx->iface_buf = dalloc<double>(static_cast<size_t>(std::max<int64_t>(num_global, 1)) * 3, "interface buffer");
        if (num_local > 0) {
            ctx->iface_nodes = dalloc<int32_t>(num_local, "interface nodes");
            ctx->iface_rows = dalloc<int32_t>(num_local, "interface rows");
            ck(cudaMemcpy(ctx->iface_nodes, local_nodes, num_local * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemcpy(ctx->iface_rows, rows, num_local * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        }
    });
}

int am_set_neighbors(am_ctx* ctx, int32_t rank, int32_t num_neighbors, const int32_t* neighbor_ranks,
                     const int64_t* shared_ptr, const int32_t* shared_nodes) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        ctx->require_finalized();
        if (!ctx->mass_from_caller)
            fail(AM_ESTATE, "a decomposed mesh needs the global lumped mass from am_set_mass before am_finalize");
        if (ctx->iface_row_of) fail(AM_ESTATE, "interface already set");
        if (ctx->rk_ptr) fail(AM_ESTATE, "a decomposed mesh with the two-pass coupling is not built");
        if (ctx->lagr) fail(AM_ESTATE, "a decomposed mesh runs the total formulation");
        if (rank < 0 || num_neighbors < 1 || !neighbor_ranks || !shared_ptr || !shared_nodes || shared_ptr[0] != 0)
            fail(AM_EINVAL, "bad neighbour arrays");
        const int64_t S = shared_ptr[num_neighbors];
        if (S >= (int64_t(1) << 31)) fail(AM_ERANGE, "shared entries beyond int32 indexing");
        // Rows: this rank's interface nodes (every node shared with a neighbour), ascending.
        std::vector<int32_t> row_of(ctx->N, -1), nodes;
        for (int32_t j = 0; j < num_neighbors; ++j) {
            if (shared_ptr[j + 1] < shared_ptr[j]) fail(AM_EINVAL, "shared_ptr must not decrease");
            if (j > 0 && neighbor_ranks[j] <= neighbor_ranks[j - 1]) fail(AM_EINVAL, "neighbour ranks must ascend");
            for (int64_t k = shared_ptr[j]; k < shared_ptr[j + 1]; ++k) {
                const int32_t i = shared_nodes[k];
                if (i < 0 || i >= ctx->N) fail(AM_EINVAL, "shared node out of range");
                if (row_of[i] < 0) {
                    row_of[i] = 0;
                    nodes.push_back(i);
                }
            }
        }
        std::sort(nodes.begin(), nodes.end());
        const int64_t R = static_cast<int64_t>(nodes.size());
        for (int64_t r = 0; r < R; ++r) row_of[nodes[r]] = static_cast<int32_t>(r);
        // Per row: its sources in ascending holder rank; this rank's own partial (index r)
        // at its place, a neighbour's entry k as R + k.
        std::vector<std::vector<std::pair<int32_t, int32_t>>> src(R);
        std::vector<int32_t> send_rows(S);
        for (int64_t r = 0; r < R; ++r) src[r].emplace_back(rank, static_cast<int32_t>(r));
        for (int32_t j = 0; j < num_neighbors; ++j)
            for (int64_t k = shared_ptr[j]; k < shared_ptr[j + 1]; ++k) {
                const int32_t r = row_of[shared_nodes[k]];
                send_rows[k] = r;
                src[r].emplace_back(neighbor_ranks[j], static_cast<int32_t>(R + k));
            }
        std::vector<int32_t> cptr(R + 1, 0), cidx;
        for (int64_t r = 0; r < R; ++r) {
            std::stable_sort(src[r].begin(), src[r].end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            for (const auto& e : src[r]) cidx.push_back(e.second);
            cptr[r + 1] = static_cast<int32_t>(cidx.size());
        }
        std::vector<int32_t> rows(R);
        for (int64_t r = 0; r < R; ++r) rows[r] = static_cast<int32_t>(r);
        ctx->my_rank = rank;
        ctx->nbr_ranks.assign(neighbor_ranks, neighbor_ranks + num_neighbors);
        ctx->nbr_off.assign(shared_ptr, shared_ptr + num_neighbors + 1);
        ctx->iface_local = R;
        ctx->iface_global = R;
        ctx->iface_row_of = dalloc<int32_t>(ctx->N, "interface rows");
        ck(cudaMemcpy(ctx->iface_row_of, row_of.data(), ctx->N * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        const size_t R1 = static_cast<size_t>(std::max<int64_t>(R, 1)), S1 = static_cast<size_t>(std::max<int64_t>(S, 1));
        ctx->iface_buf = dalloc<double>(R1 * 3, "interface buffer");
        ctx->nbr_own = dalloc<double>(R1 * 3, "interface partials");
        ctx->nbr_send = dalloc<double>(S1 * 3, "send buffer");
        ctx->nbr_recv = dalloc<double>(S1 * 3, "receive buffer");
        ctx->nbr_send_rows = dalloc<int32_t>(S1, "send rows");
        ctx->comb_ptr = dalloc<int32_t>(R + 1, "combine offsets");
        ctx->comb_idx = dalloc<int32_t>(std::max<size_t>(cidx.size(), 1), "combine sources");
        ctx->iface_nodes = dalloc<int32_t>(R1, "interface nodes");
        ctx->iface_rows = dalloc<int32_t>(R1, "interface rows");
        if (S > 0) ck(cudaMemcpy(ctx->nbr_send_rows, send_rows.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(ctx->comb_ptr, cptr.data(), (R + 1) * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        if (!cidx.empty())
            ck(cudaMemcpy(ctx->comb_idx, cidx.data(), cidx.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        if (R > 0) {
            ck(cudaMemcpy(ctx->iface_nodes, nodes.data(), R * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
            ck(cudaMemcpy(ctx->iface_rows, rows.data(), R * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        }
        const char* ov = std::getenv("APERI_B200_EXCHANGE_OVERLAP");
        ctx->overlap = !(ov && ov[0] == '0');
        if (ctx->overlap) {
            ck(cudaStreamCreateWithFlags(&ctx->xstream, cudaStreamNonBlocking), "stream create");
            ck(cudaEventCreateWithFlags(&ctx->ev_ready, cudaEventDisableTiming), "event create");
            ck(cudaEventCreateWithFlags(&ctx->ev_done, cudaEventDisableTiming), "event create");
        }
    });
}

int am_set_formulation(am_ctx* ctx, int32_t formulation, int32_t update_interval) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        // Before the blocks: the element state is per element, so Tet4 blocks keep one
        // slot per element node instead of element patches.
        if (ctx->finalized || !ctx->blocks.empty()) fail(AM_ESTATE, "am_set_formulation comes before am_add_block");
        if (formulation < 0 || formulation > 2) fail(AM_EINVAL, "formulation: 0 total, 1 updated, 2 semi");
        if (formulation == 2 && update_interval < 1) fail(AM_EINVAL, "update_interval must be at least 1");
        ctx->lagr = formulation;
        ctx->lagr_interval = formulation == 2 ? update_interval : 1;
    });
}

int am_set_rk_points(am_ctx* ctx, int64_t num_points) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        if (ctx->finalized || !ctx->blocks.empty()) fail(AM_ESTATE, "am_set_rk_points comes before am_add_block");
        if (num_points < ctx->N) fail(AM_EINVAL, "the points start with the nodes: num_points >= num_nodes");
        if (num_points >= (int64_t(1) << 31)) fail(AM_ERANGE, "point count beyond int32 indexing");
        if (ctx->lagr) fail(AM_ESTATE, "refinement points are built for the total formulation");
        ctx->num_points = num_points;
    });
}

int am_set_rk_functions(am_ctx* ctx, const int64_t* nbr_ptr, const int32_t* nbr, const double* values) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        ctx->require_finalized();
        if (ctx->rk_ptr) fail(AM_ESTATE, "reproducing-kernel functions already set");
        if (ctx->iface_row_of) fail(AM_ESTATE, "a decomposed mesh with the two-pass coupling is not built");
        if (!ctx->mass_from_caller)
            fail(AM_ESTATE, "the two-pass coupling needs the generalized lumped mass from am_set_mass before am_finalize");
        if (!nbr_ptr) fail(AM_EINVAL, "null neighbour offsets");
        // One row per point: the nodes, then any refinement points (am_set_rk_points).
        const int64_t N = ctx->N, NP = ctx->points(), K = nbr_ptr[NP];
        if (nbr_ptr[0] != 0 || K < 0 || (K > 0 && (!nbr || !values))) fail(AM_EINVAL, "bad neighbour arrays");
        for (int64_t i = 0; i < NP; ++i)
            if (nbr_ptr[i + 1] < nbr_ptr[i]) fail(AM_EINVAL, "neighbour offsets must not decrease");
        for (int64_t k = 0; k < K; ++k)
            if (nbr[k] < 0 || nbr[k] >= N) fail(AM_EINVAL, "neighbour out of range");
        // Transposed functions: column j lists (i, psi_j(x_i)) for ascending i; a node row
        // without neighbours contributes a unit entry to its own column (a refinement point
        // without neighbours contributes nothing).
        std::vector<int64_t> tptr(N + 1, 0);
        for (int64_t i = 0; i < NP; ++i) {
            if (nbr_ptr[i] == nbr_ptr[i + 1] && i < N) ++tptr[i + 1];
            for (int64_t k = nbr_ptr[i]; k < nbr_ptr[i + 1]; ++k) ++tptr[nbr[k] + 1];
        }
        for (int64_t j = 0; j < N; ++j) tptr[j + 1] += tptr[j];
        const int64_t T = tptr[N];
        if (T >= (int64_t(1) << 31)) fail(AM_ERANGE, "functions beyond int32 indexing");
        std::vector<int32_t> tsrc(static_cast<size_t>(T));
        std::vector<double> tval(static_cast<size_t>(T));
        std::vector<int64_t> fill(tptr.begin(), tptr.end() - 1);
        for (int64_t i = 0; i < NP; ++i) {
            if (nbr_ptr[i] == nbr_ptr[i + 1] && i < N) {
                tsrc[fill[i]] = static_cast<int32_t>(i);
                tval[fill[i]++] = 1.0;
            }
            for (int64_t k = nbr_ptr[i]; k < nbr_ptr[i + 1]; ++k) {
                tsrc[fill[nbr[k]]] = static_cast<int32_t>(i);
                tval[fill[nbr[k]]++] = values[k];
            }
        }
        auto up = [&](auto*& dst, const auto* src, int64_t n, const char* what) {
            using T0 = std::remove_reference_t<decltype(*dst)>;
            dst = dalloc<T0>(static_cast<size_t>(std::max<int64_t>(n, 1)), what);
            if (n > 0) ck(cudaMemcpy(dst, src, n * sizeof(T0), cudaMemcpyHostToDevice), "upload");
        };
        if (ctx->rk_octets) {
            // rows sorted by node and columns (ascending point already) in warp octets
            auto octets = [&](int64_t count, const std::vector<int32_t>& ptr, const std::vector<int32_t>& part,
                              const std::vector<double>& w, int32_t*& optr, double2*& rec, int64_t& n_oct) {
                const OctetRows o = octet_rows(count, ptr, part);
                std::vector<double2> h(o.src.size());
                for (size_t q = 0; q < h.size(); ++q) {
                    const int32_t e = o.src[q];
                    h[q] = e < 0 ? make_double2(0.0, bits64(-1)) : make_double2(w[e], bits64(part[e]));
                }
                n_oct = static_cast<int64_t>(o.ptr.size()) - 1;
                up(optr, o.ptr.data(), static_cast<int64_t>(o.ptr.size()), "function octet rows");
                up(rec, h.data(), static_cast<int64_t>(h.size()), "function octet records");
            };
            std::vector<int32_t> rptr(NP + 1), rpart(static_cast<size_t>(K));
            std::vector<double> rval(static_cast<size_t>(K));
            std::vector<int64_t> perm;
            for (int64_t i = 0; i < NP; ++i) {
                rptr[i] = static_cast<int32_t>(nbr_ptr[i]);
                perm.resize(static_cast<size_t>(nbr_ptr[i + 1] - nbr_ptr[i]));
                for (size_t q = 0; q < perm.size(); ++q) perm[q] = nbr_ptr[i] + static_cast<int64_t>(q);
                std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return nbr[a] < nbr[b]; });
                for (size_t q = 0; q < perm.size(); ++q) {
                    rpart[nbr_ptr[i] + q] = nbr[perm[q]];
                    rval[nbr_ptr[i] + q] = values[perm[q]];
                }
            }
            rptr[NP] = static_cast<int32_t>(K);
            std::vector<int32_t> cptr(tptr.begin(), tptr.end());
            octets(NP, rptr, rpart, rval, ctx->rko_ptr, ctx->rko_rec, ctx->rko_count);
            octets(N, cptr, tsrc, tval, ctx->rkto_ptr, ctx->rkto_rec, ctx->rkto_count);
        }
        up(ctx->rk_ptr, nbr_ptr, NP + 1, "function offsets");
        up(ctx->rk_nbr, nbr, K, "function neighbours");
        up(ctx->rk_val, values, K, "function values");
        up(ctx->rkt_ptr, tptr.data(), N + 1, "transposed offsets");
        up(ctx->rkt_src, tsrc.data(), T, "transposed sources");
        up(ctx->rkt_val, tval.data(), T, "transposed values");
        ctx->rk_u = dalloc<double4>(NP, "physical displacement");
        ctx->rk_f_local = dalloc<double4>(NP, "local force");
        ctx->rk_l = dalloc<double4>(NP, "cotangent at the points");
        ctx->rk_f = dalloc<double>(3 * N, "generalized force");
    });
}

int am_nccl_unique_id(unsigned char id[128]) {
    am_ctx* none = nullptr;
    const int rc = guarded(none, [&] {
        if (!id) fail(AM_EINVAL, "null id");
        static_assert(sizeof(ncclUniqueId) == 128, "ncclUniqueId is 128 bytes");
        ncclUniqueId u;
        nccl_check(nccl().get_unique_id(&u), "ncclGetUniqueId");
        std::memcpy(id, &u, sizeof(u));
    });
    return rc;
}

int am_set_nccl(am_ctx* ctx, const unsigned char id[128], int32_t rank, int32_t nranks) {
    if (!ctx) return AM_EINVAL;
    return guarded(ctx, [&] {
        ctx->drop_graphs();
        if (!id || nranks < 1 || rank < 0 || rank >= nranks) fail(AM_EINVAL, "bad NCCL rank or id");
        if (!ctx->iface_row_of) fail(AM_ESTATE, "am_set_interface or am_set_neighbors first");
        if (!ctx->nbr_ranks.empty()) {
            if (rank != ctx->my_rank) fail(AM_EINVAL, "rank differs from the one given to am_set_neighbors");
            for (int32_t q : ctx->nbr_ranks)
                if (q >= nranks) fail(AM_EINVAL, "neighbour rank beyond the communicator");
            if (!nccl().group_start || !nccl().group_end || !nccl().send || !nccl().recv)
                fail(AM_ESTATE, "libnccl.so.2 lacks the point-to-point calls");
        }
        if (ctx->comm) fail(AM_ESTATE, "communicator already set");
        ncclUniqueId u;
        std::memcpy(&u, id, sizeof(u));
        nccl_check(nccl().comm_init_rank(&ctx->comm, nranks, u, rank), "ncclCommInitRank");
    });
}

int am_profile_enable(am_ctx* ctx, int enable) {
    if (!ctx) return AM_EINVAL;
    const int rc = guarded(ctx, [&] { ctx->collect_marks(); });
    if (rc != AM_OK) return rc;
    ctx->profiling = enable != 0;
    if (ctx->profiling) {
        const int rc2 = guarded(ctx, [&] { ctx->reserve_marks(4096); });
        if (rc2 != AM_OK) return rc2;
    }
    for (int k = 0; k < 5; ++k) {
        ctx->prof_ms[k] = 0.0;
        ctx->prof_launches[k] = 0;
    }
    return AM_OK;
}

int am_profile_read(am_ctx* ctx, double ms[5], int64_t launches[5]) {
    if (!ctx) return AM_EINVAL;
    const int rc = guarded(ctx, [&] { ctx->collect_marks(); });
    if (rc != AM_OK) return rc;
    for (int k = 0; k < 5; ++k) {
        if (ms) ms[k] = ctx->prof_ms[k];
        if (launches) launches[k] = ctx->prof_launches[k];
    }
    return AM_OK;
}

}  // extern "C"
