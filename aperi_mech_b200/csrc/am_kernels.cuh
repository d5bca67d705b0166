// am_kernels.cuh -- device kernels of the explicit-dynamics hot path and their launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/aperi_b200.h"

namespace am {

// Per-step parameters of the central-difference loop, built on the host from the
// time stepper and the boundary-condition time functions (device table).
struct StepParams {
    double dt;                 // time increment of the step
    double half;               // 0.5 * dt
    uint32_t vact;             // bit k: BC k active at t_mid (velocity overwrite)
    uint32_t aact;             // bit k: BC k active at t_next (acceleration overwrite)
    double vscale[AM_MAX_BCS]; // velocity time-function value of BC k at t_mid
    double ascale[AM_MAX_BCS]; // acceleration time-function value of BC k at t_next
};

// Device status word: [0] = first am_status error code, [1] = offending entity.
enum StatusSlot { kStatusCode = 0, kStatusIndex = 1 };

// Force slots are stored node-major: the contributions to node i occupy the
// contiguous range [node_ptr[i], node_ptr[i+1]) of the slot array, in ascending
// logical slot order (block, then element / patch / entry). Writers map a logical
// slot s of a block to its position with slot_pos[s] (block-local pointer).

// Gauss-element block on the device.
struct GaussBlockDev {
    int32_t kind;      // AM_TET4_GAUSS / AM_HEX8_GAUSS
    int32_t material;
    double lambda, mu;
    int64_t num_elems;
    const int32_t* conn;
    const double* mu_field;     // may be null
    const double* kappa_field;  // may be null
    const int32_t* slot_pos;    // logical slot -> node-major position (-1: unused)
    // Tet4 element patches: at most 6 consecutive tets on at most 8 nodes, whose
    // contributions are summed per patch node before they are written (8 logical
    // slots per patch).
    int32_t patched;             // 0: per element, 1: generic patches, 2: split-hex patches
    int64_t num_patches;
    const int32_t* patch_first;  // num_patches + 1 element offsets
    const int32_t* patch_nodes;  // num_patches x 8 (unused entries repeat entry 0)
    const uint32_t* patch_local; // per element: 4 local node ids, one byte each
    const uint32_t* patch_gather;// per patch node: bits 0-7 tets touching it, bits 8+2t: its slot in tet t
    // Split-hex patches: reference differences X_a - X_0 of patch-local nodes a = 1..7
    // (formed in FP64; rounded once to FP32 for the mixed path), component-major:
    // entry (3 (a - 1) + i) * num_patches + patch. Run-invariant; read by the kernels
    // in place of the coordinate gathers. null where not built.
    const float* patch_dx32;
    const double* patch_dx64;
    // Per-tet geometry of a Tet4 block run one thread per tet under the total formulation:
    // J^-1 (row-major) and w = det J / 6 of every tet, formed in FP64 at set-up (an FP32 copy
    // for the mixed path), in three component blocks: values 0-3 and 4-7 of J^-1 (a vec4
    // each, num_elems apiece), then (J^-1[8], w) pairs. Read in place of the coordinate
    // gathers. null where not built.
    const float* geo32;
    const double* geo64;
    // Warp chunks (such Tet4 blocks, and split-hex patches, whose thread r of patch p, unit
    // 2p + r, writes patch nodes 1, 2, 4, 0 or 5, 6, 7, 3): the 32 units [32c, 32c + 32) of
    // chunk c sum their four nodal forces on each node they share and write one slot per
    // distinct node; the node of rank k (order of first appearance over the entry codes
    // q = 32 a + lane, corner a of the chunk's unit lane) has logical slot chunk_ptr[c] + k.
    // The chunk's 128 entries sorted by (rank, code), four to a lane: word 32 c + l of
    // chunk_code / chunk_rank holds lane l's, one byte each (rank 0xFF past the last unit).
    // null: one slot per element (or patch) node.
    const int32_t* chunk_ptr;
    const uint32_t* chunk_code;
    const uint32_t* chunk_rank;
    int64_t chunk_units;  // the units chunked: tets, or split-hex half patches (two per patch)
    // nn per lane (the lane's word order): the slot position of each entry that ends its
    // node's run, else -1; resolved at am_finalize
    const int32_t* chunk_pos;
    // Updated / semi-Lagrangian formulations: element displacement gradient of the last
    // force evaluation (9 per element; for Hex8 the last Gauss point's) and the semi
    // formulation's reference gradient. null under the total formulation.
    double* hstate;
    double* href;
};

struct CellBlockDev {
    int32_t material;
    double lambda, mu;
    int64_t num_cells;
    const int32_t* ptr;         // num_cells + 1 (entry offsets, block-local)
    const int32_t* nodes;       // entries
    const double* grads64;      // entries x 3
    const float* grads32;       // entries x 3 (mixed path), may be null
    const double* volumes;
    const double* mu_field;
    const double* kappa_field;
    const int32_t* slot_pos;    // entry -> node-major position
    int64_t num_entries;        // ptr[num_cells]
    int32_t max_entries;        // longest cell (selects thread- or group-per-cell)
    // Four-entry cells grouped as split hexes (patched == 2, see GaussBlockDev): cell
    // patch_first[q] + t holds tet t of patch q; one slot per patch node.
    int32_t patched;
    int64_t num_patches;
    const int32_t* patch_first;
    const int32_t* patch_nodes;
    // F-bar (ComputeInternalForceSmoothedCell.h:354-413): the cells above are subcells,
    // grouped into num_groups cells by group_ptr; fbar is the per-subcell scratch
    // (kFbarStride values of the slot precision: H, J, then the stress). null: no F-bar.
    int64_t num_groups;
    const int64_t* group_ptr;
    void* fbar;
    int32_t max_group;          // most subcells in one cell
    int32_t fused;              // 1: one warp per cell, one lane per subcell (max_group <= 32)
    // Cell-stress form (gather = 1): per-cell M = -V P into cmat (three component arrays:
    // values 0-3, 4-7 and 8 of the num_cells cells, slot precision), then per node the block
    // touches (t_count of them, logical slot i) the sum of M b over its entries. Both
    // kernels walk octets of eight items: octet o's rows are o_ptr[o] .. o_ptr[o+1] (cells)
    // or n_ptr (nodes), row r of item j at record 8 r + j: gradient in x, y, z, the partner
    // index (node, or cell) in w, -1 for padding. c_ref: a node of each cell (-1: empty).
    // With group_items 1 instead of 8 a side's warps take one item each (rows = its entries).
    int32_t gather;
    int64_t num_octets;
    const int32_t* o_ptr;
    const float4* orec32;
    const double4* orec64;
    const int32_t* c_ref;
    int64_t t_count;
    int64_t num_node_octets;
    const int32_t* n_ptr;
    const float4* nrec32;
    const double4* nrec64;
    void* cmat;
    int32_t group_items[2];  // items per warp (8, or 1 for items of many entries): cell side, node side
    int32_t unroll[2];  // rows per lane in flight (1, 2 or 4): cell kernel, gather kernel
    // Warp chunks of cells grouped as split hexes (patched == 2), as GaussBlockDev's for
    // split-hex tet patches: units are half patches. null: one slot per patch node.
    const int32_t* chunk_ptr;
    const uint32_t* chunk_code;
    const uint32_t* chunk_rank;
    const int32_t* chunk_pos;
    int64_t chunk_units;
};
constexpr int kFbarStride = 20;

// Node gather + nodal update configuration.
struct NodeDev {
    int64_t num_nodes;
    const int32_t* node_ptr;    // num_nodes + 1: node-major slot ranges
    const double* mass;
    const uint32_t* bcword;     // per node: 3 x 10-bit masks of BCs prescribing x, y, z
    const double* bcvalues;     // AM_MAX_BCS x 3 prescribed values
    double g[3];                // body acceleration
    int32_t has_g;
    int64_t num_slots;          // node_ptr[num_nodes]: force slots in use
    // Domain decomposition: interface nodes take their force from the exchanged
    // buffer (row iface_row[i], FP64 x 3) instead of their own slots.
    const int32_t* iface_row;   // per node: row in iface_f, or -1; null when not decomposed
    const double* iface_f;
    // Two-pass reproducing-kernel coupling: every node takes its force from this FP64
    // x 3 array (the scattered generalized force) instead of its slots; null otherwise.
    const double* f_given;
    // Updated (1) / semi (2) Lagrangian formulation, 0 = total: the displacement update
    // also advances the element kernels' coordinates xc and the increment inc.
    int32_t lagr;
    double4* xc;
    double4* inc;
    // Node subset of a k_node_step launch, for overlapping the interface exchange: with
    // subset_nodes the launch runs those nodes (thread t takes subset_nodes[t]); with
    // skip_iface it runs every node except the interface ones. Neither: every node.
    const int32_t* subset_nodes;
    int64_t subset_count;
    int32_t skip_iface;
    int32_t lanes;              // lanes per node in the node kernels; 0: chosen from the slots per node
};

// ---- launchers (am_kernels.cu) ----
void launch_gauss_force(const GaussBlockDev& b, int mixed, const double4* X4, const double4* U4, void* slots,
                        int* status, cudaStream_t s);
// Returns the number of kernels launched (3 for an F-bar block).
int launch_cell_force(const CellBlockDev& b, int mixed, const double4* U4, void* slots, int* status, cudaStream_t s);
void launch_tet4_geometry(const int32_t* conn, int64_t num_elems, const double4* X4, float* geo32, double* geo64,
                          cudaStream_t s);
void launch_gauss_vjp(const GaussBlockDev& b, const double4* X4, const double4* U4, const double4* L4, double4* slots,
                      double* gmu, double* gkappa, int accumulate, cudaStream_t s);
// Lm: scratch of 9 doubles per cell for F-bar blocks (null otherwise). Returns the launch count.
int launch_cell_vjp(const CellBlockDev& b, const double4* U4, const double4* L4, double* Lm, double4* slots,
                    double* gmu, double* gkappa, int accumulate, cudaStream_t s);
void launch_hex6_patch_dx(const int32_t* patch_nodes, int64_t num_patches, const double4* X4, float* dx32,
                          double* dx64, cudaStream_t stream);
void launch_gauss_volume_slots(const GaussBlockDev& b, double density, const double4* X4, double4* slots,
                               cudaStream_t s);
// Chunked blocks: per-corner values (scratch[nn e + a]) summed into the block's slots.
void launch_chunk_sum(const GaussBlockDev& b, const double4* scratch, double4* slots, cudaStream_t s);
void launch_chunk_sum(const CellBlockDev& b, const double4* scratch, double4* slots, cudaStream_t s);
// Chunked blocks: the run-end slot positions of every lane (at am_finalize, after the layout).
void launch_chunk_positions(const GaussBlockDev& b, int32_t* out, cudaStream_t s);
void launch_chunk_positions(const CellBlockDev& b, int32_t* out, cudaStream_t s);

// f (N x 3, row-major) = gather of the slots (FP64 or FP32 slots), overwrite or accumulate.
void launch_gather_force(const NodeDev& nd, int mixed, const void* slots, double* f, int accumulate, cudaStream_t s);
void launch_gather_force4(const NodeDev& nd, int mixed, const void* slots, double4* f, cudaStream_t s);
// Partial force of each local interface node (own slots only) into its row of the
// exchange buffer (rows of nodes this rank does not hold are left as they are).
void launch_iface_gather(const NodeDev& nd, int mixed, const void* slots, int64_t num_local,
                         const int32_t* local_nodes, const int32_t* rows, double* buf, cudaStream_t s);
// Updated / semi-Lagrangian element forces (FP64): coordinates xc, displacement inc, the
// element's reference gradient (rebase: the semi formulation's reference update takes the
// last stored H first).
void launch_gauss_force_lagr(const GaussBlockDev& b, int32_t lagr, int rebase, const double4* XC, const double4* INC,
                             void* slots, int* status, cudaStream_t s);
// a = (f + g m) / m with no boundary condition (pre-loop acceleration).
void launch_init_accel(const NodeDev& nd, int mixed, const void* slots, double4* A4, int* status, cudaStream_t s);
// First half-step of a run: vh = v + h a ; BC(vh) ; u += dt vh.
// rebase (semi formulation): the reference configuration moves first (xc += inc, inc = 0);
// the updated formulation always advances xc by the last increment.
void launch_prologue(const NodeDev& nd, const StepParams* table, double4* U4, double4* V4, const double4* A4,
                     double4* u_copy, int rebase, cudaStream_t s);
// Gather + a = f/m ; BC(a) ; v = vh + h a ; then either advance (next vh, BC, u) or store (v, a).
void launch_node_step(const NodeDev& nd, int mixed, const void* slots, const StepParams* table, int64_t step,
                      int advance, double4* U4, double4* V4, double4* A4, double4* u_copy, int* status,
                      cudaStream_t s, int rebase = 0);
// Adjoint node kernels.
void launch_adj_prep(const NodeDev& nd, const StepParams* table, int64_t step, const double4* VB, const double4* AB,
                     double4* L4, cudaStream_t s);
void launch_adj_update(const NodeDev& nd, const double4* slots, const StepParams* table, int64_t step, double4* UB,
                       double4* VB, double4* AB, double4* L4, cudaStream_t s);
// Power method for the stable time increment (PowerMethodProcessor.h:196-330):
// W = U + V l eps on the free dofs (U on the prescribed ones); then
// V = (f_eps - f_u) / (l eps m) on the free dofs (0 on the prescribed), with the
// squares of V summed per block into partial[blockIdx] (fixed order); then V *= s.
void launch_pm_perturb(const NodeDev& nd, const double4* U4, const double4* V4, const double* l, double eps,
                       double4* W4, cudaStream_t s);
int64_t launch_pm_next(const NodeDev& nd, const double* f_eps, const double* f_u, const double* l, double eps,
                       double4* V4, double* partial, cudaStream_t s);
void launch_pm_scale(int64_t n, double4* V4, double scale, cudaStream_t s);
// Two-pass reproducing-kernel coupling (FunctionEvaluationProcessor): Psi in CSR rows
// (row i: psi_j(x_i) for the neighbours j of node i, n rows: one per node, or one per
// refinement point with the nodes first). rows4: P = Psi U, a row without neighbours
// copying U[i] (zero past the nodes); cols3: f = Psi^T f_local from the transposed CSR
// (column j: the rows i that hold j, ascending i, with a unit entry for each empty node row).
void launch_rk_rows4(int64_t n, int64_t num_nodes, const int64_t* ptr, const int32_t* nbr, const double* val,
                     const double4* U4, double4* P4, cudaStream_t s);
void launch_rk_cols3(int64_t n, const int64_t* tptr, const int32_t* tsrc, const double* tval, const double4* f_local,
                     double* f, cudaStream_t s);
void launch_sensor_seed(const double4* U4, int32_t num_sensors, const int32_t* sensors, double4* UB, double* loss,
                        cudaStream_t s);

// Layout conversion.
void launch_rk_octets(int64_t count, int64_t num_octets, const int32_t* optr, const double2* rec, const double4* in,
                      const int64_t* row_ptr, int64_t num_nodes, double4* out4, double* out3, cudaStream_t s);
void launch_pack4(const double* aos3, double4* out, int64_t n, cudaStream_t s);
void launch_unpack4(const double4* in, double* aos3, int64_t n, cudaStream_t s);
void launch_zero4(double4* out, int64_t n, cudaStream_t s);

// Batched point kernels.
void launch_stress_batch(int32_t mat, double lambda, double mu, int64_t n, const double* H, double* P,
                         cudaStream_t s);
void launch_quadrature_batch(int32_t kind, int32_t smoothed, int64_t n, const double* X, double* B, double* w,
                             cudaStream_t s);

// dst[order[k]] = src[k] for k < n (per-element results back into the caller's order).
void launch_scatter_elems(const int32_t* order, int64_t n, const double* src, double* dst, cudaStream_t s);
// Neighbour exchange: send[k] = own[rows[k]] (3 doubles each) for k < n.
void launch_iface_pack(int64_t n, const int32_t* rows, const double* own, double* send, cudaStream_t s);
// out[r] = sum over e in [ptr[r], ptr[r+1]) of src(idx[e]) in that order, src(j) = own[j]
// for j < num_own and recv[j - num_own] after: each interface node's partial forces
// summed in ascending rank of their holders.
void launch_iface_combine(int64_t rows, const int32_t* ptr, const int32_t* idx, int64_t num_own, const double* own,
                          const double* recv, double* out, cudaStream_t s);

}  // namespace am
