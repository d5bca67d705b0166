/*
 * aperi_b200.h -- C ABI of the B200-native explicit-dynamics hot path.
 *
 * The library replaces, for one GPU, the per-step path of aperi-mech's
 * explicit solver: the internal-force contributions of the parts
 * (InternalForceContribution -> ElementBase::ComputeInternalForceAllElements),
 * their material stress update (Material::StressFunctor::GetStress) and the
 * central-difference nodal update (ExplicitTimeIntegrator), in the step order of
 * ExplicitSolver::Solve. Reference interfaces are cited as file:line of the
 * aperi-mech source tree.
 *
 * Conventions
 *  - Every call returns an am_status code; no C++ exception crosses the ABI.
 *    am_last_error() gives the message of the last failing call on a context.
 *  - Nodal vectors are row-major N x 3 FP64 arrays (the layout of an aperi
 *    3-component node field, Field.h:129-136). Tensors are row-major 3 x 3.
 *  - Pointers are host or device pointers as selected by the am_memory
 *    argument. Host arrays passed to am_add_block / am_set_boundary_conditions /
 *    am_create are copied; the caller keeps ownership.
 *  - One context owns its device buffers and one CUDA stream (or the stream
 *    given to am_set_stream). Calls are stream-ordered; the host blocks only
 *    in am_get_* with AM_HOST, in am_run/am_solve/am_adjoint when the device
 *    status word must be read, and on errors. A context is not thread-safe.
 *  - Forces are assembled by a deterministic node-centric gather (no atomics):
 *    results are bitwise reproducible run to run.
 */
#ifndef APERI_B200_H
#define APERI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AM_MAX_BCS 10

typedef enum {
    AM_OK = 0,
    AM_EINVAL = 1,      /* invalid argument (std::runtime_error in the reference) */
    AM_ENOMEM = 2,      /* device allocation failed */
    AM_ECUDA = 3,       /* CUDA runtime error */
    AM_ENONPOS_J = 4,   /* an element / cell reached det F <= 0 or det J <= 0 */
    AM_ENAN = 5,        /* a non-finite nodal acceleration was produced */
    AM_ESTATE = 6,      /* call out of order (e.g. before am_finalize) */
    AM_ERANGE = 7       /* size beyond a compiled limit */
} am_status;

typedef enum { AM_FP64 = 0, AM_MIXED = 1 } am_precision;
typedef enum { AM_HOST = 0, AM_DEVICE = 1 } am_memory;

/* Element kinds: ElementTetrahedron4 (1-pt Gauss), ElementHexahedron8 (2x2x2
 * Gauss), and strain-smoothed / RKPM cells (ElementSmoothedTetrahedron4,
 * ElementReproducingKernel; include/Element.h:32-86). */
typedef enum { AM_TET4_GAUSS = 0, AM_HEX8_GAUSS = 1, AM_SMOOTHED_CELLS = 2 } am_block_kind;

/* Materials/Base.h MaterialType: LINEAR_ELASTIC, NEO_HOOKEAN, ELASTIC (SVK). */
typedef enum { AM_LINEAR_ELASTIC = 0, AM_NEO_HOOKEAN = 1, AM_ELASTIC_SVK = 2 } am_material_kind;

typedef enum { AM_BC_DISPLACEMENT = 0, AM_BC_VELOCITY = 1 } am_bc_kind;
typedef enum { AM_TF_RAMP = 0, AM_TF_SMOOTH_STEP = 1 } am_time_function;

/* One part: replaces InternalForceContribution (include/InternalForceContribution.h:26-159)
 * with its Material (include/Materials/Factory.h:43). lambda/mu are the completed
 * Lame parameters (LinearElasticProperties::CompleteProperties, Materials/Base.h:47-129).
 * mu_field / kappa_field (per element or cell, optional) replace them element-wise
 * with lambda_e = kappa_e - 2/3 mu_e. */
typedef struct {
    int32_t kind;               /* am_block_kind */
    int32_t material;           /* am_material_kind */
    double lambda, mu, density;
    const double* mu_field;     /* host, num_elems, or NULL */
    const double* kappa_field;  /* host, num_elems, or NULL */
    int64_t num_elems;          /* elements, or cells for AM_SMOOTHED_CELLS */
    const int32_t* conn;        /* Gauss: num_elems x (4|8), reference node order */
    const int64_t* cell_ptr;    /* cells: num_elems+1 offsets into the entry arrays */
    const int32_t* cell_nodes;  /* cells: node of each entry (SmoothedCellData node CSR) */
    const double* cell_grads;   /* cells: entry x 3 smoothed gradients (function derivatives) */
    const double* cell_volumes; /* cells: num_elems subcell volumes */
} am_block_desc;

/* Displacement / velocity boundary condition (src/BoundaryCondition.cpp:14-222).
 * values = magnitude x normalized direction, or the component values. Later
 * entries win where node sets overlap, as in the reference's in-order apply. */
typedef struct {
    int64_t num_nodes;
    const int32_t* nodes;       /* host */
    int32_t component_mask;     /* bit c: component c prescribed */
    int32_t kind;               /* am_bc_kind */
    int32_t time_function;      /* am_time_function */
    int32_t num_points;
    double values[3];
    const double* abscissa;     /* host, num_points */
    const double* ordinate;     /* host, num_points */
    double active_start, active_end;
} am_bc_desc;

typedef struct am_ctx am_ctx;

/* ---- context set-up (replaces Application::CreateSolver / Preprocessor) ---- */
int am_create(int64_t num_nodes, const double* coords, am_ctx** out);
void am_destroy(am_ctx* ctx);
int am_set_stream(am_ctx* ctx, void* cuda_stream);
int am_add_block(am_ctx* ctx, const am_block_desc* desc, int32_t* block_id);
int am_set_boundary_conditions(am_ctx* ctx, int32_t num_bcs, const am_bc_desc* bcs);
/* Replace the per-element shear / bulk modulus fields of a block (host arrays of
 * num_elems; NULL leaves that field unchanged). Allowed after am_finalize. */
int am_set_block_fields(am_ctx* ctx, int32_t block_id, const double* mu_field, const double* kappa_field);
/* F-bar smoothed cells (use_f_bar; ComputeInternalForceSmoothedCell.h:120-183 J-bar and
 * F-bar, :227-309 the stress un-barring, :354-413 the pass order). The block's cells
 * become subcells, grouped into num_cells cells: cell g holds subcells
 * [group_ptr[g], group_ptr[g+1]) (host array). Per force evaluation: H and J of every
 * subcell, Jbar = sum J_s V_s / V_cell per cell, the subcells' stresses at
 * Fbar = (Jbar / J_s)^(1/3) F, the cell's dual pressure, the un-barred stresses, and the
 * subcell forces -V_s b P^T. As in the reference, when num_cells equals the subcell
 * count the call changes nothing. Before am_finalize. am_vjp_force and am_adjoint take
 * F-bar blocks in the cell-stress form (every cell of at most 32 subcells, the default
 * layout; AM_ESTATE otherwise): the VJP is the F-bar force's derivative along lam, the
 * force being the gradient of sum_s V_s psi(Fbar_s). */
int am_set_cell_groups(am_ctx* ctx, int32_t block_id, int64_t num_cells, const int64_t* group_ptr);
int am_set_body_acceleration(am_ctx* ctx, const double g[3]);
int am_set_mass(am_ctx* ctx, const double* mass);
int am_finalize(am_ctx* ctx);

/* ---- state (the *_coefficients node fields, states N and NP1 folded) ---- */
int am_set_state(am_ctx* ctx, am_memory where, const double* u, const double* v, const double* a);
int am_get_state(am_ctx* ctx, am_memory where, double* u, double* v, double* a);
int am_get_mass(am_ctx* ctx, double* mass_host);

/* ---- the hot path ---- */
/* Internal force f = F(u) over all parts: replaces ComputeInternalForceGaussian::operator()
 * (include/ComputeInternalForceGaussian.h:57-131) and
 * ComputeInternalForceSmoothedCellBase::ForEachCellComputeForce
 * (include/ComputeInternalForceSmoothedCell.h:416-442). accumulate=0 overwrites f,
 * accumulate=1 adds to it (the reference accumulates into a zeroed field). */
int am_internal_force(am_ctx* ctx, am_precision prec, am_memory where, const double* u, double* f, int accumulate);
/* Pre-loop force + acceleration of ExplicitSolver::Solve (src/Solvers/Explicit.cpp:357-368). */
int am_init_acceleration(am_ctx* ctx, am_precision prec);
/* nsteps central-difference steps at fixed dt from time t0 (loop body of
 * src/Solvers/Explicit.cpp:383-483 with ExplicitTimeIntegrator.h:97-364). */
int am_run(am_ctx* ctx, am_precision prec, int64_t nsteps, double dt, double t0);
/* The same with a per-step time increment. */
int am_run_schedule(am_ctx* ctx, am_precision prec, int64_t nsteps, const double* dts, double t0);
/* ExplicitSolver::Solve with a DirectTimeStepper (include/TimeStepper.h:97-128):
 * initial acceleration, then steps until time >= t_end. */
int am_solve(am_ctx* ctx, am_precision prec, double dt, double t_end, int64_t max_steps, int64_t* steps_done);

/* ---- adjoint (no counterpart in the reference) ---- */
/* gu = (dF/du)^T lam ; gmu/gkappa (per element, all parts concatenated, may be NULL)
 * = (dF/dmu_e)^T lam, (dF/dkappa_e)^T lam. FP64. */
int am_vjp_force(am_ctx* ctx, am_memory where, const double* u, const double* lam, double* gu, double* gmu,
                 double* gkappa);
/* Loss L = sum_s |u_s(nsteps)|^2 over the sensor nodes after nsteps steps from the
 * current state, and its gradient with respect to the per-element shear and bulk
 * moduli, by a reverse pass with checkpoints every ckpt_every steps. FP64. The
 * state is left at the end of the forward trajectory. Host outputs. */
int am_adjoint(am_ctx* ctx, int64_t nsteps, double dt, int32_t ckpt_every, int32_t num_sensors,
               const int32_t* sensors, double* loss, double* gmu, double* gkappa);

/* ---- batched point kernels (for the reference's unit-level known answers) ---- */
/* Material::StressFunctor::GetStress (Materials/Base.h:205-213) on n displacement gradients. */
int am_stress(int32_t material, double lambda, double mu, int64_t n, am_memory where, const double* H, double* P);
/* Quadrature::ComputeBMatrixAndWeight (QuadratureGaussian.h:17-39) for each element
 * and Gauss point of kind (Tet4: 1 point, Hex8: 8 points), or the smoothed
 * quadrature (QuadratureSmoothed.h:32-142) when smoothed != 0.
 * X: n x nodes x 3; B: n x points x nodes x 3; w: n x points. */
int am_quadrature(int32_t kind, int32_t smoothed, int64_t n, am_memory where, const double* X, double* B,
                  double* w);

/* ---- RKPM one-pass nodal smoothing cells (set-up) ----
 * Replaces the reproducing-kernel preprocessing of ElementReproducingKernel with
 * nodal_smoothing_cell on a thex mesh: the neighbour search
 * (NeighborSearchProcessor.h:224-319, capped at max_neighbors; the reference caps at
 * 40, Constants.h:15), the function values (FunctionCreationProcessor.h:72-134, the
 * 4x4 moment matrices solved in FP64 on the GPU), the one-pass smoothed gradients
 * (SmoothedCellDataProcessor.h:541-675) and the lumped mass scattered through the
 * functions (src/MassUtils.cpp:79-112). The thex refinement is implicit: every tet
 * contributes, at each vertex, the hex through its edge midpoints, face centroids
 * and centroid; one cell per tet vertex (the active nodes). kernel_radius is per
 * vertex. The result feeds am_add_block (AM_SMOOTHED_CELLS) and am_set_mass. Host
 * arrays; errors via am_last_error(NULL). */
typedef struct am_cells am_cells;
int am_rkpm_nodal_cells(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                        const double* kernel_radius, int32_t max_neighbors, double density, am_cells** out);
/* RKPM one-pass element smoothing cells (element_smoothing_cell, subdomains 1, with the
 * reproducing_kernel approximation space): one cell per tet, whose entries are the
 * union of its four vertices' neighbours, gradients b_{t,j} = sum_k B_{t,k} psi_k(j)
 * (SmoothedCellDataProcessor.h:541-675 one-pass, QuadratureSmoothed.h:32-63), the
 * functions evaluated at the vertices only, and the mass rho V_t / 4 to the vertices
 * scattered through the functions. Same outputs and accessors as the nodal cells
 * (the points are the vertices). */
/* Nodal cells split into subcells (nodal_smoothing_cell with subdomains 0,
 * MeshLabelerProcessor.h:832-853): every corner hex is a subcell with its own one-pass
 * gradients sum_k B_hex,k psi_k(j) and volume; the cell arrays hold the subcells
 * (vertex order, then tet order), am_cells_groups gives the vertex cells they form
 * (for am_set_cell_groups). Same functions and mass as am_rkpm_nodal_cells. */
int am_rkpm_nodal_subcells(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                           const double* kernel_radius, int32_t max_neighbors, double density, am_cells** out);
/* Cells formed by the subcells: num_groups (0 when every cell is one subcell) and, when
 * group_ptr is not NULL, its num_groups + 1 offsets. */
int am_cells_groups(const am_cells* cells, int64_t* num_groups, int64_t* group_ptr);
int am_rkpm_element_cells(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                          const double* kernel_radius, int32_t max_neighbors, double density, am_cells** out);
/* Two-pass nodal cells (nodal_smoothing_cell with force_two_pass_method,
 * InternalForceContributionParameters.h:164-194; ExplicitSolver::ComputeForce's two
 * passes, src/Solvers/Explicit.cpp:146-186): the vertex cells of am_rkpm_nodal_cells,
 * whose entries are now their corner-hex points (point ids; the first num_nodes points
 * are the vertices) with the hexes' own smoothed gradients b_p = sum_hex B_hex(p) V_hex /
 * V_cell (SmoothedCellDataProcessor.h:541-675 without the functions). The functions at
 * all points (am_cells_get_points) couple them to the vertices at run time: declare the
 * points with am_set_rk_points before am_add_block, add the cells, pass the mass (as
 * above) to am_set_mass, finalize, then hand the functions to am_set_rk_functions. */
int am_rkpm_nodal_cells_two_pass(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                                 const double* kernel_radius, int32_t max_neighbors, double density, am_cells** out);
/* The same for Hex8 elements (ElementReproducingKernelHex8 with element_smoothing_cell, the
 * reference's rkpm_hex inputs): one cell per hex (reference node order), gradients from the
 * smoothed Hex8 quadrature (QuadratureSmoothed.h:97-142) through the vertices' functions,
 * mass rho V / 8 to the vertices scattered through the functions. */
int am_rkpm_hex8_element_cells(int64_t num_nodes, const double* coords, int64_t num_hexes, const int32_t* hexes,
                               const double* kernel_radius, int32_t max_neighbors, double density, am_cells** out);
/* Finite-element strain smoothing with element cells (element_smoothing_cell with
 * finite_element, subdomains 1; ElementSmoothedTetrahedron4, include/Element.h:45-47):
 * one cell per Tet4 or Hex8 element holding its own nodes, with the smoothed gradients
 * of QuadratureSmoothed.h:32-63 (Tet4) / :97-142 (Hex8) and the element volume, and the
 * lumped mass rho V / nodes_per_elem to the vertices (src/MassUtils.cpp:17-46). Host
 * only. Read it with am_cells_sizes / am_cells_get, add it with am_add_block
 * (AM_SMOOTHED_CELLS) and pass the mass to am_set_mass. */
int am_smoothed_element_cells(int64_t num_nodes, const double* coords, int64_t num_elems, int32_t nodes_per_elem,
                              const int32_t* conn, double density, am_cells** out);
int am_cells_sizes(const am_cells* cells, int64_t* num_cells, int64_t* num_entries, int64_t* num_points,
                   int64_t* num_nbr_entries);
/* cell_ptr (num_cells+1), cell_nodes/cell_grads (entries, x3), cell_volumes (num_cells)
 * and mass (one per mesh node). */
int am_cells_get(const am_cells* cells, int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                 double* cell_volumes, double* mass);
/* The refinement points (x3), their neighbour CSR and function values. */
int am_cells_get_points(const am_cells* cells, double* points, int64_t* nbr_ptr, int32_t* nbr, double* values);
void am_cells_destroy(am_cells* cells);

/* ---- allocation-free Tet4 internal force (no counterpart in the reference) ----
 * For callers that cannot allocate device memory, e.g. a host framework that owns
 * every device allocation through its own pool, or a step that must not pay the
 * latency and implicit synchronization of cudaMalloc/cudaFree. Computes
 * f = F(u) (overwritten) for one Tet4 1-point-Gauss part without allocating:
 * all arguments are device pointers owned by the caller, and the per-element
 * force slots live in a fixed 16 MiB device array inside this library that every
 * GPU loading it keeps until process exit. Hence at most AM_NOALLOC_MAX_TETS tets;
 * larger inputs return AM_ERANGE with the reason in am_last_error(NULL).
 *   coords, u, f : num_nodes x 3 row-major FP64;  conn : num_elems x 4 (reference node order)
 *   node_ptr (num_nodes+1) / node_slots (4 num_elems): for each node, the slots
 *   4e+a (element e, local node a) that touch it, ascending. node_ptr[num_nodes]
 *   must equal 4 num_elems and every slot id must be below it: only those slots
 *   are written by this call, so a range or id beyond them would read what an
 *   earlier call left in the shared array. Such entries are skipped and reported
 *   as AM_EINVAL through am_noalloc_status (index = the node).
 * The first call on a device, and the first after a device reset, looks up the
 * scratch array's device address (so make that call before any stream capture).
 * All calls share the array: each call overwrites the slots it reads, so nothing
 * needs clearing, but calls that overlap on the GPU race on it and must be ordered
 * by the caller. Stream-ordered on cuda_stream (NULL = legacy default stream);
 * nothing is synchronized, and device-side checks do not change the return code:
 * read them with am_noalloc_status. */
#define AM_NOALLOC_MAX_TETS 174762
int am_tet4_internal_force_noalloc(int32_t material, double lambda, double mu, int64_t num_nodes, int64_t num_elems,
                                   const double* coords, const double* u, const int32_t* conn,
                                   const int32_t* node_ptr, const int32_t* node_slots, double* f, void* cuda_stream);
/* Device-side status of the most recent am_tet4_internal_force_noalloc call on the
 * current device (no counterpart in the reference; the context path reports the same
 * checks through its own return codes): *status = AM_OK, AM_ENONPOS_J (a tet with
 * det J <= 0, or J <= 0 for neo-Hookean; *index = the tet) or AM_EINVAL (a node ->
 * slot CSR entry outside the call's slots; *index = the node, or num_nodes when
 * node_ptr[num_nodes] != 4 num_elems). The first error of a call wins. The word lives
 * beside the scratch array, in fixed device memory shared by every caller, and each
 * force call clears it before its kernels run; so read it on the same stream, after
 * the call and before the next one. Synchronizes cuda_stream; allocates nothing. */
int am_noalloc_status(void* cuda_stream, int32_t* status, int64_t* index);

/* LinearElasticProperties::CompleteProperties (Materials/Base.h:47-158): props =
 * {youngs_modulus, poissons_ratio, shear_modulus, lambda, bulk_modulus} with NaN for
 * the undefined ones; exactly two must be defined. Fills the rest, checks the physical
 * bounds; on failure returns AM_EINVAL and writes the reason to msg. Host only. */
int am_complete_properties(double props[5], char* msg, int msg_len);

/* The order in which the library runs a Gauss block's elements (no counterpart in the
 * reference, whose Kokkos loops run elements in mesh order). Host only. order[k] = the
 * caller's index of the k-th element run. Chosen from the mesh alone, so every
 * numbering of one mesh gets the same order (and bitwise the same results): with
 * try_rings, Tet4 blocks whose tets all lie on six-tet rings around an edge (a tet
 * (c0, a, b, c3) on the ring of the tets sharing its first and last node, as in the
 * six-tet split of a hex) run ring by ring in the Morton order of the ring axes, each
 * ring in its chain order (*rings = 1: the split-hex patches); otherwise the elements
 * run in the Morton order of their centroids (*rings = 0). am_add_block applies it
 * unless APERI_B200_ELEMENT_ORDER=input; per-element inputs and outputs of the ABI stay
 * in the caller's order. */
int am_element_order(int64_t num_nodes, const double* coords, int64_t num_elems, int32_t nodes_per_elem,
                     const int32_t* conn, int32_t try_rings, int32_t* order, int32_t* rings);

/* ---- diagnostics ---- */
const char* am_last_error(const am_ctx* ctx);
const char* am_status_string(int status);
/* Force-slot layout after am_finalize: node-major slots referenced by nodes (one per
 * element node, patch node, cell entry or, for blocks run in warp chunks, distinct node of
 * a chunk; APERI_B200_WARP_CHUNKS=0 turns the chunks off), and the number of Tet4 blocks
 * assembled through element patches. */
int am_get_layout(const am_ctx* ctx, int64_t* used_slots, int32_t* patched_tet4_blocks);
/* Kernel launches issued by this context so far (all kinds). */
int64_t am_launch_count(const am_ctx* ctx);
/* Per-kernel device timing: when enabled, every launch of the hot loop is
 * bracketed by CUDA events on the context stream (recorded asynchronously; the
 * elapsed times are collected, with one synchronization, by am_profile_read).
 * Slot 0: element/cell force kernels, 1: node gather + update kernels, 2: VJP
 * kernels, 3: adjoint node kernels, 4: interface exchange (decomposed meshes).
 * Milliseconds and launch counts accumulate until am_profile_enable is called again. */
int am_profile_enable(am_ctx* ctx, int enable);
int am_profile_read(am_ctx* ctx, double ms[5], int64_t launches[5]);
/* Measured FMA throughput of the current device (no counterpart in the reference): FP64
 * (fp64 != 0) or FP32 fused multiply-adds in independent chains over the whole GPU,
 * one launch timed with CUDA events on cuda_stream after a warm-up launch; writes
 * flop/s (an FMA counts 2). The compute-roofline denominator for the element kernels,
 * which FP32 issue or the FP64 pipe bind rather than HBM. Synchronizes cuda_stream. */
int am_measure_fma_peak(int32_t fp64, void* cuda_stream, double* flops_per_s);

/* ---- stable time increment by the power method (PowerMethodProcessor,
 * include/PowerMethodProcessor.h:87-480, and PowerMethodTimeStepper, TimeStepper.h:138-221) ----
 * am_set_power_method: the start vector (num_nodes x 3, e.g. uniform in [-1, 1]; the
 * reference draws it per node from its id) and each node's longest edge to a node of a
 * connected element (MaxEdgeLengthProcessor). The first increment scales the start
 * vector by epsilon times the edge length; later ones continue from the last estimate.
 * am_stable_time_increment: 2 / sqrt(lambda_max(M^-1 K)) at the current displacement,
 * by power iteration on finite differences of the internal force with the reference's
 * stopping rules; previous is the last (unscaled) increment, 0 at the start.
 * am_solve_power_method: Solve() with the power-method time stepper: initial
 * acceleration, then every update_interval steps the increment is recomputed
 * (50 iterations, epsilon 1e-5, tolerance 1e-3, variation tolerance 1e-7, the
 * reference's defaults) and multiplied by scale_factor; the last step ends at t_end.
 * FP64 increments; not available on a decomposed mesh. */
int am_set_power_method(am_ctx* ctx, const double* start, const double* max_edge_length);
int am_stable_time_increment(am_ctx* ctx, double previous, int32_t num_iterations, double epsilon, double tolerance,
                             double variation_tolerance, double* dt, int32_t* iterations, int32_t* converged);
int am_solve_power_method(am_ctx* ctx, am_precision prec, double scale_factor, int64_t update_interval, double t_end,
                          int64_t max_steps, int64_t* steps_done, double* last_increment);

/* ---- updated / semi-Lagrangian formulations (LagrangianFormulationType; the Gauss force
 * ComputeInternalForceGaussian.h:57-131 with ComputeInternalForceBase.h:158-174; the displacement
 * update ExplicitTimeIntegrator.h:141-244,461-551; the reference-configuration schedule
 * src/Application.cpp:301-308 and src/Solvers/Explicit.cpp:195-214) ----
 * formulation 0 total (the default), 1 updated, 2 semi with a reference update every
 * update_interval steps. The element kernels then take shape-function gradients on the
 * current coordinates (updated: those at the start of the step) or on the reference
 * coordinates of the last update (semi), the displacement increment of the step (updated)
 * or since the last update (semi), and compose H = dH + Href + dH Href with the element's
 * stored reference gradient; forces map back through F_ref = I + Href. As in the reference,
 * an element keeps one H: for Hex8 the last Gauss point's serves as every Gauss point's
 * reference (Tet4, with one point, matches the total formulation to round-off). State
 * starts undeformed and is reset by every am_set_state (whose displacement, null meaning
 * zero, should be zero); FP64 only; Gauss blocks only; not with am_internal_force, the VJP, the adjoint,
 * the power method, the two-pass coupling or a decomposed mesh (AM_ESTATE). Call after
 * am_create and before am_add_block (Tet4 blocks then keep per-element slots). */
int am_set_formulation(am_ctx* ctx, int32_t formulation, int32_t update_interval);

/* ---- two-pass reproducing-kernel coupling (the solver's generalized-field path with the
 * two-pass method, src/Solvers/Explicit.cpp:146-186; FunctionEvaluationProcessor::ComputeValues
 * and ScatterValues, include/FunctionEvaluationProcessor.h:70-174) ----
 * The state (u, v, a) holds the generalized coefficients. Row i of Psi (nbr_ptr num_nodes+1,
 * nbr, values; host arrays) lists psi_j(x_i) for the neighbours j of node i, as
 * am_cells_get_points returns them for element cells. Every force evaluation then runs
 * the blocks (FEM smoothed cells, Gauss elements) on the physical displacement Psi u
 * (a row without neighbours copies its coefficient), gathers their forces per node and
 * scatters them to the coefficients as Psi^T f (a row without neighbours passes its
 * force through), summed in a fixed order instead of the reference's atomics. Needs the
 * generalized lumped mass (the element mass scattered through the functions, as
 * am_cells_get returns it) from am_set_mass before am_finalize; call once after
 * am_finalize. am_vjp_force and am_adjoint then apply Psi^T VJP(Psi u, Psi lam) (the VJP of
 * the composed force; the modulus gradients are the blocks' at the physical fields). Not
 * available on a decomposed mesh (AM_ESTATE). */
int am_set_rk_functions(am_ctx* ctx, const int64_t* nbr_ptr, const int32_t* nbr, const double* values);
/* Points for cells coupled through the functions (two-pass nodal cells): the cell entries
 * of this context then index num_points points, the first num_nodes being the nodes and
 * the rest refinement points. The functions of am_set_rk_functions then have one row per
 * point (nbr_ptr of num_points + 1), the physical displacement lives on the points and
 * the cells' forces reach the nodes through the functions' transpose. Before am_add_block. */
int am_set_rk_points(am_ctx* ctx, int64_t num_points);

/* ---- domain decomposition (replaces the reference's ParallelSum of the force field
 * after the element loop, src/Solvers/Explicit.cpp:190-193) ----
 * A context holds one rank's slab of elements and every node they touch; nodes held by
 * several ranks are interface nodes. local_nodes[k] (this context's node ids) owns row
 * rows[k] of an exchange buffer of num_global rows (FP64 x 3, the interface nodes of the
 * whole mesh). Each step the element kernels run, every interface node's partial force
 * goes to its row, the rows are summed over the ranks (NCCL all-reduce on the context
 * stream when a communicator is set; a single rank without one sums nothing), and the
 * node kernel takes the summed force for interface nodes. Needs the global lumped mass
 * (am_set_mass before am_finalize); call after am_finalize. The VJP and the adjoint are
 * not available on a decomposed mesh (AM_ESTATE). */
int am_set_interface(am_ctx* ctx, int64_t num_local, const int32_t* local_nodes, const int32_t* rows,
                     int64_t num_global);
/* The same decomposition with a neighbour exchange in place of the all-rank sum: this
 * context is rank `rank`; it shares nodes with num_neighbors ranks neighbor_ranks
 * (ascending), the nodes shared with neighbour j being shared_nodes[shared_ptr[j] ..
 * shared_ptr[j+1]) (this context's node ids, in the order both ranks of the pair use,
 * e.g. ascending global id). Each step this rank's partial forces of the shared nodes go
 * to the neighbours that hold them (grouped ncclSend / ncclRecv, payload a few MB at
 * most for slabs), and every interface node sums its holders' partials in ascending rank
 * (its own at its place), so all holders of a node get the same bits. In am_run /
 * am_solve the exchange runs on a second stream while the interior nodes update, and the
 * interface nodes update once it lands (APERI_B200_EXCHANGE_OVERLAP=0 runs the two in
 * sequence on the context stream, with bitwise the same result). Call after am_finalize
 * instead of am_set_interface, then am_set_nccl with the same rank. */
int am_set_neighbors(am_ctx* ctx, int32_t rank, int32_t num_neighbors, const int32_t* neighbor_ranks,
                     const int64_t* shared_ptr, const int32_t* shared_nodes);
/* ncclGetUniqueId (libnccl.so.2 is opened at run time): rank 0 makes the id, the host
 * sends it to the other ranks, every rank passes it to am_set_nccl. */
int am_nccl_unique_id(unsigned char id[128]);
int am_set_nccl(am_ctx* ctx, const unsigned char id[128], int32_t rank, int32_t nranks);

#ifdef __cplusplus
}
#endif
#endif
