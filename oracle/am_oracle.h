/*
 * am_oracle.h -- CPU FP64 restatement of aperi-mech's explicit-dynamics hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker for the CUDA
 * path in aperi_mech_b200: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it. The product never links,
 * calls or falls back to it.
 *
 * Each routine cites the reference function it restates (paths are relative
 * to the aperi-mech source tree). The arithmetic is plain FP64 with no Eigen;
 * 3x3 inverses use the adjugate formula (Eigen's fixed-size inverse is the
 * same closed form, so results agree to a few ulps).
 *
 * Parity pins: the oracle is checked against the known answers of the
 * reference's own unit tests (QuadratureTests.cpp, MaterialDriverTest.cpp,
 * SolverTest.cpp gravity/free-flight, ForceTest.cpp/PatchTestFixture.h shear
 * and tension patch tests, LinearElasticPropertiesTest.cpp) in tests/.
 * Hex8 2x2x2 Gauss force and the adjoint have no reference known answer
 * (parity unpinned there); they are pinned by analytic patch/rigid-motion
 * checks and by finite differences instead.
 */
#ifndef AM_ORACLE_H
#define AM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OB_TET4_GAUSS = 0, OB_HEX8_GAUSS = 1, OB_CELLS = 2 };
enum { OB_LINEAR_ELASTIC = 0, OB_NEO_HOOKEAN = 1, OB_SVK = 2 };
enum { OB_BC_DISPLACEMENT = 0, OB_BC_VELOCITY = 1 };
enum { OB_TF_RAMP = 0, OB_TF_SMOOTH_STEP = 1 };

/* One part (InternalForceContribution): element kind + material (+ optional
 * per-element shear/bulk fields, which replace lambda/mu element-wise with
 * lambda_e = kappa_e - 2/3 mu_e, mu_e). */
typedef struct {
    int32_t kind;
    int32_t material;
    double lambda, mu, density;
    const double* mu_field;     /* per element / cell, or NULL */
    const double* kappa_field;  /* per element / cell, or NULL */
    int64_t num_elems;          /* elements (Gauss) or cells (OB_CELLS) */
    const int32_t* conn;        /* Gauss: num_elems * nodes_per_elem */
    const int64_t* cell_ptr;    /* cells: num_elems + 1 */
    const int32_t* cell_nodes;  /* cells: cell_ptr[num_elems] */
    const double* cell_grads;   /* cells: 3 per entry, row-major */
    const double* cell_volumes; /* cells: num_elems */
    /* F-bar (ComputeInternalForceSmoothedCell.h:354-413): the cells above are subcells,
     * grouped into num_groups cells by group_ptr (num_groups + 1 offsets); NULL = none. */
    int64_t num_groups;
    const int64_t* group_ptr;
} ob_block;

/* One displacement/velocity boundary condition (BoundaryCondition.cpp). */
typedef struct {
    int64_t num_nodes;
    const int32_t* nodes;
    int32_t component_mask; /* bit c: component c prescribed */
    int32_t kind;           /* OB_BC_DISPLACEMENT / OB_BC_VELOCITY */
    int32_t time_function;  /* OB_TF_RAMP / OB_TF_SMOOTH_STEP */
    int32_t num_points;
    double values[3];
    const double* abscissa;
    const double* ordinate;
    double active_start, active_end;
} ob_bc;

typedef struct {
    int64_t num_nodes;
    const double* coords; /* num_nodes * 3 */
    int32_t num_blocks;
    const ob_block* blocks;
    int32_t num_bcs;
    const ob_bc* bcs;
    const double* mass;    /* lumped nodal mass, or NULL = from Gauss blocks */
    double body_accel[3];  /* gravity vector (ExternalForceContributionGravity) */
    /* Two-pass reproducing-kernel coupling, or NULL: row i of Psi (rk_ptr rk_rows+1,
     * rk_nbr / rk_values) holds the functions psi_j(x_i) at point i. The blocks then see
     * the physical displacement Psi u at the points and their forces reach the nodes as
     * Psi^T f. rk_rows = 0 means one point per node (element cells: the points are the
     * nodes); more points than nodes are the thex refinement points of two-pass nodal
     * cells, the first num_nodes of them the nodes. Cell entries index the points. */
    const int64_t* rk_ptr;
    const int32_t* rk_nbr;
    const double* rk_values;
    int64_t rk_rows;
} ob_problem;

/* ---- quadrature (QuadratureGaussian.h, QuadratureSmoothed.h) ---- */
void ob_tet4_gauss_bw(const double X[12], double B[12], double* w);
void ob_hex8_gauss_bw(const double X[24], int gp, double B[24], double* w);
void ob_tet4_smoothed_bw(const double X[12], double B[12], double* volume);
void ob_hex8_smoothed_bw(const double X[24], double B[24], double* volume);

/* ---- materials (Materials/Base.h, LinearElastic.h, NeoHooke.h, Elastic.h) ---- */
/* props = {E, nu, mu, lambda, K}; NaN = undefined. Returns 0, or -1 with msg. */
int ob_complete_properties(double props[5], char* msg, int msg_len);
void ob_stress(int material, double lambda, double mu, int64_t n, const double* H, double* P);

/* ---- forces, mass, time integration ---- */
void ob_internal_force(const ob_problem* p, const double* u, double* f);
void ob_element_volumes(const ob_problem* p, int32_t block, double* vol);
void ob_lumped_mass(const ob_problem* p, double* m);
int64_t ob_direct_time_schedule(double dt, double t_end, int64_t max_steps, double* dts);
int ob_explicit_solve(const ob_problem* p, double dt, double t_end, int64_t max_steps,
                      double* u, double* v, double* a, int64_t* steps_done);
int ob_init_acceleration(const ob_problem* p, const double* u, double* a);
int ob_explicit_steps(const ob_problem* p, int64_t nsteps, const double* dts, double t0,
                      double* u, double* v, double* a);

/* ---- adjoint (new capability; no reference counterpart) ---- */
void ob_vjp_force(const ob_problem* p, const double* u, const double* lam, double* gu,
                  double* gmu, double* gkappa);
int ob_adjoint(const ob_problem* p, int64_t nsteps, double dt, const double* u0,
               const double* v0, int32_t num_sensors, const int32_t* sensors, double* loss,
               double* gmu, double* gkappa);

/* ---- RKPM setup (ShapeFunctionsFunctorReproducingKernel.h, MathUtils.h,
 *      FunctionCreationProcessor.h, NeighborSearchProcessor) ---- */
double ob_rk_kernel(const double d[3], double R);
int ob_rk_function_values(int64_t num_points, const double* points, const double* coords,
                          const double* kernel_radius, const int64_t* nbr_ptr,
                          const int32_t* nbr, double* values);

/* RKPM one-pass nodal smoothing cells on the tet-corner hexes (the thex
 * refinement: each tet splits into 4 hexes at its corners through edge
 * midpoints, face centroids and the centroid; only the tet vertices are active).
 * Two calls: sizes first (outputs NULL), then the arrays.
 *   points (P x 3) and the neighbour CSR (nbr_ptr P+1, nbr) with function values,
 *   cells (one per vertex): cell_ptr (N+1), cell_nodes, cell_grads (x3), cell_volumes (N),
 *   mass (N): rho V_hex / 8 to the hex points, scattered through the functions. */
int ob_rkpm_nodal_cells(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                        const double* kernel_radius, int32_t max_neighbors, double density,
                        int64_t* num_points, int64_t* num_nbr_entries, int64_t* num_cell_entries,
                        double* points, int64_t* nbr_ptr, int32_t* nbr, double* values,
                        int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads, double* cell_volumes,
                        double* mass);

/* The two-pass form of the same cells (force_two_pass_method with nodal_smoothing_cell):
 * a vertex cell's entries are its corner-hex points (point ids, the first num_nodes
 * points being the vertices) with the hexes' own smoothed gradients b_p = sum_hex
 * B_hex,k(p) V_hex / V_cell; points, functions and mass as above. */
int ob_rkpm_nodal_cells_two_pass(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                                 const double* kernel_radius, int32_t max_neighbors, double density,
                                 int64_t* num_points, int64_t* num_nbr_entries, int64_t* num_cell_entries,
                                 double* points, int64_t* nbr_ptr, int32_t* nbr, double* values,
                                 int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads, double* cell_volumes,
                                 double* mass);

/* RKPM one-pass element smoothing cells (each tet a cell; functions at the vertices).
 * Two calls: sizes first (outputs NULL), then the arrays: the vertices' neighbour CSR
 * (nbr_ptr N+1, nbr) with function values, cells (one per tet): cell_ptr (T+1),
 * cell_nodes, cell_grads (x3), cell_volumes (T), mass (N): rho V_t / 4 to the vertices,
 * scattered through the functions. */
/* The same set-up with every corner hex its own subcell (nodal_smoothing_cell with
 * subdomains 0, LabelSubcellIds in MeshLabelerProcessor.h:832-853): the cell arrays hold
 * one entry per corner hex (vertex order, then tet order) with its own one-pass
 * gradients b = sum_k B_hex,k psi_k and volume, and group_ptr (num_nodes + 1) groups the
 * hexes of each vertex into its cell. num_cell_entries counts the subcell entries. */
int ob_rkpm_nodal_subcells(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                           const double* kernel_radius, int32_t max_neighbors, double density,
                           int64_t* num_cell_entries, int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                           double* cell_volumes, int64_t* group_ptr);

int ob_rkpm_element_cells(int64_t num_nodes, const double* coords, int64_t num_tets, const int32_t* tets,
                          const double* kernel_radius, int32_t max_neighbors, double density,
                          int64_t* num_nbr_entries, int64_t* num_cell_entries, int64_t* nbr_ptr, int32_t* nbr,
                          double* values, int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                          double* cell_volumes, double* mass);

/* The same for Hex8 elements: smoothed Hex8 gradients, mass rho V / 8 to the vertices. */
int ob_rkpm_hex8_element_cells(int64_t num_nodes, const double* coords, int64_t num_hexes, const int32_t* hexes,
                               const double* kernel_radius, int32_t max_neighbors, double density,
                               int64_t* num_nbr_entries, int64_t* num_cell_entries, int64_t* nbr_ptr, int32_t* nbr,
                               double* values, int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                               double* cell_volumes, double* mass);

/* Stable time increment by the power method (PowerMethodProcessor.h:331-480) at the
 * displacement u; v (num_nodes x 3) is the eigenvector estimate, updated in place; l is
 * each node's longest edge. Returns the increment. */
double ob_stable_time_increment(const ob_problem* p, const double* u, double* v, const double* l, double previous,
                                int32_t num_iterations, double eps, double tol, double vartol, int32_t* iterations,
                                int32_t* converged);

/* ---- updated / semi-Lagrangian formulations (Gauss blocks) ----
 * State (ExplicitTimeIntegrator.h:50-90, ComputeInternalForceBase.h:158-174): x holds the
 * current coordinates at the start of the step (updated) or the reference coordinates
 * (semi), inc the displacement increment (of the step, or since the last reference
 * update), H the element displacement gradients of the last force evaluation (one per
 * element: the last Gauss point's, as the reference's element field) and Href the semi
 * formulation's reference gradients; n counts completed steps. Start: x = coordinates,
 * inc = H = Href = 0, n = 0. */
enum { OB_TOTAL = 0, OB_UPDATED = 1, OB_SEMI = 2 };
typedef struct {
    int32_t formulation;
    int32_t update_interval; /* semi: reference update every update_interval steps */
    int64_t n;
    double* x;    /* num_nodes x 3 */
    double* inc;  /* num_nodes x 3 */
    double* H;    /* 9 per Gauss element, blocks in order */
    double* Href; /* 9 per Gauss element (semi) */
} ob_lagrangian;
/* Internal force of the formulation at the state (stores H). */
int ob_lagrangian_force(const ob_problem* p, ob_lagrangian* s, double* f);
/* Initial acceleration (the force at the state, no acceleration BC). */
int ob_lagrangian_init(const ob_problem* p, ob_lagrangian* s, double* a);
/* nsteps central-difference steps in the order of ExplicitSolver::Solve with the
 * formulation's displacement update and reference-configuration updates. */
int ob_lagrangian_steps(const ob_problem* p, ob_lagrangian* s, int64_t nsteps, const double* dts, double t0, double* u,
                        double* v, double* a);

/* ---- threads ---- */
void ob_set_threads(int n);
int ob_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
