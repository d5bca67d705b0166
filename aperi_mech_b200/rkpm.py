"""RKPM smoothing cells (ElementReproducingKernel, include/ElementReproducingKernel.h)
built by the library's set-up: neighbour search, FP64 reproducing-kernel functions on
the GPU, one-pass smoothed gradients, lumped mass scattered through the functions.
Nodal cells (nodal_smoothing_cell) live on the tet-corner hexes of the thex refinement
(am_rkpm_nodal_cells); element cells (element_smoothing_cell) are the tets themselves
(am_rkpm_element_cells). The two-pass method on element cells keeps the tets' own
smoothed FEM gradients and couples them to the coefficients through the functions at
the vertices (two_pass_element_cells, ExplicitDynamics.set_rk_functions)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .capi import check
from .model import Material, Part


@dataclass
class RKPMCells:
    part: Part
    mass: np.ndarray
    points: np.ndarray | None = None
    nbr_ptr: np.ndarray | None = None
    nbr: np.ndarray | None = None
    values: np.ndarray | None = None

    @property
    def entries_per_cell(self) -> float:
        return float(self.part.cell_ptr[-1]) / (len(self.part.cell_ptr) - 1)

    def functions(self):
        """(nbr_ptr, nbr, values) of the functions at the mesh nodes, for the two-pass
        coupling (element cells: the points are the vertices)."""
        if self.nbr_ptr is None:
            raise ValueError("built without keep_points")
        if self.points is not None and self.points.shape[0] != self.mass.shape[0] and \
                int(self.part.cell_nodes.max()) < self.mass.shape[0]:
            raise ValueError("the functions live on refinement points the cells do not use")
        return self.nbr_ptr, self.nbr, self.values


def thex_max_edge_length(coords: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """MaxEdgeLengthFunctor (src/MaxEdgeLengthProcessor.cpp:36-60) on the thex refinement:
    for each vertex, the longest distance to a point of its corner hexes, doubled for
    inactive points (edge midpoints, face centroids, centroids)."""
    x = coords[tets]  # T x 4 x 3
    cen = x.mean(axis=1)
    out = np.zeros(coords.shape[0])
    for i in range(4):
        v = x[:, i]
        cand = [2.0 * np.linalg.norm(cen - v, axis=1)]
        others = [j for j in range(4) if j != i]
        for j in others:
            cand.append(2.0 * np.linalg.norm((x[:, j] + v) * 0.5 - v, axis=1))
        for a in range(3):
            for b in range(a + 1, 3):
                f = (v + x[:, others[a]] + x[:, others[b]]) / 3.0
                cand.append(2.0 * np.linalg.norm(f - v, axis=1))
        np.maximum.at(out, tets[:, i], np.max(np.stack(cand), axis=0))
    return out


def tet_max_edge_length(coords: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """MaxEdgeLengthFunctor (src/MaxEdgeLengthProcessor.cpp:36-60) on a tet mesh whose
    nodes are all active: per node, the longest distance to a node of a connected tet."""
    from .mesh import max_edge_length

    return max_edge_length(coords, tets)


def nodal_cells(coords: np.ndarray, tets: np.ndarray, material: Material, kernel_radius: np.ndarray,
                max_neighbors: int = 40, keep_points: bool = False, mu_field=None, kappa_field=None,
                name: str = "block_1") -> RKPMCells:
    """One cell per vertex on the thex corner hexes (nodal_smoothing_cell)."""
    return _cells("am_rkpm_nodal_cells", coords, tets, material, kernel_radius, max_neighbors, keep_points,
                  mu_field, kappa_field, name)


def nodal_subcells(coords: np.ndarray, tets: np.ndarray, material: Material, kernel_radius: np.ndarray,
                   max_neighbors: int = 40, keep_points: bool = False, fbar: bool = True, mu_field=None,
                   kappa_field=None, name: str = "block_1") -> RKPMCells:
    """Nodal cells split into one subcell per corner hex (nodal_smoothing_cell with
    subdomains 0); with fbar the part carries the vertex cells they form (use_f_bar),
    otherwise every subcell integrates on its own."""
    return _cells("am_rkpm_nodal_subcells", coords, tets, material, kernel_radius, max_neighbors, keep_points,
                  mu_field, kappa_field, name, groups=fbar)


def two_pass_nodal_cells(coords: np.ndarray, tets: np.ndarray, material: Material, kernel_radius: np.ndarray,
                         max_neighbors: int = 40, mu_field=None, kappa_field=None,
                         name: str = "block_1") -> RKPMCells:
    """Two-pass nodal cells (nodal_smoothing_cell with force_two_pass_method): the vertex
    cells' entries are their corner-hex points with the hexes' own smoothed gradients;
    functions() then returns one row per point (the vertices first), which
    ExplicitDynamics(..., rk=cells.functions()) takes as the coupling."""
    return _cells("am_rkpm_nodal_cells_two_pass", coords, tets, material, kernel_radius, max_neighbors, True,
                  mu_field, kappa_field, name)


def element_cells(coords: np.ndarray, tets: np.ndarray, material: Material, kernel_radius: np.ndarray,
                  max_neighbors: int = 40, keep_points: bool = False, mu_field=None, kappa_field=None,
                  name: str = "block_1") -> RKPMCells:
    """One cell per element (element_smoothing_cell with the reproducing_kernel space):
    Tet4 (4 columns) or Hex8 (8 columns, reference node order) connectivity."""
    entry = "am_rkpm_hex8_element_cells" if np.asarray(tets).shape[1] == 8 else "am_rkpm_element_cells"
    return _cells(entry, coords, tets, material, kernel_radius, max_neighbors, keep_points, mu_field, kappa_field,
                  name)


def two_pass_element_cells(coords: np.ndarray, tets: np.ndarray, material: Material, kernel_radius: np.ndarray,
                           max_neighbors: int = 40, mu_field=None, kappa_field=None, name: str = "block_1") -> RKPMCells:
    """element_smoothing_cell with the reproducing_kernel space and the two-pass method
    (the reference's default for element cells): the cells are the tets with their own
    smoothed gradients (SmoothedCellDataProcessor.h:541-675, two-pass branch), the mass is
    rho V_t / 4 scattered through the functions, and functions() gives the coupling."""
    from .smoothing import element_smoothing_part

    rk = element_cells(coords, tets, material, kernel_radius, max_neighbors, keep_points=True, name=name)
    part, _ = element_smoothing_part(np.asarray(coords, dtype=np.float64), np.asarray(tets), material,
                                     mu_field=mu_field, kappa_field=kappa_field, name=name)
    return RKPMCells(part, rk.mass, rk.points, rk.nbr_ptr, rk.nbr, rk.values)


def apply_functions(functions, d: np.ndarray) -> np.ndarray:
    """Physical field Psi d at the points (the nodes, or the refinement points with the
    nodes first) from generalized coefficients d (N x 3): row i sums psi_j(x_i) d_j over
    its neighbours; a node row without neighbours copies d_i, any other empty row is 0."""
    ptr, nbr, val = (np.asarray(a) for a in functions)
    d = np.asarray(d, dtype=np.float64)
    counts = np.diff(ptr)
    out = np.zeros((counts.size,) + d.shape[1:])
    np.add.at(out, np.repeat(np.arange(counts.size), counts), val[:, None] * d[nbr])
    empty = np.nonzero(counts[: d.shape[0]] == 0)[0]
    out[empty] = d[empty]
    return out


def _cells(entry: str, coords, tets, material, kernel_radius, max_neighbors, keep_points, mu_field, kappa_field,
           name, groups: bool = False) -> RKPMCells:
    lib = capi.load()
    X = np.ascontiguousarray(coords, dtype=np.float64)
    T = np.ascontiguousarray(tets, dtype=np.int32)
    R = np.ascontiguousarray(kernel_radius, dtype=np.float64)
    h = C.c_void_p()
    check(getattr(lib, entry)(X.shape[0], capi._ptr(X), T.shape[0], capi._ptr(T, C.c_int32), capi._ptr(R),
                              int(max_neighbors), float(material.density), C.byref(h)))
    try:
        nc, ne, npnt, nn = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(lib.am_cells_sizes(h, C.byref(nc), C.byref(ne), C.byref(npnt), C.byref(nn)))
        ptr = np.empty(nc.value + 1, dtype=np.int64)
        nodes = np.empty(ne.value, dtype=np.int32)
        grads = np.empty((ne.value, 3))
        vols = np.empty(nc.value)
        mass = np.empty(X.shape[0])
        check(lib.am_cells_get(h, capi._ptr(ptr, C.c_int64), capi._ptr(nodes, C.c_int32), capi._ptr(grads),
                               capi._ptr(vols), capi._ptr(mass)))
        cell_groups = None
        if groups:
            ng = C.c_int64()
            check(lib.am_cells_groups(h, C.byref(ng), None))
            cell_groups = np.empty(ng.value + 1, dtype=np.int64)
            check(lib.am_cells_groups(h, C.byref(ng), capi._ptr(cell_groups, C.c_int64)))
        res = RKPMCells(Part("cells", material, cell_ptr=ptr, cell_nodes=nodes, cell_grads=grads, cell_volumes=vols,
                             mu_field=mu_field, kappa_field=kappa_field, name=name, cell_groups=cell_groups), mass)
        if keep_points:
            res.points = np.empty((npnt.value, 3))
            res.nbr_ptr = np.empty(npnt.value + 1, dtype=np.int64)
            res.nbr = np.empty(nn.value, dtype=np.int32)
            res.values = np.empty(nn.value)
            check(lib.am_cells_get_points(h, capi._ptr(res.points), capi._ptr(res.nbr_ptr, C.c_int64),
                                          capi._ptr(res.nbr, C.c_int32), capi._ptr(res.values)))
        return res
    finally:
        lib.am_cells_destroy(h)
