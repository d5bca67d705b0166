"""Smoothed-cell data (the SmoothedCellData CSR, include/SmoothedCellData.h:72-659)
for strain-smoothed elements: one cell per element with the element's smoothed
gradients from the divergence theorem (QuadratureSmoothed.h:32-63 for Tet4,
:97-142 for Hex8) and the element volume as the cell volume.

This is one-time host set-up feeding the smoothed-cell force kernel.
"""
from __future__ import annotations

import numpy as np

from .model import Material, Part

_TET_FACES = np.array([[0, 1, 3], [1, 2, 3], [0, 3, 2], [0, 2, 1]])
_HEX_FACES = np.array([[0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [0, 4, 7, 3], [0, 3, 2, 1], [4, 5, 6, 7]])


def smoothed_gradients(coords: np.ndarray, conn: np.ndarray):
    """Smoothed B (E, n_en, 3) and volume (E,) of Tet4 or Hex8 elements."""
    X = coords[conn]
    E, nn, _ = X.shape
    B = np.zeros((E, nn, 3))
    vol = np.zeros(E)
    if nn == 4:
        for f in _TET_FACES:
            p0, p1, p2 = X[:, f[0]], X[:, f[1]], X[:, f[2]]
            nrm = np.cross(p1 - p0, p2 - p0) / 2.0
            vol += np.einsum("ij,ij->i", p0, nrm)
            for l in range(3):
                B[:, f[l]] += nrm / 3.0
    else:
        for f in _HEX_FACES:
            mid = X[:, f].sum(axis=1) / 4.0
            km1 = 3
            for k in range(4):
                nrm = np.cross(X[:, f[km1]] - mid, X[:, f[k]] - mid) / 2.0
                vol += np.einsum("ij,ij->i", mid, nrm)
                for l in range(4):
                    w = 5.0 / 12.0 if (l == k or l == km1) else 1.0 / 12.0
                    B[:, f[l]] += nrm * w
                km1 = k
    vol /= 3.0
    B /= vol[:, None, None]
    return B, vol


def element_smoothing_part(coords: np.ndarray, conn: np.ndarray, material: Material, mu_field=None,
                           kappa_field=None, name: str = "block_1"):
    """Part of element smoothing cells (element_smoothing_cell, subdomains 1) and its
    lumped nodal mass rho V_e / n_en (src/MassUtils.cpp:17-46)."""
    B, vol = smoothed_gradients(coords, conn)
    E, nn = conn.shape
    part = Part("cells", material, cell_ptr=np.arange(E + 1, dtype=np.int64) * nn,
                cell_nodes=conn.reshape(-1).astype(np.int32), cell_grads=B.reshape(-1, 3),
                cell_volumes=vol, mu_field=mu_field, kappa_field=kappa_field, name=name)
    mass = np.zeros(coords.shape[0])
    np.add.at(mass, conn.reshape(-1), np.repeat(vol * material.density / nn, nn))
    return part, mass


def element_smoothing_part_library(coords: np.ndarray, conn: np.ndarray, material: Material, mu_field=None,
                                   kappa_field=None, name: str = "block_1"):
    """The same cells and mass from the library's host set-up (am_smoothed_element_cells),
    the call a C++ host makes without Python."""
    import ctypes as C

    from . import capi
    from .capi import check

    lib = capi.load()
    X = np.ascontiguousarray(coords, dtype=np.float64)
    T = np.ascontiguousarray(conn, dtype=np.int32)
    h = C.c_void_p()
    check(lib.am_smoothed_element_cells(X.shape[0], capi._ptr(X), T.shape[0], T.shape[1], capi._ptr(T, C.c_int32),
                                        float(material.density), C.byref(h)))
    try:
        nc, ne = C.c_int64(), C.c_int64()
        check(lib.am_cells_sizes(h, C.byref(nc), C.byref(ne), None, None))
        ptr = np.empty(nc.value + 1, dtype=np.int64)
        nodes = np.empty(ne.value, dtype=np.int32)
        grads = np.empty((ne.value, 3))
        vols = np.empty(nc.value)
        mass = np.empty(X.shape[0])
        check(lib.am_cells_get(h, capi._ptr(ptr, C.c_int64), capi._ptr(nodes, C.c_int32), capi._ptr(grads),
                               capi._ptr(vols), capi._ptr(mass)))
    finally:
        lib.am_cells_destroy(h)
    part = Part("cells", material, cell_ptr=ptr, cell_nodes=nodes, cell_grads=grads, cell_volumes=vols,
                mu_field=mu_field, kappa_field=kappa_field, name=name)
    return part, mass
