"""Host-side set-up of the library (no GPU). The element processing order it applies
to Gauss blocks (am_element_order): split-hex rings are found by topology whatever the
numbering, the order depends on the mesh alone (a renumbered mesh gets the same
elements in the same order), and meshes without rings fall back to a Morton order of
the centroids that keeps elements sharing nodes close together. The finite-element
element smoothing cells (am_smoothed_element_cells) against the numpy set-up and the
oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from aperi_mech_b200 import mesh


def element_order(coords, conn, try_rings=True):
    from aperi_mech_b200 import capi

    lib = capi.load()
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    order = np.empty(conn.shape[0], dtype=np.int32)
    rings = C.c_int32(-1)
    rc = lib.am_element_order(coords.shape[0], coords.ctypes.data_as(C.POINTER(C.c_double)), conn.shape[0],
                              conn.shape[1], conn.ctypes.data_as(C.POINTER(C.c_int32)), int(try_rings),
                              order.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(rings))
    assert rc == 0, lib.am_last_error(None)
    return order, rings.value


def permuted(coords, conn, seed):
    """The same mesh with its nodes and elements renumbered at random."""
    rng = np.random.default_rng(seed)
    pn = rng.permutation(coords.shape[0])  # new node k is old node pn[k]
    inv = np.empty_like(pn)
    inv[pn] = np.arange(pn.size)
    pe = rng.permutation(conn.shape[0])    # new element k is old element pe[k]
    return coords[pn], inv[conn[pe]].astype(np.int32), pn, pe


@pytest.fixture(scope="module")
def tet_mesh():
    rng = np.random.default_rng(3)
    coords, hexes = mesh.box_hex(6, 5, 4)
    coords = mesh.jitter_interior(coords, 0.2 / 6, rng)
    return coords, mesh.hex_to_tets(hexes), hexes


def test_split_hex_rings_found_and_canonical(capi_lib, tet_mesh):
    coords, tets, _ = tet_mesh
    order, rings = element_order(coords, tets)
    assert rings == 1
    assert np.array_equal(np.sort(order), np.arange(tets.shape[0]))
    t = tets[order].reshape(-1, 6, 4)
    # each ring: six tets on one axis (first and last node), chained b_k = a_{k+1}
    assert np.all(t[:, :, 0] == t[:, :1, 0]) and np.all(t[:, :, 3] == t[:, :1, 3])
    assert np.array_equal(t[:, :, 2], np.roll(t[:, :, 1], -1, axis=1))
    # a ring is one hex's split: its eight nodes are the hex's
    hex_of = np.arange(tets.shape[0]) // 6
    for r in range(t.shape[0]):
        h = hex_of[order[6 * r]]
        assert set(t[r].ravel()) == set(tet_mesh[2][h])


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
def test_order_independent_of_numbering(capi_lib, tet_mesh, kind):
    coords, tets, hexes = tet_mesh
    conn = tets if kind == "tet4" else hexes
    base, r0 = element_order(coords, conn)
    for seed in (1, 2):
        c2, conn2, pn, pe = permuted(coords, conn, seed)
        order2, r2 = element_order(c2, conn2)
        assert r2 == r0
        # the k-th element run is the same element of the mesh in both numberings
        assert np.array_equal(pe[order2], base)


def test_generic_order_keeps_neighbours_close(capi_lib, tet_mesh):
    coords, tets, _ = tet_mesh
    c2, t2, pn, pe = permuted(coords, tets, 5)
    order, rings = element_order(c2, t2, try_rings=False)
    assert rings == 0
    cen = c2[t2[order]].mean(axis=1)
    step = np.linalg.norm(np.diff(cen, axis=0), axis=1).mean()
    rand = np.linalg.norm(np.diff(c2[t2].mean(axis=1), axis=0), axis=1).mean()
    assert step < 0.25 * rand


def test_rings_rejected_when_the_split_is_broken(capi_lib, tet_mesh):
    coords, tets, _ = tet_mesh
    t = tets.copy()
    t[0] = t[0][[1, 2, 0, 3]]  # an even permutation: same tet, no longer on its hex's ring
    _, rings = element_order(coords, t)
    assert rings == 0


def test_element_order_rejects_bad_input(capi_lib):
    coords = np.zeros((4, 3))
    bad = np.array([[0, 1, 2, 9]], dtype=np.int32)
    from aperi_mech_b200 import capi

    lib = capi.load()
    order = np.empty(1, dtype=np.int32)
    rc = lib.am_element_order(4, coords.ctypes.data_as(C.POINTER(C.c_double)), 1, 4,
                              bad.ctypes.data_as(C.POINTER(C.c_int32)), 1, order.ctypes.data_as(C.POINTER(C.c_int32)),
                              None)
    assert rc == capi.AM_EINVAL


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
def test_smoothed_element_cells_from_the_library(capi_lib, tet_mesh, kind):
    """am_smoothed_element_cells (host C++ set-up of finite-element element smoothing
    cells) against the numpy set-up and the oracle's smoothed quadrature."""
    from aperi_mech_b200 import smoothing
    from aperi_mech_b200.model import Material
    from oracle import oracle

    coords, tets, hexes = tet_mesh
    conn = tets if kind == "tet4" else hexes
    mat = Material("neo_hookean", 1000.0, 5.8e8, 3.85e8)
    want, mass_w = smoothing.element_smoothing_part(coords, conn, mat)
    got, mass_g = smoothing.element_smoothing_part_library(coords, conn, mat)
    assert np.array_equal(got.cell_ptr, want.cell_ptr) and np.array_equal(got.cell_nodes, want.cell_nodes)
    scale = np.abs(want.cell_grads).max()
    assert np.abs(got.cell_grads - want.cell_grads).max() < 1e-13 * scale
    assert np.abs(got.cell_volumes - want.cell_volumes).max() < 1e-14 * want.cell_volumes.max()
    assert np.abs(mass_g - mass_w).max() < 1e-13 * mass_w.max()
    for e in (0, conn.shape[0] // 2, conn.shape[0] - 1):
        B, w = oracle.smoothed_bw(kind, coords[conn[e]])
        nn = conn.shape[1]
        assert np.abs(got.cell_grads[nn * e: nn * (e + 1)] - B.reshape(nn, 3)).max() < 1e-12 * scale
        assert abs(got.cell_volumes[e] - float(w)) < 1e-14
