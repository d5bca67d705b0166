"""Structured mesh generation for the synthetic workloads.

Stands in for STK's generated meshes ("NXxNYxNZ|sideset:xXyYzZ|tets",
src/IoMesh.cpp:145-156), whose hex->tet split is not available here:
  - hexes use aperi-mech's Hex8 node order (ShapeFunctionsFunctorHex8.h:17-33),
  - the tet split is the conforming 6-tet split about each hex's 0->6 diagonal,
  - side sets surface_1..6 are the x-, x+, y-, y+, z-, z+ faces.
Nodes and elements are numbered lexicographically (x fastest), which already
gives the gather kernels spatial locality on these boxes.
"""
from __future__ import annotations

import math

import numpy as np

# Six tets around the 0->6 diagonal of a Hex8; every face diagonal passes
# through the face's lowest or highest corner, so neighbouring hexes conform.
TET6_OF_HEX = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]],
                       dtype=np.int64)


def box_hex(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0):
    """Coordinates (N,3) and Hex8 connectivity (E,8) of an nx x ny x nz brick."""
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))  # x fastest

    def nid(a, b, c):
        return a + (nx + 1) * (b + (ny + 1) * c)

    conn = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                     nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)],
                    axis=1).astype(np.int32)
    return coords, conn


def hex_to_tets(conn_hex: np.ndarray) -> np.ndarray:
    """(E,8) Hex8 -> (6E,4) Tet4, the six tets of each hex consecutive."""
    return conn_hex[:, TET6_OF_HEX].reshape(-1, 4).astype(np.int32)


def side_sets(coords: np.ndarray, tol: float = 1e-12) -> dict[str, np.ndarray]:
    lo = coords.min(axis=0)
    hi = coords.max(axis=0)
    sets = {}
    for d in range(3):
        sets[f"surface_{2 * d + 1}"] = np.nonzero(np.abs(coords[:, d] - lo[d]) < tol)[0].astype(np.int32)
        sets[f"surface_{2 * d + 2}"] = np.nonzero(np.abs(coords[:, d] - hi[d]) < tol)[0].astype(np.int32)
    return sets


def boundary_mask(coords: np.ndarray, tol: float = 1e-12) -> np.ndarray:
    lo = coords.min(axis=0)
    hi = coords.max(axis=0)
    return np.any((np.abs(coords - lo) < tol) | (np.abs(coords - hi) < tol), axis=1)


def jitter_interior(coords: np.ndarray, amplitude: float, rng: np.random.Generator) -> np.ndarray:
    """Uniform [-amplitude, amplitude]^3 perturbation of the interior nodes."""
    out = coords.copy()
    interior = ~boundary_mask(coords)
    out[interior] += rng.uniform(-amplitude, amplitude, size=(int(interior.sum()), 3))
    return out


def tet_volumes(coords: np.ndarray, conn: np.ndarray) -> np.ndarray:
    x = coords[conn]
    d = x[:, 1:, :] - x[:, :1, :]
    return np.einsum("ij,ij->i", d[:, 0], np.cross(d[:, 1], d[:, 2])) / 6.0


def tet_char_length(coords: np.ndarray, conn: np.ndarray) -> np.ndarray:
    """3 V / A_max per tet (the stable-time-step length of a linear tet)."""
    x = coords[conn]
    faces = [(1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2)]
    amax = np.zeros(conn.shape[0])
    for a, b, c in faces:
        area = 0.5 * np.linalg.norm(np.cross(x[:, b] - x[:, a], x[:, c] - x[:, a]), axis=1)
        amax = np.maximum(amax, area)
    return 3.0 * np.abs(tet_volumes(coords, conn)) / amax


def check_orientation(coords: np.ndarray, conn: np.ndarray) -> None:
    if conn.shape[1] == 4:
        v = tet_volumes(coords, conn)
        if np.any(v <= 0):
            raise ValueError(f"{int((v <= 0).sum())} tets with non-positive volume")


def hex8_volumes(coords: np.ndarray, conn: np.ndarray) -> np.ndarray:
    """sum over the 2x2x2 Gauss points of det J (ElementHexahedron8.h:107-117)."""
    s = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=float)
    x = coords[conn]  # E x 8 x 3
    vol = np.zeros(conn.shape[0])
    for g in s / math.sqrt(3.0):
        dN = np.stack([s[:, 0] * (1 + s[:, 1] * g[1]) * (1 + s[:, 2] * g[2]),
                       s[:, 1] * (1 + s[:, 0] * g[0]) * (1 + s[:, 2] * g[2]),
                       s[:, 2] * (1 + s[:, 0] * g[0]) * (1 + s[:, 1] * g[1])], axis=1) / 8.0
        vol += np.linalg.det(np.einsum("eai,aj->eij", x, dN))
    return vol


def lumped_mass(coords: np.ndarray, conn: np.ndarray, density: float) -> np.ndarray:
    """Lumped nodal mass rho V_e / n_en summed over the elements (src/MassUtils.cpp:17-46),
    on the host: for Gauss parts that share a model with cell parts (whose mass comes
    from their own set-up) and for the global mass of a decomposed mesh."""
    m = np.zeros(coords.shape[0])
    x = coords[conn]
    if conn.shape[1] == 4:
        vol = np.abs(np.einsum("ij,ij->i", x[:, 1] - x[:, 0], np.cross(x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]))) / 6.0
    else:
        vol = hex8_volumes(coords, conn)
    np.add.at(m, conn.ravel(), np.repeat(density * vol / conn.shape[1], conn.shape[1]))
    return m


def max_edge_length(coords: np.ndarray, conns) -> np.ndarray:
    """MaxEdgeLengthFunctor (src/MaxEdgeLengthProcessor.cpp:36-60) with every node active:
    per node, the longest distance to any node of an element it belongs to (for a hex
    this includes the face and body diagonals). conns: one connectivity array or a list."""
    if isinstance(conns, np.ndarray):
        conns = [conns]
    out = np.zeros(coords.shape[0])
    for conn in conns:
        conn = np.asarray(conn)
        x = coords[conn]
        for a in range(conn.shape[1]):
            d = np.linalg.norm(x - x[:, a:a + 1], axis=2).max(axis=1)
            np.maximum.at(out, conn[:, a], d)
    return out
