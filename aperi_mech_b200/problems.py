"""Seeded synthetic workloads (no public dataset is involved; these arrays are the
whole workload). Sizes follow the five benchmark configurations:

  hex8_le_cube      20^3 Hex8, linear elastic E=1e9, nu=0.3, rho=1000, bottom fixed,
                    v0 ~ U[-0.01, 0.01], dt = 0.5 h_min / c, 100 steps
  tet4_nh_shear     70^3 hexes -> 6 tets each (2,058,000 tets), neo-Hookean mu=3.85e8,
                    kappa=8.33e8, rho=1000, interior jitter U[-0.2h, 0.2h]^3, bottom fixed,
                    v0_x = z + U[-0.01, 0.01] noise, dt = 0.5 min(3V/A_max)/c, 1000 steps
  hex8_nh_lognormal 64^3 (or 128^3) Hex8 neo-Hookean with lognormal per-element shear
                    (and bulk) modulus fields, sigma 0.3, bottom fixed

The density of the neo-Hookean workloads, the bottom support and the shear-profile
direction are not fixed by the configuration text; the values here are the stated
assumptions (rho = 1000, z = 0 face held, shear velocity along x growing with z).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import mesh
from .model import BoundaryCondition, Material, Part


@dataclass
class Problem:
    name: str
    coords: np.ndarray
    parts: list
    bcs: list
    v0: np.ndarray
    dt: float
    nsteps: int
    seed: int
    meta: dict = field(default_factory=dict)

    @property
    def num_elems(self) -> int:
        return sum(p.num_elems for p in self.parts)

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])


def wave_speed(lam: float, mu: float, rho: float) -> float:
    return math.sqrt((lam + 2.0 * mu) / rho)


def _initial_velocity(coords, fixed, rng, amplitude=0.01, shear=0.0):
    v = rng.uniform(-amplitude, amplitude, size=coords.shape)
    v[:, 0] += shear * coords[:, 2]
    v[fixed] = 0.0
    return v


def hex8_le_cube(n: int = 20, seed: int = 0, nsteps: int = 100) -> Problem:
    rng = np.random.default_rng(seed)
    coords, conn = mesh.box_hex(n, n, n)
    mat = Material.create("linear_elastic", 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng)
    dt = 0.5 * (1.0 / n) / wave_speed(mat.lam, mat.mu, mat.density)
    return Problem(f"hex8_le_cube_{n}", coords, [Part("hex8", mat, conn=conn)], [BoundaryCondition.fixed(fixed)],
                   v0, dt, nsteps, seed, {"config": "Hex8 2x2x2 Gauss, linear elastic"})


def tet4_nh_shear(n: int = 70, seed: int = 0, nsteps: int = 1000, jitter: float = 0.2, complete=None) -> Problem:
    """complete: property completion to use instead of the library's (Material.create)."""
    rng = np.random.default_rng(seed)
    coords, conn_hex = mesh.box_hex(n, n, n)
    h = 1.0 / n
    coords = mesh.jitter_interior(coords, jitter * h, rng)
    conn = mesh.hex_to_tets(conn_hex)
    mesh.check_orientation(coords, conn)
    mat = Material.create("neo_hookean", 1000.0, complete=complete, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng, shear=1.0)
    c = wave_speed(mat.lam, mat.mu, mat.density)
    dt = 0.5 * float(mesh.tet_char_length(coords, conn).min()) / c
    return Problem(f"tet4_nh_shear_{n}", coords, [Part("tet4", mat, conn=conn)], [BoundaryCondition.fixed(fixed)],
                   v0, dt, nsteps, seed, {"config": "Tet4 1-pt Gauss, neo-Hookean, 6-tet split, jittered"})


def hex8_nh_lognormal(n: int = 64, seed: int = 0, nsteps: int = 200, sigma: float = 0.3,
                      bulk_field: bool = False, num_sensors: int = 512) -> Problem:
    rng = np.random.default_rng(seed)
    coords, conn = mesh.box_hex(n, n, n)
    E = conn.shape[0]
    mu_e = 3.85e8 * np.exp(sigma * rng.standard_normal(E))
    kappa_e = 8.33e8 * np.exp(sigma * rng.standard_normal(E)) if bulk_field else np.full(E, 8.33e8)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng)
    lam_e = kappa_e - 2.0 / 3.0 * mu_e
    cmax = float(np.sqrt((lam_e + 2.0 * mu_e) / mat.density).max())
    dt = 0.5 * (1.0 / n) / cmax
    free = np.setdiff1d(np.arange(coords.shape[0]), fixed)
    sensors = np.sort(rng.choice(free, size=min(num_sensors, free.size), replace=False)).astype(np.int32)
    part = Part("hex8", mat, conn=conn, mu_field=mu_e, kappa_field=kappa_e)
    return Problem(f"hex8_nh_lognormal_{n}", coords, [part], [BoundaryCondition.fixed(fixed)], v0, dt, nsteps, seed,
                   {"sensors": sensors, "config": "Hex8 2x2x2 Gauss, neo-Hookean, lognormal fields"})


def _box_tets(n: int, seed: int, jitter: float, lz: float = 2.0):
    rng = np.random.default_rng(seed)
    nz = int(round(n * lz))
    coords, conn_hex = mesh.box_hex(n, n, nz, 1.0, 1.0, lz)
    coords = mesh.jitter_interior(coords, jitter / n, rng)
    tets = mesh.hex_to_tets(conn_hex)
    mesh.check_orientation(coords, tets)
    return rng, coords, tets


def smoothed_tet4_box(n: int = 46, seed: int = 0, nsteps: int = 500, jitter: float = 0.2) -> Problem:
    """Strain-smoothed Tet4 (element smoothing cells, one cell per tet) on the jittered
    1 x 1 x 2 lattice of spacing h = 1/n, neo-Hookean as tet4_nh_shear."""
    from .smoothing import element_smoothing_part

    rng, coords, tets = _box_tets(n, seed, jitter)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    part, mass = element_smoothing_part(coords, tets, mat)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng, shear=1.0)
    dt = 0.5 * float(mesh.tet_char_length(coords, tets).min()) / wave_speed(mat.lam, mat.mu, mat.density)
    return Problem(f"smoothed_tet4_box_{n}", coords, [part], [BoundaryCondition.fixed(fixed)], v0, dt, nsteps, seed,
                   {"mass": mass, "config": "strain-smoothed Tet4 element cells, neo-Hookean"})


def rkpm_box(n: int = 46, seed: int = 0, nsteps: int = 500, jitter: float = 0.2, radius: float = 1.8,
             max_neighbors: int = 40) -> Problem:
    """RKPM one-pass nodal smoothing cells on the same lattice: linear basis, cubic
    B-spline kernel of support radius `radius` x h, neighbours capped at max_neighbors
    (40 in the reference), neo-Hookean. The cell set-up runs on the GPU."""
    from .rkpm import nodal_cells

    rng, coords, tets = _box_tets(n, seed, jitter)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    R = np.full(coords.shape[0], radius / n)
    cells = nodal_cells(coords, tets, mat, R, max_neighbors=max_neighbors)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng, shear=1.0)
    dt = 0.5 * float(mesh.tet_char_length(coords, tets).min()) / wave_speed(mat.lam, mat.mu, mat.density)
    return Problem(f"rkpm_box_{n}", coords, [cells.part], [BoundaryCondition.fixed(fixed)], v0, dt, nsteps, seed,
                   {"mass": cells.mass, "tets": tets, "entries_per_cell": cells.entries_per_cell,
                    "config": f"RKPM one-pass nodal cells, R={radius}h, cap {max_neighbors}, neo-Hookean"})


def rkpm_fbar_box(n: int = 32, seed: int = 0, nsteps: int = 500, jitter: float = 0.2, radius: float = 1.8,
                  max_neighbors: int = 40) -> Problem:
    """RKPM nodal cells split into one subcell per corner hex with F-bar over each
    vertex's subcells (nodal_smoothing_cell subdomains 0 + use_f_bar, the reference's
    rkpm_fbar Taylor-bar formulation) on the jittered 1 x 1 x 2 lattice, neo-Hookean."""
    from .rkpm import nodal_subcells

    rng, coords, tets = _box_tets(n, seed, jitter)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    cells = nodal_subcells(coords, tets, mat, np.full(coords.shape[0], radius / n), max_neighbors=max_neighbors)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng, shear=1.0)
    dt = 0.5 * float(mesh.tet_char_length(coords, tets).min()) / wave_speed(mat.lam, mat.mu, mat.density)
    return Problem(f"rkpm_fbar_box_{n}", coords, [cells.part], [BoundaryCondition.fixed(fixed)], v0, dt, nsteps, seed,
                   {"mass": cells.mass, "entries_per_cell": cells.entries_per_cell,
                    "config": f"RKPM nodal subcells (corner hexes) with F-bar, R={radius}h, cap {max_neighbors}, "
                              "neo-Hookean"})


def rkpm_two_pass_box(n: int = 46, seed: int = 0, nsteps: int = 500, jitter: float = 0.2, scale: float = 1.1,
                      max_neighbors: int = 40) -> Problem:
    """RKPM element cells with the two-pass method (the reference's default for
    element_smoothing_cell): FEM smoothed tets on the physical displacement, coupled to
    the coefficients through the functions at the vertices, kernel radius scale x the
    longest edge, neo-Hookean."""
    from .rkpm import tet_max_edge_length, two_pass_element_cells

    rng, coords, tets = _box_tets(n, seed, jitter)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    cells = two_pass_element_cells(coords, tets, mat, scale * tet_max_edge_length(coords, tets),
                                   max_neighbors=max_neighbors)
    fixed = mesh.side_sets(coords)["surface_5"]
    v0 = _initial_velocity(coords, fixed, rng, shear=1.0)
    dt = 0.5 * float(mesh.tet_char_length(coords, tets).min()) / wave_speed(mat.lam, mat.mu, mat.density)
    return Problem(f"rkpm_two_pass_box_{n}", coords, [cells.part], [BoundaryCondition.fixed(fixed)], v0, dt, nsteps,
                   seed, {"mass": cells.mass, "rk": cells.functions(),
                          "config": f"RKPM two-pass element cells, scale {scale}, cap {max_neighbors}, neo-Hookean"})


def tet4_nh_shear_slab(n: int = 70, rank: int = 0, world: int = 1, seed: int = 0, nsteps: int = 1000,
                       jitter: float = 0.2) -> Problem:
    """One rank's slab of the weak-scaled tet4_nh_shear mesh: world slabs of n^3 hexes
    (6 tets each) stacked along z on a box 1 x 1 x world (h = 1/n), built locally
    without the global mesh. Interior jitter and the initial-velocity noise are drawn
    per z-plane of nodes from seed and the plane index, so the two slabs sharing an
    interface plane generate identical nodes. meta holds the interface (local ids and
    rows of the exchange buffer, one plane of (n+1)^2 rows per slab boundary) and the
    slab's own lumped mass (interface rows still to be summed over the neighbours)."""
    h = 1.0 / n
    m1 = n + 1
    coords, conn_hex = mesh.box_hex(n, n, n, 1.0, 1.0, 1.0)
    z0 = n * rank
    coords[:, 2] += rank  # global z
    kz = np.rint(coords[:, 2] * n).astype(np.int64)
    noise = np.empty_like(coords)
    for p in range(m1):
        sel = slice(p * m1 * m1, (p + 1) * m1 * m1)
        rng = np.random.default_rng([seed, z0 + p])
        jit = rng.uniform(-jitter * h, jitter * h, size=(m1 * m1, 3))
        noise[sel] = rng.uniform(-0.01, 0.01, size=(m1 * m1, 3))
        xy = coords[sel, :2]
        interior = ((xy > 1e-12) & (xy < 1.0 - 1e-12)).all(axis=1) & (z0 + p > 0) & (z0 + p < n * world)
        block = coords[sel]
        block[interior] += jit[interior]
        coords[sel] = block
    conn = mesh.hex_to_tets(conn_hex)
    mesh.check_orientation(coords, conn)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    fixed = np.nonzero(kz == 0)[0].astype(np.int32)
    v0 = noise.copy()
    v0[:, 0] += coords[:, 2]
    v0[fixed] = 0.0
    c = wave_speed(mat.lam, mat.mu, mat.density)
    dt = 0.5 * float(mesh.tet_char_length(coords, conn).min()) / c
    local, rows = [], []
    if rank > 0:
        local.append(np.arange(m1 * m1))
        rows.append((rank - 1) * m1 * m1 + np.arange(m1 * m1))
    if rank < world - 1:
        local.append(n * m1 * m1 + np.arange(m1 * m1))
        rows.append(rank * m1 * m1 + np.arange(m1 * m1))
    iface_local = np.concatenate(local).astype(np.int32) if local else np.zeros(0, np.int32)
    iface_rows = np.concatenate(rows).astype(np.int32) if rows else np.zeros(0, np.int32)
    # neighbour exchange: the bottom plane is shared with rank - 1, the top with rank + 1,
    # both listed in ascending global id (the order the neighbour lists them in too)
    neighbors = [q for q in (rank - 1, rank + 1) if 0 <= q < world]
    planes = [np.arange(m1 * m1) if q < rank else n * m1 * m1 + np.arange(m1 * m1) for q in neighbors]
    meta = {"config": f"Tet4 1-pt Gauss, neo-Hookean, slab {rank} of {world}", "iface_local": iface_local,
            "iface_rows": iface_rows, "num_iface": (world - 1) * m1 * m1,
            "slab_mass": mesh.lumped_mass(coords, conn, mat.density),
            "neighbors": np.asarray(neighbors, dtype=np.int32),
            "shared_ptr": np.arange(len(neighbors) + 1, dtype=np.int64) * m1 * m1,
            "shared_nodes": (np.concatenate(planes) if planes else np.zeros(0)).astype(np.int32)}
    return Problem(f"tet4_nh_shear_{n}_slab{rank}of{world}", coords, [Part("tet4", mat, conn=conn)],
                   [BoundaryCondition.fixed(fixed)], v0, dt, nsteps, seed, meta)


def renumbered(p: Problem, seed: int = 1) -> tuple[Problem, np.ndarray, list]:
    """The same workload with its nodes and its elements renumbered at random (seeded):
    an unstructured mesh's numbering carries no locality. Returns the problem, pn (new
    node k is old node pn[k]) and per part pe (new element k of the part is old element
    pe[k]). Gauss parts only."""
    rng = np.random.default_rng(seed)
    pn = rng.permutation(p.num_nodes)
    inv = np.empty_like(pn)
    inv[pn] = np.arange(pn.size)
    parts, pes = [], []
    for q in p.parts:
        if q.kind == "cells":
            raise ValueError("renumbered() takes Gauss parts only")
        pe = rng.permutation(q.num_elems)
        pes.append(pe)
        parts.append(Part(q.kind, q.material, conn=inv[q.conn[pe]].astype(np.int32),
                          mu_field=None if q.mu_field is None else q.mu_field[pe],
                          kappa_field=None if q.kappa_field is None else q.kappa_field[pe], name=q.name))
    bcs = [BoundaryCondition(nodes=np.sort(inv[b.nodes]).astype(np.int32), values=b.values,
                             component_mask=b.component_mask, kind=b.kind, time_function=b.time_function,
                             abscissa=b.abscissa, ordinate=b.ordinate, active_range=b.active_range) for b in p.bcs]
    meta = dict(p.meta)
    if "sensors" in meta:
        meta["sensors"] = inv[meta["sensors"]].astype(np.int32)
    meta["config"] = f"{p.meta.get('config')}, nodes and elements renumbered at random (seed {seed})"
    return (Problem(f"{p.name}_renumbered", p.coords[pn].copy(), parts, bcs, p.v0[pn].copy(), p.dt, p.nsteps, p.seed,
                    meta), pn, pes)
