"""Element-partitioned domain decomposition of one mesh over ranks.

Each rank owns a slab of elements (or smoothing cells) and every node they touch.
Nodes touched by more than one rank are interface nodes: every rank holding one
sums its own elements' partial force there, the partial forces are summed across
ranks (the reference's ParallelSum of the force field after the element loop,
src/Solvers/Explicit.cpp:190-193), and then every holder applies the same nodal
update to the same state, so the copies stay identical without a second exchange.

The exchange buffer has one FP64 x 3 row per interface node of the whole mesh
(global interface index = rank of the node among all interface nodes in global
order); a rank writes only its own rows, the buffer is summed across ranks, and
each rank reads its rows back. The lumped mass is the global one (sliced), so the
interface nodes see the mass of all their elements.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import mesh as _mesh
from .model import BoundaryCondition, Part


@dataclass
class Subdomain:
    rank: int
    world: int
    global_nodes: np.ndarray  # local -> global node id (ascending)
    coords: np.ndarray
    parts: list
    bcs: list
    v0: np.ndarray
    mass: np.ndarray
    iface_local: np.ndarray   # local ids of this rank's interface nodes
    iface_ids: np.ndarray     # their global interface index
    num_iface: int            # interface nodes of the whole mesh
    owned: np.ndarray         # per local node: this rank is the lowest rank holding it
    elements: list = field(default_factory=list)  # per part: global element (cell) ids held here
    # Neighbour exchange: the ranks sharing interface nodes with this one (ascending) and,
    # per neighbour, the local ids of the shared nodes in ascending global id, the order
    # both sides of the pair agree on.
    neighbors: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    shared_ptr: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int64))
    shared_nodes: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def num_elems(self) -> int:
        return sum(p.num_elems for p in self.parts)


def _element_nodes(p: Part):
    """Per element (cell) of a part: its node list, as (flat nodes, offsets)."""
    if p.kind == "cells":
        return np.asarray(p.cell_nodes, dtype=np.int64), np.asarray(p.cell_ptr, dtype=np.int64)
    conn = np.asarray(p.conn, dtype=np.int64)
    return conn.ravel(), np.arange(0, conn.size + 1, conn.shape[1], dtype=np.int64)


def _element_ranks(coords, p: Part, world: int, axis: int, lo: float, hi: float) -> np.ndarray:
    flat, off = _element_nodes(p)
    counts = np.diff(off)
    centroid = np.add.reduceat(coords[flat, axis], off[:-1]) / np.maximum(counts, 1) if flat.size else np.zeros(0)
    r = np.floor((centroid - lo) / max(hi - lo, 1e-300) * world).astype(np.int64)
    return np.clip(r, 0, world - 1)


def _sub_part(p: Part, sel: np.ndarray, g2l: np.ndarray) -> Part:
    mu = None if p.mu_field is None else np.ascontiguousarray(p.mu_field[sel])
    ka = None if p.kappa_field is None else np.ascontiguousarray(p.kappa_field[sel])
    if p.kind == "cells":
        ptr = np.asarray(p.cell_ptr, dtype=np.int64)
        lens = ptr[sel + 1] - ptr[sel]
        new_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        idx = np.concatenate([np.arange(ptr[c], ptr[c + 1]) for c in sel]) if sel.size else np.zeros(0, np.int64)
        grads = np.asarray(p.cell_grads).reshape(-1, 3)
        return Part("cells", p.material, cell_ptr=new_ptr, cell_nodes=g2l[np.asarray(p.cell_nodes)[idx]].astype(np.int32),
                    cell_grads=np.ascontiguousarray(grads[idx]), cell_volumes=np.ascontiguousarray(p.cell_volumes[sel]),
                    mu_field=mu, kappa_field=ka, name=p.name)
    return Part(p.kind, p.material, conn=g2l[np.asarray(p.conn)[sel]].astype(np.int32), mu_field=mu, kappa_field=ka,
                name=p.name)


def decompose(coords: np.ndarray, parts: list, bcs: list, v0: np.ndarray, world: int, mass: np.ndarray | None = None,
              axis: int | None = None) -> list:
    """Slabs of elements along `axis` (default: the longest extent), by element
    centroid; returns one Subdomain per rank. `mass` is the global lumped mass (needed
    when a part is made of cells; computed from the Gauss parts otherwise)."""
    coords = np.asarray(coords, dtype=np.float64)
    N = coords.shape[0]
    if world < 1:
        raise ValueError("world must be >= 1")
    if any(getattr(p, "cell_groups", None) is not None for p in parts):
        raise ValueError("F-bar cells are not decomposed (a cell's subcells must stay on one rank)")
    if mass is None:
        if any(p.kind == "cells" for p in parts):
            raise ValueError("cell parts need the global lumped mass")
        mass = np.zeros(N)
        for p in parts:
            mass += _mesh.lumped_mass(coords, np.asarray(p.conn), p.material.density)
    lo_c, hi_c = coords.min(axis=0), coords.max(axis=0)
    if axis is None:
        axis = int(np.argmax(hi_c - lo_c))
    ranks = [_element_ranks(coords, p, world, axis, lo_c[axis], hi_c[axis]) for p in parts]
    # Which ranks touch each node.
    touch = np.zeros((world, N), dtype=bool)
    for p, r in zip(parts, ranks):
        flat, off = _element_nodes(p)
        touch[np.repeat(r, np.diff(off)), flat] = True
    holders = touch.sum(axis=0)
    iface_global = np.nonzero(holders > 1)[0]
    iface_index = np.full(N, -1, dtype=np.int64)
    iface_index[iface_global] = np.arange(iface_global.size)
    owner = np.argmax(touch, axis=0)  # lowest rank holding the node
    subs = []
    for k in range(world):
        gnodes = np.nonzero(touch[k])[0]
        g2l = np.full(N, -1, dtype=np.int64)
        g2l[gnodes] = np.arange(gnodes.size)
        sub_parts, elems = [], []
        for p, r in zip(parts, ranks):
            sel = np.nonzero(r == k)[0]
            elems.append(sel)
            if sel.size:
                sub_parts.append(_sub_part(p, sel, g2l))
        sub_bcs = []
        for bc in bcs:
            loc = g2l[np.asarray(bc.nodes, dtype=np.int64)]
            sub_bcs.append(BoundaryCondition(nodes=loc[loc >= 0].astype(np.int32), values=bc.values,
                                             component_mask=bc.component_mask, kind=bc.kind,
                                             time_function=bc.time_function, abscissa=bc.abscissa,
                                             ordinate=bc.ordinate, active_range=bc.active_range))
        il = np.nonzero(iface_index[gnodes] >= 0)[0]
        nbrs, ptr, shared = [], [0], []
        for q in range(world):
            if q == k:
                continue
            common = np.nonzero(touch[k] & touch[q])[0]  # ascending global ids
            if common.size:
                nbrs.append(q)
                shared.append(g2l[common])
                ptr.append(ptr[-1] + common.size)
        subs.append(Subdomain(k, world, gnodes, np.ascontiguousarray(coords[gnodes]), sub_parts, sub_bcs,
                              np.ascontiguousarray(np.asarray(v0)[gnodes]), np.ascontiguousarray(mass[gnodes]),
                              il.astype(np.int32), iface_index[gnodes[il]].astype(np.int32), int(iface_global.size),
                              owner[gnodes] == k, elems, np.asarray(nbrs, dtype=np.int32),
                              np.asarray(ptr, dtype=np.int64),
                              np.concatenate(shared).astype(np.int32) if shared else np.zeros(0, np.int32)))
    return subs


def neighbor_sum(sub: Subdomain, own: np.ndarray, received: list) -> np.ndarray:
    """The interface nodes' summed force after a neighbour exchange, as every holder
    forms it: own is this rank's partial force (local nodes x 3), received[j] the partial
    forces neighbour j sent for the nodes it shares with this rank (in the shared order).
    Each interface node sums its holders' partials in ascending rank order (this rank's
    own partial at its place), so all holders of a node get the same bits. Returns the
    local array with the interface rows replaced."""
    out = np.array(own, dtype=np.float64, copy=True)
    parts = {}  # local node -> [(rank, partial)]
    for i in sub.iface_local:
        parts[int(i)] = [(sub.rank, own[i])]
    for j, q in enumerate(sub.neighbors):
        nodes = sub.shared_nodes[sub.shared_ptr[j]:sub.shared_ptr[j + 1]]
        for t, i in enumerate(nodes):
            parts[int(i)].append((int(q), received[j][t]))
    for i, lst in parts.items():
        lst.sort(key=lambda x: x[0])
        acc = np.zeros(3)
        for _, v in lst:
            acc = acc + v
        out[i] = acc
    return out


def assemble(subs: list, arrays: list, num_nodes: int) -> np.ndarray:
    """Global nodal array from per-rank local arrays (each node from its owner)."""
    out = np.zeros((num_nodes,) + np.asarray(arrays[0]).shape[1:])
    for s, a in zip(subs, arrays):
        out[s.global_nodes[s.owned]] = np.asarray(a)[s.owned]
    return out
