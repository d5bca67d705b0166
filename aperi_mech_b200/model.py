"""Python front-end over the C ABI, shaped like aperi-mech's solver objects.

    Material        ~ aperi::Material (Materials/Base.h:174-323) built by CreateMaterial
                      (Materials/Factory.h:43): kind + density + completed Lame parameters.
    Part            ~ aperi::InternalForceContribution (include/InternalForceContribution.h:26-159):
                      one element block with its material and formulation.
    BoundaryCondition ~ aperi::BoundaryCondition (src/BoundaryCondition.cpp).
    ExplicitDynamics ~ aperi::ExplicitSolver (src/Solvers/Explicit.cpp): owns the device
                      context; Solve() / run() advance the central-difference loop on the GPU.

All compute goes through libaperi_b200.so; this module only marshals arrays.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .capi import check

MATERIAL_KINDS = {"linear_elastic": capi.AM_LINEAR_ELASTIC, "neo_hookean": capi.AM_NEO_HOOKEAN,
                  "elastic": capi.AM_ELASTIC_SVK}
PRECISIONS = {"fp64": capi.AM_FP64, "mixed": capi.AM_MIXED}
_PROPS = ("youngs_modulus", "poissons_ratio", "shear_modulus", "lambda", "bulk_modulus")


def nccl_unique_id() -> bytes:
    """ncclGetUniqueId through the library (rank 0 makes it and sends it to the others)."""
    buf = C.create_string_buffer(128)
    check(capi.load().am_nccl_unique_id(buf))
    return buf.raw


def complete_properties(**props) -> dict:
    """LinearElasticProperties::CompleteProperties (Materials/Base.h:47-158), run by the
    library's C++ host code: exactly two of youngs_modulus, poissons_ratio, shear_modulus,
    lambda, bulk_modulus -> all five; raises ValueError where the reference throws."""
    vals = (C.c_double * 5)(*[float(props[k]) if props.get(k) is not None else math.nan for k in _PROPS])
    msg = C.create_string_buffer(256)
    rc = capi.load().am_complete_properties(vals, msg, 256)
    if rc != capi.AM_OK:
        raise ValueError(msg.value.decode())
    return dict(zip(_PROPS, list(vals)))


@dataclass
class Material:
    kind: str  # linear_elastic | neo_hookean | elastic
    density: float
    lam: float
    mu: float

    @classmethod
    def create(cls, kind: str, density: float, complete=None, **props) -> "Material":
        """CreateMaterial: kind, density and two elastic constants. `complete` replaces the
        library's property completion (a callable taking the constants as keywords and
        returning all five), for callers that build problems without loading the CUDA
        library."""
        if kind not in MATERIAL_KINDS:
            raise ValueError(f"unknown material {kind!r}")
        p = (complete or complete_properties)(**props)
        return cls(kind, float(density), p["lambda"], p["shear_modulus"])

    @property
    def kappa(self) -> float:
        return self.lam + 2.0 * self.mu / 3.0


@dataclass
class Part:
    """One element block. kind: 'tet4' (1-pt Gauss), 'hex8' (2x2x2 Gauss) or 'cells'
    (strain-smoothed / RKPM cells given as a CSR of (node, gradient) entries). With
    cell_groups (offsets into the cells) the cells are subcells of F-bar cells."""
    kind: str
    material: Material
    conn: np.ndarray | None = None
    cell_ptr: np.ndarray | None = None
    cell_nodes: np.ndarray | None = None
    cell_grads: np.ndarray | None = None
    cell_volumes: np.ndarray | None = None
    mu_field: np.ndarray | None = None
    kappa_field: np.ndarray | None = None
    name: str = "block_1"
    cell_groups: np.ndarray | None = None  # F-bar: the cells above are subcells of these cells

    @property
    def num_elems(self) -> int:
        if self.kind == "cells":
            return int(len(self.cell_ptr) - 1)
        return int(self.conn.shape[0])


@dataclass
class BoundaryCondition:
    nodes: np.ndarray
    values: tuple  # (vx, vy, vz): magnitude*direction or component values
    component_mask: int = 7
    kind: str = "displacement"  # displacement | velocity
    time_function: str = "ramp_function"  # ramp_function | smooth_step_function
    abscissa: tuple = (0.0, 1.0)
    ordinate: tuple = (0.0, 1.0)
    active_range: tuple = (0.0, 1.7976931348623157e308)

    @classmethod
    def fixed(cls, nodes: np.ndarray) -> "BoundaryCondition":
        """Homogeneous displacement BC (all components held at zero)."""
        return cls(nodes=np.asarray(nodes, dtype=np.int32), values=(0.0, 0.0, 0.0))


class ExplicitDynamics:
    """Device-resident explicit-dynamics model (one am_ctx)."""

    def __init__(self, coords: np.ndarray, parts: list[Part], bcs: list[BoundaryCondition] = (),
                 body_accel=None, mass: np.ndarray | None = None, stream=None, rk=None, formulation=None):
        """rk = (nbr_ptr, nbr, values) sets the two-pass reproducing-kernel coupling
        (set_rk_functions); mass is then the generalized lumped mass. With more rows than
        nodes (two-pass nodal cells: one row per refinement point, the nodes first) the
        cells index the points (am_set_rk_points). formulation =
        ('updated', 1) or ('semi', update_interval) selects the updated or semi-Lagrangian
        formulation of the Gauss blocks (FP64 runs only); None or ('total', ...) the total one."""
        self.lib = capi.load()
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.N = int(self.coords.shape[0])
        self.parts = list(parts)
        h = C.c_void_p()
        check(self.lib.am_create(self.N, self.coords.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)))
        self.ctx = h
        self._keep = []
        try:
            if stream is not None:
                check(self.lib.am_set_stream(self.ctx, stream), self.ctx)
            if formulation is not None and formulation[0] != "total":
                code = {"updated": 1, "semi": 2}[formulation[0]]
                interval = int(formulation[1]) if len(formulation) > 1 else 1
                check(self.lib.am_set_formulation(self.ctx, code, interval), self.ctx)
            if rk is not None and len(rk[0]) - 1 > self.N:
                # functions with a row per refinement point: the cells index the points
                check(self.lib.am_set_rk_points(self.ctx, len(rk[0]) - 1), self.ctx)
            for p in self.parts:
                self._add_part(p)
            if bcs:
                self._set_bcs(list(bcs))
            if body_accel is not None:
                g = np.ascontiguousarray(body_accel, dtype=np.float64)
                check(self.lib.am_set_body_acceleration(self.ctx, g.ctypes.data_as(C.POINTER(C.c_double))), self.ctx)
            if mass is not None:
                m = np.ascontiguousarray(mass, dtype=np.float64)
                check(self.lib.am_set_mass(self.ctx, m.ctypes.data_as(C.POINTER(C.c_double))), self.ctx)
            check(self.lib.am_finalize(self.ctx), self.ctx)
            if rk is not None:
                self.set_rk_functions(*rk)
        except Exception:
            self.close()
            raise
        self._keep = []
        self.num_elems = sum(p.num_elems for p in self.parts)

    # -- set-up ------------------------------------------------------------
    def _add_part(self, p: Part) -> None:
        d = capi.BlockDesc()
        d.kind = {"tet4": capi.AM_TET4_GAUSS, "hex8": capi.AM_HEX8_GAUSS, "cells": capi.AM_SMOOTHED_CELLS}[p.kind]
        d.material = MATERIAL_KINDS[p.material.kind]
        d.lam, d.mu, d.density = p.material.lam, p.material.mu, p.material.density
        d.num_elems = p.num_elems

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        if p.kind == "cells":
            d.cell_ptr = capi._ptr(arr(p.cell_ptr, np.int64), C.c_int64)
            d.cell_nodes = capi._ptr(arr(p.cell_nodes, np.int32), C.c_int32)
            d.cell_grads = capi._ptr(arr(p.cell_grads, np.float64))
            d.cell_volumes = capi._ptr(arr(p.cell_volumes, np.float64))
        else:
            d.conn = capi._ptr(arr(p.conn, np.int32), C.c_int32)
        d.mu_field = capi._ptr(arr(p.mu_field, np.float64))
        d.kappa_field = capi._ptr(arr(p.kappa_field, np.float64))
        bid = C.c_int32()
        check(self.lib.am_add_block(self.ctx, C.byref(d), C.byref(bid)), self.ctx)
        if p.kind == "cells" and p.cell_groups is not None:
            g = arr(p.cell_groups, np.int64)
            check(self.lib.am_set_cell_groups(self.ctx, bid.value, g.size - 1, capi._ptr(g, C.c_int64)), self.ctx)

    def _set_bcs(self, bcs: list[BoundaryCondition]) -> None:
        arr_t = capi.BCDesc * len(bcs)
        descs = arr_t()
        for d, bc in zip(descs, bcs):
            nodes = np.ascontiguousarray(bc.nodes, dtype=np.int32)
            ab = np.ascontiguousarray(bc.abscissa, dtype=np.float64)
            od = np.ascontiguousarray(bc.ordinate, dtype=np.float64)
            self._keep += [nodes, ab, od]
            d.num_nodes = nodes.size
            d.nodes = capi._ptr(nodes, C.c_int32)
            d.component_mask = bc.component_mask
            d.kind = capi.AM_BC_DISPLACEMENT if bc.kind == "displacement" else capi.AM_BC_VELOCITY
            d.time_function = capi.AM_TF_RAMP if bc.time_function == "ramp_function" else capi.AM_TF_SMOOTH_STEP
            d.num_points = ab.size
            for c in range(3):
                d.values[c] = float(bc.values[c])
            d.abscissa = capi._ptr(ab)
            d.ordinate = capi._ptr(od)
            d.active_start, d.active_end = float(bc.active_range[0]), float(bc.active_range[1])
        check(self.lib.am_set_boundary_conditions(self.ctx, len(bcs), descs), self.ctx)

    def set_block_fields(self, block: int, mu_field=None, kappa_field=None) -> None:
        m = None if mu_field is None else np.ascontiguousarray(mu_field, dtype=np.float64)
        k = None if kappa_field is None else np.ascontiguousarray(kappa_field, dtype=np.float64)
        check(self.lib.am_set_block_fields(self.ctx, int(block), capi._ptr(m), capi._ptr(k)), self.ctx)

    # -- state ---------------------------------------------------------------
    def set_state(self, u=None, v=None, a=None, where: int = capi.AM_HOST) -> None:
        args = []
        for x in (u, v, a):
            if x is None:
                args.append(None)
            elif where == capi.AM_HOST:
                x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.N, 3)
                self._keep.append(x)
                args.append(x.ctypes.data)
            else:
                args.append(capi._vp(x))
        check(self.lib.am_set_state(self.ctx, where, *args), self.ctx)
        self._keep = []

    def get_state(self):
        u, v, a = (np.empty((self.N, 3)) for _ in range(3))
        check(self.lib.am_get_state(self.ctx, capi.AM_HOST, u.ctypes.data, v.ctypes.data, a.ctypes.data), self.ctx)
        return u, v, a

    def get_state_into(self, u=None, v=None, a=None, where: int = capi.AM_DEVICE) -> None:
        check(self.lib.am_get_state(self.ctx, where, capi._vp(u), capi._vp(v), capi._vp(a)), self.ctx)

    def mass(self) -> np.ndarray:
        m = np.empty(self.N)
        check(self.lib.am_get_mass(self.ctx, m.ctypes.data_as(C.POINTER(C.c_double))), self.ctx)
        return m

    # -- hot path ------------------------------------------------------------
    def internal_force(self, u, precision: str = "fp64", out=None, accumulate: bool = False) -> np.ndarray:
        if isinstance(u, np.ndarray):
            u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.N, 3)
            f = np.zeros((self.N, 3)) if out is None else out
            check(self.lib.am_internal_force(self.ctx, PRECISIONS[precision], capi.AM_HOST, u.ctypes.data,
                                             f.ctypes.data, int(accumulate)), self.ctx)
            return f
        check(self.lib.am_internal_force(self.ctx, PRECISIONS[precision], capi.AM_DEVICE, capi._vp(u),
                                         capi._vp(out), int(accumulate)), self.ctx)
        return out

    def init_acceleration(self, precision: str = "fp64") -> None:
        check(self.lib.am_init_acceleration(self.ctx, PRECISIONS[precision]), self.ctx)

    def run(self, nsteps: int, dt: float, precision: str = "fp64", t0: float = 0.0) -> None:
        check(self.lib.am_run(self.ctx, PRECISIONS[precision], int(nsteps), float(dt), float(t0)), self.ctx)

    def run_schedule(self, dts, precision: str = "fp64", t0: float = 0.0) -> None:
        d = np.ascontiguousarray(dts, dtype=np.float64)
        check(self.lib.am_run_schedule(self.ctx, PRECISIONS[precision], d.size, capi._ptr(d), float(t0)), self.ctx)

    def solve(self, dt: float, t_end: float, precision: str = "fp64", max_steps: int = 1 << 40) -> int:
        n = C.c_int64()
        check(self.lib.am_solve(self.ctx, PRECISIONS[precision], float(dt), float(t_end), int(max_steps),
                                C.byref(n)), self.ctx)
        return n.value

    def vjp_force(self, u: np.ndarray, lam: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        gu = np.empty((self.N, 3))
        gm = np.empty(self.num_elems)
        gk = np.empty(self.num_elems)
        check(self.lib.am_vjp_force(self.ctx, capi.AM_HOST, u.ctypes.data, lam.ctypes.data, gu.ctypes.data,
                                    gm.ctypes.data, gk.ctypes.data), self.ctx)
        return gu, gm, gk

    def adjoint(self, nsteps: int, dt: float, ckpt_every: int, sensors: np.ndarray):
        s = np.ascontiguousarray(sensors, dtype=np.int32)
        loss = C.c_double()
        gm = np.empty(self.num_elems)
        gk = np.empty(self.num_elems)
        check(self.lib.am_adjoint(self.ctx, int(nsteps), float(dt), int(ckpt_every), s.size, capi._ptr(s, C.c_int32),
                                  C.byref(loss), capi._ptr(gm), capi._ptr(gk)), self.ctx)
        return loss.value, gm, gk

    # -- power-method time stepper ------------------------------------------------
    def set_power_method(self, start: np.ndarray, max_edge_length: np.ndarray) -> None:
        st = np.ascontiguousarray(start, dtype=np.float64).reshape(self.N, 3)
        le = np.ascontiguousarray(max_edge_length, dtype=np.float64)
        check(self.lib.am_set_power_method(self.ctx, capi._ptr(st), capi._ptr(le)), self.ctx)

    def stable_time_increment(self, previous: float = 0.0, num_iterations: int = 50, epsilon: float = 1e-5,
                              tolerance: float = 1e-3, variation_tolerance: float = 1e-7):
        dt, its, conv = C.c_double(), C.c_int32(), C.c_int32()
        check(self.lib.am_stable_time_increment(self.ctx, float(previous), int(num_iterations), float(epsilon),
                                                float(tolerance), float(variation_tolerance), C.byref(dt),
                                                C.byref(its), C.byref(conv)), self.ctx)
        return dt.value, its.value, bool(conv.value)

    def solve_power_method(self, scale_factor: float, update_interval: int, t_end: float, precision: str = "fp64",
                           max_steps: int = 1 << 40):
        n, last = C.c_int64(), C.c_double()
        check(self.lib.am_solve_power_method(self.ctx, PRECISIONS[precision], float(scale_factor),
                                             int(update_interval), float(t_end), int(max_steps), C.byref(n),
                                             C.byref(last)), self.ctx)
        return n.value, last.value

    # -- domain decomposition -------------------------------------------------
    def set_interface(self, local_nodes: np.ndarray, rows: np.ndarray, num_global: int) -> None:
        """This rank's interface nodes and their rows of the exchange buffer
        (partition.Subdomain.iface_local / iface_ids / num_iface)."""
        ln = np.ascontiguousarray(local_nodes, dtype=np.int32)
        rw = np.ascontiguousarray(rows, dtype=np.int32)
        check(self.lib.am_set_interface(self.ctx, ln.size, capi._ptr(ln, C.c_int32), capi._ptr(rw, C.c_int32),
                                        int(num_global)), self.ctx)

    def set_neighbors(self, rank: int, neighbors: np.ndarray, shared_ptr: np.ndarray, shared_nodes: np.ndarray) -> None:
        """am_set_neighbors: neighbour exchange of the shared nodes' partial forces (the
        lists of partition.Subdomain: neighbors, shared_ptr, shared_nodes)."""
        nb = np.ascontiguousarray(neighbors, dtype=np.int32)
        sp = np.ascontiguousarray(shared_ptr, dtype=np.int64)
        sn = np.ascontiguousarray(shared_nodes, dtype=np.int32)
        check(self.lib.am_set_neighbors(self.ctx, int(rank), int(nb.size), capi._ptr(nb, C.c_int32),
                                        capi._ptr(sp, C.c_int64), capi._ptr(sn, C.c_int32)), self.ctx)

    def set_rk_functions(self, nbr_ptr: np.ndarray, nbr: np.ndarray, values: np.ndarray) -> None:
        """Two-pass reproducing-kernel coupling: the state holds generalized coefficients,
        the blocks run on the physical displacement Psi u and their forces reach the
        coefficients as Psi^T f. Row i of Psi: values[nbr_ptr[i]:nbr_ptr[i+1]] at the
        neighbours nbr[...] of point i, one row per node or, for two-pass nodal cells, per
        refinement point with the nodes first (rkpm.RKPMCells.functions())."""
        ptr = np.ascontiguousarray(nbr_ptr, dtype=np.int64)
        nb = np.ascontiguousarray(nbr, dtype=np.int32)
        val = np.ascontiguousarray(values, dtype=np.float64)
        if ptr.size < self.N + 1 or nb.size != val.size or nb.size != ptr[-1]:
            raise ValueError("nbr_ptr needs one offset per point plus one (the nodes first) and nbr/values "
                             "nbr_ptr[-1] entries")
        check(self.lib.am_set_rk_functions(self.ctx, capi._ptr(ptr, C.c_int64), capi._ptr(nb, C.c_int32),
                                           capi._ptr(val)), self.ctx)

    def set_nccl(self, unique_id: bytes, rank: int, nranks: int) -> None:
        check(self.lib.am_set_nccl(self.ctx, unique_id, int(rank), int(nranks)), self.ctx)

    # -- diagnostics -----------------------------------------------------------
    def layout(self) -> dict:
        n, k = C.c_int64(), C.c_int32()
        check(self.lib.am_get_layout(self.ctx, C.byref(n), C.byref(k)), self.ctx)
        return {"used_slots": n.value, "patched_tet4_blocks": k.value}

    def launch_count(self) -> int:
        return int(self.lib.am_launch_count(self.ctx))

    def profile(self, enable: bool) -> None:
        check(self.lib.am_profile_enable(self.ctx, int(enable)), self.ctx)

    def profile_read(self):
        ms = (C.c_double * 5)()
        n = (C.c_int64 * 5)()
        check(self.lib.am_profile_read(self.ctx, ms, n), self.ctx)
        return list(ms), list(n)

    def close(self) -> None:
        if getattr(self, "ctx", None) is not None and self.ctx.value:
            self.lib.am_destroy(self.ctx)
        self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
