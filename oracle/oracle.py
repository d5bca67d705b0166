"""ctypes binding of the CPU FP64 oracle (oracle/am_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py as the parity checker. The product
(aperi_mech_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libamoracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)

KIND = {"tet4": 0, "hex8": 1, "cells": 2}
MATERIAL = {"linear_elastic": 0, "neo_hookean": 1, "elastic": 2}


class OBlock(C.Structure):
    _fields_ = [("kind", C.c_int32), ("material", C.c_int32), ("lam", C.c_double), ("mu", C.c_double),
                ("density", C.c_double), ("mu_field", _dp), ("kappa_field", _dp), ("num_elems", C.c_int64),
                ("conn", _ip), ("cell_ptr", _lp), ("cell_nodes", _ip), ("cell_grads", _dp), ("cell_volumes", _dp),
                ("num_groups", C.c_int64), ("group_ptr", _lp)]


class OLagrangian(C.Structure):
    _fields_ = [("formulation", C.c_int32), ("update_interval", C.c_int32), ("n", C.c_int64), ("x", _dp),
                ("inc", _dp), ("H", _dp), ("Href", _dp)]


FORMULATION = {"total": 0, "updated": 1, "semi": 2}


class LagrangianState:
    """Updated / semi-Lagrangian state of the oracle: coordinates x (current or reference),
    displacement increment, element H and reference H, completed steps."""

    def __init__(self, coords, num_elems, formulation, update_interval=1):
        self.x = np.array(coords, dtype=np.float64, order="C", copy=True)
        self.inc = np.zeros_like(self.x)
        self.H = np.zeros((num_elems, 9))
        self.Href = np.zeros((num_elems, 9))
        self.s = OLagrangian(FORMULATION[formulation], int(update_interval), 0, _p(self.x), _p(self.inc), _p(self.H),
                             _p(self.Href))

    @property
    def n(self) -> int:
        return int(self.s.n)


class OBC(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("nodes", _ip), ("component_mask", C.c_int32), ("kind", C.c_int32),
                ("time_function", C.c_int32), ("num_points", C.c_int32), ("values", C.c_double * 3),
                ("abscissa", _dp), ("ordinate", _dp), ("active_start", C.c_double), ("active_end", C.c_double)]


class OProblem(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("coords", _dp), ("num_blocks", C.c_int32), ("blocks", C.POINTER(OBlock)),
                ("num_bcs", C.c_int32), ("bcs", C.POINTER(OBC)), ("mass", _dp), ("body_accel", C.c_double * 3),
                ("rk_ptr", _lp), ("rk_nbr", _ip), ("rk_values", _dp), ("rk_rows", C.c_int64)]


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.ob_tet4_gauss_bw.argtypes = [_dp, _dp, _dp]
        L.ob_hex8_gauss_bw.argtypes = [_dp, C.c_int, _dp, _dp]
        L.ob_tet4_smoothed_bw.argtypes = [_dp, _dp, _dp]
        L.ob_hex8_smoothed_bw.argtypes = [_dp, _dp, _dp]
        L.ob_complete_properties.argtypes = [_dp, C.c_char_p, C.c_int]
        L.ob_stress.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int64, _dp, _dp]
        L.ob_internal_force.argtypes = [C.POINTER(OProblem), _dp, _dp]
        L.ob_element_volumes.argtypes = [C.POINTER(OProblem), C.c_int32, _dp]
        L.ob_lumped_mass.argtypes = [C.POINTER(OProblem), _dp]
        L.ob_direct_time_schedule.argtypes = [C.c_double, C.c_double, C.c_int64, _dp]
        L.ob_direct_time_schedule.restype = C.c_int64
        L.ob_explicit_solve.argtypes = [C.POINTER(OProblem), C.c_double, C.c_double, C.c_int64, _dp, _dp, _dp, _lp]
        L.ob_init_acceleration.argtypes = [C.POINTER(OProblem), _dp, _dp]
        L.ob_explicit_steps.argtypes = [C.POINTER(OProblem), C.c_int64, _dp, C.c_double, _dp, _dp, _dp]
        L.ob_vjp_force.argtypes = [C.POINTER(OProblem), _dp, _dp, _dp, _dp, _dp]
        L.ob_adjoint.argtypes = [C.POINTER(OProblem), C.c_int64, C.c_double, _dp, _dp, C.c_int32, _ip, _dp, _dp, _dp]
        L.ob_rk_kernel.argtypes = [_dp, C.c_double]
        L.ob_rk_kernel.restype = C.c_double
        L.ob_rk_function_values.argtypes = [C.c_int64, _dp, _dp, _dp, _lp, _ip, _dp]
        L.ob_rkpm_nodal_cells.argtypes = [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, _lp, _lp, _lp,
                                          _dp, _lp, _ip, _dp, _lp, _ip, _dp, _dp, _dp]
        L.ob_rkpm_nodal_cells_two_pass.argtypes = [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, _lp,
                                                   _lp, _lp, _dp, _lp, _ip, _dp, _lp, _ip, _dp, _dp, _dp]
        L.ob_rkpm_element_cells.argtypes = [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, _lp, _lp,
                                            _lp, _ip, _dp, _lp, _ip, _dp, _dp, _dp]
        L.ob_rkpm_nodal_subcells.argtypes = [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, _lp, _lp,
                                             _ip, _dp, _dp, _lp]
        L.ob_lagrangian_force.argtypes = [C.POINTER(OProblem), C.POINTER(OLagrangian), _dp]
        L.ob_lagrangian_init.argtypes = [C.POINTER(OProblem), C.POINTER(OLagrangian), _dp]
        L.ob_lagrangian_steps.argtypes = [C.POINTER(OProblem), C.POINTER(OLagrangian), C.c_int64, _dp, C.c_double, _dp,
                                          _dp, _dp]
        L.ob_rkpm_hex8_element_cells.argtypes = [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, _lp,
                                                 _lp, _lp, _ip, _dp, _lp, _ip, _dp, _dp, _dp]
        L.ob_stable_time_increment.argtypes = [C.POINTER(OProblem), _dp, _dp, _dp, C.c_double, C.c_int32, C.c_double,
                                               C.c_double, C.c_double, _ip, _ip]
        L.ob_stable_time_increment.restype = C.c_double
        L.ob_set_threads.argtypes = [C.c_int]
        L.ob_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class OracleProblem:
    """Holds the ctypes view of a problem (coords, parts, BCs) and its buffers."""

    def __init__(self, coords, parts, bcs=(), mass=None, body_accel=(0.0, 0.0, 0.0), rk=None):
        """rk = (nbr_ptr, nbr, values): the two-pass reproducing-kernel functions at the
        nodes (row i: psi_j(x_i) for the neighbours j of node i), or None."""
        self.keep = []
        self.coords = self._arr(coords, np.float64)
        self.N = self.coords.shape[0]
        blocks = (OBlock * len(parts))()
        for b, p in zip(blocks, parts):
            b.kind = KIND[p.kind]
            b.material = MATERIAL[p.material.kind]
            b.lam, b.mu, b.density = p.material.lam, p.material.mu, p.material.density
            b.num_elems = p.num_elems
            b.mu_field = _p(self._arr(p.mu_field, np.float64))
            b.kappa_field = _p(self._arr(p.kappa_field, np.float64))
            if p.kind == "cells":
                b.cell_ptr = _p(self._arr(p.cell_ptr, np.int64), C.c_int64)
                b.cell_nodes = _p(self._arr(p.cell_nodes, np.int32), C.c_int32)
                b.cell_grads = _p(self._arr(p.cell_grads, np.float64))
                b.cell_volumes = _p(self._arr(p.cell_volumes, np.float64))
                if getattr(p, "cell_groups", None) is not None:
                    g = self._arr(p.cell_groups, np.int64)
                    b.num_groups = g.size - 1
                    b.group_ptr = _p(g, C.c_int64)
            else:
                b.conn = _p(self._arr(p.conn, np.int32), C.c_int32)
        obcs = (OBC * max(1, len(bcs)))()
        for o, bc in zip(obcs, bcs):
            nodes = self._arr(bc.nodes, np.int32)
            ab = self._arr(bc.abscissa, np.float64)
            od = self._arr(bc.ordinate, np.float64)
            o.num_nodes = nodes.size
            o.nodes = _p(nodes, C.c_int32)
            o.component_mask = bc.component_mask
            o.kind = 0 if bc.kind == "displacement" else 1
            o.time_function = 0 if bc.time_function == "ramp_function" else 1
            o.num_points = ab.size
            for c in range(3):
                o.values[c] = float(bc.values[c])
            o.abscissa, o.ordinate = _p(ab), _p(od)
            o.active_start, o.active_end = float(bc.active_range[0]), float(bc.active_range[1])
        self.blocks, self.obcs = blocks, obcs
        self.mass = self._arr(mass, np.float64)
        self.num_elems = sum(p.num_elems for p in parts)
        self.s = OProblem(self.N, _p(self.coords), len(parts), blocks, len(bcs), obcs, _p(self.mass),
                          (C.c_double * 3)(*body_accel))
        if rk is not None:
            ptr, nbr, val = (self._arr(a, t) for a, t in zip(rk, (np.int64, np.int32, np.float64)))
            assert ptr.size >= self.N + 1 and nbr.size == val.size == ptr[-1]
            self.s.rk_ptr, self.s.rk_nbr, self.s.rk_values = _p(ptr, C.c_int64), _p(nbr, C.c_int32), _p(val)
            self.s.rk_rows = ptr.size - 1

    def _arr(self, a, dt):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dt)
        self.keep.append(a)
        return a

    @classmethod
    def from_problem(cls, prob, mass=None):
        return cls(prob.coords, prob.parts, prob.bcs, mass=mass)

    def internal_force(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        f = np.empty((self.N, 3))
        lib().ob_internal_force(C.byref(self.s), _p(u), _p(f))
        return f

    def lumped_mass(self):
        m = np.empty(self.N)
        lib().ob_lumped_mass(C.byref(self.s), _p(m))
        return m

    def element_volumes(self, block=0):
        v = np.empty(self.s.blocks[block].num_elems)
        lib().ob_element_volumes(C.byref(self.s), block, _p(v))
        return v

    def init_acceleration(self, u):
        a = np.empty((self.N, 3))
        lib().ob_init_acceleration(C.byref(self.s), _p(np.ascontiguousarray(u, dtype=np.float64)), _p(a))
        return a

    def steps(self, u, v, a, dts, t0=0.0):
        u, v, a = (np.array(x, dtype=np.float64, order="C", copy=True) for x in (u, v, a))
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        lib().ob_explicit_steps(C.byref(self.s), dts.size, _p(dts), t0, _p(u), _p(v), _p(a))
        return u, v, a

    def solve(self, u, v, dt, t_end, max_steps=1 << 40):
        u, v = (np.array(x, dtype=np.float64, order="C", copy=True) for x in (u, v))
        a = np.zeros_like(u)
        n = C.c_int64()
        lib().ob_explicit_solve(C.byref(self.s), dt, t_end, max_steps, _p(u), _p(v), _p(a), C.byref(n))
        return u, v, a, n.value

    def stable_time_increment(self, u, v, max_edge_length, previous=0.0, num_iterations=50, epsilon=1e-5,
                              tolerance=1e-3, variation_tolerance=1e-7):
        """Returns (dt, iterations, converged); v (the eigenvector estimate) is updated in place."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert v.flags.c_contiguous and v.dtype == np.float64
        le = np.ascontiguousarray(max_edge_length, dtype=np.float64)
        its, conv = C.c_int32(), C.c_int32()
        dt = lib().ob_stable_time_increment(C.byref(self.s), _p(u), _p(v), _p(le), previous, num_iterations, epsilon,
                                            tolerance, variation_tolerance, C.byref(its), C.byref(conv))
        return dt, its.value, bool(conv.value)

    def lagrangian_state(self, formulation, update_interval=1):
        return LagrangianState(self.coords, self.num_elems, formulation, update_interval)

    def lagrangian_force(self, state):
        f = np.empty((self.N, 3))
        assert lib().ob_lagrangian_force(C.byref(self.s), C.byref(state.s), _p(f)) == 0
        return f

    def lagrangian_init(self, state):
        a = np.empty((self.N, 3))
        assert lib().ob_lagrangian_init(C.byref(self.s), C.byref(state.s), _p(a)) == 0
        return a

    def lagrangian_steps(self, state, u, v, a, dts, t0=0.0):
        u, v, a = (np.array(x, dtype=np.float64, order="C", copy=True) for x in (u, v, a))
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        assert lib().ob_lagrangian_steps(C.byref(self.s), C.byref(state.s), dts.size, _p(dts), t0, _p(u), _p(v),
                                         _p(a)) == 0
        return u, v, a

    def vjp_force(self, u, lam):
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        gu = np.empty((self.N, 3))
        gm = np.empty(self.num_elems)
        gk = np.empty(self.num_elems)
        lib().ob_vjp_force(C.byref(self.s), _p(u), _p(lam), _p(gu), _p(gm), _p(gk))
        return gu, gm, gk

    def adjoint(self, nsteps, dt, u0, v0, sensors):
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        v0 = np.ascontiguousarray(v0, dtype=np.float64)
        s = np.ascontiguousarray(sensors, dtype=np.int32)
        loss = C.c_double()
        gm = np.empty(self.num_elems)
        gk = np.empty(self.num_elems)
        lib().ob_adjoint(C.byref(self.s), nsteps, dt, _p(u0), _p(v0), s.size, _p(s, C.c_int32), C.byref(loss),
                         _p(gm), _p(gk))
        return loss.value, gm, gk


def direct_time_schedule(dt, t_end, max_steps=1 << 40):
    n = lib().ob_direct_time_schedule(dt, t_end, max_steps, None)
    d = np.empty(n)
    lib().ob_direct_time_schedule(dt, t_end, max_steps, _p(d))
    return d


def stress(material: str, lam: float, mu: float, H):
    H = np.ascontiguousarray(H, dtype=np.float64).reshape(-1, 9)
    P = np.empty_like(H)
    lib().ob_stress(MATERIAL[material], lam, mu, H.shape[0], _p(H), _p(P))
    return P.reshape(-1, 3, 3)


def complete_properties(**props):
    keys = ("youngs_modulus", "poissons_ratio", "shear_modulus", "lambda", "bulk_modulus")
    v = np.array([float(props[k]) if props.get(k) is not None else np.nan for k in keys])
    msg = C.create_string_buffer(256)
    rc = lib().ob_complete_properties(_p(v), msg, 256)
    if rc != 0:
        raise ValueError(msg.value.decode())
    return dict(zip(keys, v))


def gauss_bw(kind: str, X, gp: int = 0):
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = 8 if kind == "hex8" else 4
    B = np.empty((n, 3))
    w = C.c_double()
    if kind == "hex8":
        lib().ob_hex8_gauss_bw(_p(X), gp, _p(B), C.byref(w))
    else:
        lib().ob_tet4_gauss_bw(_p(X), _p(B), C.byref(w))
    return B, w.value


def smoothed_bw(kind: str, X):
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = 8 if kind == "hex8" else 4
    B = np.empty((n, 3))
    w = C.c_double()
    (lib().ob_hex8_smoothed_bw if kind == "hex8" else lib().ob_tet4_smoothed_bw)(_p(X), _p(B), C.byref(w))
    return B, w.value


def rkpm_nodal_cells(coords, tets, kernel_radius, max_neighbors=40, density=1000.0, two_pass=False):
    """Oracle RKPM nodal cells: dict with points, nbr_ptr, nbr, values, cell_ptr, cell_nodes,
    cell_grads, cell_volumes, mass. two_pass: the cells hold the corner-hex points with
    their own smoothed gradients (the entries index the points)."""
    X = np.ascontiguousarray(coords, dtype=np.float64)
    T = np.ascontiguousarray(tets, dtype=np.int32)
    R = np.ascontiguousarray(kernel_radius, dtype=np.float64)
    P, S, K = C.c_int64(), C.c_int64(), C.c_int64()
    args = (X.shape[0], _p(X), T.shape[0], _p(T, C.c_int32), _p(R), int(max_neighbors), float(density))
    fn = lib().ob_rkpm_nodal_cells_two_pass if two_pass else lib().ob_rkpm_nodal_cells
    fn(*args, C.byref(P), C.byref(S), C.byref(K), *([None] * 9))
    N = X.shape[0]
    out = {"points": np.empty((P.value, 3)), "nbr_ptr": np.empty(P.value + 1, dtype=np.int64),
           "nbr": np.empty(S.value, dtype=np.int32), "values": np.empty(S.value),
           "cell_ptr": np.empty(N + 1, dtype=np.int64), "cell_nodes": np.empty(K.value, dtype=np.int32),
           "cell_grads": np.empty((K.value, 3)), "cell_volumes": np.empty(N), "mass": np.empty(N)}
    fn(*args, None, None, None, _p(out["points"]), _p(out["nbr_ptr"], C.c_int64), _p(out["nbr"], C.c_int32),
       _p(out["values"]), _p(out["cell_ptr"], C.c_int64), _p(out["cell_nodes"], C.c_int32), _p(out["cell_grads"]),
       _p(out["cell_volumes"]), _p(out["mass"]))
    return out


def rkpm_element_cells(coords, tets, kernel_radius, max_neighbors=40, density=1000.0):
    """Oracle RKPM element cells (Tet4 or Hex8 elements, from the connectivity's width):
    dict with nbr_ptr, nbr, values (at the vertices), cell_ptr, cell_nodes, cell_grads,
    cell_volumes, mass."""
    X = np.ascontiguousarray(coords, dtype=np.float64)
    T = np.ascontiguousarray(tets, dtype=np.int32)
    R = np.ascontiguousarray(kernel_radius, dtype=np.float64)
    fn = lib().ob_rkpm_hex8_element_cells if T.shape[1] == 8 else lib().ob_rkpm_element_cells
    S, K = C.c_int64(), C.c_int64()
    args = (X.shape[0], _p(X), T.shape[0], _p(T, C.c_int32), _p(R), int(max_neighbors), float(density))
    fn(*args, C.byref(S), C.byref(K), *([None] * 8))
    N, E = X.shape[0], T.shape[0]
    out = {"nbr_ptr": np.empty(N + 1, dtype=np.int64), "nbr": np.empty(S.value, dtype=np.int32),
           "values": np.empty(S.value), "cell_ptr": np.empty(E + 1, dtype=np.int64),
           "cell_nodes": np.empty(K.value, dtype=np.int32), "cell_grads": np.empty((K.value, 3)),
           "cell_volumes": np.empty(E), "mass": np.empty(N)}
    fn(*args, None, None, _p(out["nbr_ptr"], C.c_int64), _p(out["nbr"], C.c_int32),
                                _p(out["values"]), _p(out["cell_ptr"], C.c_int64), _p(out["cell_nodes"], C.c_int32),
                                _p(out["cell_grads"]), _p(out["cell_volumes"]), _p(out["mass"]))
    return out


def rkpm_nodal_subcells(coords, tets, kernel_radius, max_neighbors=40, density=1000.0):
    """Oracle RKPM nodal cells split into corner-hex subcells: dict with cell_ptr,
    cell_nodes, cell_grads, cell_volumes (per subcell) and group_ptr (per vertex)."""
    X = np.ascontiguousarray(coords, dtype=np.float64)
    T = np.ascontiguousarray(tets, dtype=np.int32)
    R = np.ascontiguousarray(kernel_radius, dtype=np.float64)
    K = C.c_int64()
    args = (X.shape[0], _p(X), T.shape[0], _p(T, C.c_int32), _p(R), int(max_neighbors), float(density))
    lib().ob_rkpm_nodal_subcells(*args, C.byref(K), *([None] * 5))
    S = 4 * T.shape[0]
    out = {"cell_ptr": np.empty(S + 1, dtype=np.int64), "cell_nodes": np.empty(K.value, dtype=np.int32),
           "cell_grads": np.empty((K.value, 3)), "cell_volumes": np.empty(S),
           "group_ptr": np.empty(X.shape[0] + 1, dtype=np.int64)}
    lib().ob_rkpm_nodal_subcells(*args, None, _p(out["cell_ptr"], C.c_int64), _p(out["cell_nodes"], C.c_int32),
                                 _p(out["cell_grads"]), _p(out["cell_volumes"]), _p(out["group_ptr"], C.c_int64))
    return out


def set_threads(n: int) -> None:
    lib().ob_set_threads(n)


def get_threads() -> int:
    return lib().ob_get_threads()
