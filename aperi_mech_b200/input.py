"""aperi-mech YAML input for the explicit-dynamics hot path.

Reads the reference's input schema (include/AperiInputSchema/AperiInputSchema.h, consumed in
the reference by include/IoInputFile.h and the factories it feeds) for the part of it this
library computes, and builds an ExplicitDynamics model on the GPU:

    procedures:
      - explicit_dynamics_procedure:
          geometry:
            mesh: generated:NxMxK[|sideset:xXyYzZ][|tets][|bbox:x0,y0,z0,x1,y1,z1]  or  <mesh>.npz
            parts:
              - part:
                  set: block_1
                  formulation:                      (InternalForceContributionParameters.h:58-246)
                    integration_scheme:
                      gauss_quadrature: {integration_order: 1}
                      | strain_smoothing: {element_smoothing_cell | nodal_smoothing_cell: {subdomains: 1 | 0},
                                           force_one_pass_method | force_two_pass_method: true,
                                           use_f_bar: true}
                    approximation_space:
                      finite_element: ~ | reproducing_kernel: {kernel_radius_scale_factor: s}
                  material:                         (Materials/Factory.h:19-160)
                    linear_elastic | neo_hookean | elastic: {density, two elastic constants}
          initial_conditions: [- velocity: {sets, components: {X, Y, Z} | vector: {magnitude, direction}}]
          loads: [- gravity_load: {sets, components | vector}]
          time_stepper: {direct_time_stepper: {time_increment, time_end}
                         | power_method_time_stepper: {scale_factor, update_interval, time_end}}
          boundary_conditions:                      (src/BoundaryCondition.cpp:197-220)
            - displacement | velocity: {sets, components | vector,
                                        time_function: {ramp_function | smooth_step_function:
                                                        {abscissa_values, ordinate_values}},
                                        active_time_range: {time_start, time_end}}
          output: {file, time_start, time_end, time_increment}
                                                    (fields at the output times, as an .npz of frames)
          lagrangian_formulation: {total: ~ | updated: ~ | semi: {update_interval: k}}
                                                    (IoInputFile.h:188-262; Gauss parts and Tet4
                                                    finite-element element cells, FP64)
          x_b200: {precision: fp64 | mixed, seed, jitter, velocity_noise, max_steps,
                   fields: {<part set>: {shear_modulus | bulk_modulus: {lognormal_sigma}}}}

Keys this build adds live under `x_b200`. Generated meshes follow STK's "generated:" form:
unit-size hexes on [0,N]x[0,M]x[0,K] (or the bbox), nodes numbered x fastest, block "block_1",
side sets named surface_1, surface_2, ... in the order their letters appear (x = min-x face,
X = max-x face, ...), and "|tets" splits each hex into six tets (this library's conforming
split; STK's own split is not available here). An .npz mesh holds `coords` (N x 3),
`block_<name>` (E x 4 or E x 8, zero-based) and `set_<name>` (zero-based node ids).
Element cells with the reproducing_kernel space use the two-pass method unless
force_one_pass_method is set, nodal cells the one-pass method unless force_two_pass_method is
set (the reference's defaults and switches).
Nodal cells with subdomains 0 split into one subcell per corner hex, and use_f_bar then
applies F-bar over each vertex's subcells; with one subcell per cell (subdomains 1, or
element cells) use_f_bar changes nothing, as in the reference. Anything else (Exodus
meshes, two-pass nodal cells split into subcells, other materials) raises InputError naming the key.
"""
from __future__ import annotations

import json
import math
import re
import sys
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import yaml

from . import mesh as _mesh
from .model import BoundaryCondition, ExplicitDynamics, Material, Part

_AXES = {"X": 0, "Y": 1, "Z": 2}
_FACES = {"x": (0, 0), "X": (0, 1), "y": (1, 0), "Y": (1, 1), "z": (2, 0), "Z": (2, 1)}


class InputError(ValueError):
    """An input the reference would reject, or one outside this library's path."""


@dataclass
class Simulation:
    """Everything the explicit solve needs, as arrays (the GPU model is built from it)."""
    name: str
    coords: np.ndarray
    parts: list
    bcs: list
    v0: np.ndarray
    dt: float
    time_end: float
    precision: str = "fp64"
    body_accel: np.ndarray | None = None
    mass: np.ndarray | None = None
    max_steps: int = 1 << 40
    sets: dict = field(default_factory=dict)
    meta: dict = field(default_factory=dict)
    power_method: tuple | None = None  # (scale_factor, update_interval) of power_method_time_stepper
    rk: tuple | None = None  # (nbr_ptr, nbr, values): two-pass reproducing-kernel coupling
    output: tuple | None = None  # (file, time_start, time_end, time_increment) of the output block
    formulation: tuple = ("total", 1)  # lagrangian_formulation and the semi update_interval

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def num_elems(self) -> int:
        return sum(p.num_elems for p in self.parts)

    def model(self, stream=None) -> ExplicitDynamics:
        return ExplicitDynamics(self.coords, self.parts, self.bcs, body_accel=self.body_accel, mass=self.mass,
                                stream=stream, rk=self.rk, formulation=self.formulation)

    def problem(self):
        """The same inputs as a problems.Problem (for the oracle and the benchmark)."""
        from .problems import Problem

        if self.power_method is not None:
            raise InputError("the power-method time stepper has no precomputed step list")
        nsteps = len(direct_time_steps(self.dt, self.time_end))
        meta = dict(self.meta)
        if self.mass is not None:
            meta["mass"] = self.mass
        if self.body_accel is not None:
            meta["body_accel"] = self.body_accel
        if self.rk is not None:
            meta["rk"] = self.rk
        if self.formulation[0] != "total":
            meta["formulation"] = self.formulation
        return Problem(self.name, self.coords, self.parts, self.bcs, self.v0, self.dt, nsteps,
                       int(self.meta.get("seed", 0)), meta)


class TimeIncrementScheduler:
    """TimeIncrementScheduler (include/Scheduler.h:51-89): an event at time_start, then every
    time_increment, while the next event point does not pass time_end; a call that finds
    the event point reached (within 1e-15) moves it past the given time."""

    def __init__(self, time_start: float, time_end: float, time_increment: float):
        self.time_end = float(time_end)
        self.increment = float(time_increment)
        self.next_event = float(time_start)

    def at_next_event(self, time: float) -> bool:
        at_event = time + 1.0e-15 >= self.next_event
        if at_event:
            self.next_event += self.increment
            self.at_next_event(time)
            if self.next_event > self.time_end:
                self.next_event = sys.float_info.max
        return at_event


def output_steps(dts, output) -> list:
    """Step counts (0 = the initial state) after which ExplicitSolver::Solve writes output
    (src/Solvers/Explicit.cpp:375,472): the scheduler asked at time 0, then after each step
    with the accumulated time."""
    _, t0, t1, inc = output
    sched = TimeIncrementScheduler(t0, t1, inc)
    out = [0] if sched.at_next_event(0.0) else []
    time = 0.0
    for n, d in enumerate(dts, start=1):
        time += d
        if sched.at_next_event(time):
            out.append(n)
    return out


def direct_time_steps(dt: float, time_end: float, max_steps: int = 1 << 40) -> list:
    """Step sizes of DirectTimeStepper::GetTimeIncrement (include/TimeStepper.h:97-128) under
    the `while (!AtEnd(time)) { ...; time += dt; }` loop of ExplicitSolver::Solve: dt while
    time + dt <= t_end, then the remainder. Floating-point accumulation can leave a tiny
    remainder and hence one extra short step, exactly as in the reference (am_solve follows
    the same rule in C++)."""
    out, t = [], 0.0
    while not (t >= time_end) and len(out) < max_steps:
        h = dt if t + dt <= time_end else (0.0 if t > time_end else time_end - t)
        out.append(h)
        t += h
    return out


# ---------------------------------------------------------------------------
# meshes
def generated_mesh(spec: str, rng=None, jitter: float = 0.0):
    """STK-style generated box: returns (coords, {block: conn}, {set: node ids})."""
    body = spec[len("generated:"):] if spec.startswith("generated:") else spec
    tokens = body.split("|")
    m = re.fullmatch(r"\s*(\d+)x(\d+)x(\d+)\s*", tokens[0])
    if not m:
        raise InputError(f"generated mesh {spec!r}: expected NxMxK")
    n = [int(v) for v in m.groups()]
    lo, hi = np.zeros(3), np.array(n, dtype=float)
    tets, faces = False, ""
    for tok in tokens[1:]:
        key, _, val = tok.partition(":")
        key = key.strip()
        if key == "tets":
            tets = True
        elif key == "sideset":
            faces = val.strip()
        elif key == "bbox":
            b = [float(v) for v in val.split(",")]
            if len(b) != 6:
                raise InputError(f"bbox needs six values: {tok!r}")
            lo, hi = np.array(b[:3]), np.array(b[3:])
        else:
            raise InputError(f"generated mesh option {key!r} is not supported")
    coords, conn = _mesh.box_hex(n[0], n[1], n[2], *(hi - lo))
    coords = coords + lo
    sets = {}
    for k, ch in enumerate(faces):
        if ch not in _FACES:
            raise InputError(f"side set letter {ch!r} (expected one of xXyYzZ)")
        d, side = _FACES[ch]
        target = hi[d] if side else lo[d]
        tol = 1e-9 * max(1.0, float(np.abs(hi - lo).max()))
        sets[f"surface_{k + 1}"] = np.nonzero(np.abs(coords[:, d] - target) < tol)[0].astype(np.int32)
    if jitter > 0.0:
        h = float(((hi - lo) / np.array(n)).min())
        coords = _mesh.jitter_interior(coords, jitter * h, rng if rng is not None else np.random.default_rng(0))
    blocks = {"block_1": _mesh.hex_to_tets(conn) if tets else conn}
    return coords, blocks, sets


def npz_mesh(path: Path):
    d = np.load(path)
    if "coords" not in d:
        raise InputError(f"{path}: no 'coords' array")
    coords = np.ascontiguousarray(d["coords"], dtype=np.float64)
    blocks = {k[len("block_"):]: np.ascontiguousarray(d[k], dtype=np.int32) for k in d.files if k.startswith("block_")}
    sets = {k[len("set_"):]: np.ascontiguousarray(d[k], dtype=np.int32) for k in d.files if k.startswith("set_")}
    if not blocks:
        raise InputError(f"{path}: no 'block_<name>' arrays")
    return coords, blocks, sets


# ---------------------------------------------------------------------------
# the procedure
def _one_key(node, what: str):
    if not isinstance(node, dict) or len(node) != 1:
        raise InputError(f"{what}: expected a map with exactly one key, got {node!r}")
    return next(iter(node.items()))


def _components(node: dict, what: str):
    """GetComponentsAndValues (include/IoInputFile.h:280-304): `vector` (magnitude times the
    normalised direction, all three components) or `components` (the listed X, Y, Z)."""
    if "vector" in node:
        vec = node["vector"]
        d = np.asarray(vec["direction"], dtype=float)
        n = float(np.linalg.norm(d))
        if d.shape != (3,) or n == 0.0:
            raise InputError(f"{what}: vector direction must be three numbers, not all zero")
        vals = float(vec["magnitude"]) * d / n
        return vals, 7
    if "components" in node:
        vals, mask = np.zeros(3), 0
        for k, v in node["components"].items():
            if k not in _AXES:
                raise InputError(f"{what}: component {k!r} (expected X, Y or Z)")
            vals[_AXES[k]] = float(v)
            mask |= 1 << _AXES[k]
        return vals, mask
    raise InputError(f"{what}: needs a 'vector' or 'components' node")


def _set_nodes(names, sets: dict, what: str) -> np.ndarray:
    if isinstance(names, str):
        names = [names]
    ids = []
    for s in names:
        if s not in sets:
            raise InputError(f"{what}: unknown set {s!r} (known: {sorted(sets)})")
        ids.append(sets[s])
    return np.unique(np.concatenate(ids)).astype(np.int32) if ids else np.zeros(0, np.int32)


def _material(node: dict) -> Material:
    kind, props = _one_key(node, "material")
    if kind not in ("linear_elastic", "neo_hookean", "elastic"):
        raise InputError(f"material {kind!r} is not on this path (linear_elastic, neo_hookean, elastic)")
    props = dict(props or {})
    if "density" not in props:
        raise InputError(f"material {kind}: density is required")
    density = float(props.pop("density"))
    try:
        return Material.create(kind, density, **{k: float(v) for k, v in props.items()})
    except ValueError as e:
        raise InputError(f"material {kind}: {e}") from None


def _lagrangian_formulation(proc: dict) -> tuple:
    """lagrangian_formulation (IoInputFile.h:195-252): ("total", 1),
    ("updated", 1) or ("semi", update_interval)."""
    lnode = proc.get("lagrangian_formulation")
    if lnode is None:
        return ("total", 1)
    if not isinstance(lnode, dict):
        raise InputError("'lagrangian_formulation' must be a map")
    if "total" in lnode:
        return ("total", 1)
    if "updated" in lnode:
        return ("updated", 1)
    if "semi" in lnode:
        k = (lnode.get("semi") or {}).get("update_interval")
        if k is None:
            raise InputError("lagrangian_formulation.semi needs update_interval")
        if int(k) < 1:
            raise InputError("lagrangian_formulation.semi.update_interval must be at least 1")
        return ("semi", int(k))
    raise InputError("lagrangian_formulation must have 'total', 'updated', or 'semi' key")


def _part(pnode: dict, blocks: dict, coords, ext: dict, rng, formulation=("total", 1)):
    """One InternalForceContribution: block connectivity + formulation + material.
    Returns (part, lumped mass or None, two-pass functions or None)."""
    name = pnode.get("set")
    if name not in blocks:
        raise InputError(f"part set {name!r} is not a block of the mesh (blocks: {sorted(blocks)})")
    conn = blocks[name]
    mat = _material(pnode.get("material", {}))
    form = pnode.get("formulation", {}) or {}
    scheme, snode = _one_key(form.get("integration_scheme", {"gauss_quadrature": {"integration_order": 1}}),
                             "integration_scheme")
    space, spnode = _one_key(form.get("approximation_space", {"finite_element": None}), "approximation_space")
    fields = (ext.get("fields") or {}).get(name, {})
    mu_f = kappa_f = None
    E = conn.shape[0]
    if fields:
        for key in fields:
            if key not in ("shear_modulus", "bulk_modulus"):
                raise InputError(f"x_b200.fields.{name}: {key!r} (shear_modulus or bulk_modulus)")
        if "shear_modulus" in fields:
            mu_f = mat.mu * np.exp(float(fields["shear_modulus"]["lognormal_sigma"]) * rng.standard_normal(E))
        if "bulk_modulus" in fields:
            kappa_f = mat.kappa * np.exp(float(fields["bulk_modulus"]["lognormal_sigma"]) * rng.standard_normal(E))
    if scheme == "gauss_quadrature":
        if space != "finite_element":
            raise InputError("gauss_quadrature needs approximation_space: finite_element")
        order = int((snode or {}).get("integration_order", 1))
        if order != 1:
            raise InputError(f"gauss_quadrature integration_order {order}: only 1 is defined")
        kind = {4: "tet4", 8: "hex8"}.get(conn.shape[1])
        if kind is None:
            raise InputError(f"block {name}: {conn.shape[1]}-node elements (Tet4 or Hex8 only)")
        return Part(kind, mat, conn=conn, mu_field=mu_f, kappa_field=kappa_f, name=name), None, None
    if scheme != "strain_smoothing":
        raise InputError(f"integration_scheme {scheme!r} (gauss_quadrature or strain_smoothing)")
    snode = snode or {}
    use_f_bar = bool(snode.get("use_f_bar", False))
    # IntegrationSchemeStrainSmoothingParameters (InternalForceContributionParameters.h:164-194):
    # one-pass by default, two-pass for element cells, either forced by a key.
    force_one, force_two = bool(snode.get("force_one_pass_method")), bool(snode.get("force_two_pass_method"))
    if force_one and force_two:
        raise InputError("Cannot force both one pass and two pass methods")
    one_pass = force_one or (not force_two and "element_smoothing_cell" not in snode)
    cell = "nodal_smoothing_cell" if "nodal_smoothing_cell" in snode else "element_smoothing_cell"
    sub = int(((snode.get(cell) or {}).get("subdomains", 1)))
    # MeshLabelerProcessor.h:832-870: element cells always hold one subcell (other values
    # only warn); nodal cells split into one subcell per element for subdomains < 1 and
    # refuse more than one.
    if cell == "nodal_smoothing_cell" and sub > 1:
        raise InputError(f"nodal_smoothing_cell.subdomains = {sub}: num_subcells > 1 is not implemented")
    if cell == "element_smoothing_cell":
        sub = 1
    # include/Element.h:32-86: Hex8 blocks take strain smoothing only with the
    # reproducing-kernel space; nodal cells are built here from a tet mesh's thex refinement.
    if conn.shape[1] not in (4, 8):
        raise InputError(f"block {name}: {conn.shape[1]}-node elements (Tet4 or Hex8 only)")
    if conn.shape[1] == 8 and space == "finite_element":
        raise InputError("Strain Smoothing is not supported for finite elements and Hexahedron8")
    if conn.shape[1] == 8 and cell == "nodal_smoothing_cell":
        raise InputError(f"nodal_smoothing_cell on the Hex8 block {name}: nodal cells are built from the tet mesh "
                         "(its thex refinement is formed here)")
    if space == "finite_element" and cell == "element_smoothing_cell" and formulation[0] != "total":
        # Updated / semi (ElementSmoothedTetrahedron4.h:73-122, ComputeInternalForceSmoothedCell.h:
        # 326-350): the cell gradients and volume are rebuilt on the reference configuration of
        # each update, H composes with the stored reference gradient and the force maps back by
        # F_ref / det F_ref, as for a Gauss element. A Tet4 cell's divergence-theorem gradients
        # are the tet's exact constant gradients and its volume the tet's, so the cell is the
        # one-point Gauss tet in every configuration and runs as one.
        part = Part("tet4", mat, conn=conn, mu_field=mu_f, kappa_field=kappa_f, name=name)
        return part, None, None
    if formulation[0] != "total":
        raise InputError(f"{formulation[0]} Lagrangian formulation: built for Gauss parts and Tet4 "
                         "finite-element element cells only")
    if space == "finite_element" and cell == "element_smoothing_cell":
        from .smoothing import element_smoothing_part

        part, mass = element_smoothing_part(coords, conn, mat, mu_field=mu_f, kappa_field=kappa_f)
        part.name = name
        return part, mass, None
    if space == "reproducing_kernel" and cell == "nodal_smoothing_cell":
        if mu_f is not None or kappa_f is not None:
            raise InputError("x_b200.fields on RKPM nodal cells: per-cell fields are not supported")
        from .rkpm import nodal_cells, nodal_subcells, thex_max_edge_length, two_pass_nodal_cells

        scale = float((spnode or {}).get("kernel_radius_scale_factor", 1.0))
        radius = scale * thex_max_edge_length(coords, conn)
        if not one_pass:
            # force_two_pass_method: the vertex cells hold their corner-hex points, coupled to
            # the vertices by the functions at every point of the thex refinement.
            if sub < 1:
                raise InputError("force_two_pass_method with nodal_smoothing_cell.subdomains 0: not built "
                                 "(two-pass nodal cells integrate whole vertex cells)")
            cells = two_pass_nodal_cells(coords, conn, mat, radius, max_neighbors=int(ext.get("max_neighbors", 40)),
                                         name=name)
            return cells.part, cells.mass, cells.functions()
        if sub < 1:
            cells = nodal_subcells(coords, conn, mat, radius, max_neighbors=int(ext.get("max_neighbors", 40)),
                                   fbar=use_f_bar)
        else:
            cells = nodal_cells(coords, conn, mat, radius, max_neighbors=int(ext.get("max_neighbors", 40)))
        cells.part.name = name
        return cells.part, cells.mass, None
    if space == "reproducing_kernel" and cell == "element_smoothing_cell" and not one_pass:
        from .rkpm import tet_max_edge_length, two_pass_element_cells

        scale = float((spnode or {}).get("kernel_radius_scale_factor", 1.0))
        cells = two_pass_element_cells(coords, conn, mat, scale * tet_max_edge_length(coords, conn),
                                       max_neighbors=int(ext.get("max_neighbors", 40)), mu_field=mu_f,
                                       kappa_field=kappa_f, name=name)
        return cells.part, cells.mass, cells.functions()
    if space == "reproducing_kernel" and cell == "element_smoothing_cell":
        if mu_f is not None or kappa_f is not None:
            raise InputError("x_b200.fields on RKPM element cells: per-cell fields are not supported")
        from .rkpm import element_cells, tet_max_edge_length

        scale = float((spnode or {}).get("kernel_radius_scale_factor", 1.0))
        cells = element_cells(coords, conn, mat, scale * tet_max_edge_length(coords, conn),
                              max_neighbors=int(ext.get("max_neighbors", 40)))
        cells.part.name = name
        return cells.part, cells.mass, None
    raise InputError(f"{space} with {cell}: not built")


def load(source, base_dir: Path | None = None) -> Simulation:
    """Parse an input (a YAML path, YAML text, or the parsed dict) into a Simulation."""
    if isinstance(source, dict):
        doc = source
    else:
        text = str(source)
        p = Path(text)
        if "\n" not in text and p.suffix in (".yaml", ".yml") and p.exists():
            base_dir = base_dir or p.parent
            text = p.read_text()
        doc = yaml.safe_load(text)
    base_dir = base_dir or Path.cwd()
    procs = doc.get("procedures") if isinstance(doc, dict) else None
    if not procs or not isinstance(procs, list):
        raise InputError("input needs a 'procedures' sequence")
    if len(procs) != 1:
        raise InputError(f"{len(procs)} procedures: one explicit_dynamics_procedure is supported")
    kind, proc = _one_key(procs[0], "procedure")
    if kind != "explicit_dynamics_procedure":
        raise InputError(f"procedure {kind!r} (explicit_dynamics_procedure only)")
    ext = proc.get("x_b200", {}) or {}
    seed = int(ext.get("seed", 0))
    rng = np.random.default_rng(seed)

    geo = proc.get("geometry") or {}
    mesh_spec = geo.get("mesh")
    if not isinstance(mesh_spec, str):
        raise InputError("geometry.mesh is required")
    if mesh_spec.startswith("generated:"):
        coords, blocks, sets = generated_mesh(mesh_spec, rng, float(ext.get("jitter", 0.0)))
    elif mesh_spec.endswith(".npz"):
        coords, blocks, sets = npz_mesh((base_dir / mesh_spec) if not Path(mesh_spec).is_absolute() else Path(mesh_spec))
    else:
        raise InputError(f"mesh {mesh_spec!r}: Exodus files are outside this library (use generated: or .npz)")
    sets = dict(sets)
    for b, conn in blocks.items():
        sets.setdefault(b, np.unique(conn).astype(np.int32))

    formulation = _lagrangian_formulation(proc)
    parts, masses, rk = [], [], None
    for entry in geo.get("parts") or []:
        _, pnode = _one_key(entry, "parts entry")
        part, mass, functions = _part(pnode, blocks, coords, ext, rng, formulation)
        parts.append(part)
        masses.append(mass)
        if functions is not None:
            if rk is not None:
                raise InputError("two-pass reproducing-kernel coupling on more than one part is not built")
            rk = functions
    if not parts:
        raise InputError("geometry.parts is empty")
    if rk is not None and len(parts) > 1:
        raise InputError("two-pass reproducing-kernel parts beside other parts are not built")
    mass = None
    if any(m is not None for m in masses):
        mass = np.zeros(coords.shape[0])
        for part, m in zip(parts, masses):
            mass += m if m is not None else _mesh.lumped_mass(coords, part.conn, part.material.density)

    v0 = np.zeros_like(coords)
    for entry in proc.get("initial_conditions") or []:
        kind, node = _one_key(entry, "initial_conditions entry")
        if kind != "velocity":
            raise InputError(f"initial condition {kind!r} (velocity only)")
        vals, mask = _components(node, "initial velocity")
        ids = _set_nodes(node.get("sets", []), sets, "initial velocity")
        for d in range(3):
            if mask >> d & 1:
                v0[ids, d] = vals[d]
    noise = float(ext.get("velocity_noise", 0.0))
    if noise > 0.0:
        v0 += rng.uniform(-noise, noise, size=v0.shape)

    body = None
    for entry in proc.get("loads") or []:
        kind, node = _one_key(entry, "loads entry")
        if kind != "gravity_load":
            raise InputError(f"load {kind!r} (gravity_load only)")
        ids = _set_nodes(node.get("sets", []), sets, "gravity_load")
        if ids.size != coords.shape[0]:
            raise InputError("gravity_load on part of the mesh: only whole-mesh gravity is built")
        if "time_function" in node:
            raise InputError("gravity_load time_function: only constant gravity is built")
        vals, _ = _components(node, "gravity_load")
        body = vals if body is None else body + vals

    bcs = []
    for entry in proc.get("boundary_conditions") or []:
        kind, node = _one_key(entry, "boundary_conditions entry")
        if kind not in ("displacement", "velocity"):
            raise InputError(f"boundary condition {kind!r} (displacement or velocity)")
        vals, mask = _components(node, f"{kind} boundary condition")
        ids = _set_nodes(node.get("sets", []), sets, f"{kind} boundary condition")
        tf_kind, tf = _one_key(node.get("time_function", {"ramp_function": {"abscissa_values": [0.0, 1.0],
                                                                             "ordinate_values": [1.0, 1.0]}}),
                               "time_function")
        if tf_kind not in ("ramp_function", "smooth_step_function"):
            raise InputError(f"time_function {tf_kind!r}")
        atr = node.get("active_time_range") or {}
        bcs.append(BoundaryCondition(nodes=ids, values=tuple(float(v) for v in vals), component_mask=mask,
                                     kind=kind, time_function=tf_kind,
                                     abscissa=tuple(float(v) for v in tf["abscissa_values"]),
                                     ordinate=tuple(float(v) for v in tf["ordinate_values"]),
                                     active_range=(float(atr.get("time_start", 0.0)),
                                                   float(atr.get("time_end", 1.7976931348623157e308)))))

    ts_kind, ts = _one_key(proc.get("time_stepper") or {}, "time_stepper")
    power = None
    if ts_kind == "direct_time_stepper":
        dt, t_end = float(ts["time_increment"]), float(ts["time_end"])
        if not (dt > 0.0 and t_end >= 0.0):
            raise InputError("direct_time_stepper needs time_increment > 0 and time_end >= 0")
    elif ts_kind == "power_method_time_stepper":
        dt, t_end = 0.0, float(ts["time_end"])
        power = (float(ts["scale_factor"]), int(ts["update_interval"]))
        if not (power[0] > 0.0 and power[1] >= 1 and t_end >= 0.0):
            raise InputError("power_method_time_stepper needs scale_factor > 0, update_interval >= 1, time_end >= 0")
    else:
        raise InputError(f"time_stepper {ts_kind!r} (direct_time_stepper or power_method_time_stepper)")
    precision = str(ext.get("precision", "fp64"))
    if precision not in ("fp64", "mixed"):
        raise InputError(f"x_b200.precision {precision!r} (fp64 or mixed)")
    name = Path(str(source)).stem if isinstance(source, (str, Path)) and "\n" not in str(source) else "input"
    element_blocks = [blocks[(e.get("part") or {}).get("set")] for e in (geo.get("parts") or [])]
    if formulation[0] != "total":
        if precision != "fp64":
            raise InputError(f"{formulation[0]} Lagrangian formulation runs in FP64 (x_b200.precision: fp64)")
        if power is not None:
            raise InputError(f"{formulation[0]} Lagrangian formulation with the power-method time stepper is not built")
    output = None
    onode = proc.get("output")
    if onode:
        inc = float(onode.get("time_increment", 0.0))
        if not inc > 0.0:
            raise InputError("output.time_increment must be positive")
        output = (str(onode.get("file", "results.exo")), float(onode.get("time_start", 0.0)),
                  float(onode.get("time_end", t_end)), inc)
    return Simulation(name, coords, parts, bcs, v0, dt, t_end, precision, body, mass,
                      int(ext.get("max_steps", 1 << 40)), sets,
                      {"seed": seed, "mesh": mesh_spec, "element_blocks": element_blocks, "base_dir": str(base_dir)},
                      power, rk, output, formulation)


def power_method_inputs(sim: Simulation):
    """Start vector (uniform in [-1, 1] per node component, from the x_b200 seed; the
    reference draws it per node from the node id) and each node's longest edge."""
    rng = np.random.default_rng([int(sim.meta.get("seed", 0)), 1])
    return rng.uniform(-1.0, 1.0, size=sim.coords.shape), _mesh.max_edge_length(sim.coords, sim.meta["element_blocks"])


def run(source, stream=None, power_method_start=None) -> dict:
    """Parse, build the GPU model, and Solve(): the initial acceleration, then the time
    stepper's steps (ExplicitSolver::Solve, src/Solvers/Explicit.cpp:308-483); with the
    power-method stepper the increment is recomputed on the GPU every update_interval steps.
    With an output block and the direct stepper the run stops at the output steps and the
    result holds the frames (times and nodal fields) the reference would write there.
    power_method_start (N x 3) replaces the seeded start vector of the power method."""
    sim = source if isinstance(source, Simulation) else load(source)
    dt = sim.dt
    frames = None
    with sim.model(stream) as m:
        m.set_state(np.zeros_like(sim.coords), sim.v0)
        if sim.power_method is not None and sim.output is not None:
            # The schedule of am_solve_power_method driven from here, so that the run can
            # stop at the output steps: every update_interval steps the stable increment
            # is recomputed at the current state and scaled; runs are cut where the output
            # scheduler fires, with the same time accumulation.
            start, edges = power_method_inputs(sim)
            m.set_power_method(start if power_method_start is None else power_method_start, edges)
            scale, interval = sim.power_method
            m.init_acceleration(sim.precision)
            sched = TimeIncrementScheduler(*sim.output[1:])
            frames = {"step": [], "time": [], "displacement": [], "velocity": [], "acceleration": []}

            def record(n, t):
                fu, fv, fa = m.get_state()
                for k, x in zip(("step", "time", "displacement", "velocity", "acceleration"), (n, t, fu, fv, fa)):
                    frames[k].append(x)

            if sched.at_next_event(0.0):
                record(0, 0.0)
            time, dt, steps = 0.0, 0.0, 0
            while not time >= sim.time_end and steps < sim.max_steps:
                full, _, _ = m.stable_time_increment(dt / scale)
                dt = full * scale
                seg, t_seg = [], time
                for _ in range(interval):
                    if time >= sim.time_end or steps >= sim.max_steps:
                        break
                    d = dt if time + dt <= sim.time_end else (0.0 if time > sim.time_end else sim.time_end - time)
                    seg.append(d)
                    time += d
                    steps += 1
                    if sched.at_next_event(time):
                        m.run_schedule(seg, sim.precision, t0=t_seg)
                        seg, t_seg = [], time
                        record(steps, time)
                if seg:
                    m.run_schedule(seg, sim.precision, t0=t_seg)
        elif sim.power_method is not None:
            start, edges = power_method_inputs(sim)
            m.set_power_method(start if power_method_start is None else power_method_start, edges)
            steps, dt = m.solve_power_method(sim.power_method[0], sim.power_method[1], sim.time_end, sim.precision,
                                             sim.max_steps)
        elif sim.output is not None:
            dts = direct_time_steps(sim.dt, sim.time_end, sim.max_steps)
            at = output_steps(dts, sim.output)
            m.init_acceleration(sim.precision)
            frames = {"step": [], "time": [], "displacement": [], "velocity": [], "acceleration": []}
            done, time = 0, 0.0
            for n in at + [len(dts)]:
                if n > done:
                    m.run_schedule(dts[done:n], sim.precision, t0=time)
                    for d in dts[done:n]:
                        time += d
                    done = n
                if n in at and (not frames["step"] or frames["step"][-1] != n):
                    fu, fv, fa = m.get_state()
                    for k, x in zip(("step", "time", "displacement", "velocity", "acceleration"), (n, time, fu, fv, fa)):
                        frames[k].append(x)
            steps = len(dts)
        else:
            steps = m.solve(sim.dt, sim.time_end, sim.precision, sim.max_steps)
        u, v, a = m.get_state()
    out = {"simulation": sim, "steps": steps, "time_increment": dt, "displacement": u, "velocity": v,
           "acceleration": a}
    if sim.rk is not None:
        # The state holds generalized coefficients; the physical displacement is Psi u.
        from .rkpm import apply_functions

        out["physical_displacement"] = apply_functions(sim.rk, u)
    if frames is not None:
        out["frames"] = {k: np.asarray(x) for k, x in frames.items()}
        if sim.rk is not None:
            out["frames"]["physical_displacement"] = np.stack(
                [apply_functions(sim.rk, fu) for fu in frames["displacement"]]) if frames["displacement"] else \
                np.zeros((0,) + sim.coords.shape)
    return out


def write_output(result: dict, directory: Path | str = ".") -> Path:
    """The output frames as <output file stem>.npz in `directory`: step, time and the nodal
    fields (N x 3 per frame) at every output time, with the coordinates."""
    sim = result["simulation"]
    if sim.output is None or "frames" not in result:
        raise InputError("no output block")
    path = Path(directory) / (Path(sim.output[0]).stem + ".npz")
    np.savez(path, coordinates=sim.coords, **result["frames"])
    return path


def main(argv=None) -> int:
    import argparse

    ap = argparse.ArgumentParser(description="Run an aperi-mech explicit-dynamics input on the GPU.")
    ap.add_argument("input")
    ap.add_argument("--save", help="write the final u, v, a to this .npz")
    ap.add_argument("--output-dir", default=".", help="where the output block's frames are written (.npz)")
    a = ap.parse_args(argv)
    r = run(a.input)
    sim = r["simulation"]
    if "frames" in r:
        write_output(r, a.output_dir)
    if a.save:
        np.savez(a.save, displacement=r["displacement"], velocity=r["velocity"], acceleration=r["acceleration"])
    print(json.dumps({"input": a.input, "nodes": sim.num_nodes, "elements": sim.num_elems, "steps": r["steps"],
                      "precision": sim.precision, "max_abs_displacement": float(np.abs(r["displacement"]).max())}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
