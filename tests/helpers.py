"""Shared builders for the parity tests: the reference's patch/shear/gravity
fixtures restated on this repo's generated meshes, and error norms."""
from __future__ import annotations

import numpy as np

from aperi_mech_b200 import mesh
from aperi_mech_b200.model import BoundaryCondition, Material, Part


def rel_err(a, b) -> float:
    """max |a - b| / max |b| (max-norm relative error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / (den if den > 0 else 1.0)


def l2_rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def brick(kind: str, nx: int, ny: int, nz: int, unit: bool = True):
    """STK-style generated brick: elements of unit size (coordinates 0..n)."""
    lx, ly, lz = (nx, ny, nz) if unit else (1.0, 1.0, 1.0)
    coords, conn = mesh.box_hex(nx, ny, nz, lx, ly, lz)
    if kind == "tet4":
        conn = mesh.hex_to_tets(conn)
    return coords, conn


def svk_patch_material(E: float = 1.0, nu: float = 0.0, rho: float = 0.08) -> Material:
    # PatchTestFixture.h:432-434 (E=1, nu=0) and :74 (density 0.08).
    return Material.create("elastic", rho, youngs_modulus=E, poissons_ratio=nu)


def prescribed_patch(kind: str, dims, load_direction: int, load_surface: int, magnitude: float,
                     final_time: float = 10.0, material: Material | None = None):
    """PatchTestFixture::RunFullyPrescribedBoundaryConditionProblem (PatchTestFixture.h:48-172):
    smooth-step displacement BCs of -/+ 2*magnitude on the two faces normal to
    load_surface, over [0, 2*final_time] (half the step is run), dt = 0.1."""
    coords, conn = brick(kind, *dims)
    sets = mesh.side_sets(coords)
    s0 = sets[f"surface_{2 * load_surface + 1}"]
    s1 = sets[f"surface_{2 * load_surface + 2}"]
    d = np.zeros(3)
    d[load_direction] = 1.0
    mat = material or svk_patch_material()
    common = dict(kind="displacement", time_function="smooth_step_function", abscissa=(0.0, 2.0 * final_time),
                  ordinate=(0.0, 1.0), component_mask=7)
    bcs = [BoundaryCondition(nodes=s0, values=tuple(-2.0 * magnitude * d), **common),
           BoundaryCondition(nodes=s1, values=tuple(2.0 * magnitude * d), **common)]
    return coords, [Part(kind, mat, conn=conn)], bcs, sets


def expected_pk1(H: np.ndarray, material: Material) -> np.ndarray:
    """PatchTestFixture::GetExpectedFirstPKStress (SVK): P = F S(E)."""
    F = H + np.eye(3)
    Eg = 0.5 * (F.T @ F - np.eye(3))
    S = material.lam * np.trace(Eg) * np.eye(3) + 2.0 * material.mu * Eg
    return F @ S


def integrate_gravity(dt: float, g: np.ndarray, end_time: float):
    """SolverTest.cpp IntegrateKinematics (no ramp): the expected displacement and velocity
    increments of central differences under a constant body acceleration."""
    u = np.zeros(3)
    v = np.zeros(3)
    t = dt
    while t < end_time:
        v += g * dt
        u += v * dt
        t += dt
    u -= v * dt * 0.5
    return u, v
