"""The CPU oracle against the reference's own known answers (no GPU)."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from helpers import expected_pk1, integrate_gravity, prescribed_patch, rel_err, svk_patch_material

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    return json.loads((GOLD / name).read_text())


# ---- QuadratureTests.cpp ---------------------------------------------------------
@pytest.mark.parametrize("case", _load("quadrature_tet4.json"), ids=lambda c: c["name"])
def test_tet4_gauss_quadrature(oracle_lib, case):
    B, w = oracle_lib.gauss_bw("tet4", np.array(case["X"]))
    assert np.max(np.abs(B - np.array(case["B"]))) < 1e-12
    assert abs(w - case["w"]) < 1e-12
    assert np.all(np.abs(B.sum(axis=0)) < 1e-12)  # partition of nullity


@pytest.mark.parametrize("case", _load("quadrature_tet4.json"), ids=lambda c: c["name"])
def test_tet4_smoothed_quadrature(oracle_lib, case):
    B, w = oracle_lib.smoothed_bw("tet4", np.array(case["X"]))
    assert np.max(np.abs(B - np.array(case["B"]))) < 1e-12
    assert abs(w - case["w"]) < 1e-12


@pytest.mark.parametrize("case", _load("quadrature_hex8_smoothed.json"), ids=lambda c: c["name"])
def test_hex8_smoothed_quadrature(oracle_lib, case):
    B, w = oracle_lib.smoothed_bw("hex8", np.array(case["X"]))
    assert np.max(np.abs(B - np.array(case["B"]))) < 1e-12
    assert abs(w - case["w"]) < 1e-12


@pytest.mark.parametrize("case", _load("quadrature_hex8_smoothed.json")[:5], ids=lambda c: c["name"])
def test_hex8_gauss_quadrature_affine(oracle_lib, case):
    # For an affine hex every Gauss weight is V/8 and the volume average of the Gauss-point
    # B matrices is the smoothed (cell-average) B of the golden case.
    X = np.array(case["X"])
    avg = np.zeros((8, 3))
    for gp in range(8):
        B, w = oracle_lib.gauss_bw("hex8", X, gp)
        avg += w * B
        assert abs(w - case["w"] / 8.0) < 1e-12
    assert np.max(np.abs(avg / case["w"] - np.array(case["B"]))) < 1e-12


# ---- MaterialDriverTest.cpp, LinearElasticPropertiesTest.cpp ---------------------
def test_material_driver_neo_hookean(oracle_lib):
    g = _load("material_driver_nh.json")
    p = oracle_lib.complete_properties(youngs_modulus=g["youngs_modulus"], poissons_ratio=g["poissons_ratio"])
    for k, H in enumerate(g["displacement_gradients"]):
        H = np.array(H)
        P = oracle_lib.stress("neo_hookean", p["lambda"], p["shear_modulus"], H)[0]
        F = H + np.eye(3)
        sigma = P @ F.T / np.linalg.det(F)
        tol = g["expected_cauchy_diagonal"] * g["rel_tol"]
        for i in range(3):
            for j in range(3):
                want = g["expected_cauchy_diagonal"] if (i == j == k) else 0.0
                assert abs(sigma[i, j] - want) < tol


def test_linear_elastic_properties(oracle_lib):
    g = _load("linear_elastic_properties.json")
    vals = g["values"]
    for a, b in g["valid_pairs"]:
        out = oracle_lib.complete_properties(**{a: vals[a], b: vals[b]})
        for k, v in vals.items():
            assert abs(out[k] - v) < g["tol"], (a, b, k)
    for bad in g["invalid"]:
        with pytest.raises(ValueError):
            oracle_lib.complete_properties(**bad)


# ---- analytic element checks (Hex8 Gauss force has no reference known answer) ----
@pytest.mark.parametrize("kind", ["hex8", "tet4"])
@pytest.mark.parametrize("material", ["linear_elastic", "neo_hookean", "elastic"])
def test_linear_field_patch_and_rigid_rotation(oracle_lib, kind, material):
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import Material, Part

    rng = np.random.default_rng(3)
    coords, conn = mesh.box_hex(4, 4, 4)
    coords = mesh.jitter_interior(coords, 0.2 / 4, rng)
    if kind == "tet4":
        conn = mesh.hex_to_tets(conn)
    mat = Material.create(material, 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)
    prob = oracle_lib.OracleProblem(coords, [Part(kind, mat, conn=conn)])
    interior = ~mesh.boundary_mask(coords)
    # Constant stress: interior nodal forces vanish (patch test), forces sum to zero.
    A = 1e-3 * rng.standard_normal((3, 3))
    f = prob.internal_force(coords @ A.T)
    scale = np.abs(f).max()
    assert np.abs(f[interior]).max() < 1e-11 * scale
    assert np.abs(f.sum(axis=0)).max() < 1e-11 * scale
    # Rigid rotation: zero stress for the finite-strain models.
    if material != "linear_elastic":
        from golden.make_golden import rotation

        R = rotation([0.3, -1.0, 0.7], 0.9)
        f = prob.internal_force(coords @ R.T - coords)
        assert np.abs(f).max() < 1e-6 * scale


# ---- ForceTest.cpp shear patch tests (Tet4, fully prescribed, SVK E=1 nu=0) -------
SHEAR = [(1, 0), (2, 0), (0, 1), (2, 1), (0, 2), (1, 2)]


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("direction,surface", SHEAR)
def test_shear_patch(oracle_lib, kind, direction, surface):
    mag = 0.1
    coords, parts, bcs, sets = prescribed_patch(kind, (1, 1, 1), direction, surface, mag)
    prob = oracle_lib.OracleProblem(coords, parts, bcs)
    u, v, a, n = prob.solve(np.zeros_like(coords), np.zeros_like(coords), 0.1, 10.0)
    assert n == len(oracle_lib.direct_time_schedule(0.1, 10.0))
    H = np.zeros((3, 3))
    H[direction, surface] = 2.0 * mag
    mass = prob.lumped_mass()
    assert abs(mass.sum() - 0.08 * 1.0) < 1e-12  # PatchTestFixture::CheckMass
    f = prob.internal_force(u)
    P = expected_pk1(H, parts[0].material)
    s_lo, s_hi = sets[f"surface_{2 * surface + 1}"], sets[f"surface_{2 * surface + 2}"]
    # Displacement field is the linear patch: every element's H equals the expected one.
    conn = parts[0].conn
    for e in range(conn.shape[0]):
        B, _ = oracle_lib.gauss_bw(kind, coords[conn[e]])
        assert np.abs(u[conn[e]].T @ B - H).max() < 1e-9
    assert np.abs(a).max() < 1e-12
    assert np.abs(f[np.union1d(s_lo, s_hi)].sum(axis=0)).max() < 1e-8
    for i in range(3):
        n_i = np.zeros(3)
        n_i[i] = 1.0
        expected = P @ n_i * 1.0
        assert np.abs(f[sets[f"surface_{2 * i + 1}"]].sum(axis=0) - expected).max() < 1e-8
        assert np.abs(f[sets[f"surface_{2 * i + 2}"]].sum(axis=0) + expected).max() < 1e-8
    d = np.zeros(3)
    d[direction] = mag
    assert np.abs(u[s_hi] - d).max() < 1e-9 and np.abs(u[s_lo] + d).max() < 1e-9
    assert np.abs(v[s_hi] - 1.875 * d / 10.0).max() < 1e-4


# ---- PatchTest.cpp tension / compression (2x2x2, free interior nodes) --------------
@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("mag", [0.1, -0.1])
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_tension_compression_patch(oracle_lib, kind, mag, axis):
    coords, parts, bcs, sets = prescribed_patch(kind, (2, 2, 2), axis, axis, mag)
    prob = oracle_lib.OracleProblem(coords, parts, bcs)
    u, v, a, _ = prob.solve(np.zeros_like(coords), np.zeros_like(coords), 0.1, 10.0)
    H = np.zeros((3, 3))
    H[axis, axis] = 2.0 * mag / 2.0
    com = np.array([1.0, 1.0, 1.0])
    assert np.abs(u - (coords - com) @ H.T).max() < 1e-9
    assert np.abs(v - (coords - com) @ (H * 1.875 / 10.0).T).max() < 1e-4
    assert np.abs(a).max() < 1e-9
    f = prob.internal_force(u)
    assert np.abs(f.sum(axis=0)).max() < 1e-12
    P = expected_pk1(H, parts[0].material)
    for i in range(3):
        n_i = np.zeros(3)
        n_i[i] = 1.0
        area = 4.0
        assert np.abs(f[sets[f"surface_{2 * i + 1}"]].sum(axis=0) - P @ n_i * area).max() < 1e-8
        assert np.abs(f[sets[f"surface_{2 * i + 2}"]].sum(axis=0) + P @ n_i * area).max() < 1e-8


# ---- SolverTest.cpp free flight and gravity ---------------------------------------
@pytest.mark.parametrize("gravity", [False, True])
def test_free_flight_and_gravity(oracle_lib, gravity):
    # SolverTest.cpp:12-32 and :110-154 use a "1x1x1|tets" mesh; dt = 0.1 is far beyond the
    # stable step, so the test relies on rigid motion producing exactly zero stress.
    kind = "tet4"
    from helpers import brick
    from aperi_mech_b200.model import Part

    coords, conn = brick(kind, 1, 1, 1)
    rho = 7850.0 * (1e4 if gravity else 1.0)
    mat = svk_patch_material(E=2.1e11, nu=0.3, rho=rho)
    d = np.array([1.4, -2.5, 2.9])
    v0 = np.tile(1.23 * d / np.linalg.norm(d), (coords.shape[0], 1))
    g = np.array([0.0, 0.0, -9.81]) if gravity else np.zeros(3)
    prob = oracle_lib.OracleProblem(coords, [Part(kind, mat, conn=conn)], body_accel=tuple(g))
    u, v, a, n = prob.solve(np.zeros_like(coords), v0, 0.1, 1.0)
    du, dv = integrate_gravity(0.1, g, 1.0)
    assert np.abs(u - (v0 * 1.0 + du)).max() < 1e-12
    assert np.abs(v - (v0 + dv)).max() < 1e-12
    assert np.abs(a - g).max() < 1e-11
    assert abs(prob.lumped_mass().sum() - rho * 1.0) < 1e-12 * rho


def test_direct_time_schedule(oracle_lib):
    d = oracle_lib.direct_time_schedule(0.1, 1.0)
    assert len(d) == 11 and abs(d[-1]) < 1e-15  # accumulated time falls short of t_end by one ulp
    assert len(oracle_lib.direct_time_schedule(0.25, 1.0)) == 4


# ---- adjoint on the oracle: central finite differences --------------------------
def test_oracle_vjp_matches_finite_differences(oracle_lib):
    from aperi_mech_b200.problems import hex8_nh_lognormal

    prob = hex8_nh_lognormal(n=3, seed=1, nsteps=5, bulk_field=True, num_sensors=8)
    op = oracle_lib.OracleProblem.from_problem(prob)
    rng = np.random.default_rng(0)
    u = 1e-3 * rng.standard_normal(prob.coords.shape)
    lam = rng.standard_normal(prob.coords.shape)
    gu, gm, gk = op.vjp_force(u, lam)
    eps = 1e-7
    du = rng.standard_normal(prob.coords.shape)
    fd = (np.sum(lam * op.internal_force(u + eps * du)) - np.sum(lam * op.internal_force(u - eps * du))) / (2 * eps)
    assert abs(np.sum(gu * du) - fd) < 1e-6 * abs(fd)
    part = prob.parts[0]
    mu0, k0 = part.mu_field.copy(), part.kappa_field.copy()
    for e in [0, 7, 20]:
        for field, g, base in (("mu_field", gm, mu0), ("kappa_field", gk, k0)):
            h = 1e-6 * base[e]
            vals = []
            for s in (1, -1):
                arr = base.copy()
                arr[e] += s * h
                setattr(part, field, arr)
                vals.append(np.sum(lam * oracle_lib.OracleProblem.from_problem(prob).internal_force(u)))
            setattr(part, field, base)
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(g[e] - fd) < 1e-5 * max(abs(fd), 1e-30), (field, e)


def test_oracle_adjoint_matches_finite_differences(oracle_lib):
    from aperi_mech_b200.problems import hex8_nh_lognormal

    prob = hex8_nh_lognormal(n=3, seed=2, nsteps=20, bulk_field=True, num_sensors=10)
    sens = prob.meta["sensors"]
    op = oracle_lib.OracleProblem.from_problem(prob)
    loss, gm, gk = op.adjoint(prob.nsteps, prob.dt, np.zeros_like(prob.coords), prob.v0, sens)
    part = prob.parts[0]
    for e in [1, 13]:
        for field, g in (("mu_field", gm), ("kappa_field", gk)):
            base = getattr(part, field).copy()
            h = 1e-6 * base[e]
            Ls = []
            for s in (1, -1):
                arr = base.copy()
                arr[e] += s * h
                setattr(part, field, arr)
                Ls.append(oracle_lib.OracleProblem.from_problem(prob).adjoint(
                    prob.nsteps, prob.dt, np.zeros_like(prob.coords), prob.v0, sens)[0])
            setattr(part, field, base)
            fd = (Ls[0] - Ls[1]) / (2 * h)
            assert abs(g[e] - fd) <= 1e-4 * abs(fd), (field, e, g[e], fd)
