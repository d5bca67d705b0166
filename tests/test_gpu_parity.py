"""Parity of the CUDA path (through the C ABI) with the CPU FP64 oracle.

Tolerances: the FP64 path must agree with the oracle to 1e-12 relative (max-norm
relative to the largest entry); the mixed FP32-element / FP64-state path to the
per-test tolerance written below."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from helpers import expected_pk1, integrate_gravity, prescribed_patch, rel_err, svk_patch_material

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
FP64_TOL = 1e-12
MIXED_FORCE_TOL = 5e-5


def _load(name):
    return json.loads((GOLD / name).read_text())


def _mesh(kind, n, seed=0, jitter=0.2):
    from aperi_mech_b200 import mesh

    rng = np.random.default_rng(seed)
    coords, conn = mesh.box_hex(n, n, n)
    coords = mesh.jitter_interior(coords, jitter / n, rng)
    if kind == "tet4":
        conn = mesh.hex_to_tets(conn)
    return coords, conn


def _material(name):
    from aperi_mech_b200.model import Material

    if name == "neo_hookean":
        return Material.create(name, 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    return Material.create(name, 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)


def _fields(E, seed, with_fields):
    if not with_fields:
        return None, None
    rng = np.random.default_rng(seed)
    return 3.85e8 * np.exp(0.3 * rng.standard_normal(E)), 8.33e8 * np.exp(0.3 * rng.standard_normal(E))


# ---- point kernels against the reference's unit-test known answers --------------------
def test_quadrature_gpu_golden(gpu):
    from aperi_mech_b200 import capi

    tets = _load("quadrature_tet4.json")
    X = np.array([c["X"] for c in tets])
    for smoothed in (False, True):
        B, w = capi.quadrature(capi.AM_TET4_GAUSS, X, smoothed=smoothed)
        for k, c in enumerate(tets):
            assert np.abs(B[k, 0] - np.array(c["B"])).max() < 1e-12, c["name"]
            assert abs(w[k, 0] - c["w"]) < 1e-12
    hexes = _load("quadrature_hex8_smoothed.json")
    X = np.array([c["X"] for c in hexes])
    B, w = capi.quadrature(capi.AM_HEX8_GAUSS, X, smoothed=True)
    for k, c in enumerate(hexes):
        assert np.abs(B[k, 0] - np.array(c["B"])).max() < 1e-12, c["name"]
        assert abs(w[k, 0] - c["w"]) < 1e-12
    Bg, wg = capi.quadrature(capi.AM_HEX8_GAUSS, X[:5])
    for k in range(5):
        avg = np.einsum("g,gaj->aj", wg[k], Bg[k]) / wg[k].sum()
        assert np.abs(avg - np.array(hexes[k]["B"])).max() < 1e-12


def test_material_driver_gpu(gpu, oracle_lib):
    from aperi_mech_b200 import capi
    from aperi_mech_b200.model import complete_properties

    g = _load("material_driver_nh.json")
    p = complete_properties(youngs_modulus=g["youngs_modulus"], poissons_ratio=g["poissons_ratio"])
    P = capi.stress(capi.AM_NEO_HOOKEAN, p["lambda"], p["shear_modulus"], np.array(g["displacement_gradients"]))
    for k, H in enumerate(g["displacement_gradients"]):
        F = np.array(H) + np.eye(3)
        sigma = P[k] @ F.T / np.linalg.det(F)
        want = np.zeros((3, 3))
        want[k, k] = g["expected_cauchy_diagonal"]
        assert np.abs(sigma - want).max() < g["expected_cauchy_diagonal"] * g["rel_tol"]
    rng = np.random.default_rng(5)
    H = 0.05 * rng.standard_normal((64, 3, 3))
    for name, code in (("linear_elastic", 0), ("neo_hookean", 1), ("elastic", 2)):
        mat = _material(name)
        got = capi.stress(code, mat.lam, mat.mu, H)
        want = oracle_lib.stress(name, mat.lam, mat.mu, H)
        assert rel_err(got, want) < 1e-14, name


def test_neo_hookean_log_j_across_series_range(gpu, oracle_lib):
    """The neo-Hookean log J uses a series for |J - 1| <= 1/16 and CUDA's log1p beyond:
    the volumetric stress of pure dilatations H = a I, J - 1 from -0.5 to 1 (both sides of
    the switch, and tiny |J - 1|), matches the oracle's std::log1p to a few ulp."""
    from aperi_mech_b200 import capi

    jm1 = np.concatenate([np.linspace(-0.5, 1.0, 301), [-0.0625, 0.0625, -0.0624999, 0.0625001],
                          np.geomspace(1e-14, 1e-2, 25), -np.geomspace(1e-14, 1e-2, 25)])
    a = np.cbrt(1.0 + jm1) - 1.0
    H = a[:, None, None] * np.eye(3)[None]
    mat = _material("neo_hookean")
    got = capi.stress(capi.AM_NEO_HOOKEAN, mat.lam, mat.mu, H)
    want = oracle_lib.stress("neo_hookean", mat.lam, mat.mu, H)
    scale = np.abs(want).reshape(len(a), -1).max(axis=1)
    assert (np.abs(got - want).reshape(len(a), -1).max(axis=1) <= 1e-14 * scale + 1e-300).all()


# ---- internal force ------------------------------------------------------------------
@pytest.mark.parametrize("kind,n", [("tet4", 5), ("hex8", 6)])
@pytest.mark.parametrize("material", ["linear_elastic", "neo_hookean", "elastic"])
@pytest.mark.parametrize("with_fields", [False, True])
def test_internal_force_parity(gpu, oracle_lib, kind, n, material, with_fields):
    from aperi_mech_b200.model import ExplicitDynamics, Part

    coords, conn = _mesh(kind, n, seed=1)
    mu_f, k_f = _fields(conn.shape[0], 2, with_fields)
    parts = [Part(kind, _material(material), conn=conn, mu_field=mu_f, kappa_field=k_f)]
    rng = np.random.default_rng(4)
    u = 2e-3 * rng.standard_normal(coords.shape) + 1e-3 * coords @ rng.standard_normal((3, 3))
    want = oracle_lib.OracleProblem(coords, parts).internal_force(u)
    with ExplicitDynamics(coords, parts) as m:
        f64 = m.internal_force(u, "fp64")
        f32 = m.internal_force(u, "mixed")
        assert rel_err(m.mass(), oracle_lib.OracleProblem(coords, parts).lumped_mass()) < 1e-14
    assert rel_err(f64, want) < FP64_TOL
    assert rel_err(f32, want) < MIXED_FORCE_TOL


def test_internal_force_two_parts_accumulate(gpu, oracle_lib):
    """Two parts (InternalForceContributions) sharing nodes, and accumulate=1."""
    from aperi_mech_b200.model import ExplicitDynamics, Part

    coords, conn = _mesh("hex8", 6, seed=3)
    half = conn.shape[0] // 2
    parts = [Part("hex8", _material("neo_hookean"), conn=conn[:half]),
             Part("hex8", _material("elastic"), conn=conn[half:])]
    u = 1e-3 * np.random.default_rng(0).standard_normal(coords.shape)
    want = oracle_lib.OracleProblem(coords, parts).internal_force(u)
    with ExplicitDynamics(coords, parts) as m:
        f = m.internal_force(u)
        base = np.ones_like(f)
        g = m.internal_force(u, out=base.copy(), accumulate=True)
    assert rel_err(f, want) < FP64_TOL
    assert rel_err(g - 1.0, want) < 1e-11


def test_smoothed_cells_parity(gpu, oracle_lib):
    from aperi_mech_b200.model import ExplicitDynamics
    from aperi_mech_b200.smoothing import element_smoothing_part

    coords, conn = _mesh("tet4", 5, seed=7)
    part, mass = element_smoothing_part(coords, conn, _material("neo_hookean"))
    u = 1e-3 * np.random.default_rng(1).standard_normal(coords.shape)
    op = oracle_lib.OracleProblem(coords, [part], mass=mass)
    want = op.internal_force(u)
    with ExplicitDynamics(coords, [part], mass=mass) as m:
        assert rel_err(m.internal_force(u), want) < FP64_TOL
        assert rel_err(m.internal_force(u, "mixed"), want) < MIXED_FORCE_TOL


@pytest.mark.parametrize("material", ["neo_hookean", "elastic", "linear_elastic"])
def test_element_cells_grouped_as_split_hexes(gpu, oracle_lib, monkeypatch, material):
    """Element smoothing cells of a split-hex tet mesh run as patches (one slot per patch
    node, a third of the slots; with warp chunks, the default, one per distinct node of a
    warp's 16 patches): the force (FP64 and mixed), the VJP and 30 steps with per-cell
    moduli against the oracle, grouped with and without chunks and with patching off."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics
    from aperi_mech_b200.smoothing import element_smoothing_part

    coords, conn = _mesh("tet4", 5, seed=11)
    mu_f, k_f = _fields(conn.shape[0], 7, True)
    mat = _material(material)
    part, mass = element_smoothing_part(coords, conn, mat, mu_field=mu_f, kappa_field=k_f)
    bcs = [BoundaryCondition.fixed(mesh.side_sets(coords)["surface_5"])]
    rng = np.random.default_rng(12)
    u = 1e-3 * rng.standard_normal(coords.shape)
    lam = rng.standard_normal(coords.shape)
    v0 = rng.uniform(-0.01, 0.01, size=coords.shape)
    v0[bcs[0].nodes] = 0.0
    cmax = np.sqrt((k_f.max() + 4.0 / 3.0 * mu_f.max()) / mat.density)
    dt = 0.2 * float(mesh.tet_char_length(coords, conn).min()) / cmax
    op = oracle_lib.OracleProblem(coords, [part], bcs, mass=mass)
    want_f, want_v = op.internal_force(u), op.vjp_force(u, lam)
    zero = np.zeros_like(coords)
    want_s = op.steps(zero, v0, op.init_acceleration(zero), np.full(30, dt))
    slots = {}
    # split-hex grouping with warp chunks (the default), without them, and no grouping
    for patches, chunks in (("2", "1"), ("2", "0"), ("0", "1")):
        monkeypatch.setenv("APERI_B200_TET4_PATCHES", patches)
        monkeypatch.setenv("APERI_B200_WARP_CHUNKS", chunks)
        with ExplicitDynamics(coords, [part], bcs, mass=mass) as m:
            slots[patches + chunks] = m.layout()["used_slots"]
            assert rel_err(m.internal_force(u), want_f) < FP64_TOL
            assert rel_err(m.internal_force(u, "mixed"), want_f) < MIXED_FORCE_TOL
            for g, w in zip(m.vjp_force(u, lam), want_v):
                assert rel_err(g, w) < 1e-11
            m.set_state(None, v0)
            m.init_acceleration()
            m.run(30, dt)
            for g, w in zip(m.get_state(), want_s):
                assert rel_err(g, w) < FP64_TOL
    assert 3 * slots["20"] == slots["01"] == 4 * conn.shape[0]
    assert slots["21"] < slots["20"] // 2


# ---- time integration ----------------------------------------------------------------
def _small_problem(name):
    from aperi_mech_b200 import problems

    if name == "hex8_le":
        return problems.hex8_le_cube(n=6, seed=3, nsteps=100)
    if name == "tet4_nh":
        return problems.tet4_nh_shear(n=5, seed=3, nsteps=100)
    return problems.hex8_nh_lognormal(n=5, seed=3, nsteps=60, bulk_field=True)


@pytest.mark.parametrize("name", ["hex8_le", "tet4_nh", "hex8_nh_fields"])
def test_run_fp64_matches_oracle(gpu, oracle_lib, name):
    from aperi_mech_b200.model import ExplicitDynamics

    p = _small_problem(name)
    u0 = np.zeros_like(p.coords)
    op = oracle_lib.OracleProblem.from_problem(p)
    a0 = op.init_acceleration(u0)
    want = op.steps(u0, p.v0, a0, np.full(p.nsteps, p.dt))
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_state(u0, p.v0)
        m.init_acceleration()
        m.run(p.nsteps // 3, p.dt)
        m.run(p.nsteps - p.nsteps // 3, p.dt, t0=(p.nsteps // 3) * p.dt)  # two calls == one run
        got = m.get_state()
    for g, w in zip(got, want):
        assert rel_err(g, w) < FP64_TOL


def test_run_is_bitwise_deterministic(gpu):
    from aperi_mech_b200.model import ExplicitDynamics

    p = _small_problem("tet4_nh")
    outs = []
    for _ in range(3):
        with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
            m.set_state(None, p.v0)
            m.init_acceleration("mixed")
            m.run(50, p.dt, "mixed")
            outs.append(m.get_state())
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert np.array_equal(a, b)


def test_mixed_accuracy_after_1000_steps(gpu):
    """Mixed path vs the GPU FP64 path (itself 1e-12 from the oracle) on the neo-Hookean
    Tet4 shear workload, 1000 steps: relative displacement error (L2) <= 1e-5."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics
    from helpers import l2_rel

    p = problems.tet4_nh_shear(n=12, seed=0, nsteps=1000)
    res = {}
    for prec in ("fp64", "mixed"):
        with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
            m.set_state(None, p.v0)
            m.init_acceleration(prec)
            m.run(p.nsteps, p.dt, prec)
            res[prec] = m.get_state()
    assert l2_rel(res["mixed"][0], res["fp64"][0]) < 1e-5


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("direction,surface", [(1, 0), (2, 1), (0, 2)])
def test_shear_patch_gpu(gpu, oracle_lib, kind, direction, surface):
    from aperi_mech_b200.model import ExplicitDynamics

    mag = 0.1
    coords, parts, bcs, sets = prescribed_patch(kind, (1, 1, 1), direction, surface, mag)
    op = oracle_lib.OracleProblem(coords, parts, bcs)
    zero = np.zeros_like(coords)
    wu, wv, wa, wn = op.solve(zero, zero, 0.1, 10.0)
    with ExplicitDynamics(coords, parts, bcs) as m:
        m.set_state(zero, zero)
        n = m.solve(0.1, 10.0)
        u, v, a = m.get_state()
        f = m.internal_force(u)
    assert n == wn
    assert rel_err(u, wu) < FP64_TOL and rel_err(v, wv) < FP64_TOL
    assert np.abs(a - wa).max() < 1e-12
    H = np.zeros((3, 3))
    H[direction, surface] = 2 * mag
    P = expected_pk1(H, parts[0].material)
    for i in range(3):
        e = np.eye(3)[i]
        assert np.abs(f[sets[f"surface_{2 * i + 1}"]].sum(axis=0) - P @ e).max() < 1e-8


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
def test_tension_patch_gpu(gpu, oracle_lib, kind):
    from aperi_mech_b200.model import ExplicitDynamics

    coords, parts, bcs, sets = prescribed_patch(kind, (2, 2, 2), 0, 0, 0.1)
    zero = np.zeros_like(coords)
    with ExplicitDynamics(coords, parts, bcs) as m:
        m.set_state(zero, zero)
        m.solve(0.1, 10.0)
        u, v, a = m.get_state()
    H = np.zeros((3, 3))
    H[0, 0] = 0.1
    assert np.abs(u - (coords - 1.0) @ H.T).max() < 1e-9
    assert np.abs(a).max() < 1e-9
    wu, wv, wa, _ = oracle_lib.OracleProblem(coords, parts, bcs).solve(zero, zero, 0.1, 10.0)
    assert rel_err(u, wu) < FP64_TOL and rel_err(v, wv) < FP64_TOL


@pytest.mark.parametrize("gravity", [False, True])
def test_free_flight_and_gravity_gpu(gpu, gravity):
    from helpers import brick
    from aperi_mech_b200.model import ExplicitDynamics, Part

    coords, conn = brick("tet4", 1, 1, 1)
    rho = 7850.0 * (1e4 if gravity else 1.0)
    mat = svk_patch_material(E=2.1e11, nu=0.3, rho=rho)
    d = np.array([1.4, -2.5, 2.9])
    v0 = np.tile(1.23 * d / np.linalg.norm(d), (coords.shape[0], 1))
    g = np.array([0.0, 0.0, -9.81]) if gravity else np.zeros(3)
    with ExplicitDynamics(coords, [Part("tet4", mat, conn=conn)], body_accel=g) as m:
        m.set_state(None, v0)
        assert m.solve(0.1, 1.0) == 11
        u, v, a = m.get_state()
        assert abs(m.mass().sum() - rho) < 1e-12 * rho
    du, dv = integrate_gravity(0.1, g, 1.0)
    assert np.abs(u - (v0 + du)).max() < 1e-12
    assert np.abs(v - (v0 + dv)).max() < 1e-12
    assert np.abs(a - g).max() < 1e-11


def test_velocity_bc_with_active_range(gpu, oracle_lib):
    """Velocity BC (ramp) active only on [0.2, 0.8], overlapping a fixed support."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics, Part

    coords, conn = _mesh("hex8", 4, seed=9)
    sets = mesh.side_sets(coords)
    mat = _material("linear_elastic")
    dt = 0.5 * 0.25 / np.sqrt((mat.lam + 2 * mat.mu) / mat.density)
    T = 40 * dt
    bcs = [BoundaryCondition.fixed(sets["surface_5"]),
           BoundaryCondition(nodes=sets["surface_6"], values=(0.0, 0.0, 0.5), component_mask=4, kind="velocity",
                             abscissa=(0.0, T), ordinate=(0.0, 1.0), active_range=(0.2 * T, 0.8 * T)),
           BoundaryCondition(nodes=sets["surface_2"], values=(0.01, 0.0, 0.0), component_mask=1)]
    parts = [Part("hex8", mat, conn=conn)]
    zero = np.zeros_like(coords)
    wu, wv, wa, wn = oracle_lib.OracleProblem(coords, parts, bcs).solve(zero, zero, dt, T)
    with ExplicitDynamics(coords, parts, bcs) as m:
        m.set_state(zero, zero)
        assert m.solve(dt, T) == wn
        u, v, a = m.get_state()
    assert rel_err(u, wu) < FP64_TOL and rel_err(v, wv) < FP64_TOL and rel_err(a, wa) < FP64_TOL


def test_inverted_element_reports_status(gpu):
    from aperi_mech_b200.capi import AM_ENONPOS_J, AmError
    from aperi_mech_b200.model import ExplicitDynamics, Part

    coords, conn = _mesh("tet4", 2, seed=0, jitter=0.0)
    with ExplicitDynamics(coords, [Part("tet4", _material("neo_hookean"), conn=conn)]) as m:
        u = np.zeros_like(coords)
        u[0] = [2.0, 2.0, 2.0]  # drives the corner tets through themselves: J < 0
        with pytest.raises(AmError) as e:
            m.internal_force(u)
        assert e.value.code == AM_ENONPOS_J
        m.internal_force(np.zeros_like(coords))  # the context stays usable


# ---- adjoint ---------------------------------------------------------------------------
@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("material", ["linear_elastic", "neo_hookean", "elastic"])
def test_vjp_matches_oracle(gpu, oracle_lib, kind, material):
    from aperi_mech_b200.model import ExplicitDynamics, Part

    coords, conn = _mesh(kind, 4, seed=2)
    mu_f, k_f = _fields(conn.shape[0], 3, True)
    parts = [Part(kind, _material(material), conn=conn, mu_field=mu_f, kappa_field=k_f)]
    rng = np.random.default_rng(8)
    u = 1e-3 * rng.standard_normal(coords.shape)
    lam = rng.standard_normal(coords.shape)
    want = oracle_lib.OracleProblem(coords, parts).vjp_force(u, lam)
    with ExplicitDynamics(coords, parts) as m:
        got = m.vjp_force(u, lam)
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-11


def test_adjoint_matches_oracle(gpu, oracle_lib):
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.hex8_nh_lognormal(n=4, seed=5, nsteps=31, bulk_field=True, num_sensors=20)
    sens = p.meta["sensors"]
    wl, wm, wk = oracle_lib.OracleProblem.from_problem(p).adjoint(p.nsteps, p.dt, np.zeros_like(p.coords), p.v0, sens)
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_state(None, p.v0)
        loss, gm, gk = m.adjoint(p.nsteps, p.dt, 7, sens)
    assert abs(loss - wl) < 1e-12 * abs(wl)
    assert rel_err(gm, wm) < 1e-10 and rel_err(gk, wk) < 1e-10


def test_adjoint_finite_differences_hex8_64(gpu):
    """Hex8 neo-Hookean 64^3 with a lognormal shear-modulus field, 200 steps, checkpoints
    every 20: adjoint gradient vs central finite differences (step 1e-6 relative) on 32
    seeded elements, relative error <= 1e-4."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.hex8_nh_lognormal(n=64, seed=0, nsteps=200)
    sens = p.meta["sensors"]
    mu0 = p.parts[0].mu_field.copy()
    elems = np.sort(np.random.default_rng(11).choice(mu0.size, size=32, replace=False))
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_state(None, p.v0)
        loss, gm, _ = m.adjoint(p.nsteps, p.dt, 20, sens)

        def L(mu):
            m.set_block_fields(0, mu_field=mu)
            m.set_state(None, p.v0)
            m.init_acceleration()
            m.run(p.nsteps, p.dt)
            u = m.get_state()[0][sens]
            return float(np.sum(u * u))

        assert abs(L(mu0) - loss) < 1e-12 * loss
        errs = []
        for e in elems:
            h = 1e-6 * mu0[e]
            mp, mm = mu0.copy(), mu0.copy()
            mp[e] += h
            mm[e] -= h
            fd = (L(mp) - L(mm)) / (2 * h)
            errs.append(abs(gm[e] - fd) / abs(fd))
    assert max(errs) <= 1e-4, max(errs)


# ---- Tet4 one thread per tet: reference geometry table ------------------------------------
@pytest.mark.parametrize("material", ["neo_hookean", "elastic", "linear_elastic"])
def test_tet4_geometry_table(gpu, oracle_lib, monkeypatch, material):
    """One thread per tet with the reference J^-1 and weight set up once (the default) and
    with the coordinates gathered and J inverted every step (APERI_B200_TET4_GEOMETRY=0):
    both match the oracle, FP64 forces and 30 steps, and agree with each other to
    round-off; mixed forces within the mixed bar."""
    from aperi_mech_b200.model import ExplicitDynamics, Part

    monkeypatch.setenv("APERI_B200_TET4_PATCHES", "0")
    coords, conn = _mesh("tet4", 5, seed=9)
    conn = conn[np.random.default_rng(1).permutation(conn.shape[0])]
    parts = [Part("tet4", _material(material), conn=conn)]
    rng = np.random.default_rng(4)
    u = 1e-3 * rng.standard_normal(coords.shape)
    v0 = 10.0 * rng.standard_normal(coords.shape)
    op = oracle_lib.OracleProblem(coords, parts)
    want_f = op.internal_force(u)
    out = {}
    for geo in ("1", "0"):
        monkeypatch.setenv("APERI_B200_TET4_GEOMETRY", geo)
        with ExplicitDynamics(coords, parts) as m:
            f = m.internal_force(u)
            assert rel_err(f, want_f) < FP64_TOL
            assert rel_err(m.internal_force(u, "mixed"), want_f) < MIXED_FORCE_TOL
            dt = 1e-7
            m.set_state(None, v0)
            m.init_acceleration()
            m.run(30, dt)
            out[geo] = (f, m.get_state())
    z = np.zeros_like(coords)
    want = op.steps(z, v0, op.init_acceleration(z), np.full(30, 1e-7))
    for g, w in zip(out["1"][1], want):
        assert rel_err(g, w) < 1e-12
    assert rel_err(out["1"][0], out["0"][0]) < 1e-13


@pytest.mark.parametrize("path", ["per_tet", "split_hex"])
@pytest.mark.parametrize("material", ["neo_hookean", "elastic", "linear_elastic"])
def test_warp_chunks(gpu, oracle_lib, monkeypatch, material, path):
    """Warp chunks, where each warp sums its nodal forces on shared nodes before writing one
    slot per distinct node (the default), against one slot per tet or patch node
    (APERI_B200_WARP_CHUNKS=0), on one thread per tet (32 tets a warp) and on the split-hex
    patches (16 patches a warp): FP64 and mixed forces, the lumped mass, the VJP with
    modulus fields and 30 steps against the oracle, on 750 tets (125 patches: partial last
    chunks); the chunked layout writes fewer slots and repeats bit for bit."""
    from aperi_mech_b200.model import ExplicitDynamics, Part

    monkeypatch.setenv("APERI_B200_TET4_PATCHES", "0" if path == "per_tet" else "2")
    coords, conn = _mesh("tet4", 5, seed=13)
    assert conn.shape[0] % 32 != 0 and (conn.shape[0] // 3) % 32 != 0
    mu_f, k_f = _fields(conn.shape[0], 8, True)
    parts = [Part("tet4", _material(material), conn=conn, mu_field=mu_f, kappa_field=k_f)]
    rng = np.random.default_rng(5)
    u = 1e-3 * rng.standard_normal(coords.shape)
    lam = rng.standard_normal(coords.shape)
    v0 = 10.0 * rng.standard_normal(coords.shape)
    op = oracle_lib.OracleProblem(coords, parts)
    want_f, want_v = op.internal_force(u), op.vjp_force(u, lam)
    z = np.zeros_like(coords)
    want_s = op.steps(z, v0, op.init_acceleration(z), np.full(30, 1e-7))
    slots = {}
    for chunks in ("1", "0"):
        monkeypatch.setenv("APERI_B200_WARP_CHUNKS", chunks)
        with ExplicitDynamics(coords, parts) as m:
            slots[chunks] = m.layout()["used_slots"]
            assert m.layout()["patched_tet4_blocks"] == (path == "split_hex")
            f = m.internal_force(u)
            assert rel_err(f, want_f) < FP64_TOL
            assert np.array_equal(f, m.internal_force(u))
            assert rel_err(m.internal_force(u, "mixed"), want_f) < MIXED_FORCE_TOL
            assert rel_err(m.mass(), op.lumped_mass()) < 1e-14
            for g, w in zip(m.vjp_force(u, lam), want_v):
                assert rel_err(g, w) < 1e-11
            m.set_state(None, v0)
            m.init_acceleration()
            m.run(30, 1e-7)
            for g, w in zip(m.get_state(), want_s):
                assert rel_err(g, w) < 1e-12
    per_node = 4 if path == "per_tet" else 8 / 6
    assert slots["0"] == per_node * conn.shape[0] and slots["1"] < slots["0"] // 2


def test_warp_chunks_fan_mesh(gpu, oracle_lib, monkeypatch):
    """Every tet shares node 0 (a fan of 100 tets about it, with neighbouring tets sharing two
    more nodes), so in each warp chunk node 0's run holds 32 entries over eight lanes and is
    summed by the scan across lanes: FP64 force, lumped mass and VJP against the oracle, with
    and without warp chunks."""
    from aperi_mech_b200.model import ExplicitDynamics, Part

    monkeypatch.setenv("APERI_B200_TET4_PATCHES", "0")
    rng = np.random.default_rng(21)
    n = 102
    t = np.linspace(0.0, 6.0 * np.pi, n)
    ring = np.stack([np.cos(t), np.sin(t), 0.3 * t / np.pi + 0.2 * rng.standard_normal(n)], axis=1)
    coords = np.vstack([np.zeros((1, 3)), ring + 0.05 * rng.standard_normal(ring.shape)])
    conn = np.array([[0, i, i + 1, i + 2] for i in range(1, n - 1)], dtype=np.int32)
    x = coords[conn]
    det = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    conn[det < 0, 1], conn[det < 0, 2] = conn[det < 0, 2], conn[det < 0, 1].copy()
    parts = [Part("tet4", _material("neo_hookean"), conn=conn)]
    u = 1e-3 * rng.standard_normal(coords.shape)
    lam = rng.standard_normal(coords.shape)
    op = oracle_lib.OracleProblem(coords, parts)
    want_f, want_v = op.internal_force(u), op.vjp_force(u, lam)
    for chunks in ("1", "0"):
        monkeypatch.setenv("APERI_B200_WARP_CHUNKS", chunks)
        with ExplicitDynamics(coords, parts) as m:
            # FP64 only: the spiral's sliver tets would test the mixed path's conditioning, not
            # the chunk sums (the same code in both precisions, checked by test_warp_chunks)
            assert rel_err(m.internal_force(u), want_f) < FP64_TOL
            assert rel_err(m.mass(), op.lumped_mass()) < 1e-14
            for g, w in zip(m.vjp_force(u, lam), want_v):
                assert rel_err(g, w) < 1e-11


# ---- Tet4 element patches ----------------------------------------------------------------
@pytest.mark.parametrize("layout", ["unpatched", "irregular_patches", "shuffled"])
def test_tet4_patch_layouts(gpu, oracle_lib, monkeypatch, layout):
    """The patched Tet4 kernel (contributions summed per patch of tets on <= 8 nodes) and the
    per-element kernel agree with the oracle: patching disabled, patches of uneven size
    (every 7th tet removed), and a shuffled element order (patches too small, so the
    per-element kernel is chosen)."""
    from aperi_mech_b200.model import ExplicitDynamics, Part

    coords, conn = _mesh("tet4", 5, seed=6)
    if layout == "unpatched":
        monkeypatch.setenv("APERI_B200_TET4_PATCHES", "0")
    elif layout == "irregular_patches":
        conn = conn[np.arange(conn.shape[0]) % 7 != 3]
    else:
        conn = conn[np.random.default_rng(0).permutation(conn.shape[0])]
    mu_f, k_f = _fields(conn.shape[0], 5, True)
    parts = [Part("tet4", _material("neo_hookean"), conn=conn, mu_field=mu_f, kappa_field=k_f)]
    rng = np.random.default_rng(2)
    u = 1e-3 * rng.standard_normal(coords.shape)
    lam = rng.standard_normal(coords.shape)
    op = oracle_lib.OracleProblem(coords, parts)
    with ExplicitDynamics(coords, parts) as m:
        assert rel_err(m.internal_force(u), op.internal_force(u)) < FP64_TOL
        assert rel_err(m.internal_force(u, "mixed"), op.internal_force(u)) < MIXED_FORCE_TOL
        assert rel_err(m.mass(), op.lumped_mass()) < 1e-14
        for g, w in zip(m.vjp_force(u, lam), op.vjp_force(u, lam)):
            assert rel_err(g, w) < 1e-11


# ---- domain decomposition on one GPU --------------------------------------------------
@pytest.mark.parametrize("use_nccl", [False, True])
def test_interface_exchange_single_rank_is_exact(gpu, use_nccl):
    """With one rank, the decomposed step (interface gather into the exchange buffer,
    the all-reduce, the node kernel reading interface rows back) must reproduce the
    plain step bit for bit; rows are a random injection into a larger buffer."""
    import os

    from aperi_mech_b200 import mesh, problems
    from aperi_mech_b200.model import ExplicitDynamics, nccl_unique_id

    p = problems.tet4_nh_shear(n=8, seed=3, nsteps=25)
    mass = mesh.lumped_mass(p.coords, p.parts[0].conn, p.parts[0].material.density)
    rng = np.random.default_rng(0)
    iface = np.sort(rng.choice(p.num_nodes, size=p.num_nodes // 3, replace=False)).astype(np.int32)
    rows = rng.permutation(2 * iface.size)[: iface.size].astype(np.int32)
    out = {}
    for decomposed in (False, True):
        with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
            if decomposed:
                m.set_interface(iface, rows, 2 * iface.size)
                if use_nccl:
                    os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")
                    m.set_nccl(nccl_unique_id(), 0, 1)
            for prec in ("fp64", "mixed"):
                m.set_state(None, p.v0)
                m.init_acceleration(prec)
                m.run(p.nsteps, p.dt, prec)
                out[(decomposed, prec)] = m.get_state()
            out[(decomposed, "f")] = m.internal_force(out[(decomposed, "fp64")][0])
    for key in ("fp64", "mixed"):
        for a, b in zip(out[(False, key)], out[(True, key)]):
            assert np.array_equal(a, b), key
    assert np.array_equal(out[(False, "f")], out[(True, "f")])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_neighbor_exchange_single_rank_self_neighbor(gpu, prec, monkeypatch):
    """The neighbour exchange on one GPU, with the rank as its own neighbour for a subset
    S of the nodes (NCCL sends to self): each node of S then sums its own partial twice
    (own, then the received copy), so the internal force doubles exactly on S and stays
    bitwise equal elsewhere; and the step with the exchange on a second stream under the
    interior nodes' update equals the same step run in sequence, bit for bit."""
    import os

    from aperi_mech_b200 import mesh, problems
    from aperi_mech_b200.model import ExplicitDynamics, nccl_unique_id

    p = problems.tet4_nh_shear(n=8, seed=5, nsteps=20)
    mass = mesh.lumped_mass(p.coords, p.parts[0].conn, p.parts[0].material.density)
    rng = np.random.default_rng(3)
    shared = np.sort(rng.choice(p.num_nodes, size=p.num_nodes // 4, replace=False)).astype(np.int32)
    u = 1e-4 * rng.standard_normal(p.coords.shape)
    os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")
    with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
        f_plain = m.internal_force(u, prec)
    runs = {}
    for overlap in ("1", "0"):
        monkeypatch.setenv("APERI_B200_EXCHANGE_OVERLAP", overlap)
        with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
            m.set_neighbors(0, np.array([0]), np.array([0, shared.size]), shared)
            m.set_nccl(nccl_unique_id(), 0, 1)
            f = m.internal_force(u, prec)
            m.set_state(None, p.v0)
            m.init_acceleration(prec)
            m.run(p.nsteps, p.dt, prec)
            runs[overlap] = m.get_state()
        mask = np.zeros(p.num_nodes, dtype=bool)
        mask[shared] = True
        assert np.array_equal(f[mask], 2.0 * f_plain[mask])
        assert np.array_equal(f[~mask], f_plain[~mask])
    for a, b in zip(runs["1"], runs["0"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["tet4_nh", "hex8_le", "cells", "rkpm", "fbar"])
def test_graph_replay_is_bitwise_identical(gpu, monkeypatch, name):
    """The step loop replayed from captured CUDA graphs (chunks of 32 steps, captured at
    the end of a precision's first run and replayed from its second) gives bitwise the
    same states as the same runs launched kernel by kernel (APERI_B200_GRAPHS=0). A body
    acceleration set between runs (a kernel argument of the node kernel) reaches the
    replayed steps: the setter drops the captured graphs."""
    import ctypes as C

    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = {"cells": lambda: problems.smoothed_tet4_box(n=4, seed=2, nsteps=80),
         "rkpm": lambda: problems.rkpm_box(n=4, seed=2, nsteps=80),
         "fbar": lambda: problems.rkpm_fbar_box(n=3, seed=2, nsteps=80)}.get(name, lambda: _small_problem(name))()
    mass = p.meta.get("mass")
    g = np.array([0.0, -3.0e2, 1.0e2])
    out = {}
    for graphs in ("1", "0"):
        monkeypatch.setenv("APERI_B200_GRAPHS", graphs)
        res = []
        with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
            for prec in ("fp64", "mixed"):
                for k in range(3):  # the second and third runs of a precision replay a graph
                    if k == 2:
                        rc = m.lib.am_set_body_acceleration(m.ctx, g.ctypes.data_as(C.POINTER(C.c_double)))
                        assert rc == 0
                    m.set_state(None, p.v0)
                    m.init_acceleration(prec)
                    m.run(75, p.dt, prec)
                    res.append(m.get_state())
                rc = m.lib.am_set_body_acceleration(m.ctx, np.zeros(3).ctypes.data_as(C.POINTER(C.c_double)))
                assert rc == 0
        out[graphs] = res
    # the body acceleration changed the third run's state
    assert not np.array_equal(out["0"][1][0], out["0"][2][0])
    for a, b in zip(out["1"], out["0"]):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
