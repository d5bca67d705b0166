"""RKPM one-pass nodal smoothing cells: the oracle's reproducing conditions (CPU) and
the library's GPU set-up, force and time stepping against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err


def _box(n=4, seed=0, jitter=0.2):
    from aperi_mech_b200 import problems

    _, X, T = problems._box_tets(n, seed, jitter)
    return X, T


def _rows(ptr):
    return np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))


@pytest.mark.parametrize("cap", [40, 12])
def test_oracle_rk_reproducing_conditions(oracle_lib, cap):
    """ShapeFunctionsFunctorsTest.cpp:138-272 (partition of unity, linear completeness) and
    SmoothedCellDataTest (partition of nullity of the smoothed gradients), plus exact
    gradients of linear fields, total cell volume and total mass."""
    X, T = _box()
    r = oracle_lib.rkpm_nodal_cells(X, T, np.full(X.shape[0], 1.8 / 4), max_neighbors=cap, density=1000.0)
    P, ptr, nb, v = r["points"], r["nbr_ptr"], r["nbr"], r["values"]
    assert np.all(np.diff(ptr) <= cap)
    rows = _rows(ptr)
    pu = np.bincount(rows, weights=v, minlength=P.shape[0])
    assert np.abs(pu - 1.0).max() < 4e-12
    lc = np.zeros_like(P)
    np.add.at(lc, rows, v[:, None] * X[nb])
    assert np.abs(lc - P).max() < 4e-11
    g, cp, cn = r["cell_grads"], r["cell_ptr"], r["cell_nodes"]
    crow = _rows(cp)
    nul = np.zeros_like(X)
    np.add.at(nul, crow, g)
    assert np.abs(nul).max() < 1e-9
    A = np.random.default_rng(1).standard_normal((3, 3))
    H = np.zeros((X.shape[0], 3, 3))
    np.add.at(H, crow, (X[cn] @ A.T)[:, :, None] * g[:, None, :])
    assert np.abs(H - A).max() < 1e-9
    assert abs(r["cell_volumes"].sum() - 2.0) < 1e-12
    assert abs(r["mass"].sum() - 2000.0) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("cap", [40, 80])
def test_rkpm_setup_matches_oracle(gpu, oracle_lib, cap):
    from aperi_mech_b200.model import Material
    from aperi_mech_b200.rkpm import nodal_cells

    X, T = _box(n=4, seed=3)
    R = np.full(X.shape[0], 1.8 / 4)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    got = nodal_cells(X, T, mat, R, max_neighbors=cap, keep_points=True)
    want = oracle_lib.rkpm_nodal_cells(X, T, R, max_neighbors=cap, density=1000.0)
    assert np.array_equal(got.points, want["points"])
    assert np.array_equal(got.nbr_ptr, want["nbr_ptr"]) and np.array_equal(got.nbr, want["nbr"])
    assert rel_err(got.values, want["values"]) < 1e-12
    part = got.part
    assert np.array_equal(part.cell_ptr, want["cell_ptr"]) and np.array_equal(part.cell_nodes, want["cell_nodes"])
    assert rel_err(part.cell_grads, want["cell_grads"]) < 1e-12
    assert rel_err(part.cell_volumes, want["cell_volumes"]) < 1e-13
    assert rel_err(got.mass, want["mass"]) < 1e-12


@pytest.mark.gpu
def test_rkpm_force_and_steps_match_oracle(gpu, oracle_lib):
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.rkpm_box(n=4, seed=2, nsteps=40)
    mass = p.meta["mass"]
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=mass)
    rng = np.random.default_rng(0)
    u = 1e-3 * rng.standard_normal(p.coords.shape)
    lam = rng.standard_normal(p.coords.shape)
    want_f = op.internal_force(u)
    with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
        assert rel_err(m.internal_force(u), want_f) < 1e-12
        assert rel_err(m.internal_force(u, "mixed"), want_f) < 5e-5
        for g, w in zip(m.vjp_force(u, lam), op.vjp_force(u, lam)):
            assert rel_err(g, w) < 1e-11
        m.set_state(None, p.v0)
        m.init_acceleration()
        m.run(p.nsteps, p.dt)
        got = m.get_state()
    zero = np.zeros_like(p.coords)
    want = op.steps(zero, p.v0, op.init_acceleration(zero), np.full(p.nsteps, p.dt))
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-12


@pytest.mark.gpu
def test_rkpm_cell_stress_form(gpu, oracle_lib, monkeypatch):
    """The generic cell path runs in the cell-stress form by default (per cell -V P, then a
    node-major gather into one slot per node). With one, two or four rows per lane in flight
    (APERI_B200_CELL_UNROLL) every lane sums its rows in the same order, so the
    forces, gradients and states are bitwise equal; the per-entry slot form
    (APERI_B200_CELL_GATHER=0) sums in another order and agrees with the oracle as closely."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.rkpm_box(n=4, seed=5, nsteps=30)
    mass = p.meta["mass"]
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=mass)
    rng = np.random.default_rng(3)
    u = 1e-3 * rng.standard_normal(p.coords.shape)
    lam = rng.standard_normal(p.coords.shape)
    want_f = op.internal_force(u)
    out = {}
    for gather, unroll in (("1", "1111"), ("1", "2222"), ("1", "4444"), ("0", "4444")):
        monkeypatch.setenv("APERI_B200_CELL_GATHER", gather)
        monkeypatch.setenv("APERI_B200_CELL_UNROLL", unroll)
        with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
            f = m.internal_force(u)
            fm = m.internal_force(u, "mixed")
            g = m.vjp_force(u, lam)
            m.set_state(None, p.v0)
            m.init_acceleration("mixed")
            m.run(p.nsteps, p.dt, "mixed")
            out[gather, unroll] = (f, fm, *g, *m.get_state())
        assert rel_err(f, want_f) < 1e-12
        assert rel_err(fm, want_f) < 5e-5
    for key in (("1", "1111"), ("1", "2222")):
        for a, b in zip(out[key], out["1", "4444"]):
            assert np.array_equal(a, b)
    for a, b in zip(out["0", "4444"][2:5], out["1", "4444"][2:5]):
        assert rel_err(a, b) < 1e-11


@pytest.mark.gpu
def test_rkpm_linear_field_patch(gpu):
    """Linear displacement -> every nodal cell's displacement gradient is exact, so the
    forces of a linear-elastic body in constant stress vanish away from the boundary."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import ExplicitDynamics, Material
    from aperi_mech_b200.rkpm import nodal_cells

    X, T = _box(n=8, seed=4)
    mat = Material.create("linear_elastic", 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)
    cells = nodal_cells(X, T, mat, np.full(X.shape[0], 1.8 / 8))
    A = 1e-3 * np.random.default_rng(5).standard_normal((3, 3))
    with ExplicitDynamics(X, [cells.part], mass=cells.mass) as m:
        f = m.internal_force(X @ A.T)
    # nodes whose cell and neighbours stay off the boundary (2 layers in)
    lo, hi = X.min(axis=0), X.max(axis=0)
    deep = np.all((X > lo + 2.5 / 8) & (X < hi - 2.5 / 8), axis=1)
    assert deep.sum() > 0
    assert np.abs(f[deep]).max() < 1e-9 * np.abs(f).max()


# ---- element smoothing cells with the reproducing-kernel space --------------------------
def _tet_radius(X, T, scale):
    from aperi_mech_b200.rkpm import tet_max_edge_length

    return scale * tet_max_edge_length(X, T)


def test_oracle_rk_element_cells_reproducing_conditions(oracle_lib):
    """Element cells: partition of unity and linear completeness of the vertex functions,
    partition of nullity and exact linear-field gradients per tet cell, total volume and
    total mass, entries capped by the four vertices' neighbour lists."""
    X, T = _box(n=4, seed=1)
    r = oracle_lib.rkpm_element_cells(X, T, _tet_radius(X, T, 1.1), max_neighbors=40, density=1000.0)
    ptr, nb, v = r["nbr_ptr"], r["nbr"], r["values"]
    rows = _rows(ptr)
    assert np.abs(np.bincount(rows, weights=v, minlength=X.shape[0]) - 1.0).max() < 4e-12
    lc = np.zeros_like(X)
    np.add.at(lc, rows, v[:, None] * X[nb])
    assert np.abs(lc - X).max() < 4e-11
    g, cp, cn = r["cell_grads"], r["cell_ptr"], r["cell_nodes"]
    assert len(cp) == T.shape[0] + 1
    crow = _rows(cp)
    nul = np.zeros((T.shape[0], 3))
    np.add.at(nul, crow, g)
    assert np.abs(nul).max() < 1e-9
    A = np.random.default_rng(2).standard_normal((3, 3))
    H = np.zeros((T.shape[0], 3, 3))
    np.add.at(H, crow, (X[cn] @ A.T)[:, :, None] * g[:, None, :])
    assert np.abs(H - A).max() < 1e-9
    assert np.all(np.diff(cp) <= 4 * 40)
    assert abs(r["cell_volumes"].sum() - 2.0) < 1e-12
    assert abs(r["mass"].sum() - 2000.0) < 1e-9


@pytest.mark.gpu
def test_rkpm_element_cells_setup_force_and_steps_match_oracle(gpu, oracle_lib):
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics, Material
    from aperi_mech_b200.rkpm import element_cells

    X, T = _box(n=4, seed=5)
    R = _tet_radius(X, T, 1.1)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    got = element_cells(X, T, mat, R, keep_points=True)
    want = oracle_lib.rkpm_element_cells(X, T, R, max_neighbors=40, density=1000.0)
    assert np.array_equal(got.nbr_ptr, want["nbr_ptr"]) and np.array_equal(got.nbr, want["nbr"])
    assert rel_err(got.values, want["values"]) < 1e-12
    part = got.part
    assert np.array_equal(part.cell_ptr, want["cell_ptr"]) and np.array_equal(part.cell_nodes, want["cell_nodes"])
    assert rel_err(part.cell_grads, want["cell_grads"]) < 1e-12
    assert rel_err(part.cell_volumes, want["cell_volumes"]) < 1e-13
    assert rel_err(got.mass, want["mass"]) < 1e-12
    fixed = mesh.side_sets(X)["surface_5"]
    bcs = [BoundaryCondition.fixed(fixed)]
    rng = np.random.default_rng(3)
    v0 = rng.uniform(-0.01, 0.01, size=X.shape)
    v0[:, 0] += X[:, 2]
    v0[fixed] = 0.0
    u = 1e-3 * rng.standard_normal(X.shape)
    op = oracle_lib.OracleProblem(X, [part], bcs, mass=got.mass)
    dt = 0.5 * float(mesh.tet_char_length(X, T).min()) / np.sqrt((mat.lam + 2 * mat.mu) / mat.density)
    with ExplicitDynamics(X, [part], bcs, mass=got.mass) as m:
        assert rel_err(m.internal_force(u), op.internal_force(u)) < 1e-12
        assert rel_err(m.internal_force(u, "mixed"), op.internal_force(u)) < 5e-5
        m.set_state(None, v0)
        m.init_acceleration()
        m.run(30, dt)
        got_state = m.get_state()
    zero = np.zeros_like(X)
    want_state = op.steps(zero, v0, op.init_acceleration(zero), np.full(30, dt))
    for g, w in zip(got_state, want_state):
        assert rel_err(g, w) < 1e-12


# ---- two-pass method on element cells (the reference's default for element cells) ------
def _two_pass_inputs(oracle_lib, X, T, mat, scale=1.1):
    """Oracle functions and generalized mass at the vertices, FEM smoothed tet cells."""
    from aperi_mech_b200.smoothing import element_smoothing_part

    r = oracle_lib.rkpm_element_cells(X, T, _tet_radius(X, T, scale), max_neighbors=40, density=mat.density)
    part, _ = element_smoothing_part(X, T, mat)
    return part, r["mass"], (r["nbr_ptr"], r["nbr"], r["values"])


def _dense(rk, N):
    ptr, nb, v = rk
    Psi = np.zeros((N, N))
    np.add.at(Psi, (_rows(ptr), nb), v)
    return Psi


def test_oracle_two_pass_is_psi_transpose_fem_psi(oracle_lib):
    """ExplicitSolver::ComputeForce with the two-pass method: f = Psi^T F_fem(Psi d); the
    work identity d . f = (Psi d) . F_fem and a zero force sum (partition of unity)."""
    from aperi_mech_b200.model import Material

    X, T = _box(n=4, seed=6)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    part, mass, rk = _two_pass_inputs(oracle_lib, X, T, mat)
    Psi = _dense(rk, X.shape[0])
    d = 1e-3 * np.random.default_rng(2).standard_normal(X.shape)
    fem = oracle_lib.OracleProblem(X, [part]).internal_force(Psi @ d)
    got = oracle_lib.OracleProblem(X, [part], mass=mass, rk=rk).internal_force(d)
    assert rel_err(got, Psi.T @ fem) < 1e-13
    assert abs(np.sum(got * d) - np.sum(fem * (Psi @ d))) < 1e-12 * np.abs(fem).max() * np.abs(d).max() * d.size
    assert np.abs(got.sum(axis=0)).max() < 1e-9 * np.abs(got).max()
    assert abs(mass.sum() - 2000.0) < 1e-9


def test_oracle_two_pass_vjp_is_psi_transpose_fem_vjp(oracle_lib):
    """The VJP of the composed force f = Psi^T F(Psi d): Psi^T VJP_F(Psi d, Psi lam), with the
    modulus gradients of F at (Psi d, Psi lam); and lam . f against central differences."""
    from aperi_mech_b200.model import Material

    X, T = _box(n=3, seed=7)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    part, mass, rk = _two_pass_inputs(oracle_lib, X, T, mat)
    Psi = _dense(rk, X.shape[0])
    rng = np.random.default_rng(5)
    d = 1e-3 * rng.standard_normal(X.shape)
    lam = rng.standard_normal(X.shape)
    op = oracle_lib.OracleProblem(X, [part], mass=mass, rk=rk)
    gu, gm, gk = op.vjp_force(d, lam)
    fu, fm, fk = oracle_lib.OracleProblem(X, [part]).vjp_force(Psi @ d, Psi @ lam)
    assert rel_err(gu, Psi.T @ fu) < 1e-13
    assert rel_err(gm, fm) < 1e-13 and rel_err(gk, fk) < 1e-13
    dirn = rng.standard_normal(X.shape)
    h = 1e-6
    fd = (np.sum(lam * op.internal_force(d + h * dirn)) - np.sum(lam * op.internal_force(d - h * dirn))) / (2 * h)
    assert abs(np.sum(gu * dirn) - fd) < 1e-5 * abs(fd)


SHEAR = [(1, 0), (2, 0), (0, 1), (2, 1), (0, 2), (1, 2)]


@pytest.mark.parametrize("direction,surface", SHEAR)
def test_oracle_two_pass_shear_patch(oracle_lib, direction, surface):
    """ForceTest.cpp ExplicitShearForceReproducingKernel (element smoothing cells, the
    two-pass default, kernel radius scale 1.1, PatchTestFixture.h:118-123): mass, the
    physical displacement gradient of every cell, zero acceleration, the local force of
    each surface pair +/- P n A, the physical displacement and velocity of the faces."""
    from helpers import expected_pk1, prescribed_patch

    mag = 0.1
    X, parts, bcs, sets = prescribed_patch("tet4", (1, 1, 1), direction, surface, mag)
    mat = parts[0].material
    part, mass, rk = _two_pass_inputs(oracle_lib, X, parts[0].conn, mat)
    op = oracle_lib.OracleProblem(X, [part], bcs, mass=mass, rk=rk)
    d, v, a, _ = op.solve(np.zeros_like(X), np.zeros_like(X), 0.1, 10.0)
    Psi = _dense(rk, X.shape[0])
    u, vp = Psi @ d, Psi @ v
    H = np.zeros((3, 3))
    H[direction, surface] = 2.0 * mag
    assert abs(mass.sum() - 0.08) < 1e-12
    B = part.cell_grads.reshape(-1, 4, 3)
    conn = part.cell_nodes.reshape(-1, 4)
    for c in range(conn.shape[0]):
        assert np.abs(u[conn[c]].T @ B[c] - H).max() < 1e-9
    assert np.abs(a).max() < 1e-12
    f_local = oracle_lib.OracleProblem(X, [part]).internal_force(u)
    P = expected_pk1(H, mat)
    for i in range(3):
        n_i = np.zeros(3)
        n_i[i] = 1.0
        assert np.abs(f_local[sets[f"surface_{2 * i + 1}"]].sum(axis=0) - P @ n_i).max() < 1e-8
        assert np.abs(f_local[sets[f"surface_{2 * i + 2}"]].sum(axis=0) + P @ n_i).max() < 1e-8
    s_lo, s_hi = sets[f"surface_{2 * surface + 1}"], sets[f"surface_{2 * surface + 2}"]
    dd = np.zeros(3)
    dd[direction] = mag
    assert np.abs(u[s_hi] - dd).max() < 1e-9 and np.abs(u[s_lo] + dd).max() < 1e-9
    assert np.abs(vp[s_hi] - 1.875 * dd / 10.0).max() < 1e-4


@pytest.mark.gpu
def test_rkpm_two_pass_vjp_and_adjoint_match_oracle(gpu, oracle_lib):
    """The library's VJP and checkpointed adjoint with the two-pass coupling against the
    oracle's (its reverse pass stores every state): u-VJP at 1e-11, loss at 1e-12, modulus
    gradients at 1e-10."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.rkpm_two_pass_box(n=4, seed=2, nsteps=20)
    mass, rk = p.meta["mass"], p.meta["rk"]
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=mass, rk=rk)
    rng = np.random.default_rng(8)
    u = 1e-3 * rng.standard_normal(p.coords.shape)
    lam = rng.standard_normal(p.coords.shape)
    sens = np.arange(0, p.coords.shape[0], 7, dtype=np.int32)[:16]
    with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass, rk=rk) as m:
        for g, w in zip(m.vjp_force(u, lam), op.vjp_force(u, lam)):
            assert rel_err(g, w) < 1e-11
        m.set_state(None, p.v0)
        loss, gm, gk = m.adjoint(p.nsteps, p.dt, 5, sens)
    wl, wm, wk = op.adjoint(p.nsteps, p.dt, np.zeros_like(p.coords), p.v0, sens)
    assert abs(loss - wl) < 1e-12 * abs(wl)
    assert rel_err(gm, wm) < 1e-10 and rel_err(gk, wk) < 1e-10


@pytest.mark.gpu
def test_rkpm_two_pass_force_and_steps_match_oracle(gpu, oracle_lib):
    """The library's two-pass coupling (set-up, force in FP64 and mixed precision, 30
    steps with a fixed face) against the oracle fed the same functions."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics, Material
    from aperi_mech_b200.rkpm import apply_functions, two_pass_element_cells

    X, T = _box(n=4, seed=7)
    R = _tet_radius(X, T, 1.1)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    cells = two_pass_element_cells(X, T, mat, R)
    part, mass, rk = _two_pass_inputs(oracle_lib, X, T, mat)
    assert np.array_equal(cells.part.cell_nodes, part.cell_nodes)
    assert rel_err(cells.mass, mass) < 1e-12
    assert np.array_equal(cells.nbr_ptr, rk[0]) and np.array_equal(cells.nbr, rk[1])
    assert rel_err(cells.values, rk[2]) < 1e-12
    fixed = mesh.side_sets(X)["surface_5"]
    bcs = [BoundaryCondition.fixed(fixed)]
    rng = np.random.default_rng(4)
    v0 = rng.uniform(-0.01, 0.01, size=X.shape)
    v0[:, 0] += X[:, 2]
    v0[fixed] = 0.0
    u = 1e-3 * rng.standard_normal(X.shape)
    op = oracle_lib.OracleProblem(X, [cells.part], bcs, mass=cells.mass, rk=cells.functions())
    dt = 0.5 * float(mesh.tet_char_length(X, T).min()) / np.sqrt((mat.lam + 2 * mat.mu) / mat.density)
    zero = np.zeros_like(X)
    want_state = op.steps(zero, v0, op.init_acceleration(zero), np.full(30, dt))
    with ExplicitDynamics(X, [cells.part], bcs, mass=cells.mass, rk=cells.functions()) as m:
        assert rel_err(m.internal_force(u), op.internal_force(u)) < 1e-12
        assert rel_err(m.internal_force(u, "mixed"), op.internal_force(u)) < 5e-5
        m.set_state(None, v0)
        m.init_acceleration()
        m.run(30, dt)
        got_state = m.get_state()
        m.set_state(zero, v0)
        m.init_acceleration("mixed")
        m.run(30, dt, "mixed")
        mixed_u = m.get_state()[0]
    for g, w in zip(got_state, want_state):
        assert rel_err(g, w) < 1e-12
    assert rel_err(mixed_u, want_state[0]) < 1e-5
    # the physical displacement reproduces a linear field of the coefficients
    A = 1e-3 * rng.standard_normal((3, 3))
    assert np.abs(apply_functions(cells.functions(), X @ A.T) - X @ A.T).max() < 1e-12


# ---- RKPM element cells on Hex8 meshes (ElementReproducingKernelHex8) ------------------
def _hex_box(n=3, seed=4, jitter=0.15):
    from aperi_mech_b200 import mesh

    coords, conn = mesh.box_hex(n, n, 2 * n, 1.0, 1.0, 2.0)
    return mesh.jitter_interior(coords, jitter / n, np.random.default_rng(seed)), conn


def test_oracle_rk_hex8_element_cells(oracle_lib):
    """Hex cells: partition of unity and linear completeness of the vertex functions,
    partition of nullity and exact linear-field gradients per cell, volume and mass."""
    from aperi_mech_b200.rkpm import tet_max_edge_length

    X, E = _hex_box()
    r = oracle_lib.rkpm_element_cells(X, E, 1.1 * tet_max_edge_length(X, E), max_neighbors=40, density=1000.0)
    ptr, nb, v = r["nbr_ptr"], r["nbr"], r["values"]
    rows = _rows(ptr)
    assert np.abs(np.bincount(rows, weights=v, minlength=X.shape[0]) - 1.0).max() < 4e-12
    lc = np.zeros_like(X)
    np.add.at(lc, rows, v[:, None] * X[nb])
    assert np.abs(lc - X).max() < 4e-11
    g, cp, cn = r["cell_grads"], r["cell_ptr"], r["cell_nodes"]
    assert len(cp) == E.shape[0] + 1
    crow = _rows(cp)
    nul = np.zeros((E.shape[0], 3))
    np.add.at(nul, crow, g)
    assert np.abs(nul).max() < 1e-9
    A = np.random.default_rng(2).standard_normal((3, 3))
    H = np.zeros((E.shape[0], 3, 3))
    np.add.at(H, crow, (X[cn] @ A.T)[:, :, None] * g[:, None, :])
    assert np.abs(H - A).max() < 1e-9
    assert abs(r["cell_volumes"].sum() - 2.0) < 1e-12
    assert abs(r["mass"].sum() - 2000.0) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["one_pass", "two_pass"])
def test_rk_hex8_element_cells_match_oracle(gpu, oracle_lib, method):
    """Set-up against the oracle, then force and 20 steps (one-pass cells, or the two-pass
    coupling of the smoothed hexes) at 1e-12."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics, Material
    from aperi_mech_b200.rkpm import element_cells, tet_max_edge_length, two_pass_element_cells

    X, E = _hex_box(seed=6)
    R = 1.1 * tet_max_edge_length(X, E)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    want = oracle_lib.rkpm_element_cells(X, E, R, max_neighbors=40, density=1000.0)
    if method == "one_pass":
        cells = element_cells(X, E, mat, R, keep_points=True)
        p = cells.part
        assert np.array_equal(p.cell_ptr, want["cell_ptr"]) and np.array_equal(p.cell_nodes, want["cell_nodes"])
        assert rel_err(p.cell_grads, want["cell_grads"]) < 1e-12
        rk = None
    else:
        cells = two_pass_element_cells(X, E, mat, R)
        rk = cells.functions()
    assert np.array_equal(cells.nbr_ptr, want["nbr_ptr"]) and np.array_equal(cells.nbr, want["nbr"])
    assert rel_err(cells.values, want["values"]) < 1e-12
    assert rel_err(cells.mass, want["mass"]) < 1e-12
    fixed = mesh.side_sets(X)["surface_5"]
    bcs = [BoundaryCondition.fixed(fixed)]
    rng = np.random.default_rng(8)
    v0 = rng.uniform(-0.01, 0.01, size=X.shape)
    v0[:, 0] += X[:, 2]
    v0[fixed] = 0.0
    u = 1e-3 * rng.standard_normal(X.shape)
    op = oracle_lib.OracleProblem(X, [cells.part], bcs, mass=cells.mass, rk=rk)
    dt = 0.3 * (1.0 / 3.0) / np.sqrt((mat.lam + 2 * mat.mu) / mat.density)
    zero = np.zeros_like(X)
    want_state = op.steps(zero, v0, op.init_acceleration(zero), np.full(20, dt))
    with ExplicitDynamics(X, [cells.part], bcs, mass=cells.mass, rk=rk) as m:
        assert rel_err(m.internal_force(u), op.internal_force(u)) < 1e-12
        m.set_state(None, v0)
        m.init_acceleration()
        m.run(20, dt)
        got = m.get_state()
    for g, w in zip(got, want_state):
        assert rel_err(g, w) < 1e-12


# ---- two-pass method on nodal cells (force_two_pass_method with nodal_smoothing_cell) ---
def _two_pass_nodal(oracle_lib, X, T, mat, R):
    """Oracle two-pass nodal cells: the cells over the thex points, the functions at the
    points (P rows), the generalized mass at the vertices."""
    from aperi_mech_b200.model import Part

    r = oracle_lib.rkpm_nodal_cells(X, T, R, max_neighbors=40, density=mat.density, two_pass=True)
    part = Part("cells", mat, cell_ptr=r["cell_ptr"], cell_nodes=r["cell_nodes"], cell_grads=r["cell_grads"],
                cell_volumes=r["cell_volumes"])
    return part, r["mass"], (r["nbr_ptr"], r["nbr"], r["values"]), r["points"]


def _dense_rect(rk, P, N):
    ptr, nb, v = rk
    Psi = np.zeros((P, N))
    np.add.at(Psi, (_rows(ptr), nb), v)
    return Psi


def test_oracle_two_pass_nodal_cells(oracle_lib):
    """Two-pass nodal cells: each vertex cell holds its corner-hex points with the hexes'
    smoothed gradients (partition of nullity: they sum to zero; a linear field gives its
    gradient exactly), the first N points are the vertices, and f = Psi^T F_fem(Psi d)
    with Psi the P x N functions at the points; the work identity d . f = (Psi d) . F_fem."""
    from aperi_mech_b200.model import Material

    X, T = _box(n=3, seed=8)
    N = X.shape[0]
    R = np.full(N, 1.8 / 3)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    part, mass, rk, points = _two_pass_nodal(oracle_lib, X, T, mat, R)
    P = points.shape[0]
    assert P > N and np.array_equal(points[:N], X)
    assert part.cell_nodes.max() < P
    ptr, g = part.cell_ptr, part.cell_grads
    A = np.array([[0.3, -0.1, 0.2], [0.05, 0.4, -0.3], [0.1, 0.2, -0.2]])
    for c in range(N):
        s = slice(ptr[c], ptr[c + 1])
        assert np.abs(g[s].sum(axis=0)).max() < 1e-9 * np.abs(g[s]).max()
        H = (points[part.cell_nodes[s]] @ A.T).T @ g[s]
        assert np.abs(H - A).max() < 1e-11
    Psi = _dense_rect(rk, P, N)
    d = 1e-3 * np.random.default_rng(4).standard_normal(X.shape)
    fem = oracle_lib.OracleProblem(points, [part]).internal_force(Psi @ d)
    got = oracle_lib.OracleProblem(X, [part], mass=mass, rk=rk).internal_force(d)
    assert rel_err(got, Psi.T @ fem) < 1e-13
    assert abs(np.sum(got * d) - np.sum(fem * (Psi @ d))) < 1e-12 * np.abs(fem).max() * np.abs(d).max() * d.size
    one = oracle_lib.rkpm_nodal_cells(X, T, R, max_neighbors=40, density=mat.density)
    assert rel_err(mass, one["mass"]) < 1e-14


@pytest.mark.gpu
def test_rkpm_two_pass_nodal_force_and_steps_match_oracle(gpu, oracle_lib):
    """Two-pass nodal cells through the library (set-up, P-row coupling, force, 20 steps
    in FP64 and mixed) against the oracle at 1e-12 (FP64) and 1e-5 (mixed)."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics, Material
    from aperi_mech_b200.rkpm import two_pass_nodal_cells

    X, T = _box(n=3, seed=9)
    N = X.shape[0]
    R = np.full(N, 1.8 / 3)
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    cells = two_pass_nodal_cells(X, T, mat, R)
    part, mass, rk, points = _two_pass_nodal(oracle_lib, X, T, mat, R)
    assert np.array_equal(cells.points, points)
    assert np.array_equal(cells.nbr_ptr, rk[0]) and np.array_equal(cells.nbr, rk[1])
    assert rel_err(cells.values, rk[2]) < 1e-12
    assert np.array_equal(cells.part.cell_ptr, part.cell_ptr) and np.array_equal(cells.part.cell_nodes, part.cell_nodes)
    assert rel_err(cells.part.cell_grads, part.cell_grads) < 1e-12
    assert rel_err(cells.part.cell_volumes, part.cell_volumes) < 1e-13
    assert rel_err(cells.mass, mass) < 1e-12
    bcs = [BoundaryCondition.fixed(mesh.side_sets(X)["surface_5"])]
    op = oracle_lib.OracleProblem(X, [cells.part], bcs, mass=cells.mass, rk=cells.functions())
    rng = np.random.default_rng(10)
    d = 1e-4 * rng.standard_normal(X.shape)
    v0 = rng.uniform(-0.01, 0.01, size=X.shape)
    v0[bcs[0].nodes] = 0.0
    dt = 2e-7
    z = np.zeros_like(X)
    want = op.steps(z, v0, op.init_acceleration(z), np.full(20, dt))
    with ExplicitDynamics(X, [cells.part], bcs, mass=cells.mass, rk=cells.functions()) as m:
        assert rel_err(m.internal_force(d), op.internal_force(d)) < 1e-12
        assert rel_err(m.internal_force(d, "mixed"), op.internal_force(d)) < 1e-5
        m.set_state(None, v0)
        m.init_acceleration()
        m.run(20, dt)
        got = m.get_state()
        m.set_state(None, v0)
        m.init_acceleration("mixed")
        m.run(20, dt, "mixed")
        mixed = m.get_state()
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-12
    assert rel_err(mixed[0], want[0]) < 1e-5
