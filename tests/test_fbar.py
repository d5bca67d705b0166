"""F-bar smoothed cells (use_f_bar on nodal cells split into corner-hex subcells,
subdomains 0): the oracle's restatement against properties the reference's formulation
has (linear fields reduce to the plain subcell forces, rigid rotations carry no force,
the un-barred stress is the exact derivative of the F-bar energy), and the library's
set-up and forces against the oracle (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err

RADIUS = 1.8


def _box(n=3, seed=0, jitter=0.2):
    from aperi_mech_b200 import problems

    _, X, T = problems._box_tets(n, seed, jitter)
    return X, T


def _rows(ptr):
    return np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))


def _material(kind):
    from aperi_mech_b200.model import Material

    if kind == "neo_hookean":
        return Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    if kind == "elastic":
        return Material.create("elastic", 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)
    return Material.create("linear_elastic", 1000.0, youngs_modulus=1e9, poissons_ratio=0.45)


def _oracle_parts(oracle_lib, X, T, mat, n):
    """(F-bar part, the same subcells without groups) from the oracle's set-up."""
    from aperi_mech_b200.model import Part

    r = oracle_lib.rkpm_nodal_subcells(X, T, np.full(X.shape[0], RADIUS / n), density=mat.density)
    common = dict(cell_ptr=r["cell_ptr"], cell_nodes=r["cell_nodes"], cell_grads=r["cell_grads"],
                  cell_volumes=r["cell_volumes"])
    return Part("cells", mat, cell_groups=r["group_ptr"], **common), Part("cells", mat, **common), r


def test_oracle_subcells_aggregate_to_the_nodal_cells(oracle_lib):
    """A vertex cell is the volume-weighted union of its corner-hex subcells
    (SmoothedCellDataProcessor.h:541-675): sum_s V_s b_s / V_v and sum_s V_s equal the
    one-pass nodal cell's gradients and volume."""
    n = 3
    X, T = _box(n, seed=2)
    R = np.full(X.shape[0], RADIUS / n)
    sub = oracle_lib.rkpm_nodal_subcells(X, T, R)
    cells = oracle_lib.rkpm_nodal_cells(X, T, R)
    N = X.shape[0]
    g = sub["group_ptr"]
    assert g.size == N + 1 and g[-1] == 4 * T.shape[0] == sub["cell_volumes"].size
    srow = _rows(sub["cell_ptr"])
    vol_of_group = np.add.reduceat(sub["cell_volumes"], g[:-1])
    assert rel_err(vol_of_group, cells["cell_volumes"]) < 1e-13
    group_of_sub = _rows(g)
    agg = np.zeros((N, N, 3))
    np.add.at(agg, (group_of_sub[srow], sub["cell_nodes"]),
              sub["cell_grads"] * sub["cell_volumes"][srow][:, None])
    agg /= cells["cell_volumes"][:, None, None]
    want = np.zeros((N, N, 3))
    crow = _rows(cells["cell_ptr"])
    np.add.at(want, (crow, cells["cell_nodes"]), cells["cell_grads"])
    assert np.abs(agg - want).max() < 1e-11 * np.abs(want).max()


@pytest.mark.parametrize("kind", ["neo_hookean", "linear_elastic", "elastic"])
def test_oracle_fbar_linear_field_is_the_plain_subcell_force(oracle_lib, kind):
    """Every subcell reproduces a linear field, so all J_s equal Jbar, Fbar = F and the
    un-barring adds nothing: the F-bar force equals the plain subcell force."""
    n = 3
    X, T = _box(n, seed=3)
    mat = _material(kind)
    fb, plain, _ = _oracle_parts(oracle_lib, X, T, mat, n)
    A = 2e-3 * np.random.default_rng(1).standard_normal((3, 3))
    u = X @ A.T
    f_bar = oracle_lib.OracleProblem(X, [fb]).internal_force(u)
    f_plain = oracle_lib.OracleProblem(X, [plain]).internal_force(u)
    assert rel_err(f_bar, f_plain) < 1e-11


@pytest.mark.parametrize("kind", ["neo_hookean", "elastic"])
def test_oracle_fbar_rigid_rotation_has_no_force(oracle_lib, kind):
    """KinematicsTest.cpp NodalReproducingKernelFbarSimpleRotation: a rotation leaves the
    F-bar Green-Lagrange strain at zero, so a finite-strain material carries no force."""
    n = 3
    X, T = _box(n, seed=4)
    mat = _material(kind)
    fb, _, _ = _oracle_parts(oracle_lib, X, T, mat, n)
    th = 0.3
    Rz = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]])
    op = oracle_lib.OracleProblem(X, [fb])
    f_rot = op.internal_force(X @ Rz.T - X)
    scale = np.abs(op.internal_force(1e-2 * X)).max()
    assert np.abs(f_rot).max() < 1e-8 * scale


def _energy(part, X, u, mat):
    """sum_s V_s psi(Fbar_s) for the material's strain energy."""
    ptr, g = part.cell_ptr, part.cell_groups
    rows = _rows(ptr)
    H = np.zeros((ptr.size - 1, 3, 3))
    np.add.at(H, rows, u[part.cell_nodes][:, :, None] * part.cell_grads[:, None, :])
    F = H + np.eye(3)
    J = np.linalg.det(F)
    V = part.cell_volumes
    grp = _rows(g)
    Jbar = (np.add.reduceat(J * V, g[:-1]) / np.add.reduceat(V, g[:-1]))[grp]
    Fb = np.cbrt(Jbar / J)[:, None, None] * F
    lam, mu = mat.lam, mat.mu
    if mat.kind == "neo_hookean":
        Jb = np.linalg.det(Fb)
        C = np.einsum("ski,skj->sij", Fb, Fb)
        psi = 0.5 * mu * (np.trace(C, axis1=1, axis2=2) - 3) - mu * np.log(Jb) + 0.5 * lam * np.log(Jb) ** 2
    else:
        Hb = Fb - np.eye(3)
        eps = 0.5 * (Hb + np.transpose(Hb, (0, 2, 1)))
        tr = np.trace(eps, axis1=1, axis2=2)
        psi = 0.5 * lam * tr ** 2 + mu * np.einsum("sij,sij->s", eps, eps)
    return float(np.sum(V * psi))


@pytest.mark.parametrize("kind", ["neo_hookean", "linear_elastic"])
def test_oracle_fbar_force_is_the_energy_gradient(oracle_lib, kind):
    """The un-barred stress (ComputeInternalForceSmoothedCell.h:227-309) is the exact
    derivative of the F-bar energy: -f . d equals the central difference of
    sum_s V_s psi(Fbar_s) along d."""
    n = 3
    X, T = _box(n, seed=5)
    mat = _material(kind)
    fb, _, _ = _oracle_parts(oracle_lib, X, T, mat, n)
    rng = np.random.default_rng(6)
    u = 1e-2 * rng.standard_normal(X.shape)
    f = oracle_lib.OracleProblem(X, [fb]).internal_force(u)
    for _ in range(3):
        d = rng.standard_normal(X.shape)
        h = 1e-6
        fd = (_energy(fb, X, u + h * d, mat) - _energy(fb, X, u - h * d, mat)) / (2 * h)
        assert abs(fd + np.sum(f * d)) < 1e-6 * abs(fd)


def _with_empty_subcell(p0, mat, mu_field=None, kappa_field=None):
    """The part with an empty subcell (no entries, the next subcell's volume) inserted at
    the front of the second cell."""
    from aperi_mech_b200.model import Part

    s = int(p0.cell_groups[1])
    ptr = np.insert(p0.cell_ptr, s, p0.cell_ptr[s])
    vols = np.insert(p0.cell_volumes, s, p0.cell_volumes[s])
    groups = np.array(p0.cell_groups, dtype=np.int64)
    groups[2:] += 1
    return Part("cells", mat, cell_ptr=ptr, cell_nodes=p0.cell_nodes, cell_grads=p0.cell_grads, cell_volumes=vols,
                cell_groups=groups, mu_field=mu_field, kappa_field=kappa_field), s


def _fields(mat, n, seed):
    rng = np.random.default_rng(seed)
    kappa = mat.lam + 2.0 * mat.mu / 3.0
    return mat.mu * np.exp(0.2 * rng.standard_normal(n)), kappa * np.exp(0.2 * rng.standard_normal(n))


@pytest.mark.parametrize("kind", ["neo_hookean", "linear_elastic", "elastic"])
def test_oracle_fbar_vjp_matches_finite_differences(oracle_lib, kind):
    """VJP of the F-bar force (the adjoint extension): lam . (df/du) d and the per-subcell
    shear and bulk modulus gradients of lam . f against central differences, on a part with
    modulus fields and an empty subcell (which still enters J-bar, so its moduli matter)."""
    n = 3
    X, T = _box(n, seed=10)
    mat = _material(kind)
    fb, _, _ = _oracle_parts(oracle_lib, X, T, mat, n)
    mu_f, k_f = _fields(mat, fb.cell_volumes.size + 1, 11)
    part, empty = _with_empty_subcell(fb, mat, mu_f, k_f)
    rng = np.random.default_rng(12)
    u = 1e-2 * rng.standard_normal(X.shape)
    lam = rng.standard_normal(X.shape)
    gu, gm, gk = oracle_lib.OracleProblem(X, [part]).vjp_force(u, lam)

    def lam_f(uu):
        return float(np.sum(lam * oracle_lib.OracleProblem(X, [part]).internal_force(uu)))

    h = 1e-6
    for _ in range(2):
        d = rng.standard_normal(X.shape)
        fd = (lam_f(u + h * d) - lam_f(u - h * d)) / (2 * h)
        assert abs(np.sum(gu * d) - fd) < 1e-6 * abs(fd)
    base = {"mu_field": mu_f, "kappa_field": k_f}
    for e in [0, empty, 37, mu_f.size - 1]:
        for field, g in (("mu_field", gm), ("kappa_field", gk)):
            step = 1e-6 * base[field][e]
            vals = []
            for sgn in (1, -1):
                arr = base[field].copy()
                arr[e] += sgn * step
                setattr(part, field, arr)
                vals.append(lam_f(u))
            setattr(part, field, base[field])
            fd = (vals[0] - vals[1]) / (2 * step)
            # roundoff of the differences floors the check at ~1e-9 of the largest gradient
            assert abs(g[e] - fd) < 1e-6 * abs(fd) + 1e-8 * abs(g).max(), (field, e)
    assert gm[empty] != 0.0 and gk[empty] != 0.0


@pytest.mark.gpu
def test_nodal_subcells_setup_matches_oracle(gpu, oracle_lib):
    from aperi_mech_b200.rkpm import nodal_cells, nodal_subcells

    n = 3
    X, T = _box(n, seed=7)
    R = np.full(X.shape[0], RADIUS / n)
    mat = _material("neo_hookean")
    got = nodal_subcells(X, T, mat, R)
    want = oracle_lib.rkpm_nodal_subcells(X, T, R)
    p = got.part
    assert np.array_equal(p.cell_ptr, want["cell_ptr"]) and np.array_equal(p.cell_nodes, want["cell_nodes"])
    assert np.array_equal(p.cell_groups, want["group_ptr"])
    assert rel_err(p.cell_grads, want["cell_grads"]) < 1e-12
    assert rel_err(p.cell_volumes, want["cell_volumes"]) < 1e-13
    assert rel_err(got.mass, nodal_cells(X, T, mat, R).mass) < 1e-13
    assert nodal_subcells(X, T, mat, R, fbar=False).part.cell_groups is None


@pytest.mark.gpu
@pytest.mark.parametrize("passes", ["cell_stress", "fused", "three"])
@pytest.mark.parametrize("kind", ["neo_hookean", "linear_elastic"])
def test_fbar_force_and_steps_match_oracle(gpu, oracle_lib, kind, passes, monkeypatch):
    """F-bar force (FP64 and mixed) and 20 steps with a held face against the oracle: in the
    cell-stress form (the default for cells of at most 32 subcells: H per subcell, M per
    cell, node-major gather), with the one-pass kernel writing per-entry slots
    (APERI_B200_CELL_GATHER=0) and with the three-pass form."""
    from aperi_mech_b200 import mesh

    if passes == "three":
        monkeypatch.setenv("APERI_B200_FBAR_PASSES", "3")
    if passes == "fused":
        monkeypatch.setenv("APERI_B200_CELL_GATHER", "0")
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics
    from aperi_mech_b200.rkpm import nodal_subcells

    n = 3
    X, T = _box(n, seed=8)
    mat = _material(kind)
    cells = nodal_subcells(X, T, mat, np.full(X.shape[0], RADIUS / n))
    fixed = mesh.side_sets(X)["surface_5"]
    bcs = [BoundaryCondition.fixed(fixed)]
    rng = np.random.default_rng(9)
    u = 2e-3 * rng.standard_normal(X.shape)
    v0 = rng.uniform(-0.01, 0.01, size=X.shape)
    v0[:, 0] += X[:, 2]
    v0[fixed] = 0.0
    op = oracle_lib.OracleProblem(X, [cells.part], bcs, mass=cells.mass)
    dt = 0.3 * float(mesh.tet_char_length(X, T).min()) / np.sqrt((mat.lam + 2 * mat.mu) / mat.density)
    zero = np.zeros_like(X)
    want = op.steps(zero, v0, op.init_acceleration(zero), np.full(20, dt))
    with ExplicitDynamics(X, [cells.part], bcs, mass=cells.mass) as m:
        assert rel_err(m.internal_force(u), op.internal_force(u)) < 1e-12
        assert rel_err(m.internal_force(u, "mixed"), op.internal_force(u)) < 1e-4
        m.set_state(None, v0)
        m.init_acceleration()
        m.run(20, dt)
        got = m.get_state()
    # The lane butterflies sum Jbar and the dual pressure in another order than the oracle,
    # and the cube root of Jbar / J_s carries those last bits into every subcell stress:
    # after 20 steps the acceleration differs by about 1e-12 of its size.
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["cell_stress", "fused"])
def test_fbar_empty_subcell_counts_in_jbar(gpu, oracle_lib, form, monkeypatch):
    """A subcell without entries (H = 0, J = 1) still enters its cell's J-bar with its volume:
    an empty subcell inserted at the front of one cell, both F-bar forms against the oracle."""
    from aperi_mech_b200.model import ExplicitDynamics, Part
    from aperi_mech_b200.rkpm import nodal_subcells

    if form == "fused":
        monkeypatch.setenv("APERI_B200_CELL_GATHER", "0")
    n = 3
    X, T = _box(n, seed=8)
    mat = _material("neo_hookean")
    cells = nodal_subcells(X, T, mat, np.full(X.shape[0], RADIUS / n))
    p0 = cells.part
    s = int(p0.cell_groups[1])
    ptr = np.insert(p0.cell_ptr, s, p0.cell_ptr[s])
    vols = np.insert(p0.cell_volumes, s, p0.cell_volumes[s])
    groups = np.array(p0.cell_groups, dtype=np.int64)
    groups[2:] += 1
    part = Part("cells", mat, cell_ptr=ptr, cell_nodes=p0.cell_nodes, cell_grads=p0.cell_grads, cell_volumes=vols,
                cell_groups=groups)
    u = 2e-3 * np.random.default_rng(4).standard_normal(X.shape)
    want = oracle_lib.OracleProblem(X, [part], mass=cells.mass).internal_force(u)
    with ExplicitDynamics(X, [part], mass=cells.mass) as m:
        assert rel_err(m.internal_force(u), want) < 1e-12
        assert rel_err(m.internal_force(u, "mixed"), want) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["neo_hookean", "linear_elastic", "elastic"])
def test_fbar_vjp_and_adjoint_match_oracle(gpu, oracle_lib, kind):
    """The library's F-bar VJP (H and L per subcell by the octet kernel, the per-cell
    derivative, the node-major gather) and the checkpointed adjoint over 20 steps with a
    held face, against the oracle, on a part with modulus fields and an empty subcell:
    u-VJP and modulus VJP at 1e-11, loss at 1e-12, modulus gradients at 1e-10 (the linear
    material's bulk gradient at 1e-9)."""
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, ExplicitDynamics
    from aperi_mech_b200.rkpm import nodal_subcells

    n = 3
    X, T = _box(n, seed=13)
    mat = _material(kind)
    cells = nodal_subcells(X, T, mat, np.full(X.shape[0], RADIUS / n))
    mu_f, k_f = _fields(mat, cells.part.cell_volumes.size + 1, 14)
    part, _ = _with_empty_subcell(cells.part, mat, mu_f, k_f)
    fixed = mesh.side_sets(X)["surface_5"]
    bcs = [BoundaryCondition.fixed(fixed)]
    rng = np.random.default_rng(15)
    u = 2e-3 * rng.standard_normal(X.shape)
    lam = rng.standard_normal(X.shape)
    v0 = rng.uniform(-0.01, 0.01, size=X.shape)
    v0[:, 0] += X[:, 2]
    v0[fixed] = 0.0
    dt = 0.3 * float(mesh.tet_char_length(X, T).min()) / np.sqrt(1.8 * (mat.lam + 2 * mat.mu) / mat.density)
    sens = np.arange(0, X.shape[0], 5, dtype=np.int32)[:16]
    op = oracle_lib.OracleProblem(X, [part], bcs, mass=cells.mass)
    with ExplicitDynamics(X, [part], bcs, mass=cells.mass) as m:
        for g, w in zip(m.vjp_force(u, lam), op.vjp_force(u, lam)):
            assert rel_err(g, w) < 1e-11
        m.set_state(None, v0)
        loss, gm, gk = m.adjoint(20, dt, 5, sens)
    wl, wm, wk = op.adjoint(20, dt, np.zeros_like(X), v0, sens)
    assert abs(loss - wl) < 1e-12 * abs(wl)
    assert rel_err(gm, wm) < 1e-10
    # F-bar takes the volumetric response from J-bar, so the bulk gradient is what is left of
    # the subcells' volumetric terms after they cancel: for the linear material ~1e-2 of the
    # shear gradient, with the trajectory's last bits (~1e-12) amplified into ~1e-10 of it.
    assert rel_err(gk, wk) < (1e-9 if kind == "linear_elastic" else 1e-10)


@pytest.mark.gpu
def test_fbar_vjp_refused_outside_the_cell_stress_form(gpu, oracle_lib, monkeypatch):
    """The three-pass F-bar form keeps no per-subcell L beside H: the VJP and the adjoint
    refuse it (AM_ESTATE) and the context stays usable."""
    from aperi_mech_b200.capi import AM_ESTATE, AmError
    from aperi_mech_b200.model import ExplicitDynamics
    from aperi_mech_b200.rkpm import nodal_subcells

    monkeypatch.setenv("APERI_B200_FBAR_PASSES", "3")
    n = 3
    X, T = _box(n, seed=8)
    mat = _material("neo_hookean")
    cells = nodal_subcells(X, T, mat, np.full(X.shape[0], RADIUS / n))
    u = 2e-3 * np.random.default_rng(4).standard_normal(X.shape)
    with ExplicitDynamics(X, [cells.part], mass=cells.mass) as m:
        with pytest.raises(AmError) as e:
            m.vjp_force(u, u)
        assert e.value.code == AM_ESTATE
        with pytest.raises(AmError) as e:
            m.adjoint(4, 1e-7, 2, np.arange(4, dtype=np.int32))
        assert e.value.code == AM_ESTATE
        want = oracle_lib.OracleProblem(X, [cells.part], mass=cells.mass).internal_force(u)
        assert rel_err(m.internal_force(u), want) < 1e-12


@pytest.mark.parametrize("kind", ["neo_hookean", "elastic"])
def test_oracle_fbar_vjp_is_symmetric(oracle_lib, kind):
    """The F-bar force is the gradient of sum_s V_s psi(Fbar_s), so its Jacobian is
    symmetric: mu . VJP(u, lam) equals lam . VJP(u, mu) for any two directions."""
    n = 3
    X, T = _box(n, seed=16)
    mat = _material(kind)
    fb, _, _ = _oracle_parts(oracle_lib, X, T, mat, n)
    rng = np.random.default_rng(17)
    u = 1e-2 * rng.standard_normal(X.shape)
    lam, mu = rng.standard_normal(X.shape), rng.standard_normal(X.shape)
    op = oracle_lib.OracleProblem(X, [fb])
    a = np.sum(mu * op.vjp_force(u, lam)[0])
    b = np.sum(lam * op.vjp_force(u, mu)[0])
    assert abs(a - b) < 1e-12 * max(abs(a), abs(b))
