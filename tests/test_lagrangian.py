"""Updated and semi-Lagrangian formulations (Gauss elements): the oracle's restatement
against the total formulation (Tet4 has one Gauss point, so the kinematics agree to
round-off) and against the reference's shear-patch known answers, then the library
against the oracle, including runs split where a semi reference update falls (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import expected_pk1, prescribed_patch, rel_err


def _tet_problem(nsteps=40):
    from aperi_mech_b200 import problems

    return problems.tet4_nh_shear(n=4, seed=1, nsteps=nsteps)


def _hex_problem(nsteps=30):
    from aperi_mech_b200 import problems

    return problems.hex8_nh_lognormal(n=4, seed=2, nsteps=nsteps)


@pytest.mark.parametrize("form, k", [("updated", 1), ("semi", 1), ("semi", 3)])
def test_oracle_tet4_updated_and_semi_match_total(oracle_lib, form, k):
    p = _tet_problem()
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs)
    z = np.zeros_like(p.coords)
    want = op.steps(z, p.v0, op.init_acceleration(z), np.full(p.nsteps, p.dt))
    st = op.lagrangian_state(form, k)
    got = op.lagrangian_steps(st, z, p.v0, op.lagrangian_init(st), np.full(p.nsteps, p.dt))
    assert st.n == p.nsteps
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-12
    # updated: x is the current configuration X + u; semi: the last reference one
    if form == "updated":
        assert rel_err(st.x, p.coords + got[0]) < 1e-13


@pytest.mark.parametrize("form", ["updated", "semi"])
@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("direction,surface", [(1, 0), (2, 1), (0, 2)])
def test_oracle_shear_patch_known_answers(oracle_lib, form, kind, direction, surface):
    """ForceTest.cpp ExplicitShearForceUpdated / ExplicitShearForceSemi (semi with
    update_interval 2, PatchTestFixture.h:126-130): the fully prescribed patch ends with
    the expected displacement gradient in every element, zero acceleration, the faces'
    displacements and velocities, and surface forces +/- P n A."""
    mag = 0.1
    coords, parts, bcs, sets = prescribed_patch(kind, (1, 1, 1), direction, surface, mag)
    op = oracle_lib.OracleProblem(coords, parts, bcs)
    st = op.lagrangian_state(form, 2 if form == "semi" else 1)
    z = np.zeros_like(coords)
    dts = oracle_lib.direct_time_schedule(0.1, 10.0)
    u, v, a = op.lagrangian_steps(st, z, z, op.lagrangian_init(st), dts)
    H = np.zeros((3, 3))
    H[direction, surface] = 2.0 * mag
    assert np.abs(st.H.reshape(-1, 3, 3) - H).max() < 1e-9
    assert np.abs(a).max() < 1e-12
    P = expected_pk1(H, parts[0].material)
    f = op.internal_force(u)  # the total formulation's force at the same displacement
    for i in range(3):
        n_i = np.zeros(3)
        n_i[i] = 1.0
        assert np.abs(f[sets[f"surface_{2 * i + 1}"]].sum(axis=0) - P @ n_i).max() < 1e-8
        assert np.abs(f[sets[f"surface_{2 * i + 2}"]].sum(axis=0) + P @ n_i).max() < 1e-8
    d = np.zeros(3)
    d[direction] = mag
    s_lo, s_hi = sets[f"surface_{2 * surface + 1}"], sets[f"surface_{2 * surface + 2}"]
    assert np.abs(u[s_hi] - d).max() < 1e-9 and np.abs(u[s_lo] + d).max() < 1e-9
    assert np.abs(v[s_hi] - 1.875 * d / 10.0).max() < 1e-4


def test_oracle_hex8_keeps_one_gradient_per_element(oracle_lib):
    """The reference stores one H per Hex8 (the last Gauss point's) and uses it as every
    Gauss point's reference gradient, so on a non-uniform deformation the updated
    formulation departs from the total one; the stored H is the last point's."""
    p = _hex_problem(nsteps=5)
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs)
    z = np.zeros_like(p.coords)
    want = op.steps(z, p.v0, op.init_acceleration(z), np.full(p.nsteps, p.dt))
    st = op.lagrangian_state("updated")
    got = op.lagrangian_steps(st, z, p.v0, op.lagrangian_init(st), np.full(p.nsteps, p.dt))
    assert rel_err(got[2], want[2]) > 1e-6
    assert np.isfinite(st.H).all() and np.isfinite(got[0]).all()


@pytest.mark.parametrize("extra, msg", [
    ("      lagrangian_formulation: {semi: {}}\n", "update_interval"),
    ("      lagrangian_formulation: {lagrange: ~}\n", "'total', 'updated', or 'semi'"),
    ("      lagrangian_formulation: {updated: ~}\n      x_b200: {precision: mixed}\n", "FP64"),
])
def test_yaml_lagrangian_formulation_rejections(extra, msg):
    from aperi_mech_b200 import input as inp

    text = """
procedures:
  - explicit_dynamics_procedure:
      geometry:
        mesh: generated:2x2x2|sideset:z|tets
        parts:
          - part:
              set: block_1
              material:
                neo_hookean: {density: 1000.0, shear_modulus: 3.85e8, bulk_modulus: 8.33e8}
      time_stepper:
        direct_time_stepper: {time_increment: 2.0e-7, time_end: 4.0e-6}
""" + extra
    with pytest.raises(inp.InputError, match=msg):
        inp.load(text)
    ok = inp.load(text.replace(extra, "      lagrangian_formulation: {semi: {update_interval: 4}}\n"))
    assert ok.formulation == ("semi", 4)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("form, k", [("updated", 1), ("semi", 3)])
def test_lagrangian_steps_match_oracle(gpu, oracle_lib, kind, form, k):
    """30 FP64 steps, run as 9 + 21 (a semi reference update falls at the split), against
    the oracle; the displacement, velocity and acceleration at 1e-12."""
    from aperi_mech_b200.model import ExplicitDynamics

    p = _tet_problem(30) if kind == "tet4" else _hex_problem(30)
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs)
    st = op.lagrangian_state(form, k)
    z = np.zeros_like(p.coords)
    want = op.lagrangian_steps(st, z, p.v0, op.lagrangian_init(st), np.full(p.nsteps, p.dt))
    with ExplicitDynamics(p.coords, p.parts, p.bcs, formulation=(form, k)) as m:
        assert m.layout()["patched_tet4_blocks"] == 0
        m.set_state(z, p.v0)
        m.init_acceleration()
        m.run(9, p.dt)
        m.run(21, p.dt, t0=9 * p.dt)
        got = m.get_state()
        with pytest.raises(Exception):
            m.internal_force(z)
        with pytest.raises(Exception):
            m.run(1, p.dt, "mixed")
        # a second run from rest (the displacement given as null, i.e. zero) restarts the
        # formulation's state too: bitwise the first run
        m.set_state(None, p.v0)
        m.init_acceleration()
        m.run(9, p.dt)
        m.run(21, p.dt, t0=9 * p.dt)
        again = m.get_state()
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-12
    for g, h in zip(got, again):
        assert np.array_equal(g, h)


@pytest.mark.gpu
@pytest.mark.parametrize("lagr", ["updated: ~", "semi: {update_interval: 2}"])
def test_yaml_lagrangian_formulation_matches_oracle(oracle_lib, lagr):
    from aperi_mech_b200 import input as inp

    text = f"""
procedures:
  - explicit_dynamics_procedure:
      geometry:
        mesh: generated:3x3x3|sideset:z|tets|bbox:0,0,0,1,1,1
        parts:
          - part:
              set: block_1
              material:
                neo_hookean: {{density: 1000.0, shear_modulus: 3.85e8, bulk_modulus: 8.33e8}}
      lagrangian_formulation:
        {lagr}
      initial_conditions:
        - velocity:
            sets: [block_1]
            components: {{X: 1.0, Z: -0.5}}
      time_stepper:
        direct_time_stepper: {{time_increment: 2.0e-7, time_end: 4.0e-6}}
      boundary_conditions:
        - displacement:
            sets: [surface_1]
            components: {{X: 0.0, Y: 0.0, Z: 0.0}}
"""
    sim = inp.load(text)
    r = inp.run(sim)
    form, k = sim.formulation
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs)
    st = prob.lagrangian_state(form, k)
    z = np.zeros_like(sim.coords)
    dts = inp.direct_time_steps(sim.dt, sim.time_end)
    u, v, a = prob.lagrangian_steps(st, z, sim.v0, prob.lagrangian_init(st), dts)
    assert r["steps"] == len(dts)
    assert np.linalg.norm(r["displacement"] - u) <= 1e-12 * np.linalg.norm(u)


def test_oracle_tet4_element_cell_is_the_gauss_tet(oracle_lib):
    """A Tet4 element smoothing cell (divergence-theorem gradients, QuadratureSmoothed.h:
    32-63) holds the tet's exact constant gradients and volume in any configuration, so its
    force equals the one-point Gauss tet's: on the mesh and on a deformed copy of it (the
    configuration an updated or semi reference update rebuilds the cells on)."""
    from aperi_mech_b200.model import Part
    from aperi_mech_b200.smoothing import element_smoothing_part

    p = _tet_problem()
    mat = p.parts[0].material
    T = p.parts[0].conn
    rng = np.random.default_rng(3)
    h = float(np.ptp(p.coords, axis=0).max()) / 4.0
    for X in (p.coords, p.coords + 0.05 * h * rng.standard_normal(p.coords.shape)):
        cells, mass = element_smoothing_part(X, T, mat)
        u = 1e-2 * h * rng.standard_normal(X.shape)
        f_cell = oracle_lib.OracleProblem(X, [cells]).internal_force(u)
        gauss = oracle_lib.OracleProblem(X, [Part("tet4", mat, conn=T)])
        assert rel_err(f_cell, gauss.internal_force(u)) < 1e-12
        assert rel_err(mass, gauss.lumped_mass()) < 1e-13


SMOOTHING_SEMI = """
procedures:
  - explicit_dynamics_procedure:
{lagr}      geometry:
        mesh: generated:3x3x6|sideset:z|tets|bbox:0,0,0,0.01,0.01,0.02
        parts:
          - part:
              set: block_1
              formulation:
                integration_scheme:
                  strain_smoothing:
                    element_smoothing_cell:
                      subdomains: 1
                approximation_space:
                  finite_element: ~
              material:
                elastic: {{density: 2700.0, youngs_modulus: 78.2e8, poissons_ratio: 0.3}}
      initial_conditions:
        - velocity:
            sets: [block_1]
            components: {{Z: -373.0}}
      time_stepper:
        direct_time_stepper: {{time_increment: 1.0e-7, time_end: 6.0e-6}}
      boundary_conditions:
        - displacement:
            sets: [surface_1]
            components: {{Z: 0.0}}
            time_function:
              ramp_function: {{abscissa_values: [0, 1], ordinate_values: [0, 1]}}
      x_b200: {{jitter: 0.15}}
"""


def test_yaml_element_smoothing_semi_runs_as_gauss_tets():
    """The reference's fem_strain_smoothing_semi form (element cells, finite elements,
    semi update_interval 10) loads as a Tet4 Gauss part under updated / semi and as
    element cells under the total formulation; reproducing-kernel cells stay refused."""
    from aperi_mech_b200 import input as inp

    semi = inp.load(SMOOTHING_SEMI.format(lagr="      lagrangian_formulation: {semi: {update_interval: 10}}\n"))
    assert semi.formulation == ("semi", 10) and semi.parts[0].kind == "tet4" and semi.mass is None
    total = inp.load(SMOOTHING_SEMI.format(lagr=""))
    assert total.formulation == ("total", 1) and total.parts[0].kind == "cells"
    assert np.array_equal(total.coords, semi.coords)
    rk = SMOOTHING_SEMI.format(lagr="      lagrangian_formulation: {updated: ~}\n").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 0.03}")
    with pytest.raises(inp.InputError, match="Tet4 finite-element element cells only"):
        inp.load(rk)


@pytest.mark.gpu
def test_yaml_element_smoothing_semi_matches_oracle_and_total(oracle_lib):
    """The semi run (every tenth step a reference update) against the oracle's semi run of
    the same tets at 1e-12, and against the total formulation's element-cell run (the cell
    kernel) at 1e-10: on tets the formulations agree to round-off."""
    from aperi_mech_b200 import input as inp

    sim = inp.load(SMOOTHING_SEMI.format(lagr="      lagrangian_formulation: {semi: {update_interval: 10}}\n"))
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs)
    st = prob.lagrangian_state(*sim.formulation)
    z = np.zeros_like(sim.coords)
    dts = inp.direct_time_steps(sim.dt, sim.time_end)
    u, v, a = prob.lagrangian_steps(st, z, sim.v0, prob.lagrangian_init(st), dts)
    assert r["steps"] == len(dts) == st.n >= 60
    assert np.linalg.norm(r["displacement"] - u) <= 1e-12 * np.linalg.norm(u)
    total = inp.run(inp.load(SMOOTHING_SEMI.format(lagr="")))
    assert np.linalg.norm(total["displacement"] - r["displacement"]) <= 1e-10 * np.linalg.norm(u)
