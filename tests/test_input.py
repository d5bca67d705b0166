"""The YAML front-end (aperi-mech's input schema) against the array-level set-up and the oracle."""
import sys

import numpy as np
import pytest

from aperi_mech_b200 import input as inp
from helpers import expected_pk1, prescribed_patch

PATCH_YAML = """
procedures:
  - explicit_dynamics_procedure:
      geometry:
        mesh: generated:1x1x1|sideset:xXyYzZ|tets
        parts:
          - part:
              set: block_1
              formulation:
                integration_scheme:
                  gauss_quadrature:
                    integration_order: 1
                approximation_space:
                  finite_element: ~
              material:
                elastic:
                  density: 0.08
                  youngs_modulus: 1.0
                  poissons_ratio: 0.0
      time_stepper:
        direct_time_stepper:
          time_increment: 0.1
          time_end: 10.0
      output:
        file: results.exo
        time_start: 0
        time_end: 10.0
        time_increment: 1.0
      boundary_conditions:
        - displacement:
            sets: [surface_1]
            vector: {magnitude: 0.2, direction: [0, -1, 0]}
            time_function:
              smooth_step_function: {abscissa_values: [0, 20.0], ordinate_values: [0, 1]}
        - displacement:
            sets: [surface_2]
            vector: {magnitude: 0.2, direction: [0, 1, 0]}
            time_function:
              smooth_step_function: {abscissa_values: [0, 20.0], ordinate_values: [0, 1]}
"""


def nh_yaml(n=3, mesh_opts="|sideset:z|tets", extra="", stepper="direct_time_stepper: {time_increment: 2.0e-7, time_end: 4.0e-6}"):
    return f"""
procedures:
  - explicit_dynamics_procedure:
      geometry:
        mesh: generated:{n}x{n}x{n}{mesh_opts}|bbox:0,0,0,1,1,1
        parts:
          - part:
              set: block_1
              formulation:
                integration_scheme:
                  gauss_quadrature: {{integration_order: 1}}
                approximation_space:
                  finite_element: ~
              material:
                neo_hookean: {{density: 1000.0, shear_modulus: 3.85e8, bulk_modulus: 8.33e8}}
      initial_conditions:
        - velocity:
            sets: [block_1]
            components: {{X: 1.0, Z: -0.5}}
      time_stepper:
        {stepper}
      boundary_conditions:
        - displacement:
            sets: [surface_1]
            components: {{X: 0.0, Y: 0.0, Z: 0.0}}
            time_function:
              ramp_function: {{abscissa_values: [0, 1], ordinate_values: [0, 1]}}
{extra}"""


def test_generated_mesh_and_sets():
    coords, blocks, sets = inp.generated_mesh("generated:2x3x4|sideset:xXyYzZ")
    assert coords.shape == (3 * 4 * 5, 3) and blocks["block_1"].shape == (24, 8)
    assert np.allclose(coords.max(axis=0), [2, 3, 4])  # unit-size elements
    assert sets["surface_1"].size == 4 * 5 and np.all(coords[sets["surface_1"], 0] == 0)
    assert np.all(coords[sets["surface_6"], 2] == 4)
    _, blocks, sets = inp.generated_mesh("generated:1x1x1|sideset:Zz|tets")
    assert blocks["block_1"].shape == (6, 4)
    assert sets["surface_1"].size == 4 and sets["surface_2"].size == 4
    coords, _, _ = inp.generated_mesh("generated:2x2x2|bbox:-1,-1,-1,1,1,3")
    assert np.allclose(coords.min(axis=0), [-1, -1, -1]) and np.allclose(coords.max(axis=0), [1, 1, 3])


def test_patch_yaml_matches_array_setup_and_known_answer(oracle_lib):
    sim = inp.load(PATCH_YAML)
    coords, parts, bcs, sets = prescribed_patch("tet4", (1, 1, 1), 1, 0, 0.1)
    assert np.array_equal(sim.coords, coords) and np.array_equal(sim.parts[0].conn, parts[0].conn)
    assert sim.parts[0].material == parts[0].material
    for a, b in zip(sim.bcs, bcs):
        assert np.array_equal(np.sort(a.nodes), np.sort(b.nodes))
        assert np.allclose(a.values, b.values) and a.component_mask == b.component_mask
        assert (a.kind, a.time_function, a.abscissa, a.ordinate) == (b.kind, b.time_function, b.abscissa, b.ordinate)
    # ForceTest.cpp shear patch known answer, run from the parsed input by the oracle.
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert n == len(inp.direct_time_steps(sim.dt, sim.time_end)) == len(oracle_lib.direct_time_schedule(0.1, 10.0))
    H = np.zeros((3, 3))
    H[1, 0] = 0.2
    f = prob.internal_force(u)
    P = expected_pk1(H, sim.parts[0].material)
    assert np.abs(f[sim.sets["surface_1"]].sum(axis=0) - P @ [1.0, 0.0, 0.0]).max() < 1e-8
    assert np.abs(u[sim.sets["surface_2"]] - [0.0, 0.1, 0.0]).max() < 1e-9
    assert np.abs(a).max() < 1e-12


def test_components_vector_initial_conditions_and_extensions():
    extra = """      loads:
        - gravity_load:
            sets: [block_1]
            vector: {magnitude: 9.81, direction: [0, 0, -2]}
      x_b200:
        precision: mixed
        seed: 4
        jitter: 0.2
        velocity_noise: 0.01
        fields:
          block_1:
            shear_modulus: {lognormal_sigma: 0.3}
"""
    sim = inp.load(nh_yaml(extra=extra))
    assert sim.precision == "mixed" and np.allclose(sim.body_accel, [0, 0, -9.81])
    assert np.abs(sim.v0[:, 0] - 1.0).max() <= 0.01 and np.abs(sim.v0[:, 1]).max() <= 0.01
    part = sim.parts[0]
    assert part.mu_field.shape == (part.num_elems,) and part.kappa_field is None
    assert abs(np.median(np.log(part.mu_field / 3.85e8))) < 0.2
    bc = sim.bcs[0]
    assert bc.component_mask == 7 and bc.kind == "displacement" and bc.time_function == "ramp_function"
    interior = ~np.any((sim.coords == 0) | (sim.coords == 1), axis=1)
    plain = inp.load(nh_yaml())
    assert np.abs(sim.coords[interior] - plain.coords[interior]).max() > 0  # jittered
    assert np.array_equal(sim.coords[~interior], plain.coords[~interior])  # boundary untouched


def test_time_increment_scheduler_known_answers():
    """SchedulerTest.cpp TimeIncrementSchedulerAtNextEvent (start 0, end 1, increment 0.1)."""
    sched = inp.TimeIncrementScheduler(0.0, 1.0, 0.1)
    calls = [(-0.1, False, 0.0), (0.0, True, 0.1), (0.05, False, 0.1), (0.09, False, 0.1), (0.1, True, 0.2),
             (0.19, False, 0.2), (0.21, True, 0.3), (0.3, True, 0.4), (0.75, True, 0.8), (0.76, False, 0.8),
             (0.99, True, 1.0)]
    for t, want, nxt in calls:
        assert sched.at_next_event(t) == want
        assert abs(sched.next_event - nxt) < 1e-12
    assert sched.at_next_event(1.0) and sched.next_event == sys.float_info.max
    assert not sched.at_next_event(1.1) and not sched.at_next_event(10.1)


def test_output_steps_follow_the_solver_loop():
    dts = inp.direct_time_steps(0.1, 1.0)
    assert inp.output_steps(dts, ("r.exo", 0.0, 1.0, 0.25)) == [0, 3, 5, 8, 10]
    assert inp.output_steps(dts, ("r.exo", 0.5, 0.8, 0.1)) == [5, 6, 7, 8]


@pytest.mark.parametrize("text, msg", [
    (nh_yaml(stepper="implicit_time_stepper: {time_end: 1.0}"), "time_stepper"),
    (nh_yaml(stepper="power_method_time_stepper: {scale_factor: 0.0, update_interval: 10, time_end: 1.0}"),
     "scale_factor"),
    (nh_yaml().replace("generated:3x3x3|sideset:z|tets|bbox:0,0,0,1,1,1", "../mesh/tet.e"), "Exodus"),
    (nh_yaml().replace("sets: [surface_1]", "sets: [nodeset_9]"), "unknown set"),
    (nh_yaml().replace("neo_hookean: {density: 1000.0,", "neo_hookean: {"), "density"),
    (nh_yaml().replace("neo_hookean:", "plastic:"), "not on this path"),
    (nh_yaml().replace("shear_modulus: 3.85e8, ", ""), "neo_hookean"),
    (nh_yaml().replace("gauss_quadrature: {integration_order: 1}",
                       "strain_smoothing: {nodal_smoothing_cell: {subdomains: 2}, use_f_bar: true}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}"), "num_subcells > 1"),
    (nh_yaml().replace("components: {X: 1.0, Z: -0.5}", "components: {W: 1.0}"), "component"),
    (nh_yaml(mesh_opts="|sideset:z").replace("gauss_quadrature: {integration_order: 1}",
                                             "strain_smoothing: {element_smoothing_cell: {subdomains: 1}}"),
     "finite elements and Hexahedron8"),
    (nh_yaml(mesh_opts="|sideset:z").replace("gauss_quadrature: {integration_order: 1}",
                                             "strain_smoothing: {nodal_smoothing_cell: {subdomains: 1}}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}"), "Hex8 block"),
    (nh_yaml().replace("gauss_quadrature: {integration_order: 1}",
                       "strain_smoothing: {element_smoothing_cell: {subdomains: 1}, force_one_pass_method: true, "
                       "force_two_pass_method: true}"), "Cannot force both"),
    (nh_yaml().replace("gauss_quadrature: {integration_order: 1}",
                       "strain_smoothing: {nodal_smoothing_cell: {subdomains: 0}, force_two_pass_method: true}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}"), "two-pass nodal"),
])
def test_rejected_inputs(text, msg):
    with pytest.raises(inp.InputError, match=msg):
        inp.load(text)


def test_f_bar_on_single_subcell_cells_is_a_no_op():
    """ForEachCellComputeForce_Impl uses F-bar only when the cells hold several subcells;
    element cells hold one (MeshLabelerProcessor.h:855-870), so use_f_bar changes nothing."""
    base = "strain_smoothing: {element_smoothing_cell: {subdomains: 1}%s}"
    plain = inp.load(nh_yaml().replace("gauss_quadrature: {integration_order: 1}", base % ""))
    fbar = inp.load(nh_yaml().replace("gauss_quadrature: {integration_order: 1}", base % ", use_f_bar: true"))
    assert fbar.parts[0].cell_groups is None
    assert np.array_equal(fbar.parts[0].cell_grads, plain.parts[0].cell_grads)


def test_strain_smoothing_part_from_yaml():
    text = nh_yaml().replace("gauss_quadrature: {integration_order: 1}",
                             "strain_smoothing: {element_smoothing_cell: {subdomains: 1}, force_one_pass_method: true}")
    sim = inp.load(text)
    part = sim.parts[0]
    assert part.kind == "cells" and part.num_elems == 6 * 27
    assert sim.mass is not None and abs(sim.mass.sum() - 1000.0) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_yaml_run_matches_oracle(oracle_lib, precision):
    extra = f"""      x_b200:
        precision: {precision}
        seed: 2
        jitter: 0.2
        velocity_noise: 0.01
        fields:
          block_1:
            shear_modulus: {{lognormal_sigma: 0.3}}
            bulk_modulus: {{lognormal_sigma: 0.3}}
"""
    sim = inp.load(nh_yaml(n=6, extra=extra))
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert r["steps"] == n
    tol = 1e-12 if precision == "fp64" else 1e-5
    for got, ref in ((r["displacement"], u), (r["velocity"], v)):
        assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("cell", ["nodal_smoothing_cell", "element_smoothing_cell"])
def test_yaml_rkpm_cells_run_matches_oracle(oracle_lib, cell):
    """reproducing_kernel with nodal cells (thex corner hexes) or element cells (the tets,
    as in the reference's RKPM Taylor-bar inputs)."""
    text = nh_yaml(n=4).replace(
        "gauss_quadrature: {integration_order: 1}",
        f"strain_smoothing: {{{cell}: {{subdomains: 1}}, force_one_pass_method: true}}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}")
    sim = inp.load(text)
    assert sim.parts[0].kind == "cells" and sim.mass is not None
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs, mass=sim.mass)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert r["steps"] == n
    assert np.linalg.norm(r["displacement"] - u) <= 1e-12 * np.linalg.norm(u)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_yaml_rkpm_two_pass_default_matches_oracle(oracle_lib, precision):
    """element_smoothing_cell with reproducing_kernel and no force key runs the two-pass
    method (InternalForceContributionParameters.h:164-194): FEM smoothed tet cells coupled
    to the coefficients through the vertex functions, against the oracle given them."""
    text = nh_yaml(n=4, extra=f"""      x_b200:
        precision: {precision}
""").replace(
        "gauss_quadrature: {integration_order: 1}",
        "strain_smoothing: {element_smoothing_cell: {subdomains: 1}}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}")
    sim = inp.load(text)
    assert sim.rk is not None and sim.parts[0].kind == "cells" and sim.parts[0].num_elems == 6 * 64
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs, mass=sim.mass, rk=sim.rk)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert r["steps"] == n
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.linalg.norm(r["displacement"] - u) <= tol * np.linalg.norm(u)
    from aperi_mech_b200.rkpm import apply_functions

    up = apply_functions(sim.rk, u)
    assert np.linalg.norm(r["physical_displacement"] - up) <= tol * np.linalg.norm(up)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_yaml_rkpm_two_pass_nodal_cells_match_oracle(oracle_lib, precision):
    """nodal_smoothing_cell with reproducing_kernel and force_two_pass_method: the vertex
    cells of the thex refinement hold their corner-hex points, coupled to the coefficients
    through the functions at every point (one row per point), against the oracle given them."""
    text = nh_yaml(n=3, extra=f"""      x_b200:
        precision: {precision}
""").replace(
        "gauss_quadrature: {integration_order: 1}",
        "strain_smoothing: {nodal_smoothing_cell: {subdomains: 1}, force_two_pass_method: true}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}")
    sim = inp.load(text)
    N = sim.coords.shape[0]
    assert sim.rk is not None and len(sim.rk[0]) - 1 > N and sim.parts[0].num_elems == N
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs, mass=sim.mass, rk=sim.rk)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert r["steps"] == n
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.linalg.norm(r["displacement"] - u) <= tol * np.linalg.norm(u)
    assert r["physical_displacement"].shape[0] == len(sim.rk[0]) - 1


@pytest.mark.gpu
@pytest.mark.parametrize("use_f_bar", [True, False])
def test_yaml_rkpm_nodal_subcells_match_oracle(oracle_lib, use_f_bar):
    """nodal_smoothing_cell with subdomains 0 (one subcell per corner hex), with and
    without use_f_bar, as the reference's rkpm_fbar Taylor-bar input sets it up."""
    text = nh_yaml(n=3).replace(
        "gauss_quadrature: {integration_order: 1}",
        f"strain_smoothing: {{nodal_smoothing_cell: {{subdomains: 0}}, use_f_bar: {str(use_f_bar).lower()}}}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.1}")
    sim = inp.load(text)
    part = sim.parts[0]
    assert part.num_elems == 4 * 6 * 27 and (part.cell_groups is not None) == use_f_bar
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs, mass=sim.mass)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert r["steps"] == n
    assert np.linalg.norm(r["displacement"] - u) <= 1e-12 * np.linalg.norm(u)


@pytest.mark.gpu
def test_yaml_output_frames_match_oracle(oracle_lib, tmp_path):
    """The output block: frames at the scheduler's steps equal the oracle run in the same
    segments, the last state equals the run without output, and the .npz holds them."""
    text = nh_yaml(n=4) + """      output:
        file: results.exo
        time_start: 0
        time_end: 4.0e-6
        time_increment: 1.0e-6
"""
    sim = inp.load(text)
    r = inp.run(sim)
    fr = r["frames"]
    dts = inp.direct_time_steps(sim.dt, sim.time_end)
    assert list(fr["step"]) == inp.output_steps(dts, sim.output) and len(fr["step"]) >= 4
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs)
    u = np.zeros_like(sim.coords)
    v, a = sim.v0.copy(), prob.init_acceleration(u)
    done, t = 0, 0.0
    for k, n in enumerate(fr["step"]):
        if n > done:
            u, v, a = prob.steps(u, v, a, np.array(dts[done:n]), t0=t)
            for d in dts[done:n]:
                t += d
            done = n
        assert abs(fr["time"][k] - t) <= 1e-18
        for g, w in ((fr["displacement"][k], u), (fr["velocity"][k], v), (fr["acceleration"][k], a)):
            assert np.linalg.norm(g - w) <= 1e-12 * max(np.linalg.norm(w), 1e-300)
    plain = inp.run(inp.load(nh_yaml(n=4)))
    assert np.linalg.norm(r["displacement"] - plain["displacement"]) <= 1e-13 * np.linalg.norm(plain["displacement"])
    path = inp.write_output(r, tmp_path)
    with np.load(path) as z:
        assert z["displacement"].shape == (len(fr["step"]),) + sim.coords.shape
        assert np.array_equal(z["time"], fr["time"])


@pytest.mark.gpu
@pytest.mark.parametrize("one_pass", [True, False])
def test_yaml_rkpm_hex8_element_cells_match_oracle(oracle_lib, one_pass):
    """element_smoothing_cell with reproducing_kernel on a Hex8 block (the reference's
    rkpm_hex inputs), one-pass or the two-pass default."""
    flag = ", force_one_pass_method: true" if one_pass else ""
    text = nh_yaml(n=3, mesh_opts="|sideset:z").replace(
        "gauss_quadrature: {integration_order: 1}",
        f"strain_smoothing: {{element_smoothing_cell: {{subdomains: 1}}{flag}}}").replace(
        "finite_element: ~", "reproducing_kernel: {kernel_radius_scale_factor: 1.0}")
    sim = inp.load(text)
    assert sim.parts[0].num_elems == 27 and (sim.rk is None) == one_pass
    r = inp.run(sim)
    prob = oracle_lib.OracleProblem(sim.coords, sim.parts, sim.bcs, mass=sim.mass, rk=sim.rk)
    u, v, a, n = prob.solve(np.zeros_like(sim.coords), sim.v0, sim.dt, sim.time_end)
    assert r["steps"] == n
    assert np.linalg.norm(r["displacement"] - u) <= 1e-12 * np.linalg.norm(u)


@pytest.mark.gpu
def test_yaml_power_method_stepper_matches_direct_api(gpu):
    """power_method_time_stepper from YAML equals the same run driven through the model API."""
    from aperi_mech_b200.model import ExplicitDynamics

    sim = inp.load(nh_yaml(n=4, stepper="power_method_time_stepper: {scale_factor: 0.4, update_interval: 5, "
                                        "time_end: 2.0e-6}"))
    assert sim.power_method == (0.4, 5)
    r = inp.run(sim)
    assert r["steps"] > 0 and r["time_increment"] > 0
    with ExplicitDynamics(sim.coords, sim.parts, sim.bcs) as m:
        m.set_power_method(*inp.power_method_inputs(sim))
        m.set_state(None, sim.v0)
        steps, dt = m.solve_power_method(0.4, 5, 2.0e-6)
        u = m.get_state()[0]
    assert steps == r["steps"] and dt == r["time_increment"]
    assert np.array_equal(u, r["displacement"])

