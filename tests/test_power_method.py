"""Stable time increment by the power method (PowerMethodProcessor) and the power-method
time stepper: the oracle against the exact largest eigenvalue of M^-1 K on a small
linear-elastic mesh (CPU), and the library against the oracle (GPU)."""
import numpy as np
import pytest

from helpers import rel_err


def _le_problem(kind="hex8", n=3, seed=0):
    from aperi_mech_b200 import mesh
    from aperi_mech_b200.model import BoundaryCondition, Material, Part

    rng = np.random.default_rng(seed)
    coords, conn = mesh.box_hex(n, n, n)
    coords = mesh.jitter_interior(coords, 0.15 / n, rng)
    if kind == "tet4":
        conn = mesh.hex_to_tets(conn)
    mat = Material.create("linear_elastic", 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)
    fixed = mesh.side_sets(coords)["surface_5"]
    return coords, [Part(kind, mat, conn=conn)], [BoundaryCondition.fixed(fixed)], conn


def _start(N, seed=7):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=(N, 3))


@pytest.mark.parametrize("kind", ["hex8", "tet4"])
def test_oracle_power_method_matches_largest_eigenvalue(oracle_lib, kind):
    """2 / sqrt(lambda_max(M^-1 K)) with K assembled column by column from the (linear)
    internal force, prescribed dofs removed."""
    from aperi_mech_b200 import mesh

    coords, parts, bcs, conn = _le_problem(kind)
    N = coords.shape[0]
    op = oracle_lib.OracleProblem(coords, parts, bcs)
    m = op.lumped_mass()
    free = np.ones(3 * N, dtype=bool)
    free[(3 * bcs[0].nodes[:, None] + np.arange(3)).ravel()] = False
    K = np.zeros((3 * N, 3 * N))
    for j in np.nonzero(free)[0]:
        e = np.zeros(3 * N)
        e[j] = 1e-6
        K[:, j] = -op.internal_force(e.reshape(N, 3)).ravel() / 1e-6
    Kf = K[np.ix_(free, free)]
    mf = np.repeat(m, 3)[free]
    lam = np.max(np.real(np.linalg.eigvals(Kf / mf[:, None])))
    l = mesh.max_edge_length(coords, conn)
    exact = 2.0 / np.sqrt(lam)
    # Tight stopping: the iteration converges to the exact increment (finite-difference error only).
    v = np.ascontiguousarray(_start(N) * 1e-5 * l[:, None])
    dt, its, conv = op.stable_time_increment(np.zeros_like(coords), v, l, num_iterations=2000, tolerance=1e-10,
                                             variation_tolerance=1e-16)
    assert abs(dt - exact) < 1e-3 * exact
    # The reference's defaults stop once successive estimates differ by < 1e-3 relative,
    # which on this slowly converging mesh leaves the estimate a few percent high.
    v = np.ascontiguousarray(_start(N) * 1e-5 * l[:, None])
    dt, its, conv = op.stable_time_increment(np.zeros_like(coords), v, l)
    assert conv and its < 50 and abs(dt - exact) < 0.06 * exact


@pytest.mark.gpu
@pytest.mark.parametrize("material", ["linear_elastic", "neo_hookean"])
def test_stable_time_increment_matches_oracle(gpu, oracle_lib, material):
    """Same start vector: same estimate, same iteration count, twice in a row (the second
    call continues from the first call's eigenvector), at a deformed state."""
    from aperi_mech_b200 import mesh, problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.tet4_nh_shear(n=4, seed=5, nsteps=10) if material == "neo_hookean" else \
        problems.hex8_le_cube(n=5, seed=5, nsteps=10)
    conn = p.parts[0].conn
    l = mesh.max_edge_length(p.coords, conn)
    start = _start(p.num_nodes, 3)
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs)
    u = 2e-4 * np.random.default_rng(1).standard_normal(p.coords.shape)
    v = np.ascontiguousarray(start * 1e-5 * l[:, None])
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_power_method(start, l)
        m.set_state(u, None)
        prev_g = prev_o = 0.0
        for _ in range(2):
            dt_g, its_g, conv_g = m.stable_time_increment(prev_g)
            dt_o, its_o, conv_o = op.stable_time_increment(u, v, l, previous=prev_o)
            assert its_g == its_o and conv_g == conv_o
            assert abs(dt_g - dt_o) <= 1e-9 * dt_o
            prev_g, prev_o = dt_g, dt_o


@pytest.mark.gpu
def test_power_method_solve_matches_oracle_schedule(gpu, oracle_lib):
    """Solve() with the power-method time stepper: increments recomputed every
    update_interval steps at the current state and scaled, last step cut at t_end."""
    from aperi_mech_b200 import mesh, problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.tet4_nh_shear(n=4, seed=2, nsteps=0)
    l = mesh.max_edge_length(p.coords, p.parts[0].conn)
    start = _start(p.num_nodes, 11)
    scale, interval = 0.5, 7
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs)
    u = np.zeros_like(p.coords)
    v = p.v0.copy()
    a = op.init_acceleration(u)
    ev = np.ascontiguousarray(start * 1e-5 * l[:, None])
    # the oracle's own schedule
    dt0, _, _ = op.stable_time_increment(u, ev.copy(), l)
    t_end = 23.5 * dt0 * scale
    time, inc, n = 0.0, 0.0, 0
    while not time >= t_end:
        full, _, _ = op.stable_time_increment(u, ev, l, previous=inc / scale)
        inc = full * scale
        dts = []
        t0 = time
        for _ in range(interval):
            if time >= t_end:
                break
            d = inc if time + inc <= t_end else (0.0 if time > t_end else t_end - time)
            dts.append(d)
            time += d
        u, v, a = op.steps(u, v, a, np.array(dts), t0=t0)
        n += len(dts)
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_power_method(start, l)
        m.set_state(None, p.v0)
        steps, last = m.solve_power_method(scale, interval, t_end)
        got = m.get_state()
    assert steps == n and abs(last - inc) <= 1e-9 * inc
    for g, w in zip(got, (u, v, a)):
        assert rel_err(g, w) < 1e-9
