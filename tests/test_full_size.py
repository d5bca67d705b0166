"""Parity at the benchmark sizes. The FP64 internal force of the library against the
oracle on the full workloads: 70^3 split-hex Tet4, 128^3 Hex8 with lognormal fields, the
element-cell and RKPM nodal-cell boxes at h = 1/46 and the F-bar subcell box at h = 1/32 (for the cell
workloads the oracle takes the cells the library built; their set-up is pinned against the
oracle at smaller sizes, since the oracle's full-size RKPM set-up takes minutes). The mixed
force against the same at the mixed-precision bar; size-independent properties (the nodal
forces of every element sum to zero, a repeated run is bitwise identical); the split-hex
kernel against the per-element kernel on the same mesh. Trajectories of the benchmark
configurations at their stated lengths: the 70^3 Tet4 headline for 1000 steps, the 20^3
Hex8 linear-elastic cube for 100, the h = 1/46 cell boxes for 100 (of 500), the 128^3
Hex8 for 1000 (mixed against FP64) and 50 (FP64 against the oracle), and the 64^3 Hex8
adjoint gradient against the oracle's reverse pass."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5


def _displacement(p, scale, seed):
    """A smooth shear plus small noise, `scale` times the mesh spacing h."""
    X = p.coords
    h = float(np.ptp(X[:, 0])) / round(np.cbrt(X.shape[0]))
    rng = np.random.default_rng(seed)
    u = scale * h * rng.standard_normal(X.shape)
    u[:, 0] += 1e-3 * X[:, 2]
    return u


def _forces(p, u, precs=("fp64", "mixed"), mass=None):
    from aperi_mech_b200.model import ExplicitDynamics

    with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
        layout = m.layout()
        return {prec: m.internal_force(u, prec) for prec in precs}, layout


def _check(f, want):
    assert rel_err(f["fp64"], want) < FP64_TOL
    assert rel_err(f["mixed"], want) < MIXED_TOL
    # every element's nodal forces sum to zero, so the total does too
    assert np.abs(f["fp64"].sum(axis=0)).max() < 1e-13 * np.abs(f["fp64"]).sum()


@pytest.fixture(scope="module")
def tet70():
    from aperi_mech_b200 import problems

    return problems.tet4_nh_shear(n=70, seed=0, nsteps=20)


def test_tet4_70_force_matches_oracle(gpu, oracle_lib, tet70):
    """2,058,000 neo-Hookean tets on the split-hex kernel."""
    u = _displacement(tet70, 1e-3, 1)
    f, layout = _forces(tet70, u)
    assert layout["patched_tet4_blocks"] == 1
    _check(f, oracle_lib.OracleProblem(tet70.coords, tet70.parts, tet70.bcs).internal_force(u))


def test_tet4_70_split_hex_kernel_matches_per_element_kernel(gpu, tet70, monkeypatch):
    """The pair-split patch kernel and the one-thread-per-tet kernel (patching off) are
    independent code paths over the same tets: their FP64 forces agree to round-off."""
    u = _displacement(tet70, 1e-3, 2)
    patched, lp = _forces(tet70, u, ("fp64",))
    monkeypatch.setenv("APERI_B200_TET4_PATCHES", "0")
    plain, lu = _forces(tet70, u, ("fp64",))
    assert lp["patched_tet4_blocks"] == 1 and lu["patched_tet4_blocks"] == 0
    assert rel_err(patched["fp64"], plain["fp64"]) < 1e-13


def _run(m, p, prec, nsteps):
    m.set_state(None, p.v0)
    m.init_acceleration(prec)
    m.run(nsteps, p.dt, prec)
    return m.get_state()


def _oracle_run(oracle_lib, p, nsteps, mass=None):
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=mass)
    z = np.zeros_like(p.coords)
    return op.steps(z, p.v0, op.init_acceleration(z), np.full(nsteps, p.dt))


def _check_trajectory(got, want):
    """FP64 state after a run against the oracle's: displacement and velocity within
    1e-12 (relative L2, the parity metric, and max-norm), acceleration within 1e-11. The
    acceleration is the internal force, a residual of element stresses far larger than
    itself, over the mass: it turns the round-off that two summation orders leave in u
    into a larger relative difference. Measured after 1000 steps of the 70^3 Tet4
    workload: 2.0e-12 in L2, 2.8e-12 in max-norm; u and v stay below 1e-12."""
    from helpers import l2_rel

    for name, g, w in zip("uva", got, want):
        tol = FP64_TOL if name != "a" else 10 * FP64_TOL
        assert l2_rel(g, w) < tol, (name, l2_rel(g, w), rel_err(g, w))
        assert rel_err(g, w) < tol, (name, l2_rel(g, w), rel_err(g, w))


def _mixed_errors(p, nsteps, s64, sm):
    """Mixed-vs-FP64 errors after nsteps: displacement (L2 relative), the same relative to
    the displacement the forces produced (u - v0 t: the force-free drift v0 t is
    integrated in FP64 by both paths and would hide the element arithmetic), and the
    acceleration of the last step."""
    from helpers import l2_rel

    ukin = p.v0 * (nsteps * p.dt)
    return {"disp": l2_rel(sm[0], s64[0]),
            "disp_force_part": float(np.linalg.norm(sm[0] - s64[0]) / np.linalg.norm(s64[0] - ukin)),
            "accel": l2_rel(sm[2], s64[2])}


def test_tet4_70_1000_steps_match_oracle_and_repeat_bitwise(gpu, oracle_lib):
    """The headline configuration as stated: 1000 FP64 central-difference steps of the
    70^3 x 6 neo-Hookean Tet4 shear workload against the oracle at 1e-12; the mixed path
    after the same 1000 steps within 1e-5 of FP64 in displacement, in the displacement the
    forces produced and in acceleration; a repeated mixed run bitwise identical."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.tet4_nh_shear(n=70, seed=0, nsteps=1000)
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        got = _run(m, p, "fp64", p.nsteps)
        mixed = [_run(m, p, "mixed", p.nsteps) for _ in range(2)]
    want = _oracle_run(oracle_lib, p, p.nsteps)
    _check_trajectory(got, want)
    for a, b in zip(*mixed):
        assert np.array_equal(a, b)
    err = _mixed_errors(p, p.nsteps, got, mixed[0])
    print("tet4_nh_shear_70 mixed vs FP64 after 1000 steps:", err)
    assert max(err.values()) < MIXED_TOL, err


def test_hex8_le_20_100_steps_match_oracle(gpu, oracle_lib):
    """Hex8 linear elastic 20^3 (9,261 nodes), bottom fixed, seeded U[-0.01, 0.01]
    initial velocity, 100 steps at 0.5 CFL: FP64 against the oracle at 1e-12, mixed
    against FP64 within 1e-5."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.hex8_le_cube(n=20, seed=0, nsteps=100)
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        got = _run(m, p, "fp64", p.nsteps)
        mixed = _run(m, p, "mixed", p.nsteps)
    want = _oracle_run(oracle_lib, p, p.nsteps)
    _check_trajectory(got, want)
    err = _mixed_errors(p, p.nsteps, got, mixed)
    print("hex8_le_cube_20 mixed vs FP64 after 100 steps:", err)
    assert max(err.values()) < MIXED_TOL, err


@pytest.mark.parametrize("workload", ["smoothed_tet4_box_46", "rkpm_box_46"])
def test_cells_46_100_steps_match_oracle(gpu, oracle_lib, workload):
    """The strain-smoothed Tet4 element cells and the one-pass RKPM nodal cells on the
    h = 1/46 box (205,437 nodes), 100 FP64 steps against the oracle at 1e-12 (the oracle
    takes the cells the library built), mixed against FP64 within 1e-5."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    nsteps = 100
    p = {"smoothed_tet4_box_46": lambda: problems.smoothed_tet4_box(n=46, nsteps=nsteps),
         "rkpm_box_46": lambda: problems.rkpm_box(n=46, nsteps=nsteps)}[workload]()
    mass = p.meta["mass"]
    with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass) as m:
        got = _run(m, p, "fp64", nsteps)
        mixed = _run(m, p, "mixed", nsteps)
    want = _oracle_run(oracle_lib, p, nsteps, mass=mass)
    _check_trajectory(got, want)
    err = _mixed_errors(p, nsteps, got, mixed)
    print(f"{workload} mixed vs FP64 after {nsteps} steps:", err)
    assert max(err.values()) < MIXED_TOL, err


@pytest.mark.parametrize("workload", ["rkpm_fbar_box_32", "rkpm_two_pass_box_46"])
def test_fbar_and_two_pass_full_size_steps_match_oracle(gpu, oracle_lib, workload):
    """The F-bar subcells of the h = 1/32 box (1,572,864 subcells, cell-stress form) over 20
    steps and the two-pass element cells of the h = 1/46 box (octet coupling) over 50 steps,
    FP64 against the oracle (the oracle takes the cells and functions the library built),
    mixed against FP64 within 1e-5. F-bar carries the last bits of the lane-summed J-bar
    through a cube root into every subcell stress, and the acceleration, a residual of
    those stresses, magnifies them: after 20 steps on this box the acceleration differed
    from the oracle's by 1.3e-11 (relative L2) while u and v stayed at 3e-14 and 6e-14.
    F-bar's u and v are held to the 1e-12 parity bar and its acceleration to 5e-11; the
    two-pass states to the parity bar (acceleration 1e-11, as every trajectory here)."""
    from helpers import l2_rel

    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    if workload == "rkpm_fbar_box_32":
        nsteps = 20
        p = problems.rkpm_fbar_box(n=32, nsteps=nsteps)
    else:
        nsteps = 50
        p = problems.rkpm_two_pass_box(n=46, nsteps=nsteps)
    mass, rk = p.meta["mass"], p.meta.get("rk")
    with ExplicitDynamics(p.coords, p.parts, p.bcs, mass=mass, rk=rk) as m:
        got = _run(m, p, "fp64", nsteps)
        mixed = _run(m, p, "mixed", nsteps)
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=mass, rk=rk)
    z = np.zeros_like(p.coords)
    want = op.steps(z, p.v0, op.init_acceleration(z), np.full(nsteps, p.dt))
    if workload == "rkpm_fbar_box_32":
        errs = [l2_rel(g, w) for g, w in zip(got, want)]
        print("rkpm_fbar_box_32 FP64 vs oracle after 20 steps (u, v, a):", errs)
        assert errs[0] < 1e-12 and errs[1] < 1e-12 and errs[2] < 5e-11, errs
    else:
        _check_trajectory(got, want)
    err = _mixed_errors(p, nsteps, got, mixed)
    print(f"{workload} mixed vs FP64 after {nsteps} steps:", err)
    assert max(err.values()) < MIXED_TOL, err


def test_hex8_128_1000_steps_mixed_and_50_steps_match_oracle(gpu, oracle_lib):
    """Hex8 neo-Hookean 128^3 (2,146,689 nodes) with lognormal shear and bulk fields:
    1000 steps mixed against FP64 within 1e-5 (displacement, its force-produced part and
    acceleration), and the first 50 FP64 steps against the oracle at 1e-12."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.hex8_nh_lognormal(n=128, seed=0, nsteps=1000, bulk_field=True)
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        short = _run(m, p, "fp64", 50)
        got = _run(m, p, "fp64", p.nsteps)
        mixed = _run(m, p, "mixed", p.nsteps)
    err = _mixed_errors(p, p.nsteps, got, mixed)
    print("hex8_nh_lognormal_128 mixed vs FP64 after 1000 steps:", err)
    assert max(err.values()) < MIXED_TOL, err
    want = _oracle_run(oracle_lib, p, 50)
    _check_trajectory(short, want)


def test_adjoint_hex8_64_matches_oracle_gradient(gpu, oracle_lib):
    """The adjoint configuration as stated: Hex8 neo-Hookean 64^3 with a lognormal
    shear-modulus field, 200 steps, checkpoints every 20, loss over 512 sensor nodes; the
    library's gradient against the oracle's FP64 reverse pass (all states stored) at 1e-10."""
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = problems.hex8_nh_lognormal(n=64, seed=0, nsteps=200)
    sens = p.meta["sensors"]
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_state(None, p.v0)
        loss, gm, gk = m.adjoint(p.nsteps, p.dt, 20, sens)
    wl, wm, wk = oracle_lib.OracleProblem.from_problem(p).adjoint(p.nsteps, p.dt, np.zeros_like(p.coords), p.v0,
                                                                  sens)
    assert abs(loss - wl) < 1e-12 * abs(wl)
    assert rel_err(gm, wm) < 1e-10 and rel_err(gk, wk) < 1e-10


def test_hex8_128_force_matches_oracle(gpu, oracle_lib):
    """2,097,152 neo-Hookean Hex8 with lognormal shear and bulk fields."""
    from aperi_mech_b200 import problems

    p = problems.hex8_nh_lognormal(n=128, seed=0, nsteps=1, bulk_field=True)
    u = _displacement(p, 1e-3, 3)
    f, _ = _forces(p, u)
    _check(f, oracle_lib.OracleProblem(p.coords, p.parts, p.bcs).internal_force(u))


@pytest.mark.parametrize("workload", ["smoothed_tet4_box_46", "rkpm_box_46", "rkpm_fbar_box_32"])
def test_cells_force_matches_oracle(gpu, oracle_lib, workload):
    """The element smoothing cells of the h = 1/46 box (1,168,032 tets, grouped as split
    hexes), the one-pass RKPM nodal cells (205,437 cells, 13.5 M entries) and the F-bar
    corner-hex subcells (1,572,864 subcells) built by the library, forces against the
    oracle's."""
    from aperi_mech_b200 import problems

    p = {"smoothed_tet4_box_46": lambda: problems.smoothed_tet4_box(n=46, nsteps=1),
         "rkpm_box_46": lambda: problems.rkpm_box(n=46, nsteps=1),
         "rkpm_fbar_box_32": lambda: problems.rkpm_fbar_box(n=32, nsteps=1)}[workload]()
    u = _displacement(p, 1e-3, 4)
    f, _ = _forces(p, u, mass=p.meta["mass"])
    _check(f, oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=p.meta["mass"]).internal_force(u))
