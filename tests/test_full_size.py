"""Parity at the benchmark sizes. The FP64 internal force of the library against the
oracle on the full workloads: 70^3 split-hex Tet4, 128^3 Hex8 with lognormal fields, the
element-cell and RKPM nodal-cell boxes at h = 1/46 and the F-bar subcell box at h = 1/32 (for the cell
workloads the oracle takes the cells the library built; their set-up is pinned against the
oracle at smaller sizes, since the oracle's full-size RKPM set-up takes minutes). The mixed
force against the same at the mixed-precision bar; size-independent properties (the nodal
forces of every element sum to zero, a repeated run is bitwise identical); the split-hex
kernel against the per-element kernel on the same mesh; 20 FP64 steps of the headline
workload against the oracle."""
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


def test_tet4_70_steps_match_oracle_and_repeat_bitwise(gpu, oracle_lib, tet70):
    """20 FP64 central-difference steps of the headline workload against the oracle, and
    a repeated mixed run bitwise identical to the first."""
    from aperi_mech_b200.model import ExplicitDynamics

    p = tet70
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs)
    z = np.zeros_like(p.coords)
    want = op.steps(z, p.v0, op.init_acceleration(z), np.full(p.nsteps, p.dt))
    mixed = []
    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        m.set_state(None, p.v0)
        m.init_acceleration()
        m.run(p.nsteps, p.dt)
        got = m.get_state()
        for _ in range(2):
            m.set_state(None, p.v0)
            m.init_acceleration("mixed")
            m.run(p.nsteps, p.dt, "mixed")
            mixed.append(m.get_state())
    for g, w in zip(got, want):
        assert rel_err(g, w) < FP64_TOL
    for a, b in zip(*mixed):
        assert np.array_equal(a, b)
    assert rel_err(mixed[0][0], got[0]) < MIXED_TOL


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
