"""A mesh and the same mesh renumbered at random run the same: the library orders each
Gauss block's elements from the mesh alone (split-hex rings found by topology, else a
Morton order of the centroids), so the slots, their order and every sum are the same.
Forces, trajectories, the VJP and the adjoint gradient of a renumbered mesh equal those of
the original bit for bit once mapped back; both match the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import l2_rel, rel_err

pytestmark = pytest.mark.gpu


def _problem(kind):
    from aperi_mech_b200 import problems

    if kind == "tet4":
        return problems.tet4_nh_shear(n=10, seed=2, nsteps=40)
    return problems.hex8_nh_lognormal(n=8, seed=2, nsteps=40, bulk_field=True, num_sensors=30)


def _run(p, prec, u):
    from aperi_mech_b200.model import ExplicitDynamics

    with ExplicitDynamics(p.coords, p.parts, p.bcs) as m:
        f = m.internal_force(u, prec)
        m.set_state(None, p.v0)
        m.init_acceleration(prec)
        m.run(p.nsteps, p.dt, prec)
        state = m.get_state()
        layout = m.layout()
    return f, state, layout


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_renumbered_mesh_is_bitwise_identical(gpu, kind, prec):
    from aperi_mech_b200 import problems

    p = _problem(kind)
    q, pn, pes = problems.renumbered(p, seed=7)
    rng = np.random.default_rng(1)
    u = 1e-4 * rng.standard_normal(p.coords.shape)
    f0, s0, l0 = _run(p, prec, u)
    f1, s1, l1 = _run(q, prec, u[pn])
    assert l0 == l1
    assert np.array_equal(f1, f0[pn])
    for a, b in zip(s1, s0):
        assert np.array_equal(a, b[pn])


def test_renumbered_tet4_runs_split_hex_patches(gpu, monkeypatch):
    """The rings of the six-tet split are found in the renumbered mesh too: one slot per
    patch node (8 per 6 tets) without warp chunks, fewer with them (the default)."""
    from aperi_mech_b200 import problems

    p = _problem("tet4")
    q, _, _ = problems.renumbered(p, seed=3)
    _, _, chunked = _run(q, "fp64", np.zeros_like(q.coords))
    monkeypatch.setenv("APERI_B200_WARP_CHUNKS", "0")
    _, _, layout = _run(q, "fp64", np.zeros_like(q.coords))
    assert layout["patched_tet4_blocks"] == 1 and chunked["patched_tet4_blocks"] == 1
    assert layout["used_slots"] == 8 * q.num_elems // 6
    assert chunked["used_slots"] < layout["used_slots"] // 2


def test_renumbered_vjp_and_adjoint_map_back(gpu):
    from aperi_mech_b200 import problems
    from aperi_mech_b200.model import ExplicitDynamics

    p = _problem("hex8")
    q, pn, pes = problems.renumbered(p, seed=11)
    pe = pes[0]
    rng = np.random.default_rng(4)
    u = 1e-4 * rng.standard_normal(p.coords.shape)
    lam = rng.standard_normal(p.coords.shape)
    out = []
    for prob, uu, ll in ((p, u, lam), (q, u[pn], lam[pn])):
        with ExplicitDynamics(prob.coords, prob.parts, prob.bcs) as m:
            gu, gm, gk = m.vjp_force(uu, ll)
            m.set_state(None, prob.v0)
            loss, am_, ak = m.adjoint(prob.nsteps, prob.dt, 8, prob.meta["sensors"])
        out.append((gu, gm, gk, loss, am_, ak))
    (gu0, gm0, gk0, l0, am0, ak0), (gu1, gm1, gk1, l1, am1, ak1) = out
    assert np.array_equal(gu1, gu0[pn])
    assert np.array_equal(gm1, gm0[pe]) and np.array_equal(gk1, gk0[pe])
    assert l1 == l0
    assert np.array_equal(am1, am0[pe]) and np.array_equal(ak1, ak0[pe])


@pytest.mark.parametrize("kind,patches", [("tet4", "2"), ("tet4", "1"), ("tet4", "0"), ("hex8", "2")])
def test_renumbered_mesh_matches_oracle(gpu, oracle_lib, monkeypatch, kind, patches):
    """Against the oracle, with each Tet4 path: split-hex rings (the default), generic
    patches in Morton order (APERI_B200_TET4_PATCHES=1) and one thread per tet (=0)."""
    from aperi_mech_b200 import problems

    monkeypatch.setenv("APERI_B200_TET4_PATCHES", patches)
    p = _problem(kind)
    q, pn, _ = problems.renumbered(p, seed=5)
    op = oracle_lib.OracleProblem(q.coords, q.parts, q.bcs)
    z = np.zeros_like(q.coords)
    want = op.steps(z, q.v0, op.init_acceleration(z), np.full(q.nsteps, q.dt))
    rng = np.random.default_rng(2)
    u = 1e-4 * rng.standard_normal(q.coords.shape)
    f, got, _ = _run(q, "fp64", u)
    assert rel_err(f, op.internal_force(u)) < 1e-12
    for g, w in zip(got, want):
        assert l2_rel(g, w) < 1e-12


def test_caller_order_option_matches_locality_order(gpu, monkeypatch):
    """APERI_B200_ELEMENT_ORDER=input keeps the caller's element order: the same forces
    summed in another order, equal to round-off."""
    p = _problem("hex8")
    rng = np.random.default_rng(6)
    u = 1e-4 * rng.standard_normal(p.coords.shape)
    f0, _, _ = _run(p, "fp64", u)
    monkeypatch.setenv("APERI_B200_ELEMENT_ORDER", "input")
    f1, _, _ = _run(p, "fp64", u)
    assert rel_err(f1, f0) < 1e-13

