"""The allocation-free Tet4 internal force (am_tet4_internal_force_noalloc).

It serves callers that cannot allocate device memory themselves (a framework that
owns all device memory through its own pool, or a step that must not pay
cudaMalloc's latency and implicit synchronization): every argument is the
caller's device memory, and the scratch force slots live in a fixed array inside
the library. Its device-side checks (inverted tets, CSR entries outside the call's
slots) are read back with am_noalloc_status. This file is collected last so that a
run stopping at its first failure has already run every other test; it also passes
on its own in a fresh process."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

MATERIALS = ["linear_elastic", "neo_hookean", "elastic"]


def _node_csr(conn: np.ndarray, num_nodes: int):
    slots_of = conn.reshape(-1)
    order = np.argsort(slots_of, kind="stable")  # ascending slot id within each node
    ptr = np.zeros(num_nodes + 1, dtype=np.int32)
    np.add.at(ptr, slots_of + 1, 1)
    return np.cumsum(ptr).astype(np.int32), order.astype(np.int32)


def _call(lib, material, lam, mu, N, E, X, u, conn, ptr, slots, f, stream):
    return lib.am_tet4_internal_force_noalloc(material, lam, mu, N, E, X.data_ptr(), u.data_ptr(), conn.data_ptr(),
                                              ptr.data_ptr(), slots.data_ptr(), f.data_ptr(), stream)


def _status(lib, stream):
    from aperi_mech_b200 import capi

    code, index = C.c_int32(-1), C.c_int64(-2)
    assert lib.am_noalloc_status(stream, C.byref(code), C.byref(index)) == capi.AM_OK, lib.am_last_error(None)
    return code.value, index.value


def _mesh(n=8, seed=12):
    from aperi_mech_b200 import mesh

    rng = np.random.default_rng(seed)
    coords, conn_hex = mesh.box_hex(n, n, n)
    coords = mesh.jitter_interior(coords, 0.2 / n, rng)
    return coords, mesh.hex_to_tets(conn_hex), rng


@pytest.mark.parametrize("material", MATERIALS)
def test_noalloc_matches_context_entry_point_and_oracle(gpu, material):
    """Two calls in a row (sharing the fixed scratch) against the context entry point
    and the FP64 oracle, at the 1e-12 FP64 parity bar of the other tests."""
    import torch

    from aperi_mech_b200 import capi
    from aperi_mech_b200.model import ExplicitDynamics, Material, Part
    from oracle import oracle

    lib = capi.load()
    coords, conn, rng = _mesh()
    N, E = coords.shape[0], conn.shape[0]
    mat = Material.create(material, 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    parts = [Part("tet4", mat, conn=conn)]
    ptr, slots = _node_csr(conn, N)
    dev = torch.device("cuda", 0)
    X = torch.from_numpy(coords).to(dev)
    c = torch.from_numpy(conn).to(dev)
    p = torch.from_numpy(ptr).to(dev)
    s = torch.from_numpy(slots).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    code = {"linear_elastic": capi.AM_LINEAR_ELASTIC, "neo_hookean": capi.AM_NEO_HOOKEAN,
            "elastic": capi.AM_ELASTIC_SVK}[material]
    op = oracle.OracleProblem(coords, parts)
    with ExplicitDynamics(coords, parts) as m:
        for call in range(2):
            u_h = 1e-3 * rng.standard_normal(coords.shape)
            want = m.internal_force(u_h, "fp64")
            ref = op.internal_force(u_h)
            u = torch.from_numpy(u_h).to(dev)
            f = torch.full((N, 3), float("nan"), dtype=torch.float64, device=dev)
            rc = _call(lib, code, mat.lam, mat.mu, N, E, X, u, c, p, s, f, stream)
            assert rc == capi.AM_OK, lib.am_last_error(None)
            assert _status(lib, stream) == (capi.AM_OK, -1)
            got = f.cpu().numpy()
            assert rel_err(got, want) < 1e-12, call
            assert rel_err(got, ref) < 1e-12, call


def test_noalloc_reports_inverted_tet(gpu):
    """A tet with det J < 0 is reported as AM_ENONPOS_J with its index, as the context
    path reports it; the next valid call clears the status."""
    import torch

    from aperi_mech_b200 import capi
    from aperi_mech_b200.model import Material

    lib = capi.load()
    coords, conn, rng = _mesh(n=4, seed=3)
    bad = 17
    good_conn = conn.copy()
    conn = conn.copy()
    conn[bad, [1, 2]] = conn[bad, [2, 1]]  # swapping two nodes inverts the tet
    N, E = coords.shape[0], conn.shape[0]
    mat = Material.create("neo_hookean", 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    ptr, slots = _node_csr(conn, N)
    dev = torch.device("cuda", 0)
    args = [torch.from_numpy(a).to(dev) for a in (coords, np.zeros_like(coords), conn, ptr, slots)]
    f = torch.zeros((N, 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert _call(lib, capi.AM_NEO_HOOKEAN, mat.lam, mat.mu, N, E, *args, f, stream) == capi.AM_OK
    assert _status(lib, stream) == (capi.AM_ENONPOS_J, bad)
    good = torch.from_numpy(good_conn).to(dev)
    ptr_g, slots_g = _node_csr(good_conn, N)
    assert _call(lib, capi.AM_NEO_HOOKEAN, mat.lam, mat.mu, N, E, args[0], args[1], good,
                 torch.from_numpy(ptr_g).to(dev), torch.from_numpy(slots_g).to(dev), f, stream) == capi.AM_OK
    assert _status(lib, stream) == (capi.AM_OK, -1)


def test_noalloc_reports_slot_outside_the_call(gpu):
    """A node -> slot entry at or beyond 4 num_elems is skipped and reported as
    AM_EINVAL at its node instead of reading the shared array's stale contents."""
    import torch

    from aperi_mech_b200 import capi
    from aperi_mech_b200.model import Material

    lib = capi.load()
    coords, conn, rng = _mesh(n=4, seed=5)
    N, E = coords.shape[0], conn.shape[0]
    mat = Material.create("linear_elastic", 1000.0, youngs_modulus=1e9, poissons_ratio=0.3)
    ptr, slots = _node_csr(conn, N)
    node = 9
    slots = slots.copy()
    slots[ptr[node]] = 4 * E + 3  # within node_slots' length, beyond the call's slots
    dev = torch.device("cuda", 0)
    args = [torch.from_numpy(a).to(dev) for a in (coords, 1e-4 * rng.standard_normal(coords.shape), conn, ptr, slots)]
    f = torch.zeros((N, 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert _call(lib, capi.AM_LINEAR_ELASTIC, mat.lam, mat.mu, N, E, *args, f, stream) == capi.AM_OK
    assert _status(lib, stream) == (capi.AM_EINVAL, node)


def test_noalloc_rejects_oversize_input(gpu):
    from aperi_mech_b200 import capi

    lib = capi.load()
    E = capi.AM_NOALLOC_MAX_TETS + 1
    null = C.c_void_p(8)  # never dereferenced: the size check comes first
    rc = lib.am_tet4_internal_force_noalloc(capi.AM_NEO_HOOKEAN, 1.0, 1.0, 10, E, null, null, null, null, null, null,
                                            None)
    assert rc == capi.AM_ERANGE
    assert b"AM_NOALLOC_MAX_TETS" in lib.am_last_error(None)
