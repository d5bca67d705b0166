"""The allocation-free Tet4 internal force (am_tet4_internal_force_noalloc).

It serves callers that cannot allocate device memory themselves (a framework that
owns all device memory through its own pool, or a step that must not pay
cudaMalloc's latency and implicit synchronization): every argument is the
caller's device memory, and the scratch force slots live in a fixed array inside
the library. This file is collected last so that a run stopping at its first
failure has already run every other test; it also passes on its own in a fresh
process."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _node_csr(conn: np.ndarray, num_nodes: int):
    slots_of = conn.reshape(-1)
    order = np.argsort(slots_of, kind="stable")  # ascending slot id within each node
    ptr = np.zeros(num_nodes + 1, dtype=np.int32)
    np.add.at(ptr, slots_of + 1, 1)
    return np.cumsum(ptr).astype(np.int32), order.astype(np.int32)


def _call(lib, material, lam, mu, N, E, X, u, conn, ptr, slots, f, stream):
    return lib.am_tet4_internal_force_noalloc(material, lam, mu, N, E, X.data_ptr(), u.data_ptr(), conn.data_ptr(),
                                              ptr.data_ptr(), slots.data_ptr(), f.data_ptr(), stream)


@pytest.mark.parametrize("material", ["neo_hookean", "elastic"])
def test_noalloc_matches_context_entry_point(gpu, material):
    import torch

    from aperi_mech_b200 import capi, mesh
    from aperi_mech_b200.model import ExplicitDynamics, Material, Part

    lib = capi.load()
    rng = np.random.default_rng(12)
    coords, conn_hex = mesh.box_hex(8, 8, 8)
    coords = mesh.jitter_interior(coords, 0.2 / 8, rng)
    conn = mesh.hex_to_tets(conn_hex)
    N, E = coords.shape[0], conn.shape[0]
    mat = Material.create(material, 1000.0, shear_modulus=3.85e8, bulk_modulus=8.33e8)
    ptr, slots = _node_csr(conn, N)
    dev = torch.device("cuda", 0)
    X = torch.from_numpy(coords).to(dev)
    c = torch.from_numpy(conn).to(dev)
    p = torch.from_numpy(ptr).to(dev)
    s = torch.from_numpy(slots).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    code = {"neo_hookean": capi.AM_NEO_HOOKEAN, "elastic": capi.AM_ELASTIC_SVK}[material]
    with ExplicitDynamics(coords, [Part("tet4", mat, conn=conn)]) as m:
        for call in range(2):  # two calls in a row share the fixed scratch
            u_h = 1e-3 * rng.standard_normal(coords.shape)
            want = m.internal_force(u_h, "fp64")
            u = torch.from_numpy(u_h).to(dev)
            f = torch.full((N, 3), float("nan"), dtype=torch.float64, device=dev)
            rc = _call(lib, code, mat.lam, mat.mu, N, E, X, u, c, p, s, f, stream)
            assert rc == capi.AM_OK, lib.am_last_error(None)
            torch.cuda.synchronize(dev)
            assert rel_err(f.cpu().numpy(), want) < 1e-12, call


def test_noalloc_rejects_oversize_input(gpu):
    from aperi_mech_b200 import capi

    lib = capi.load()
    E = 174762 + 1
    null = C.c_void_p(8)  # never dereferenced: the size check comes first
    rc = lib.am_tet4_internal_force_noalloc(capi.AM_NEO_HOOKEAN, 1.0, 1.0, 10, E, null, null, null, null, null, null,
                                            None)
    assert rc == capi.AM_ERANGE
    assert b"AM_NOALLOC_MAX_TETS" in lib.am_last_error(None)
