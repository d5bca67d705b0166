"""Domain decomposition: the partition bookkeeping, and a world-size-2 run on CPU (gloo)
whose per-rank forces come from the oracle and whose interface forces are summed with
torch.distributed, against the single-domain oracle."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from aperi_mech_b200 import partition, problems


def _problem(kind):
    if kind == "tet4":
        return problems.tet4_nh_shear(n=5, seed=1, nsteps=12)
    if kind == "hex8":
        return problems.hex8_nh_lognormal(n=5, seed=1, nsteps=12, bulk_field=True)
    return problems.smoothed_tet4_box(n=4, seed=1, nsteps=12)


@pytest.mark.parametrize("kind", ["tet4", "hex8", "cells"])
@pytest.mark.parametrize("world", [2, 3])
def test_decompose_bookkeeping(kind, world):
    p = _problem(kind)
    subs = partition.decompose(p.coords, p.parts, p.bcs, p.v0, world, mass=p.meta.get("mass"))
    N = p.num_nodes
    # every element (cell) in exactly one rank
    for k, part in enumerate(p.parts):
        got = np.sort(np.concatenate([s.elements[k] for s in subs]))
        assert np.array_equal(got, np.arange(part.num_elems))
    # owners partition the nodes; interface = nodes held by two or more ranks
    held = np.zeros(N, dtype=int)
    owned = np.zeros(N, dtype=int)
    for s in subs:
        held[s.global_nodes] += 1
        owned[s.global_nodes[s.owned]] += 1
        assert np.array_equal(s.coords, p.coords[s.global_nodes])
        assert np.array_equal(np.sort(s.global_nodes[s.iface_local]), s.global_nodes[s.iface_local])
    assert (held >= 1).all() and (owned == 1).all()
    iface = np.nonzero(held > 1)[0]
    assert subs[0].num_iface == iface.size > 0
    for s in subs:
        assert np.array_equal(iface[s.iface_ids], s.global_nodes[s.iface_local])
        assert np.array_equal(s.iface_local, np.nonzero(held[s.global_nodes] > 1)[0])
    # global mass sliced; boundary conditions restricted to held nodes
    mass = p.meta.get("mass")
    for s in subs:
        if mass is not None:
            assert np.array_equal(s.mass, mass[s.global_nodes])
        for bc, gbc in zip(s.bcs, p.bcs):
            assert set(s.global_nodes[bc.nodes]) == set(gbc.nodes) & set(s.global_nodes)


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def _rank_main(rank, world, port, kind, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle

        p = _problem(kind)
        s = partition.decompose(p.coords, p.parts, p.bcs, p.v0, world, mass=p.meta.get("mass"))[rank]
        op = oracle.OracleProblem(s.coords, s.parts, s.bcs, mass=s.mass)
        fixed = np.zeros(s.num_nodes, dtype=bool)
        for bc in s.bcs:
            fixed[bc.nodes] = True
        m = s.mass[:, None]

        def force(u):
            f = op.internal_force(u)
            buf = torch.zeros((s.num_iface, 3), dtype=torch.float64)
            buf[torch.from_numpy(s.iface_ids.astype(np.int64))] = torch.from_numpy(f[s.iface_local])
            dist.all_reduce(buf)
            f[s.iface_local] = buf[torch.from_numpy(s.iface_ids.astype(np.int64))].numpy()
            return f

        # ExplicitSolver::Solve order with homogeneous displacement BCs.
        u = np.zeros_like(s.coords)
        v = s.v0.copy()
        a = force(u) / m
        h = 0.5 * p.dt
        for _ in range(p.nsteps):
            v = v + h * a
            v[fixed] = 0.0
            u = u + p.dt * v
            a = force(u) / m
            a[fixed] = 0.0
            v = v + h * a
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), u=u, v=v, nodes=s.global_nodes, owned=s.owned)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["tet4", "hex8", "cells"])
def test_two_rank_gloo_run_matches_single_domain(oracle_lib, tmp_path, kind):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), kind, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    p = _problem(kind)
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=p.meta.get("mass"))
    u0 = np.zeros_like(p.coords)
    u_ref, v_ref, _ = op.steps(u0, p.v0, op.init_acceleration(u0), np.full(p.nsteps, p.dt))
    u = np.zeros_like(p.coords)
    v = np.zeros_like(p.coords)
    seen = np.zeros(p.num_nodes, dtype=int)
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        nodes, owned = d["nodes"], d["owned"]
        # interface copies agree bitwise across ranks
        if r > 0:
            common = np.intersect1d(nodes, prev_nodes)
            a_idx = np.searchsorted(nodes, common)
            b_idx = np.searchsorted(prev_nodes, common)
            assert np.array_equal(d["u"][a_idx], prev_u[b_idx])
        prev_nodes, prev_u = nodes, d["u"]
        u[nodes[owned]] = d["u"][owned]
        v[nodes[owned]] = d["v"][owned]
        seen[nodes[owned]] += 1
    assert (seen == 1).all()
    assert np.linalg.norm(u - u_ref) <= 1e-12 * np.linalg.norm(u_ref)
    assert np.linalg.norm(v - v_ref) <= 1e-12 * np.linalg.norm(v_ref)


def _slab_global_ids(prob, n, rank):
    m1 = n + 1
    k = np.arange(prob.num_nodes)
    return (k % (m1 * m1)) + m1 * m1 * (k // (m1 * m1) + n * rank)


def _slab_rank_main(rank, world, port, n, nsteps, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle

        p = problems.tet4_nh_shear_slab(n=n, rank=rank, world=world, seed=2, nsteps=nsteps)
        rows = torch.from_numpy(p.meta["iface_rows"].astype(np.int64))
        loc = p.meta["iface_local"]

        def exchange(x):  # sum the interface rows of a nodal array over the ranks
            buf = torch.zeros((p.meta["num_iface"],) + x.shape[1:], dtype=torch.float64)
            buf[rows] = torch.from_numpy(x[loc])
            dist.all_reduce(buf)
            x[loc] = buf[rows].numpy()
            return x

        mass = exchange(p.meta["slab_mass"].copy())
        dt = torch.tensor([p.dt], dtype=torch.float64)
        dist.all_reduce(dt, op=dist.ReduceOp.MIN)
        dt = float(dt)
        op = oracle.OracleProblem(p.coords, p.parts, p.bcs, mass=mass)
        fixed = p.bcs[0].nodes
        u = np.zeros_like(p.coords)
        v = p.v0.copy()
        a = exchange(op.internal_force(u)) / mass[:, None]
        for _ in range(nsteps):
            v = v + 0.5 * dt * a
            v[fixed] = 0.0
            u = u + dt * v
            a = exchange(op.internal_force(u)) / mass[:, None]
            a[fixed] = 0.0
            v = v + 0.5 * dt * a
        np.savez(os.path.join(out_dir, f"slab{rank}.npz"), u=u, dt=dt)
    finally:
        dist.destroy_process_group()


def test_weak_scaled_slabs_match_the_stacked_mesh(oracle_lib, tmp_path):
    """The per-rank slabs the multi-GPU benchmark builds (no global mesh on any rank),
    run on two gloo ranks with interface force and mass exchange, against the oracle on
    the stacked mesh assembled from the slabs."""
    from aperi_mech_b200.model import BoundaryCondition, Part

    n, world, nsteps = 4, 2, 10
    mp.start_processes(_slab_rank_main, args=(world, _free_port(), n, nsteps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    slabs = [problems.tet4_nh_shear_slab(n=n, rank=r, world=world, seed=2, nsteps=nsteps) for r in range(world)]
    m1 = n + 1
    G = m1 * m1 * (n * world + 1)
    coords, v0 = np.zeros((G, 3)), np.zeros((G, 3))
    conns, fixed = [], []
    for r, s in enumerate(slabs):
        gid = _slab_global_ids(s, n, r)
        coords[gid], v0[gid] = s.coords, s.v0
        conns.append(gid[s.parts[0].conn])
        fixed.append(gid[s.bcs[0].nodes])
    parts = [Part("tet4", slabs[0].parts[0].material, conn=np.concatenate(conns).astype(np.int32))]
    bcs = [BoundaryCondition.fixed(np.concatenate(fixed).astype(np.int32))]
    dt = min(s.dt for s in slabs)
    op = oracle_lib.OracleProblem(coords, parts, bcs)
    u0 = np.zeros_like(coords)
    u_ref, _, _ = op.steps(u0, v0, op.init_acceleration(u0), np.full(nsteps, dt))
    for r, s in enumerate(slabs):
        d = np.load(tmp_path / f"slab{r}.npz")
        assert float(d["dt"]) == dt
        ref = u_ref[_slab_global_ids(s, n, r)]
        assert np.linalg.norm(d["u"] - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("kind", ["tet4", "cells"])
@pytest.mark.parametrize("world", [2, 3])
def test_neighbor_lists_are_symmetric(kind, world):
    """Rank k's list of nodes shared with q and q's list shared with k name the same
    global nodes in the same order, and together cover each rank's interface nodes."""
    p = _problem(kind)
    subs = partition.decompose(p.coords, p.parts, p.bcs, p.v0, world, mass=p.meta.get("mass"))
    for s in subs:
        covered = set()
        for j, q in enumerate(s.neighbors):
            mine = s.global_nodes[s.shared_nodes[s.shared_ptr[j]:s.shared_ptr[j + 1]]]
            t = subs[q]
            jq = int(np.nonzero(t.neighbors == s.rank)[0][0])
            theirs = t.global_nodes[t.shared_nodes[t.shared_ptr[jq]:t.shared_ptr[jq + 1]]]
            assert np.array_equal(mine, theirs) and np.all(np.diff(mine) > 0)
            covered |= set(mine.tolist())
        assert covered == set(s.global_nodes[s.iface_local].tolist())


def _neighbor_rank_main(rank, world, port, kind, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle

        p = _problem(kind)
        s = partition.decompose(p.coords, p.parts, p.bcs, p.v0, world, mass=p.meta.get("mass"))[rank]
        op = oracle.OracleProblem(s.coords, s.parts, s.bcs, mass=s.mass)
        fixed = np.zeros(s.num_nodes, dtype=bool)
        for bc in s.bcs:
            fixed[bc.nodes] = True
        m = s.mass[:, None]

        def force(u):
            # neighbour exchange: each shared node's partial goes to the neighbours holding it
            f = op.internal_force(u)
            sends, recvs, reqs = [], [], []
            for j, q in enumerate(s.neighbors):
                nodes = s.shared_nodes[s.shared_ptr[j]:s.shared_ptr[j + 1]]
                sends.append(torch.from_numpy(np.ascontiguousarray(f[nodes])))
                recvs.append(torch.empty((nodes.size, 3), dtype=torch.float64))
                reqs.append(dist.isend(sends[-1], int(q)))
                reqs.append(dist.irecv(recvs[-1], int(q)))
            for r in reqs:
                r.wait()
            return partition.neighbor_sum(s, f, [x.numpy() for x in recvs])

        u = np.zeros_like(s.coords)
        v = s.v0.copy()
        a = force(u) / m
        h = 0.5 * p.dt
        for _ in range(p.nsteps):
            v = v + h * a
            v[fixed] = 0.0
            u = u + p.dt * v
            a = force(u) / m
            a[fixed] = 0.0
            v = v + h * a
        np.savez(os.path.join(out_dir, f"nrank{rank}.npz"), u=u, v=v, a=a, nodes=s.global_nodes, owned=s.owned)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["tet4", "cells"])
def test_three_rank_neighbor_exchange_matches_single_domain(oracle_lib, tmp_path, kind):
    """World size 3 on gloo with the neighbour exchange the library runs (point-to-point
    sends of the shared nodes' partial forces, holders summed in ascending rank order):
    every copy of an interface node is bitwise identical on all its holders, and the
    assembled state matches the single-domain oracle at 1e-12."""
    world = 3
    mp.start_processes(_neighbor_rank_main, args=(world, _free_port(), kind, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    p = _problem(kind)
    op = oracle_lib.OracleProblem(p.coords, p.parts, p.bcs, mass=p.meta.get("mass"))
    u0 = np.zeros_like(p.coords)
    u_ref, v_ref, _ = op.steps(u0, p.v0, op.init_acceleration(u0), np.full(p.nsteps, p.dt))
    data = [np.load(tmp_path / f"nrank{r}.npz") for r in range(world)]
    u = np.zeros_like(p.coords)
    for d in data:
        u[d["nodes"][d["owned"]]] = d["u"][d["owned"]]
    for r in range(world):
        for q in range(r + 1, world):
            common, ia, ib = np.intersect1d(data[r]["nodes"], data[q]["nodes"], return_indices=True)
            for key in ("u", "v", "a"):
                assert np.array_equal(data[r][key][ia], data[q][key][ib])
    assert np.linalg.norm(u - u_ref) <= 1e-12 * np.linalg.norm(u_ref)


def test_slab_neighbor_lists_pair_up():
    """The weak-scaled slabs' neighbour lists: rank r's top plane and rank r+1's bottom
    plane are the same global nodes in the same order."""
    n, world = 3, 3
    slabs = [problems.tet4_nh_shear_slab(n=n, rank=r, world=world, seed=1, nsteps=1) for r in range(world)]
    for r, s in enumerate(slabs):
        nb = list(s.meta["neighbors"])
        assert nb == [q for q in (r - 1, r + 1) if 0 <= q < world]
        gid = _slab_global_ids(s, n, r)
        ptr, nodes = s.meta["shared_ptr"], s.meta["shared_nodes"]
        for j, q in enumerate(nb):
            mine = gid[nodes[ptr[j]:ptr[j + 1]]]
            t = slabs[q]
            jq = list(t.meta["neighbors"]).index(r)
            theirs = _slab_global_ids(t, n, q)[t.meta["shared_nodes"][t.meta["shared_ptr"][jq]:t.meta["shared_ptr"][jq + 1]]]
            assert np.array_equal(mine, theirs) and np.all(np.diff(mine) > 0)
