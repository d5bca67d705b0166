"""Warp-chunk summation (the one-thread-per-tet and split-hex force kernels): a restatement of
the plan the library builds at set-up and of the per-lane reduction the kernels run, checked
against direct per-node sums on random chunks. The plan: a chunk's 128 entries (code
q = 32 a + lane, corner a of the chunk's unit lane) are ranked by the first appearance of
their node in code order and sorted by (rank, code), four to a lane. The reduction: each
lane sums the runs among its four entries, an inclusive segmented scan over the lanes
carries a run across lane boundaries, and the lane holding a node's last entry writes it.
Every distinct node of the chunk must be written exactly once with the sum of its entries,
including nodes that repeat within a unit, runs that span many lanes and partial chunks. The
library's own C++ plan builder (am_chunks.hpp, compiled here with g++) must produce the
restated plan byte for byte."""
from __future__ import annotations

import numpy as np
import pytest

PAD = 0xFF


def chunk_plan(conn: np.ndarray, c: int):
    """Sorted (code, rank) of chunk c and its distinct nodes in rank order."""
    n = min(32, conn.shape[0] - 32 * c)
    order, rank_of = [], {}
    rank = np.full(128, -1)
    for q in range(128):
        if (q & 31) >= n:
            continue
        v = int(conn[32 * c + (q & 31), q >> 5])
        if v not in rank_of:
            rank_of[v] = len(order)
            order.append(v)
        rank[q] = rank_of[v]
    codes = np.full(128, PAD)
    ranks = np.full(128, PAD)
    j = 0
    for k in range(len(order)):
        for q in np.flatnonzero(rank == k):
            codes[j], ranks[j] = q, k
            j += 1
    return codes.reshape(32, 4), ranks.reshape(32, 4), order


def chunk_reduce(values: np.ndarray, codes: np.ndarray, ranks: np.ndarray) -> dict:
    """The lanes' writes {rank: sum}; values[q] is entry q's three components."""
    out = {}

    def write(r, v):
        assert r not in out, "a node written twice"
        out[r] = v.copy()

    rnext = [ranks[lane + 1, 0] if lane < 31 else 0x100 for lane in range(32)]
    run = np.zeros((32, 3))
    head = np.zeros((32, 3))
    split = np.zeros(32, bool)
    for lane in range(32):
        for j in range(4):
            r = ranks[lane, j]
            if j > 0 and r != ranks[lane, j - 1]:
                if not split[lane]:
                    head[lane], split[lane] = run[lane], True
                elif ranks[lane, j - 1] != PAD:
                    write(ranks[lane, j - 1], run[lane])
                run[lane] = 0.0
            if r != PAD:
                run[lane] += values[codes[lane, j]]
    rprev = [ranks[lane - 1, 3] if lane > 0 else -1 for lane in range(32)]
    flag = np.array([split[lane] or lane == 0 or ranks[lane, 0] != rprev[lane] for lane in range(32)])
    d = 1
    while d < 32:  # Hillis-Steele: (a, fa) + (b, fb) = (fb ? b : a + b, fa | fb)
        up_v, up_f = np.roll(run, d, axis=0), np.roll(flag, d)
        new_v, new_f = run.copy(), flag.copy()
        for lane in range(d, 32):
            if not flag[lane]:
                new_v[lane] = up_v[lane] + run[lane]
            new_f[lane] = flag[lane] or up_f[lane]
        run, flag = new_v, new_f
        d <<= 1
    for lane in range(32):
        r0 = ranks[lane, 0]
        if split[lane] and r0 != PAD:
            cont = lane > 0 and r0 == rprev[lane]
            write(r0, head[lane] + (run[lane - 1] if cont else 0.0))
        r3 = ranks[lane, 3]
        if r3 != PAD and r3 != rnext[lane]:
            write(r3, run[lane])
    return out


CASES = ["random", "few_nodes", "fan", "partial", "repeated"]


@pytest.mark.parametrize("case", CASES)
def test_warp_chunk_sums_match_direct_sums(case):
    rng = np.random.default_rng(CASES.index(case))
    for _ in range(25):
        E = int(rng.integers(1, 33)) if case == "partial" else 32 * int(rng.integers(1, 4))
        if case == "few_nodes":
            conn = rng.integers(0, 4, size=(E, 4))
        elif case == "fan":
            conn = np.column_stack([np.zeros(E, int), rng.integers(1, 200, size=(E, 3))])
        elif case == "repeated":
            conn = rng.integers(0, 30, size=(E, 4))
            conn[:, 2] = conn[:, 0]
        else:
            conn = rng.integers(0, 500, size=(E, 4))
        vals = rng.standard_normal((E, 4, 3))
        for c in range((E + 31) // 32):
            codes, ranks, nodes = chunk_plan(conn, c)
            n = min(32, E - 32 * c)
            staged = np.zeros((128, 3))
            for q in range(128):
                if (q & 31) < n:
                    staged[q] = vals[32 * c + (q & 31), q >> 5]
            got = chunk_reduce(staged, codes, ranks)
            assert sorted(got) == list(range(len(nodes)))
            for k, node in enumerate(nodes):
                mask = conn[32 * c:32 * c + n] == node
                want = vals[32 * c:32 * c + n][mask].sum(axis=0)
                assert np.allclose(got[k], want, rtol=1e-13, atol=1e-13)


def _build_dump(tmp_path):
    import subprocess
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    exe = tmp_path / "chunk_plan_dump"
    res = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                          f"-I{root / 'aperi_mech_b200' / 'csrc'}", str(root / "tests" / "cxx" / "chunk_plan_dump.cpp"),
                          "-o", str(exe)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def _library_plan(exe, tmp_path, conn):
    import subprocess

    src, dst = tmp_path / "conn.bin", tmp_path / "plan.bin"
    with open(src, "wb") as f:
        np.array(conn.shape, dtype="<i8").tofile(f)
        np.ascontiguousarray(conn, dtype="<i4").tofile(f)
    assert subprocess.run([str(exe), str(src), str(dst)]).returncode == 0
    raw = open(dst, "rb").read()
    ok, C, G = np.frombuffer(raw[:24], dtype="<i8")
    words = 32 * C * conn.shape[1] // 4
    rest = np.frombuffer(raw[24:], dtype="<i4")
    ptr, nodes = rest[:C + 1], rest[C + 1:C + 1 + G]
    code = np.frombuffer(raw[24 + 4 * (C + 1 + G):], dtype="<u4")[:words]
    rank = np.frombuffer(raw[24 + 4 * (C + 1 + G + words):], dtype="<u4")[:words]
    return bool(ok), ptr, nodes, code, rank


def _bytes(words):
    return np.stack([(words >> (8 * k)) & 0xFF for k in range(4)], axis=-1).reshape(-1)


def test_library_plan_builder_matches_restatement(tmp_path):
    """The C++ builder the library runs at set-up (am_chunks.hpp) gives, chunk by chunk, the
    distinct nodes, the sorted entry codes and the node ranks of the restatement above."""
    exe = _build_dump(tmp_path)
    rng = np.random.default_rng(7)
    for case in CASES:
        E = int(rng.integers(1, 200))
        conn = {"few_nodes": rng.integers(0, 4, size=(E, 4)),
                "fan": np.column_stack([np.zeros(E, int), rng.integers(1, 200, size=(E, 3))])}.get(
            case, rng.integers(0, 500, size=(E, 4)))
        if case == "repeated":
            conn[:, 2] = conn[:, 0]
        ok, ptr, nodes, code, rank = _library_plan(exe, tmp_path, conn)
        assert ok and ptr[0] == 0 and ptr.size == (E + 31) // 32 + 1
        cb, rb = _bytes(code).reshape(-1, 128), _bytes(rank).reshape(-1, 128)
        for c in range(ptr.size - 1):
            codes, ranks, order = chunk_plan(conn, c)
            assert list(nodes[ptr[c]:ptr[c + 1]]) == order, (case, c)
            assert np.array_equal(cb[c], codes.reshape(-1)) and np.array_equal(rb[c], ranks.reshape(-1)), (case, c)


def test_library_plan_builder_refuses_chunks_beyond_rank_bytes(tmp_path):
    """Eight-node elements with no shared nodes put 256 distinct nodes in a chunk, more than
    the rank bytes hold: the builder reports failure (the block then keeps one slot per
    element node)."""
    exe = _build_dump(tmp_path)
    conn = np.arange(32 * 8, dtype=np.int32).reshape(32, 8)
    ok, *_ = _library_plan(exe, tmp_path, conn)
    assert not ok
    ok, *_ = _library_plan(exe, tmp_path, conn[:, :4].copy())
    assert ok
