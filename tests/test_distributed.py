"""Query sharding across ranks, on CPU with gloo and world_size 2.

Each rank evaluates its contiguous block of queries with a CPU evaluator (the
oracle for W, a numpy restatement of the boundary-edge adjoint for dL/dV);
gather_w must rebuild the serial W exactly and the all_reduce of per-vertex
partials must equal the serial dL/dV.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _edge_adjoint_numpy(V, F, O, g):
    """dL/dV, dL/dO of L = sum g W via net boundary edges (CPU restatement)."""
    nv = len(V)
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
    sgn = np.where(e[:, 0] < e[:, 1], 1, -1)
    keys, inv = np.unique(lo * nv + hi, return_inverse=True)
    m = np.zeros(len(keys), int)
    np.add.at(m, inv, sgn)
    keep = m != 0
    u, v, m = keys[keep] // nv, keys[keep] % nv, m[keep]
    dV, dO = np.zeros((nv, 3)), np.zeros((len(O), 3))
    for i, o in enumerate(O):
        p, q = V[u] - o, V[v] - o
        lp, lq = np.linalg.norm(p, axis=1), np.linalg.norm(q, axis=1)
        w = g[i] * m / (lp * lq + (p * q).sum(1)) / (4 * np.pi)
        x = np.cross(p, q)
        cp, cq = (w / lp)[:, None] * x, (w / lq)[:, None] * x
        np.add.at(dV, u, -cp)
        np.add.at(dV, v, -cq)
        dO[i] = (cp + cq).sum(0)
    return dV, dO


def _worker(rank, world, port, out_dir):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "mojo-libigl_b200", "python"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist

    import igl.synthetic as syn
    import oracle
    from igl import distributed as wd

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        V, F = syn.bumpy_icosphere(2, seed=71)
        F = syn.delete_faces(F, 0.08, seed=72)
        O = syn.mixed_queries(V, F, 301, seed=73, near_sigma=1e-2)  # odd: uneven shards
        g = np.random.default_rng(74).normal(size=len(O))
        Vt, Ft, Ot, gt = (torch.from_numpy(x) for x in (V, F, O, g))

        def forward(V_, F_, O_):
            return torch.from_numpy(oracle.winding_number(V_.numpy(), F_.numpy(), O_.numpy()))

        def backward(V_, F_, O_, g_):
            dV, dO = _edge_adjoint_numpy(V_.numpy(), F_.numpy(), O_.numpy(), g_.numpy())
            return torch.from_numpy(dV), torch.from_numpy(dO)

        W = wd.forward_sharded(forward, Vt, Ft, Ot)
        dV, dO_block, (lo, hi) = wd.backward_sharded(backward, Vt, Ft, Ot, gt)
        tree = oracle.build_aabb(V, F)

        def closest(P_):
            s, i, c = oracle.aabb_squared_distance(P_.numpy(), V, F, tree=tree)
            return torch.from_numpy(s), torch.from_numpy(i), torch.from_numpy(c)

        sq, idx, pt = wd.points_sharded(closest, Ot)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), W=W.numpy(), dV=dV.numpy(),
                 dO=dO_block.numpy(), lo=lo, hi=hi, sqrd=sq.numpy(), index=idx.numpy(),
                 closest=pt.numpy())
    finally:
        dist.destroy_process_group()


def test_shard_bounds():
    from igl.distributed import shard

    for n in (0, 1, 7, 301, 1 << 20):
        for world in (1, 2, 3, 8):
            blocks = [shard(n, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            assert max(h - l for l, h in blocks) - min(h - l for l, h in blocks) <= 1


def test_two_rank_gloo_forward_gather_and_adjoint_all_reduce(tmp_path, oracle_mod):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    import igl.synthetic as syn

    V, F = syn.bumpy_icosphere(2, seed=71)
    F = syn.delete_faces(F, 0.08, seed=72)
    O = syn.mixed_queries(V, F, 301, seed=73, near_sigma=1e-2)
    g = np.random.default_rng(74).normal(size=len(O))
    W_serial = oracle_mod.winding_number(V, F, O)
    dV_serial, dO_serial = _edge_adjoint_numpy(V, F, O, g)
    dO_parts = []
    for rank in range(world):
        r = np.load(tmp_path / f"rank{rank}.npz")
        assert np.array_equal(r["W"], W_serial)
        assert np.abs(r["dV"] - dV_serial).max() <= 1e-12 * np.abs(dV_serial).max()
        dO_parts.append((int(r["lo"]), r["dO"]))
    dO = np.concatenate([d for _, d in sorted(dO_parts, key=lambda t: t[0])])
    assert np.abs(dO - dO_serial).max() <= 1e-12 * np.abs(dO_serial).max()
    # Closest points: gathered blocks equal the serial query exactly, on every rank.
    serial = oracle_mod.aabb_squared_distance(O, V, F)
    for rank in range(world):
        r = np.load(tmp_path / f"rank{rank}.npz")
        for key, expected in zip(("sqrd", "index", "closest"), serial):
            assert np.array_equal(r[key], expected)
