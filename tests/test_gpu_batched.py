"""Batched persistent launch, CUDA-graph capture and the autotuner (needs a B200).

The batched forward of every mesh must agree with the single-mesh mixed kernel
and with the oracle (<= 1e-6), the batched adjoint with the single-mesh
boundary-edge adjoint (FP64: <= 1e-12 relative; mixed: <= 1e-6 of the mixed one,
<= 1e-4 of the FP64 one), graph replays with eager runs bit for bit, and
repeated runs with each other bit for bit.
"""

import numpy as np
import pytest

import igl
from igl import _lib
from igl import autograd as wa

pytestmark = pytest.mark.gpu


def _check_rc(rc):
    assert rc == 0, _lib.last_error()


def _small_batch(n=7, seed=5, max_level=4, max_q=3000):
    rng = np.random.default_rng(seed)
    meshes, queries = [], []
    for i in range(n):
        level = int(rng.integers(0, max_level + 1))
        V, F = igl.synthetic.bumpy_icosphere(level, seed=100 + i)
        F = igl.synthetic.delete_faces(F, float(rng.uniform(0, 0.1)), seed=200 + i)
        nq = int(rng.integers(1, max_q))
        meshes.append((V, F))
        queries.append(igl.synthetic.mixed_queries(V, F, nq, seed=300 + i, near_sigma=1e-3))
    return meshes, queries


@pytest.mark.parametrize("qpt,kappa,tile_faces", [
    (1, 4.0, 64), (2, 4.0, 64), (4, 4.0, 64), (2, 3.0, 64), (4, 3.0, 64),
    (1, 4.0, 32), (2, 4.0, 32), (4, 3.0, 32), (2, 3.0, 32)])
def test_batched_forward_matches_oracle(gpu_required, oracle_mod, qpt, kappa, tile_faces):
    """Every configuration the autotuner may pick keeps the 1e-6 bound (kappa = 3
    is the smallest refinement radius it is allowed; 32-face tiles test and sum
    each half of a tile on its own)."""
    meshes, queries = _small_batch()
    b = igl.batched.Batch(meshes, queries, qpt=qpt, target_pairs=1 << 16, kappa=kappa,
                          tile_faces=tile_faces)
    try:
        W = b.split(b.forward().clone())
        assert b.info()["work_items"] > len(meshes)
        for (V, F), O, w in zip(meshes, queries, W):
            ref = oracle_mod.winding_number(V, F, O)
            assert np.abs(w.cpu().numpy() - ref).max() <= 1e-6
    finally:
        b.close()


@pytest.mark.parametrize("adjoint,kappa", [("fp64", 4.0), ("mixed", 4.0), ("mixed", 3.0)])
def test_batched_backward_matches_single_mesh_adjoint(gpu_required, adjoint, kappa):
    """FP64: the single-mesh FP64 edge adjoint within 1e-12 (relative to the
    largest gradient). Mixed: the single-mesh mixed edge adjoint within 1e-6 (the
    same tiles and pairs; only the FP32 flush points and the FP64 partial order
    differ) and the FP64 one within 1e-4, as the single-mesh mixed path is."""
    import torch

    meshes, queries = _small_batch(seed=6)
    b = igl.batched.Batch(meshes, queries, target_pairs=1 << 16, adjoint=adjoint, kappa=kappa)
    try:
        assert b.info()["adjoint_fp64"] == (adjoint == "fp64")
        b.gW.copy_(torch.randn(b.gW.shape, dtype=torch.float64,
                               generator=torch.Generator().manual_seed(1)).cuda())
        b.forward()
        dV, dQ = b.backward()
        dVs, dQs, gs = b.split(dV.clone(), "v"), b.split(dQ.clone()), b.split(b.gW.clone())
        dV2, dQ2 = b.backward()
        assert torch.equal(dV2, dV) and torch.equal(dQ2, dQ)  # deterministic
        for (V, F), O, dv, dq, g in zip(meshes, queries, dVs, dQs, gs):
            Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
            ref_v, ref_q = wa.backward_edges(Vt, Ft, Ot, g)
            scale = max(float(ref_v.abs().max()), float(ref_q.abs().max()), 1e-30)
            tol = 1e-12 if adjoint == "fp64" else 1e-4
            assert float((dv - ref_v).abs().max()) <= tol * scale
            assert float((dq - ref_q).abs().max()) <= tol * scale
            if adjoint == "mixed":
                mv, mq = wa.backward_edges(Vt, Ft, Ot, g, precision="mixed", kappa=kappa)
                assert float((dv - mv).abs().max()) <= 1e-6 * scale
                assert float((dq - mq).abs().max()) <= 1e-6 * scale
    finally:
        b.close()


def test_graph_replay_matches_eager_and_is_deterministic(gpu_required):
    import torch

    meshes, queries = _small_batch(seed=8)
    b = igl.batched.Batch(meshes, queries, target_pairs=1 << 16)
    try:
        b.gW.normal_(generator=torch.Generator(device="cuda").manual_seed(3))
        b.step()
        torch.cuda.synchronize()
        eager = (b.W.clone(), b.dV.clone(), b.dQ.clone())
        b.step()
        torch.cuda.synchronize()
        assert torch.equal(b.W, eager[0]) and torch.equal(b.dV, eager[1])
        b.capture()
        b.W.zero_()
        b.dV.zero_()
        b.replay()
        torch.cuda.synchronize()
        assert torch.equal(b.W, eager[0])
        assert torch.equal(b.dV, eager[1]) and torch.equal(b.dQ, eager[2])
        # New query positions through the same graph.
        b.Q.add_(1e-3)
        b.replay()
        torch.cuda.synchronize()
        moved = b.W.clone()
        b.graph = None
        b.forward()
        torch.cuda.synchronize()
        assert torch.equal(b.W, moved)
    finally:
        b.close()


def test_autotuner_picks_and_caches(gpu_required, tmp_path, monkeypatch):
    monkeypatch.setenv("WN_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    meshes, queries = _small_batch(n=4, seed=9)
    space = {"qpt": (1, 2), "target_pairs": (1 << 16,), "ctas_per_sm": (0, 2),
             "kappa": (4.0,), "tile_faces": (64, 32)}
    first = igl.autotune.tune(meshes, queries, space=space, reps=1)
    assert not first["cached"] and 4 <= len(first["trials"]) <= 8
    assert {t["config"]["tile_faces"] for t in first["trials"]} == {64, 32}
    assert {t["config"]["ctas_per_sm"] for t in first["trials"]} == {0, 2}
    again = igl.autotune.tune(meshes, queries, space=space, reps=1)
    assert again["cached"] and again["config"] == first["config"]


def test_meshes_without_faces_or_queries(gpu_required, oracle_mod):
    """A mesh with no faces (W = 0 for its queries, no derivative), one with no
    queries, and ordinary ones in the same batch, forward and backward."""
    import torch

    V1, F1 = igl.synthetic.bumpy_icosphere(2, seed=31)
    V3, F3 = igl.synthetic.bumpy_icosphere(1, seed=32)
    O1 = igl.synthetic.mixed_queries(V1, F1, 700, seed=33, near_sigma=1e-3)
    O2 = np.random.default_rng(34).uniform(-1, 1, size=(300, 3))
    O4 = igl.synthetic.mixed_queries(V3, F3, 200, seed=35, near_sigma=1e-3)
    meshes = [(V1, F1), (V3, np.zeros((0, 3), np.int64)), (V3, F3), (V3, F3)]
    queries = [O1, O2, np.zeros((0, 3)), O4]
    b = igl.batched.Batch(meshes, queries, target_pairs=1 << 16)
    try:
        W = b.split(b.forward().clone())
        assert np.abs(W[0].cpu().numpy() - oracle_mod.winding_number(V1, F1, O1)).max() <= 1e-6
        assert torch.count_nonzero(W[1]) == 0 and W[2].numel() == 0
        assert np.abs(W[3].cpu().numpy() - oracle_mod.winding_number(V3, F3, O4)).max() <= 1e-6
        dV, dQ = b.backward(torch.ones_like(b.W))
        torch.cuda.synchronize()
        assert torch.isfinite(dV).all() and torch.isfinite(dQ).all()
        assert torch.count_nonzero(b.split(dQ)[1]) == 0   # no faces: no derivative
        assert torch.count_nonzero(b.split(dV, "v")[2]) == 0  # no queries: no derivative
    finally:
        b.close()


def _large_batch(seed=71, n=16, max_q=100_000):
    """16 meshes including a subdivision-7 (327,680 F) and a subdivision-6 one,
    0-10% faces deleted, queries log-uniform in [1024, 1e5], 50/50 box/near."""
    rng = np.random.default_rng(seed)
    levels = [7, 6] + [int(x) for x in rng.integers(2, 6, size=n - 2)]
    meshes, queries = [], []
    for i, level in enumerate(levels):
        V, F = igl.synthetic.bumpy_icosphere(level, seed=700 + i)
        F = igl.synthetic.delete_faces(F, float(rng.uniform(0, 0.1)), seed=800 + i)
        nq = int(np.exp(rng.uniform(np.log(1024), np.log(max_q))))
        meshes.append((V, F))
        queries.append(igl.synthetic.mixed_queries(V, F, nq, seed=900 + i, near_sigma=1e-3))
    return meshes, queries


def test_full_scale_batch_forward_backward_graph(gpu_required):
    """Configuration-5 scale: every query of every mesh against the plain FP64
    kernel (<= 1e-6), the batched FP64 adjoint against the single-mesh FP64
    boundary-edge adjoint (<= 1e-12 relative) and the mixed one against it within
    1e-4, and graph replays bit for bit equal to eager (both precisions)."""
    import torch

    meshes, queries = _large_batch()
    assert max(len(F) for _, F in meshes) > 290_000
    b = igl.batched.Batch(meshes, queries, adjoint="fp64")
    try:
        b.gW.normal_(generator=torch.Generator(device="cuda").manual_seed(72))
        b.step()
        torch.cuda.synchronize()
        eager = (b.W.clone(), b.dV.clone(), b.dQ.clone())
        assert b.info()["work_items"] > len(meshes)
        W = b.split(eager[0])
        dVs, dQs, gs = b.split(eager[1], "v"), b.split(eager[2]), b.split(b.gW.clone())
        for (V, F), O, w, dv, dq, g in zip(meshes, queries, W, dVs, dQs, gs):
            Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
            tri, ld, nf = wa.triangle_soa(Vt, Ft)
            assert float((w - wa.forward_fp64(tri, ld, nf, Ot)).abs().max()) <= 1e-6
            ref_v, ref_q = wa.backward_edges(Vt, Ft, Ot, g)
            scale = max(float(ref_v.abs().max()), float(ref_q.abs().max()), 1e-30)
            assert float((dv - ref_v).abs().max()) <= 1e-12 * scale
            assert float((dq - ref_q).abs().max()) <= 1e-12 * scale
        b.capture()
        b.W.zero_()
        b.dV.zero_()
        b.dQ.zero_()
        b.replay()
        torch.cuda.synchronize()
        assert torch.equal(b.W, eager[0])
        assert torch.equal(b.dV, eager[1]) and torch.equal(b.dQ, eager[2])
        # The mixed adjoint on the same batch: within 1e-4 of the FP64 one, and its
        # graph replay bit for bit equal to its eager run.
        b.graph = None
        _check_rc(b.handle.wn_batch_set_adjoint_fp64(b.batch, 0))
        b.step()
        torch.cuda.synchronize()
        mixed = (b.dV.clone(), b.dQ.clone())
        for dv, dq, mv, mq in zip(dVs, dQs, b.split(mixed[0], "v"), b.split(mixed[1])):
            scale = max(float(dv.abs().max()), float(dq.abs().max()), 1e-30)
            assert float((mv - dv).abs().max()) <= 1e-4 * scale
            assert float((mq - dq).abs().max()) <= 1e-4 * scale
        b.capture()
        b.dV.zero_()
        b.dQ.zero_()
        b.replay()
        torch.cuda.synchronize()
        assert torch.equal(b.dV, mixed[0]) and torch.equal(b.dQ, mixed[1])
    finally:
        b.close()
