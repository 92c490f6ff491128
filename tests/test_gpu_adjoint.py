"""Hand-written adjoint vs FP64 torch autograd and FP64 central differences (B200).

* Torch reference: autograd of the FP64 torch expression of the solid-angle sum
  (oracle.winding_torch) on the subdivision-3 mesh (1,280 F) x 4,096 queries.
* Finite differences: the subdivision-5 open mesh (8% faces deleted) with
  262,144 near-surface queries, upstream dL/dW ~ N(0, 1); central differences
  with h = 1e-6 on 64 seeded coordinates (32 of V, 32 of O) through the plain
  FP64 forward. A coordinate is usable when no query crosses the surface
  between o - h and o + h (W would jump by 1) and the h and 2h differences
  agree; at least 56 of the 64 must be usable.
"""

import numpy as np
import pytest

import igl
from igl import autograd as wa

pytestmark = pytest.mark.gpu


def _cuda(x, dtype=None):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t.to(dtype) if dtype is not None else t


@pytest.mark.parametrize("adjoint", ["faces", "edges"])
def test_matches_torch_autograd_fp64(gpu_required, oracle_mod, adjoint):
    import torch

    V, F = igl.synthetic.bumpy_icosphere(3, seed=11)
    F = igl.synthetic.delete_faces(F, 0.08, seed=12)
    O = igl.synthetic.mixed_queries(V, F, 4096, seed=13, near_sigma=1e-2)
    g = np.random.default_rng(14).normal(size=len(O))
    Vt = _cuda(V).requires_grad_(True)
    Ot = _cuda(O).requires_grad_(True)
    Ft = _cuda(F)
    W = wa.winding_number_torch(Vt, Ft, Ot, adjoint=adjoint)
    (W * _cuda(g)).sum().backward()
    dV, dO = Vt.grad.cpu().numpy(), Ot.grad.cpu().numpy()

    Vr = _cuda(V).requires_grad_(True)
    Or = _cuda(O).requires_grad_(True)
    Wr = oracle_mod.winding_torch(Vr, Ft, Or)
    (Wr * _cuda(g)).sum().backward()
    dV_ref, dO_ref = Vr.grad.cpu().numpy(), Or.grad.cpu().numpy()
    assert np.abs(W.detach().cpu().numpy() - Wr.detach().cpu().numpy()).max() < 1e-12
    assert np.abs(dV - dV_ref).max() <= 1e-9 * np.abs(dV_ref).max()
    assert np.abs(dO - dO_ref).max() <= 1e-9 * np.abs(dO_ref).max()
    del torch


@pytest.mark.parametrize("adjoint", ["faces", "edges"])
def test_central_differences_c4(gpu_required, adjoint):
    import torch

    V, F, O, _ = igl.synthetic.workload("c4_grad")
    rng = np.random.default_rng(44)
    g = rng.normal(size=len(O))
    Vt = _cuda(V).requires_grad_(True)
    Ot = _cuda(O).requires_grad_(True)
    Ft = _cuda(F)
    gt = _cuda(g)
    W = wa.winding_number_torch(Vt, Ft, Ot, adjoint=adjoint)
    (W * gt).sum().backward()
    dV, dO = Vt.grad.cpu().numpy(), Ot.grad.cpu().numpy()

    used = np.unique(F)
    picks = [("V", int(i), int(k)) for i, k in zip(rng.choice(used, 32, replace=False),
                                                   rng.integers(0, 3, 32))]
    picks += [("O", int(i), int(k)) for i, k in zip(rng.choice(len(O), 32, replace=False),
                                                    rng.integers(0, 3, 32))]

    def loss_and_w(Vx, Ox):
        tri, ld, nf = wa.triangle_soa(_cuda(Vx), Ft)
        w = wa.forward_fp64(tri, ld, nf, _cuda(Ox))
        return float((w * gt).sum()), w

    usable, worst = 0, 0.0
    for which, i, k in picks:
        fd = {}
        for h in (1e-6, 2e-6):
            Vp, Vm, Op, Om = V.copy(), V.copy(), O.copy(), O.copy()
            if which == "V":
                Vp[i, k] += h
                Vm[i, k] -= h
            else:
                Op[i, k] += h
                Om[i, k] -= h
            lp, wp = loss_and_w(Vp, Op)
            lm, wm = loss_and_w(Vm, Om)
            crossed = float((wp - wm).abs().max()) > 0.5
            fd[h] = None if crossed else (lp - lm) / (2 * h)
        if fd[1e-6] is None or fd[2e-6] is None:
            continue
        scale = max(1.0, abs(fd[1e-6]))
        if abs(fd[1e-6] - fd[2e-6]) > 1e-4 * scale:
            continue  # differences not converged at this h (a query within ~h of a face)
        usable += 1
        grad = dV[i, k] if which == "V" else dO[i, k]
        worst = max(worst, abs(grad - fd[1e-6]) / scale)
    assert usable >= 56, usable
    assert worst <= 1e-5, worst
    del torch


@pytest.mark.parametrize("adjoint", ["faces", "edges"])
def test_closed_mesh_gradients_cancel(gpu_required, adjoint):
    V, F = igl.synthetic.bumpy_icosphere(3, seed=21)
    rng = np.random.default_rng(22)
    O = np.concatenate([rng.uniform(-0.4, 0.4, size=(64, 3)), rng.normal(size=(64, 3)) * 3])
    Vt = _cuda(V).requires_grad_(True)
    Ot = _cuda(O).requires_grad_(True)
    W = wa.winding_number_torch(Vt, _cuda(F), Ot, adjoint=adjoint)
    W.sum().backward()
    # Off the surface W of a closed mesh is locally constant: every derivative cancels.
    assert float(Vt.grad.abs().max()) < 1e-9
    assert float(Ot.grad.abs().max()) < 1e-9


@pytest.mark.parametrize("adjoint", ["faces", "edges"])
def test_deterministic_and_finite_on_degenerate_queries(gpu_required, adjoint):
    V, F = igl.synthetic.bumpy_icosphere(2, seed=31)
    O = np.concatenate([V[:20], 0.5 * (V[F[:20, 0]] + V[F[:20, 1]]),
                        np.random.default_rng(32).normal(size=(200, 3))])
    grads = []
    for _ in range(2):
        Vt = _cuda(V).requires_grad_(True)
        Ot = _cuda(O).requires_grad_(True)
        W = wa.winding_number_torch(Vt, _cuda(F), Ot, adjoint=adjoint)
        (W * _cuda(np.linspace(-1, 1, len(O)))).sum().backward()
        grads.append((Vt.grad.cpu().numpy(), Ot.grad.cpu().numpy()))
    assert np.isfinite(grads[0][0]).all() and np.isfinite(grads[0][1]).all()
    assert np.array_equal(grads[0][0], grads[1][0])
    assert np.array_equal(grads[0][1], grads[1][1])


def test_empty_faces(gpu_required):
    import torch

    V = np.random.default_rng(1).normal(size=(5, 3))
    Vt = _cuda(V).requires_grad_(True)
    Ot = _cuda(np.ones((3, 3))).requires_grad_(True)
    W = wa.winding_number_torch(Vt, torch.zeros((0, 3), dtype=torch.int64, device="cuda"), Ot)
    W.sum().backward()
    assert float(W.abs().max()) == 0.0
    assert float(Vt.grad.abs().max()) == 0.0 and float(Ot.grad.abs().max()) == 0.0


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_mixed_adjoint_matches_fp64_adjoint(gpu_required, dtype):
    """Mixed-precision adjoint (FP32 far pairs, FP64 near pairs) vs the FP64 adjoint."""
    import torch

    V, F, O, _ = igl.synthetic.workload("c4_grad", n_queries=8192)
    g = np.random.default_rng(45).normal(size=len(O))
    out = {}
    for precision in ("fp64", "mixed"):
        Vt = _cuda(V).requires_grad_(True)
        Ot = _cuda(O, getattr(torch, dtype) if precision == "mixed" else None)
        Ot.requires_grad_(True)
        W = wa.winding_number_torch(Vt, _cuda(F), Ot, precision=precision, adjoint="faces")
        (W * _cuda(g, W.dtype)).sum().backward()
        out[precision] = (W.detach().double().cpu().numpy(), Vt.grad.cpu().numpy(),
                          Ot.grad.double().cpu().numpy())
    w64, dV64, dO64 = out["fp64"]
    wm, dVm, dOm = out["mixed"]
    tol_w = 1e-6 if dtype == "float64" else 1e-5  # float32 queries are rounded on input
    if dtype == "float64":
        assert np.abs(wm - w64).max() <= tol_w
        assert np.abs(dVm - dV64).max() <= 1e-4 * np.abs(dV64).max()
        assert np.abs(dOm - dO64).max() <= 1e-4 * np.abs(dO64).max()
    else:
        # float32 queries move each point by up to ~6e-8: compare the FP64 adjoint
        # evaluated at the rounded points instead.
        O32 = O.astype(np.float32).astype(np.float64)
        Vt = _cuda(V).requires_grad_(True)
        Ot = _cuda(O32).requires_grad_(True)
        W = wa.winding_number_torch(Vt, _cuda(F), Ot, precision="fp64", adjoint="faces")
        (W * _cuda(g)).sum().backward()
        assert np.abs(wm - W.detach().cpu().numpy()).max() <= 1e-6
        assert np.abs(dVm - Vt.grad.cpu().numpy()).max() <= 1e-4 * np.abs(dV64).max()
        assert np.abs(dOm - Ot.grad.cpu().numpy()).max() <= 1e-3 * np.abs(dO64).max()


def test_edge_and_face_adjoints_agree_on_nonmanifold_soup(gpu_required):
    """Inconsistent orientation and a non-manifold edge: net multiplicities still telescope."""
    import torch

    V, F = igl.synthetic.bumpy_icosphere(2, seed=61)
    F = igl.synthetic.delete_faces(F, 0.1, seed=62).copy()
    F[:7] = F[:7, [0, 2, 1]]                        # flipped faces
    O = igl.synthetic.mixed_queries(V, F, 1024, seed=63, near_sigma=1e-2)
    F = np.concatenate([F, F[20:23], [[5, 5, 9]]])  # duplicated faces, a degenerate face
    g = np.random.default_rng(64).normal(size=len(O))
    res = {}
    for adjoint in ("faces", "edges"):
        Vt = _cuda(V).requires_grad_(True)
        Ot = _cuda(O).requires_grad_(True)
        W = wa.winding_number_torch(Vt, _cuda(F), Ot, adjoint=adjoint)
        (W * _cuda(g)).sum().backward()
        res[adjoint] = (Vt.grad.cpu().numpy(), Ot.grad.cpu().numpy())
    for a, b in zip(res["faces"], res["edges"]):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()
    del torch


def test_large_fp64_forward_takes_the_prepared_mesh(gpu_required):
    """Above 1e9 pairs the torch FP64 forward runs the prepared-mesh kernel, as
    the drop-in does; it agrees with the streaming kernel within 1e-12."""
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=65536)  # 18,842 F: 1.2e9 pairs
    Vt, Ft, Ot = _cuda(V), _cuda(F), _cuda(O)
    assert wa.use_prepared_fp64(len(F), len(O))
    W = wa.winding_number_torch(Vt, Ft, Ot, precision="fp64")
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    assert (W - wa.forward_fp64(tri, ld, nf, Ot)).abs().max().item() <= 1e-12


def test_mixed_float32_queries_full_size_c4(gpu_required):
    """Configuration 4 with float32 queries at full size (262,144 near-surface
    points on the open 18,842-face mesh): the mixed forward against the plain FP64
    kernel at the rounded points (<= 1e-6 over every query), and the mixed
    per-face adjoint against the FP64 per-face adjoint there."""
    import torch

    V, F, O, _ = igl.synthetic.workload("c4_grad")
    assert len(O) == 262144
    g = np.random.default_rng(46).normal(size=len(O))
    O32 = O.astype(np.float32)
    Vt = _cuda(V).requires_grad_(True)
    Ot = _cuda(O32).requires_grad_(True)
    W = wa.winding_number_torch(Vt, _cuda(F), Ot, adjoint="faces")  # float32: mixed
    assert W.dtype == torch.float32
    (W * _cuda(g, torch.float32)).sum().backward()
    Vr = _cuda(V).requires_grad_(True)
    Or = _cuda(O32.astype(np.float64)).requires_grad_(True)
    Wr = wa.winding_number_torch(Vr, _cuda(F), Or, precision="fp64", adjoint="faces")
    (Wr * _cuda(g)).sum().backward()
    assert float((W.double() - Wr).abs().max()) <= 1e-6
    dV, dV64 = Vt.grad.cpu().numpy(), Vr.grad.cpu().numpy()
    dO, dO64 = Ot.grad.double().cpu().numpy(), Or.grad.cpu().numpy()
    assert np.isfinite(dV).all() and np.isfinite(dO).all()
    assert np.abs(dV - dV64).max() <= 1e-4 * np.abs(dV64).max()
    assert np.abs(dO - dO64).max() <= 1e-3 * np.abs(dO64).max()


def test_auto_adjoint_picks_welded_edges_on_a_soup_and_edges_on_a_mesh(gpu_required,
                                                                      monkeypatch):
    """adjoint="auto": a mixed forward on a triangle soup (three boundary edges per
    face, 1.5 welded edges per face) takes the welded-edge adjoint, one on an open
    indexed mesh the boundary-edge adjoint; both give the FP64 adjoint's gradients."""
    import torch

    V, F = igl.synthetic.bumpy_icosphere(3, seed=81)
    F = igl.synthetic.delete_faces(F, 0.05, seed=82)
    O = igl.synthetic.mixed_queries(V, F, 2048, seed=83, near_sigma=1e-2)
    g = np.random.default_rng(84).normal(size=len(O))
    Vs, Fs = igl.synthetic.unshare_vertices(V, F)
    calls = []
    real_faces = wa.PreparedMesh.backward
    real_edges = wa.backward_edges
    real_welded = wa.backward_welded_edges
    monkeypatch.setattr(wa.PreparedMesh, "backward",
                        lambda self, *a: calls.append("faces") or real_faces(self, *a))
    monkeypatch.setattr(wa, "backward_edges",
                        lambda *a, **k: calls.append("edges") or real_edges(*a, **k))
    monkeypatch.setattr(wa, "backward_welded_edges",
                        lambda *a, **k: calls.append("welded") or real_welded(*a, **k))
    for (Vx, Fx), expect in (((Vs, Fs), "welded"), ((V, F), "edges")):
        calls.clear()
        grads = {}
        for precision in ("mixed", "fp64"):
            Vt = _cuda(Vx).requires_grad_(True)
            Ot = _cuda(O).requires_grad_(True)
            W = wa.winding_number_torch(Vt, _cuda(Fx), Ot, precision=precision)
            (W * _cuda(g)).sum().backward()
            grads[precision] = (Vt.grad.cpu().numpy(), Ot.grad.cpu().numpy())
        assert calls[0] == expect, calls
        for a, b in zip(grads["mixed"], grads["fp64"]):
            assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()
    del torch


@pytest.mark.parametrize("case", ["c4", "open_c3_sample", "degenerate"])
def test_mixed_edge_adjoint_matches_fp64_edge_adjoint(gpu_required, case):
    """The mixed-precision boundary-edge adjoint (FP32 far pairs in Morton-ordered
    64-edge tiles, FP64 pairs with an endpoint within kappa |e|) against the FP64
    boundary-edge adjoint: within 1e-4 of the largest gradient, finite, and bit
    for bit repeatable; queries on vertices and edge midpoints included."""
    import torch

    if case == "c4":
        V, F, O, _ = igl.synthetic.workload("c4_grad", n_queries=16384)
    elif case == "open_c3_sample":
        V, F, O, _ = igl.synthetic.workload("c3_open", n_queries=4096)
    else:
        V, F = igl.synthetic.bumpy_icosphere(3, seed=91)
        F = igl.synthetic.delete_faces(F, 0.2, seed=92).copy()
        F[:9] = F[:9, [0, 2, 1]]
        F = np.concatenate([F, F[30:33], [[4, 4, 17]]])
        O = np.concatenate([V[:40], 0.5 * (V[F[:40, 0]] + V[F[:40, 1]]),
                            igl.synthetic.mixed_queries(V, F, 2000, seed=93, near_sigma=1e-3)])
    g = _cuda(np.random.default_rng(94).normal(size=len(O)))
    Vt, Ft, Ot = _cuda(V), _cuda(F), _cuda(O)
    edges = wa.boundary_edges(Vt, Ft)
    assert edges[1] > 0
    dV64, dO64 = wa.backward_edges(Vt, Ft, Ot, g, edges)
    dVm, dOm = wa.backward_edges(Vt, Ft, Ot, g, edges, precision="mixed")
    dVm2, dOm2 = wa.backward_edges(Vt, Ft, Ot, g, edges, precision="mixed")
    assert torch.isfinite(dVm).all() and torch.isfinite(dOm).all()
    assert torch.equal(dVm, dVm2) and torch.equal(dOm, dOm2)
    assert float((dVm - dV64).abs().max()) <= 1e-4 * float(dV64.abs().max())
    assert float((dOm - dO64).abs().max()) <= 1e-4 * float(dO64.abs().max())


@pytest.mark.parametrize("case", ["closed_soup", "open_soup", "random_soup"])
def test_welded_edge_adjoint_on_soups(gpu_required, case):
    """The soup adjoint through sides welded by position against the per-face
    FP64 adjoint: within 1e-4 of the largest gradient, for a closed mesh and an
    open one given as soups (every edge shared by two sides) and a random soup
    (no shared sides); adjoint="auto" picks it where it is cheaper than faces."""
    import torch

    V, F = igl.synthetic.bumpy_icosphere(3, seed=101)
    if case == "open_soup":
        F = igl.synthetic.delete_faces(F, 0.1, seed=102)
    if case == "random_soup":
        rng = np.random.default_rng(103)
        Vs = rng.normal(size=(3 * 900, 3))
        Fs = np.arange(3 * 900).reshape(-1, 3)
    else:
        Vs, Fs = igl.synthetic.unshare_vertices(V, F)
    O = igl.synthetic.mixed_queries(Vs, Fs, 3000, seed=104, near_sigma=1e-3)
    g = _cuda(np.random.default_rng(105).normal(size=len(O)))
    Vt, Ft, Ot = _cuda(Vs), _cuda(Fs), _cuda(O)
    welded = wa.welded_edges(Vt, Ft)
    dVw, dOw = wa.backward_welded_edges(Vt, Ft, Ot, g, welded)
    ref = {}
    Vr = _cuda(Vs).requires_grad_(True)
    Orr = _cuda(O).requires_grad_(True)
    W = wa.winding_number_torch(Vr, Ft, Orr, precision="fp64", adjoint="faces")
    (W * g).sum().backward()
    dV64, dO64 = Vr.grad, Orr.grad
    assert torch.isfinite(dVw).all() and torch.isfinite(dOw).all()
    assert float((dVw - dV64).abs().max()) <= 1e-4 * float(dV64.abs().max())
    assert float((dOw - dO64).abs().max()) <= 1e-4 * float(dO64.abs().max()) + 1e-12
    if case == "closed_soup":
        assert welded[1] == 3 * len(Fs) // 2
