"""Fast (hierarchical) winding numbers on the CPU.

The reference lists fast winding numbers as not covered (README.md:29), so
there is no reference output to match. Two checks replace it: (1) the library's
implementation against the oracle's independent numpy restatement of Barill et
al. 2018 on the same tree and beta (both FP64; the library folds the moments
into monomial coefficients, the oracle evaluates the unfolded tensors):
within 1e-12; (2) against the exact winding number (the reference's own
function, through the oracle): exact within 1e-12 when beta is so large that
no node is ever expanded, and within the expansion's error otherwise. The
error bounds below are measured on these seeded meshes with a margin of about
3x (max observed: 3.4e-3 at beta = 2, 1.1e-4 at beta = 4).
"""

import numpy as np
import pytest

import igl


def _open_s3(n=200):
    V, F = igl.synthetic.bumpy_icosphere(3, seed=11)
    F = igl.synthetic.delete_faces(F, 0.08, seed=12)
    return V, F, igl.synthetic.mixed_queries(V, F, n, seed=13, near_sigma=1e-3)


@pytest.mark.parametrize("beta", [1.0, 1.5, 2.0, 4.0])
def test_matches_oracle_restatement(oracle_mod, beta):
    V, F, O = _open_s3()
    expected = oracle_mod.fast_winding_number(V, F, O, beta)
    actual = igl.fast_winding_number(V, F, O, beta=beta)
    assert np.abs(actual - expected).max() <= 1e-12


def test_huge_beta_is_the_exact_winding_number(oracle_mod):
    V, F, O = _open_s3()
    O = np.concatenate([O, V[:10], 0.5 * (V[F[:10, 0]] + V[F[:10, 1]])])  # vertices, edges
    actual = igl.fast_winding_number(V, F, O, beta=1e9)
    assert np.abs(actual - oracle_mod.winding_number(V, F, O)).max() <= 1e-12


@pytest.mark.parametrize("beta,bound", [(2.0, 1e-2), (3.0, 2e-3), (4.0, 4e-4)])
def test_error_against_exact(oracle_mod, beta, bound):
    V, F = igl.synthetic.bumpy_icosphere(4, seed=3)
    O = igl.synthetic.mixed_queries(V, F, 400, seed=4, near_sigma=1e-3)
    err = np.abs(igl.fast_winding_number(V, F, O, beta=beta) - oracle_mod.winding_number(V, F, O))
    assert err.max() <= bound


def test_closed_mesh_inside_outside():
    V, F = igl.synthetic.bumpy_icosphere(4, seed=5)
    rng = np.random.default_rng(6)
    inside = rng.uniform(-0.5, 0.5, size=(100, 3))
    d = rng.normal(size=(100, 3))
    outside = 3.0 * d / np.linalg.norm(d, axis=1, keepdims=True)
    W = igl.fast_winding_number(V, F, np.concatenate([inside, outside]))
    assert np.abs(W[:100] - 1.0).max() < 1e-2 and np.abs(W[100:]).max() < 1e-2


def test_repeatable_and_span_independent(monkeypatch):
    V, F, O = _open_s3(3000)
    fwn = igl.FastWindingNumber(V, F)
    monkeypatch.setattr(igl, "worker_count", lambda items, work, kernel: 1)
    serial = fwn.evaluate(O)
    for workers in (2, 5):
        monkeypatch.setattr(igl, "worker_count",
                            lambda items, work, kernel, w=workers: max(1, min(items, w)))
        assert np.array_equal(fwn.evaluate(O), serial)
    assert fwn.info()["faces"] == len(F) and fwn.info()["depth"] >= 1
    fwn.close()


def test_contracts_and_edge_cases():
    V, F, O = _open_s3(5)
    with pytest.raises(ValueError):
        igl.fast_winding_number(V, F, O, beta=0.5)
    with pytest.raises(ValueError):
        igl.fast_winding_number(V, F, [[np.nan, 0, 0]])
    with pytest.raises(ValueError):
        igl.fast_winding_number(V, F, O, device="tpu")
    with pytest.raises(IndexError):
        igl.fast_winding_number(V, np.array([[0, 1, len(V)]]), O)
    assert np.array_equal(igl.fast_winding_number(V, np.zeros((0, 3), np.int64), O), np.zeros(5))
    assert igl.fast_winding_number(V, F, np.zeros((0, 3))).shape == (0,)
    w = igl.fast_winding_number(V, F, O[0])
    assert isinstance(w, float)


def _degenerate_soup():
    V, F = igl.synthetic.bumpy_icosphere(2, seed=21)
    F = np.asarray(F)
    zero = np.repeat(F[:6, :1], 3, axis=1)        # collapsed to a point
    pinched = F[6:12][:, [0, 0, 1]]               # two equal corners
    dup = F[12:40]                                # duplicated faces
    flipped = F[40:60, ::-1]                      # reversed orientation
    far_zero = np.full((9, 3), F[0, 0])           # a whole leaf of zero-area faces
    Fs = np.ascontiguousarray(np.concatenate([F, zero, pinched, dup, flipped, far_zero]))
    rng = np.random.default_rng(5)
    O = np.concatenate([V[:30], 0.5 * (V[F[:20, 0]] + V[F[:20, 1]]),
                        rng.uniform(-1.5, 1.5, size=(200, 3))])
    return V, Fs, O


@pytest.mark.parametrize("beta", [1.5, 2.0])
def test_degenerate_soup_matches_oracle(oracle_mod, beta):
    """Collapsed, pinched, duplicated and flipped faces, a leaf of zero-area
    faces, queries on vertices and edges: the host evaluator against the
    oracle's restatement (1e-12), and against the exact winding number when
    beta is so large that nothing is expanded. (Not beta = 1: a node's radius
    is the distance to its farthest vertex, so a query on that vertex sits
    exactly on the far-test boundary, and two implementations that round the
    node centre differently may expand the node or not.)"""
    V, F, O = _degenerate_soup()
    expected = oracle_mod.fast_winding_number(V, F, O, beta)
    assert np.abs(igl.fast_winding_number(V, F, O, beta=beta) - expected).max() <= 1e-12
    exact = oracle_mod.winding_number(V, F, O)
    assert np.abs(igl.fast_winding_number(V, F, O, beta=1e9) - exact).max() <= 1e-12
