"""The oracle is pinned before it is trusted (CPU only).

Pins: the reference's known answer (tetrahedron, tests/test_parity.py:74-85),
the committed golden fixtures produced by the reference's own Python package
(tests/golden/make_golden.py), the 40-digit mpmath solid-angle sums stored in
those fixtures, closed-mesh invariants, and the reference's bitwise
serial/parallel equality (tests/test_parity.py:418-427).
"""

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden, tetrahedron


def test_tetrahedron_known_answer(oracle_mod):
    V, F = tetrahedron()
    Q = np.array([[0.1, 0.1, 0.1], [2.0, 2.0, 2.0], [-1.0, 0.2, 0.2]])
    W = oracle_mod.winding_number(V, F, Q)
    assert W[0] == pytest.approx(1.0, abs=1e-14)
    assert np.abs(W[1:]).max() < 1e-14


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_shim_golden(oracle_mod, name):
    g = load_golden(name)
    W = oracle_mod.winding_number(g["V"], g["F"], g["O"])
    # Same arithmetic and order as the fixture generator: bit-for-bit.
    assert np.array_equal(W, g["W"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_mpmath(oracle_mod, name):
    g = load_golden(name)
    W = oracle_mod.winding_number(g["V"], g["F"], g["O_mp"])
    assert np.abs(W - g["W_mp"]).max() < 1e-14


def test_oracle_mpmath_on_degenerate_queries(oracle_mod):
    V, F = tetrahedron()
    # On a vertex (solid angle 1/8 of the sphere), on an edge midpoint (3/4),
    # far away (0).
    Q = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1e3, -2e3, 5e2]])
    W = oracle_mod.winding_number(V, F, Q)
    ref = oracle_mod.winding_number_mp(V, F, Q)
    assert np.abs(W - ref).max() < 1e-14
    assert W[0] == pytest.approx(0.125, abs=1e-15)
    assert W[1] == pytest.approx(0.75, abs=1e-15)
    # Inside a face the sum jumps by 1 across the surface; the signed zero of
    # det picks a side (here det = -0, atan2 = -pi), so W is one of the limits.
    w_face = oracle_mod.winding_number(V, F, [[0.3, 0.3, 0.0]])[0]
    assert min(abs(w_face), abs(w_face - 1.0)) < 1e-15


def test_closed_mesh_is_integer_off_surface(oracle_mod):
    import igl.synthetic as syn

    V, F = syn.bumpy_icosphere(2, seed=3)
    rng = np.random.default_rng(4)
    inside = rng.uniform(-0.5, 0.5, size=(64, 3))
    outside = rng.normal(size=(64, 3))
    outside *= (2.0 / np.linalg.norm(outside, axis=1))[:, None]
    assert np.abs(oracle_mod.winding_number(V, F, inside) - 1.0).max() < 1e-13
    assert np.abs(oracle_mod.winding_number(V, F, outside)).max() < 1e-13


def test_oracle_serial_and_parallel_are_bitwise_equal(oracle_mod):
    g = load_golden("serial_parallel")
    serial = oracle_mod.winding_number(g["V"], g["F"], g["O"], workers=1)
    for workers in (2, 4, 8):
        assert np.array_equal(oracle_mod.winding_number(g["V"], g["F"], g["O"], workers), serial)


def test_oracle_empty_inputs(oracle_mod):
    V, F = tetrahedron()
    assert oracle_mod.winding_number(V, F, np.zeros((0, 3))).shape == (0,)
    W = oracle_mod.winding_number(V, F[:0], np.ones((3, 3)))
    assert np.array_equal(W, np.zeros(3))
