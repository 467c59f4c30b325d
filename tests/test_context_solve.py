"""Drop-in solve_context_normal_equations: argument checks and the golden file.

The checks below run before any device call, so they need no GPU; the
device results are compared with the reference's in test_gpu_context_solve.py.
"""
import types
from pathlib import Path

import numpy as np
import pytest

from summit_b200 import jackknife as jk

GOLD = Path(__file__).resolve().parent / "golden" / "context_solve.npz"


def eq(a, b, **kw):
    return types.SimpleNamespace(matrix=a, rhs=b, **kw)


def test_rejects_non_finite_inputs_like_the_reference():
    a = np.eye(3)
    a[0, 1] = np.nan
    with pytest.raises(ValueError, match="normal matrix contains non-finite values"):
        jk.solve_context_normal_equations(eq(a, np.ones(3)))
    with pytest.raises(ValueError, match="normal RHS contains non-finite values"):
        jk.solve_context_normal_equations(eq(np.eye(3), np.array([1.0, np.inf, 0.0])))


def test_rejects_bad_shapes_and_rtol():
    with pytest.raises(ValueError, match="Normal-equation shapes are incompatible"):
        jk.solve_context_normal_equations(eq(np.eye(3), np.ones(2)))
    with pytest.raises(ValueError, match="Normal-equation shapes are incompatible"):
        jk.solve_context_normal_equations(eq(np.ones((2, 3)), np.ones(2)))
    with pytest.raises(ValueError, match="must be 2-dimensional"):
        jk.solve_context_normal_equations(eq(np.ones(3), np.ones(3)))
    for bad in (0.0, -1.0, float("nan")):
        with pytest.raises(ValueError, match="rtol must be finite and positive"):
            jk.solve_context_normal_equations(eq(np.eye(2), np.ones(2)), rtol=bad)


def test_rejects_directional_and_empty_systems():
    with pytest.raises(ValueError, match="target/source"):
        jk.solve_context_normal_equations(eq(np.eye(2), np.ones(2), target_source=True))
    with pytest.raises(ValueError, match="empty"):
        jk.solve_context_normal_equations(eq(np.zeros((0, 0)), np.zeros(0)))


def test_golden_file_is_self_consistent():
    z = np.load(GOLD)
    assert len(z["cases"]) >= 10
    for c in z["cases"]:
        if f"{c}/error" in z.files:
            continue
        a, b = z[f"{c}/matrix"], z[f"{c}/rhs"]
        s = 0.5 * (a + a.T)
        x = z[f"{c}/coefficients"]
        np.testing.assert_allclose(s @ x - b, z[f"{c}/solve_residual"], atol=1e-9 * np.abs(b).max())
        assert int(z[f"{c}/rank"]) == int(np.sum(np.abs(z[f"{c}/eigenvalues"]) > z[f"{c}/tolerance"]))
