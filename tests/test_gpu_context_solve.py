"""Device solve_context_normal_equations against the reference's own results
(golden vectors from context/fit.py:474-525, tests/golden/make_golden_context_solve.py).

Tolerances: eigenvalues, tolerance, residual and projectors are compared
relative to the matrix scale (1e-10); coefficients relative to their norm
(1e-9, scaled by the retained condition number where the system is
ill-conditioned); ranks and error messages exactly; the relative residual,
which is roundoff, within 10x of the reference's.
"""
import types
from pathlib import Path

import numpy as np
import pytest

from summit_b200 import jackknife as jk

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "context_solve.npz")
CASES = [str(c) for c in GOLD["cases"]]


def _get(c, k):
    return GOLD[f"{c}/{k}"]


@pytest.mark.parametrize("case", CASES)
def test_context_solve_matches_reference(case):
    a, b = _get(case, "matrix"), _get(case, "rhs")
    rtol = float(_get(case, "rtol"))
    kw = dict(rtol=None if np.isnan(rtol) else rtol,
              require_full_rank=bool(_get(case, "require_full_rank")))
    e = types.SimpleNamespace(matrix=a, rhs=b, component_names=tuple(f"c{i}" for i in range(len(b))))
    if f"{case}/error" in GOLD.files:
        kind, msg = str(_get(case, "error")), str(_get(case, "message"))
        exc = jk.ContextRankError if kind == "ContextRankError" else ValueError
        with pytest.raises(exc) as info:
            jk.solve_context_normal_equations(e, **kw)
        if kind == "ContextRankError":
            assert info.value.diagnostics.rank == int(_get(case, "rank"))
            assert info.value.component_names == e.component_names
            # the message carries the tolerance to 6 significant digits
            assert str(info.value).split(" at tolerance")[0] == msg.split(" at tolerance")[0]
            got_tol = float(str(info.value).split("tolerance ")[1].rstrip("."))
            want_tol = float(msg.split("tolerance ")[1].rstrip("."))
            assert got_tol == pytest.approx(want_tol, rel=1e-5)
        else:
            assert str(info.value) == msg
        return
    r = jk.solve_context_normal_equations(e, **kw)
    scale = max(np.abs(a).max(), 1.0)
    assert r.rank == int(_get(case, "rank"))
    np.testing.assert_allclose(r.diagnostics.eigenvalues, _get(case, "eigenvalues"),
                               rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(r.diagnostics.singular_values, _get(case, "singular_values"),
                               rtol=0, atol=1e-10 * scale)
    assert r.diagnostics.tolerance == pytest.approx(float(_get(case, "tolerance")), rel=1e-10)
    assert r.diagnostics.symmetry_error == float(_get(case, "symmetry_error"))
    assert r.absolute_tolerance == float(_get(case, "absolute_tolerance"))
    assert r.minimum_gram_eigenvalue == pytest.approx(float(_get(case, "minimum_gram_eigenvalue")),
                                                      rel=1e-9, abs=1e-10 * scale)
    cond = float(_get(case, "condition_number"))
    if np.isinf(cond):
        assert np.isinf(r.condition_number)
    else:
        assert r.condition_number == pytest.approx(cond, rel=1e-6)
    want = _get(case, "coefficients")
    kept = np.abs(_get(case, "eigenvalues")) > float(_get(case, "tolerance"))
    kcond = np.abs(_get(case, "eigenvalues"))[kept].max() / np.abs(_get(case, "eigenvalues"))[kept].min()
    err = np.linalg.norm(r.coefficients - want) / max(np.linalg.norm(want), 1e-300)
    assert err <= 1e-12 * max(kcond, 1.0) + 1e-9
    np.testing.assert_allclose(r.solve_residual, _get(case, "solve_residual"),
                               rtol=0, atol=1e-9 * scale * max(np.abs(want).max(), 1.0))
    np.testing.assert_allclose(r.null_space @ r.null_space.T, _get(case, "null_projector"),
                               rtol=0, atol=1e-8)
    np.testing.assert_allclose(r.retained_directions @ r.retained_directions.T,
                               _get(case, "retained_projector"), rtol=0, atol=1e-8)
    # roundoff of the solve: same order as the reference's, not the same bits
    ref_rr = float(_get(case, "relative_residual"))
    assert r.relative_residual <= max(10.0 * ref_rr, 1e-14 * max(kcond, 1.0))
