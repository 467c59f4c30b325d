"""Golden vectors of the reference's rank-revealing normal-equation solve.

Runs SUMMIT's own ``solve_context_normal_equations`` (context/fit.py:474-525)
on seeded symmetric systems - well and badly conditioned, indefinite,
rank-deficient, a custom rtol, a tolerated and a material asymmetry - and
stores its results (or its error type and message) in ``context_solve.npz``.
Run in a checkout that has the reference sources:

    SUMMIT_REFERENCE_DIR=<summit checkout> python tests/golden/make_golden_context_solve.py
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def cases():
    rng = np.random.default_rng(20261204)

    def spd(k, cond):
        q, _ = np.linalg.qr(rng.standard_normal((k, k)))
        lam = np.geomspace(1.0, 1.0 / cond, k) * 3.7
        return (q * lam) @ q.T

    out = []
    a = spd(5, 10.0)
    out.append(("spd5", a, rng.standard_normal(5), None, True))
    a = spd(24, 1e6) * 1e3
    out.append(("spd24_cond1e6", a, rng.standard_normal(24), None, True))
    q, _ = np.linalg.qr(rng.standard_normal((6, 6)))
    a = (q * np.array([-2.0, -0.5, 0.3, 1.0, 4.0, 9.0])) @ q.T
    out.append(("indefinite6", a, rng.standard_normal(6), None, True))
    b = rng.standard_normal((8, 6))
    a = b @ b.T
    rhs = rng.standard_normal(8)
    out.append(("rank6of8", a, rhs, None, False))
    out.append(("rank6of8_full", a, rhs, None, True))
    a = spd(12, 1e8)
    out.append(("rtol1e-4", a, rng.standard_normal(12), 1e-4, False))
    a = spd(7, 100.0)
    a[0, 3] += 1e-12
    out.append(("tiny_asymmetry", a, rng.standard_normal(7), None, True))
    a = spd(7, 100.0)
    a[1, 2] += 1e-3
    out.append(("material_asymmetry", a, rng.standard_normal(7), None, True))
    out.append(("scalar", np.array([[2.5]]), np.array([1.25]), None, True))
    a = spd(40, 1e4)
    out.append(("spd40", a, rng.standard_normal(40), None, True))
    return out


def main() -> None:
    ref = Path(os.environ.get("SUMMIT_REFERENCE_DIR", "/root/reference"))
    sys.path.insert(0, str(ref / "src"))
    from summit.context.fit import ContextRankError, solve_context_normal_equations

    store: dict[str, np.ndarray] = {}
    names = []
    for name, a, rhs, rtol, full in cases():
        names.append(name)
        store[f"{name}/matrix"] = a
        store[f"{name}/rhs"] = rhs
        store[f"{name}/rtol"] = np.array(np.nan if rtol is None else rtol)
        store[f"{name}/require_full_rank"] = np.array(full)
        eq = types.SimpleNamespace(matrix=a, rhs=rhs, target_source=False,
                                   component_names=tuple(f"c{i}" for i in range(a.shape[0])))
        try:
            r = solve_context_normal_equations(eq, rtol=rtol, require_full_rank=full)
        except ContextRankError as e:
            store[f"{name}/error"] = np.array("ContextRankError")
            store[f"{name}/message"] = np.array(str(e))
            store[f"{name}/rank"] = np.array(e.diagnostics.rank)
            continue
        except ValueError as e:
            store[f"{name}/error"] = np.array("ValueError")
            store[f"{name}/message"] = np.array(str(e))
            continue
        d = r.diagnostics
        store[f"{name}/coefficients"] = r.coefficients
        store[f"{name}/eigenvalues"] = d.eigenvalues
        store[f"{name}/singular_values"] = d.singular_values
        store[f"{name}/rank"] = np.array(r.rank)
        store[f"{name}/condition_number"] = np.array(r.condition_number)
        store[f"{name}/tolerance"] = np.array(d.tolerance)
        store[f"{name}/symmetry_error"] = np.array(d.symmetry_error)
        store[f"{name}/solve_residual"] = r.solve_residual
        store[f"{name}/relative_residual"] = np.array(r.relative_residual)
        store[f"{name}/minimum_gram_eigenvalue"] = np.array(r.minimum_gram_eigenvalue)
        store[f"{name}/absolute_tolerance"] = np.array(r.absolute_tolerance)
        # subspaces compared through their projectors (bases are unique only
        # up to rotation within repeated eigenvalues and sign)
        store[f"{name}/null_projector"] = r.null_space @ r.null_space.T
        store[f"{name}/retained_projector"] = r.retained_directions @ r.retained_directions.T
    store["cases"] = np.array(names)
    np.savez_compressed(HERE / "context_solve.npz", **store)
    print(f"wrote {HERE / 'context_solve.npz'} ({len(names)} cases)")


if __name__ == "__main__":
    main()
