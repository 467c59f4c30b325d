"""GPU: generalized per-variant GxE two-pass estimator against the reference.

Golden vectors come from the reference's own GeneralizedGxEPass1Executor /
GeneralizedGxEPass2Executor run on the decoded genotypes of the same BED rows
(tests/golden/make_golden_generalized_gxe.py).  Tolerances: probe signs bit
for bit; the device products against the CPU oracle's dense products 1e-8
(relative to the largest entry: the 4-digit sketch representation); every
estimator output 1e-6 per element, relative, with an absolute floor of 1e-7 of
the array's largest entry (off-diagonal pair products change sign, and the
sketch digits carry 2^-29 of a column's largest value)."""
from pathlib import Path

import numpy as np
import pytest

from conftest import assert_rel_elementwise

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "generalized_gxe.npz")
CASES = ["unprojected", "projected"]


@pytest.fixture(scope="module")
def session():
    from summit_b200.session import GwSession

    s = GwSession(GOLD["rows"], int(GOLD["n"]))
    yield s
    s.close()


@pytest.fixture(scope="module")
def decoded():
    from oracle.oracle import Oracle

    X, _m, _i = Oracle().standardize(GOLD["rows"], int(GOLD["n"]), 0, int(GOLD["m"]))
    return X


def test_device_probes_are_the_reference_stream():
    from summit_b200 import generalized_gxe as gg

    for case in CASES:
        spec = gg.GlobalVariantProbeSpec(root_seed=int(GOLD[f"{case}/root_seed"]),
                                         probe_offset=7, probe_count=11)
        want = GOLD[f"{case}/probes"]
        np.testing.assert_array_equal(gg.global_variant_probes(spec, 0, want.shape[0]), want)
        np.testing.assert_array_equal(gg.global_variant_probes(spec, 100, 57), want[100:157])
    far = gg.GlobalVariantProbeSpec(root_seed=2 ** 63 + 12345, probe_offset=2 ** 40, probe_count=5)
    np.testing.assert_array_equal(gg.global_variant_probes(far, 10 ** 12, 37), GOLD["far_probes"])


def test_device_products_match_dense_products(session, decoded):
    from oracle import generalized_oracle as go
    from summit_b200 import generalized_gxe as gg

    X = decoded
    rng = np.random.default_rng(4)
    j0, j1 = 17, 251
    annot = rng.uniform(0.0, 2.0, size=(j1 - j0, 3))
    annot[::5, 1] = 0.0
    z = np.sign(rng.normal(size=(j1 - j0, 9)))
    got = gg._source_product(session, j0, j1, annot, z)
    want = go.source_product(X, j0, j1, annot, z)
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()
    Y = rng.normal(size=(X.shape[0], 40))
    got = gg._target_product(session, j0, j1, Y)
    want = go.target_product(X, j0, j1, Y)
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()
    for r in (0, 2):
        basis = np.asfortranarray(rng.normal(size=(X.shape[0], 3)))
        fixed = np.asfortranarray(np.linalg.qr(rng.normal(size=(X.shape[0], max(r, 1))))[0][:, :r])
        coef = go.target_product(X, j0, j1, (basis[:, :, None] * fixed[:, None, :]).reshape(
            X.shape[0], 3 * r)).reshape(j1 - j0, 3, r) if r else None
        num = np.zeros((3 * 6, X.shape[0]))
        gg._component_diagonal(session, j0, j1, annot, basis, fixed, coef, num)
        ref = np.zeros_like(num)
        go.component_diagonal(X, j0, j1, annot, basis, fixed, coef, ref)
        assert np.abs(num - ref).max() <= 1e-12 * np.abs(ref).max()


def test_device_rhs_assembly_matches_host_rhs(session, decoded):
    """Pass-2 scores from the sources (right-hand side formed on the device)
    equal the scores from the host-assembled right-hand side bit for bit."""
    from oracle import generalized_oracle as go
    from summit_b200 import generalized_gxe as gg

    n, m = decoded.shape
    rng = np.random.default_rng(12)
    K, Q, B, P = 2, 3, 5, 6
    rows = rng.normal(size=(K, Q, B, n))
    basis = rng.normal(size=(n, Q))
    fam = [(t, s) for t in range(Q) for s in range(Q)]
    ft = np.array([t for t, _ in fam], np.int32)
    fs = np.array([s for _, s in fam], np.int32)
    pairs = gg.pair_order(Q)
    term_off, term_f1, term_f2 = [0], [], []
    for tp in pairs:
        for sp in pairs:
            for tl, tr in gg._orientations(tp):
                for sl, sr in gg._orientations(sp):
                    term_f1.append(tr * Q + sl)
                    term_f2.append(tl * Q + sr)
            term_off.append(len(term_f1))
    to, f1, f2 = (np.asarray(x, np.int32) for x in (term_off, term_f1, term_f2))
    annot = rng.uniform(0.0, 1.0, size=(m, K))
    rhs = go.assemble_rhs(rows, basis, ft, fs)
    want = gg._pass2_scores(session, rhs, K, B, len(fam), P, to, f1, f2, float(n - 1), annot, 97)
    got = gg._pass2_scores_sources(session, rows, basis, ft, fs, K, B, P, to, f1, f2,
                                   float(n - 1), annot, 97)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


@pytest.mark.parametrize("case", CASES)
def test_two_pass_matches_reference_executors(session, case):
    from summit_b200 import generalized_gxe as gg

    spec = gg.GlobalVariantProbeSpec(root_seed=int(GOLD[f"{case}/root_seed"]), probe_offset=7,
                                     probe_count=11)
    p1, p2 = gg.two_pass(session, GOLD[f"{case}/basis"], GOLD[f"{case}/fixed"],
                         GOLD[f"{case}/annot"], spec, variant_block_width=128)
    assert_rel_elementwise(p1.contextual_sources, GOLD[f"{case}/contextual_sources"], 1e-6,
                           "contextual_sources", atol_frac=1e-7)
    for key in ("directional_ldscores", "directed_numerator", "symmetric_numerator",
                "genetic_gram", "component_kernel_diagonal", "same_person"):
        assert_rel_elementwise(getattr(p2, key), GOLD[f"{case}/{key}"], 1e-6, key,
                               atol_frac=1e-7)


@pytest.mark.parametrize("r", [0, 2, 5])
def test_device_projection_matches_numpy(r):
    """Pass 1's projection on the device against the NumPy restatement: the
    contextual sources to 1e-12 of their scale, the leakage measures tiny on
    both sides (orthonormal fixed effects)."""
    from oracle import generalized_oracle as go
    from summit_b200 import generalized_gxe as gg

    rng = np.random.default_rng(20 + r)
    K, Q, B, n = 3, 4, 7, 5003
    base = rng.normal(size=(K, B, n))
    basis = rng.normal(size=(n, Q))
    fixed = np.linalg.qr(rng.normal(size=(n, max(r, 1))))[0][:, :r]
    got, gabs, grel = gg._project_sources(base, basis, fixed)
    want, wabs, wrel = go.project_sources(base, basis, fixed)
    assert got.shape == want.shape == (K, Q, B, n)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    if r:
        assert 0.0 < gabs < 1e-10 and 0.0 <= grel < 1e-12 and wrel < 1e-12
    else:
        np.testing.assert_array_equal(got, want)
        assert gabs == grel == 0.0
