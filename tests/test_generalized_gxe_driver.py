"""Generalized per-variant GxE two-pass driver: host-side algebra on CPU.

The device products are replaced by the CPU restatement in
oracle/generalized_oracle.py (on the oracle's standardized genotypes), so
these tests check the driver's own algebra - sources, projection, families,
orientation products, reductions, diagonals - against golden vectors written
by the reference's GeneralizedGxEPass1/Pass2Executor
(tests/golden/make_golden_generalized_gxe.py).  The device path is compared
with the same vectors in test_gpu_generalized_gxe.py."""
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import generalized_oracle as go
from oracle.oracle import Oracle
from summit_b200 import generalized_gxe as gg

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "generalized_gxe.npz")
CASES = ["unprojected", "projected"]


@pytest.fixture(scope="module")
def decoded():
    n, m = int(GOLD["n"]), int(GOLD["m"])
    X, _mean, _inv = Oracle().standardize(GOLD["rows"], n, 0, m)
    return X


def test_probe_restatement_matches_reference():
    for case in CASES:
        seed = int(GOLD[f"{case}/root_seed"])
        want = GOLD[f"{case}/probes"]
        got = go.global_probes(seed, range(want.shape[0]), range(7, 18), gg.PROBE_NAMESPACE)
        np.testing.assert_array_equal(got, want)
    far = go.global_probes(2 ** 63 + 12345, range(10 ** 12, 10 ** 12 + 37),
                           range(2 ** 40, 2 ** 40 + 5), gg.PROBE_NAMESPACE)
    np.testing.assert_array_equal(far, GOLD["far_probes"])
    assert gg.probe_namespace_key(gg.PROBE_NAMESPACE) == go.namespace_key(gg.PROBE_NAMESPACE)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("width", [64, 300, 37])
def test_driver_algebra_matches_reference(monkeypatch, decoded, case, width):
    X = decoded
    n, m = X.shape
    seed = int(GOLD[f"{case}/root_seed"])
    monkeypatch.setattr(gg, "_source_product", lambda s, a, b, ab, z: go.source_product(X, a, b, ab, z))
    monkeypatch.setattr(gg, "_target_product", lambda s, a, b, Y: go.target_product(X, a, b, Y))
    monkeypatch.setattr(gg, "_component_diagonal",
                        lambda s, a, b, ab, ba, fx, cf, num: go.component_diagonal(X, a, b, ab, ba, fx, cf, num))
    monkeypatch.setattr(gg, "_project_sources", go.project_sources)
    monkeypatch.setattr(gg, "_pass2_scores_sources",
                        lambda s, rows, bas, ft, fs, k, b, p, to, f1, f2, rr, a, blk: go.pass2_scores(
                            X, go.assemble_rhs(rows, bas, ft, fs), k, b, len(ft), p, to, f1, f2,
                            rr, a))
    monkeypatch.setattr(gg, "global_variant_probes",
                        lambda spec, v0, cnt: go.global_probes(spec.root_seed, range(v0, v0 + cnt),
                                                               range(spec.probe_offset, spec.probe_offset + spec.probe_count),
                                                               spec.namespace))
    session = SimpleNamespace(N=n, M=m, handle=None)
    spec = gg.GlobalVariantProbeSpec(root_seed=seed, probe_offset=7, probe_count=11)
    p1, p2 = gg.two_pass(session, GOLD[f"{case}/basis"], GOLD[f"{case}/fixed"],
                         GOLD[f"{case}/annot"], spec, variant_block_width=width)
    np.testing.assert_allclose(p1.contextual_sources, GOLD[f"{case}/contextual_sources"],
                               rtol=1e-12, atol=1e-12)
    for key in ("directional_ldscores", "directed_numerator", "symmetric_numerator",
                "genetic_gram", "component_kernel_diagonal", "same_person"):
        want = GOLD[f"{case}/{key}"]
        np.testing.assert_allclose(getattr(p2, key), want, rtol=1e-10,
                                   atol=1e-12 * np.abs(want).max(), err_msg=key)


def test_driver_rejects_bad_inputs():
    session = SimpleNamespace(N=4, M=3, handle=None)
    spec = gg.GlobalVariantProbeSpec(root_seed=1, probe_offset=0, probe_count=2)
    ok_basis, ok_fixed, ok_annot = np.ones((4, 1)), np.empty((4, 0)), np.ones((3, 1))
    with pytest.raises(ValueError, match="basis must have shape"):
        gg.pass1(session, np.ones((3, 1)), ok_fixed, ok_annot, spec)
    with pytest.raises(ValueError, match="nonnegative"):
        gg.pass1(session, ok_basis, ok_fixed, -ok_annot, spec)
    with pytest.raises(ValueError, match="orthonormal"):
        gg.pass1(session, ok_basis, np.ones((4, 1)), ok_annot, spec)
    with pytest.raises(ValueError, match="masses must be positive"):
        gg.pass1(session, ok_basis, ok_fixed, np.zeros((3, 1)), spec)
    with pytest.raises(ValueError, match="probe_count positive"):
        gg.GlobalVariantProbeSpec(root_seed=1, probe_offset=0, probe_count=0)
