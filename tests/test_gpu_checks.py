"""GPU: exact integrity checks of the phase-2 tensor-core products.

With checks on, every windowed estimate forms per SNP a checksum of its exact
digit products in the phase-2 epilogue (tensor cores) and the same checksum
recomputed on the CUDA cores from the sketch digits and the packed codes; the
host compares them.  Faults are injected on the host, into copied checksums,
never into a kernel."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan(sess, annot, ws, nvecs, **kw):
    from summit_b200.session import WinPlan

    return WinPlan(sess, annot, ws, nvecs, 64, 91, "rademacher", **kw)


@pytest.fixture(scope="module")
def bigger():
    """2,500 samples (N_pad 2,560: the check pass stages u in two chunks)
    x 1,500 SNPs, 1% missing."""
    from summit_b200 import gwldcore

    n, m = 2500, 1500
    return {"n": n, "m": m, "rows": gwldcore.synth_bed_rows(n, m, 20261204)}


@pytest.mark.parametrize("impute", ["mean", "hwe"])
@pytest.mark.parametrize("nvecs,vtile,batch_gb", [(50, 0, 100.0), (24, 16, 100.0),
                                                  (8, 0, 1e-6)])
def test_checks_pass_and_leave_scores_unchanged(bigger, impute, nvecs, vtile, batch_gb):
    from summit_b200.session import GwSession

    n, m = bigger["n"], bigger["m"]
    rng = np.random.default_rng(3)
    annot = (rng.random((m, 5)) < 0.3).astype(float)
    annot[:, 0] = 1.0
    ws = np.array([0, 130, 131, 700, 1111, m], dtype=np.int64)
    sess = GwSession(bigger["rows"], n, impute_mode=impute, impute_seed=2)
    kw = dict(vtile=vtile, batch_gb=batch_gb) if vtile else dict(batch_gb=batch_gb)
    plain = _plan(sess, annot, ws, nvecs, **kw)
    checked = _plan(sess, annot, ws, nvecs, **kw)
    checked.set_checks(True)
    plain.execute()
    checked.execute()
    a, b = plain.results(), checked.results()
    np.testing.assert_array_equal(a["ldscore"], b["ldscore"])
    r = checked.check_products()
    assert r["mismatches"] == 0 and r["first_snp"] == -1
    assert np.count_nonzero(r["lhs"]) > m  # the checksums are not trivially zero
    np.testing.assert_array_equal(r["lhs"], r["rhs"])
    assert r["check_ms"] > 0.0
    checked.execute()  # graph replay: the checksums restart at zero
    r2 = checked.check_products()
    assert r2["mismatches"] == 0
    np.testing.assert_array_equal(r2["lhs"], r["lhs"])
    for p in (plain, checked):
        p.close()
    sess.close()


def test_injected_product_errors_are_found(bigger):
    """A wrong product of one SNP, injected into the copied tensor-core
    checksum (or into the recomputed one), is reported for exactly that SNP."""
    from summit_b200 import _lib
    from summit_b200._lib import check, ptr
    from summit_b200.session import GwSession

    n, m = bigger["n"], bigger["m"]
    annot = np.ones((m, 2))
    annot[::3, 1] = 0.0
    ws = np.array([0, 500, m], dtype=np.int64)
    sess = GwSession(bigger["rows"], n)
    plan = _plan(sess, annot, ws, 16)
    plan.set_checks(True)
    plan.execute()
    r = plan.check_products()
    assert r["mismatches"] == 0

    def verify(lhs, rhs):
        bad, first = np.zeros(1, np.int64), np.zeros(1, np.int64)
        check(_lib.load().lds_check_vectors(ptr(np.ascontiguousarray(lhs)),
                                            ptr(np.ascontiguousarray(rhs)), m, ptr(bad),
                                            ptr(first)))
        return int(bad[0]), int(first[0])

    assert verify(r["lhs"], r["rhs"]) == (0, -1)
    for j, col, delta in [(0, 0, 1), (777, 1, 1 << 40), (m - 1, 0, -3)]:
        lhs = r["lhs"].copy()
        # a product off by delta changes the checksum by h * delta (h odd)
        lhs[j, col] = np.uint64((int(lhs[j, col]) + delta * 0x9E3779B97F4A7C15) % (1 << 64))
        assert verify(lhs, r["rhs"]) == (1, j)
    rhs = r["rhs"].copy()
    rhs[42, 1] ^= np.uint64(1)
    rhs[1000, 0] ^= np.uint64(1 << 63)
    assert verify(r["lhs"], rhs) == (2, 42)
    with pytest.raises(RuntimeError, match="product checks are off"):
        other = _plan(sess, annot, ws, 16)
        other.execute()
        other.check_products()
    with pytest.raises(RuntimeError, match="before the plan's first execute"):
        plan.set_checks(False)
    plan.close()
    other.close()
    sess.close()


@pytest.mark.parametrize("impute,vtile", [("mean", 0), ("hwe", 16)])
def test_genome_wide_plan_checks(bigger, impute, vtile):
    """The same checks on a genome-wide plan (its rows form one window)."""
    from summit_b200.session import GwSession

    n, m = bigger["n"], bigger["m"]
    rng = np.random.default_rng(8)
    annot = (rng.random((m, 3)) < 0.4).astype(float)
    annot[:, 0] = 1.0
    sess = GwSession(bigger["rows"], n, impute_mode=impute, impute_seed=4)
    kw = dict(vtile=vtile) if vtile else {}
    plain = sess.plan(annot, 40, 100, 13, "rademacher", **kw)
    checked = sess.plan(annot, 40, 100, 13, "rademacher", **kw)
    checked.set_checks(True)
    plain.execute()
    checked.execute()
    np.testing.assert_array_equal(plain.results()["ldscore"], checked.results()["ldscore"])
    r = checked.check_products()
    assert r["mismatches"] == 0 and r["first_snp"] == -1
    assert np.count_nonzero(r["lhs"]) > m
    np.testing.assert_array_equal(r["lhs"], r["rhs"])
    assert r["check_ms"] > 0.0
    checked.execute()
    assert checked.check_products()["mismatches"] == 0
    with pytest.raises(RuntimeError, match="before the plan's first execute"):
        checked.set_checks(False)
    for p in (plain, checked):
        p.close()
    sess.close()


def test_gxe_target_checks(oracle):
    """GxE reference build with the target's product checks on: the same
    accumulators as without them, every SNP's checksum pair equal, and a
    product error planted in a copy of the checksums is found."""
    import torch

    from oracle.gxe_oracle import design, rademacher_block
    from summit_b200 import _lib
    from summit_b200._lib import check, ptr
    from summit_b200.gxe import GxeReference
    from summit_b200.session import GwSession

    n, m, E, K, B, T = 600, 900, 3, 2, 8, 3
    rows = oracle.synth_bed_rows(n, m, 21)
    d = design(n, E, seed=4, categorical=1)
    rng = np.random.default_rng(6)
    probes = rademacher_block(5, 0, m, range(B))
    ann = rng.random((m, K)) + 0.05
    sx = 0.5 + rng.random((m, T))
    sw = 0.5 + rng.random((m, T))
    names = ("accum_xx", "accum_xw", "accum_wx", "accum_ww")

    def cm(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().T

    g = GwSession(rows, n)
    out = {}
    for checked in (False, True):
        ref = GxeReference(g, d["environments"], d["feature_basis"], d["power_indices"],
                           d["power_offsets"], d["ranks"], d["gram_values"], d["gram_offsets"],
                           d["e2_gram_values"], d["common_basis"], d["directions"], K,
                           product_checks=checked)
        res = ref.run(cm(probes), cm(ann), cm(sx), cm(sw), 0)
        out[checked] = {k: res[k].cpu().numpy() for k in names}
        if checked:
            r = ref.last_check(vectors=True)
            assert r["rows"] == m and r["first_row"] == 0
            assert r["mismatches"] == 0 and r["first_snp"] == -1
            assert np.count_nonzero(r["lhs"]) > m
            np.testing.assert_array_equal(r["lhs"], r["rhs"])
        else:
            with pytest.raises(RuntimeError, match="product checks are off"):
                ref.last_check()
        ref.close()
    g.close()
    for k in names:
        np.testing.assert_array_equal(out[True][k], out[False][k], err_msg=k)

    def verify(lhs, rhs):
        bad, first = np.zeros(1, np.int64), np.zeros(1, np.int64)
        check(_lib.load().lds_check_vectors(ptr(np.ascontiguousarray(lhs)),
                                            ptr(np.ascontiguousarray(rhs)), m, ptr(bad),
                                            ptr(first)))
        return int(bad[0]), int(first[0])

    lhs = r["lhs"].copy()
    lhs[311, 1] = np.uint64((int(lhs[311, 1]) + 5 * 0x9E3779B97F4A7C15) % (1 << 64))
    assert verify(lhs, r["rhs"]) == (1, 311)
