"""GPU: windowed phase 2 on SM pairs (tcgen05.mma.cta_group::2, two 128-SNP
tiles of a window sharing each sketch tile) gives the one-SM kernel's LD
scores bit for bit: windows with odd tile counts (a pair's second tile past
the window end), several bins per CTA (few probes) and two column groups per
bin (many probes)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def pairs_switch():
    from summit_b200 import gwldcore

    yield gwldcore.set_p2_pairs
    gwldcore.set_p2_pairs(False)


def _both(sess, annot, ws, nvecs, step, seed, dist, set_pairs, **kw):
    from summit_b200.session import WinPlan

    out = []
    for on in (False, True):
        set_pairs(on)
        p = WinPlan(sess, annot, ws, nvecs, step, seed, dist, **kw)
        p.execute()
        out.append(p.results())
        p.close()
    return out


@pytest.mark.parametrize("nvecs", [50, 10, 70])
def test_pairs_equal_single_sm_small(small_bed, pairs_switch, nvecs):
    from summit_b200.session import GwSession

    n, m, packed = small_bed["n"], small_bed["m"], small_bed["rows"]
    ws = np.array([0, 60, 200, 201, 333, 410], dtype=np.int64)
    rng = np.random.default_rng(3)
    annot = np.ones((m, 4))
    annot[:, 1:] = rng.random((m, 3)) < 0.4
    sess = GwSession(packed, n)
    a, b = _both(sess, annot, ws, nvecs, 50, 11, "rademacher", pairs_switch)
    sess.close()
    np.testing.assert_array_equal(b["ldscore"], a["ldscore"])
    np.testing.assert_array_equal(b["meansq_accum"], a["meansq_accum"])


def test_pairs_equal_single_sm_larger(pairs_switch):
    from summit_b200 import gwldcore
    from summit_b200.session import GwSession

    n, m = 2048, 24_000
    packed = gwldcore.synth_bed_rows(n, m, 91)
    rng = np.random.default_rng(5)
    cuts = np.sort(rng.choice(np.arange(1, m), 59, replace=False))
    ws = np.concatenate([[0], cuts, [m]]).astype(np.int64)
    annot = (rng.random((m, 6)) < 0.3).astype(np.float64)
    annot[:, 0] = 1.0
    sess = GwSession(packed, n)
    a, b = _both(sess, annot, ws, 50, 1000, 77, "rademacher", pairs_switch, with_mc=True)
    sess.close()
    np.testing.assert_array_equal(b["ldscore"], a["ldscore"])
    np.testing.assert_array_equal(b["mc_per_snp_sumsq"], a["mc_per_snp_sumsq"])
