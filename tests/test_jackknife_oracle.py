"""CPU: jackknife blocks (liblds host code) and the numpy solve/jackknife
restatement against golden vectors written by the reference's own Python."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

G = np.load(Path(__file__).parent / "golden" / "jackknife_golden.npz")


@pytest.mark.parametrize("i", range(4))
def test_equal_count_blocks_match_reference(i):
    from summit_b200.jackknife import equal_count_block_boundaries

    s, e = equal_count_block_boundaries(int(G[f"eq{i}_M"]), int(G[f"eq{i}_B"]))
    np.testing.assert_array_equal(s, G[f"eq{i}_starts"])
    np.testing.assert_array_equal(e, G[f"eq{i}_ends"])


@pytest.mark.parametrize("i", range(3))
def test_weighted_blocks_match_reference(i):
    from summit_b200.jackknife import weighted_contiguous_block_boundaries

    s, e = weighted_contiguous_block_boundaries(G["mass"], int(G[f"w{i}_B"]),
                                                min_snps=int(G[f"w{i}_min"]))
    np.testing.assert_array_equal(s, G[f"w{i}_starts"])
    np.testing.assert_array_equal(e, G[f"w{i}_ends"])


def test_block_argument_errors():
    from summit_b200.jackknife import equal_count_block_boundaries

    with pytest.raises(RuntimeError, match="1 <= nblocks <= nsnps"):
        equal_count_block_boundaries(10, 11)


@pytest.mark.parametrize("i", range(4))
def test_oracle_solve_matches_reference(i):
    from oracle.jack_oracle import solve

    x, rank = solve(G[f"s{i}_A"], G[f"s{i}_b"])
    assert rank == int(G[f"s{i}_rank"])
    np.testing.assert_allclose(x, G[f"s{i}_x"], rtol=1e-9, atol=1e-12 * np.abs(G[f"s{i}_x"]).max())


def test_oracle_jackknife_matches_reference():
    from oracle.jack_oracle import jackknife

    theta, reps, se = jackknife(G["jk_terms"], G["jk_starts"], G["jk_ends"])
    np.testing.assert_allclose(theta, G["jk_theta"], rtol=1e-12)
    np.testing.assert_allclose(reps, G["jk_reps"], rtol=1e-12)
    np.testing.assert_allclose(se, G["jk_se"], rtol=1e-10)
