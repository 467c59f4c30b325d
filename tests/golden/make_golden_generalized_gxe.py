"""Golden vectors of the generalized per-variant GxE two-pass estimator.

Runs SUMMIT's own GeneralizedGxEPass1Executor / GeneralizedGxEPass2Executor
(ldscore/generalized_gxe_pass1.py, _pass2.py) with its NumPy operators on the
standardized genotypes of a small synthetic BED fileset (decoded by the CPU
oracle, the same values as the resident image's), and its own global probe
generator; writes generalized_gxe.npz.  Run where the reference sources are:

    SUMMIT_REFERENCE_DIR=<summit checkout> python tests/golden/make_golden_generalized_gxe.py
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def main() -> None:
    ref = Path(os.environ.get("SUMMIT_REFERENCE_DIR", "/root/reference"))
    sys.path.insert(0, str(ref / "src"))
    from summit.ldscore.generalized_gxe_pass1 import (ArraySequentialGenotypeOperator,
                                                      GeneralizedGxEPass1Executor, NumpyNNOperator)
    from summit.ldscore.generalized_gxe_pass2 import GeneralizedGxEPass2Executor, NumpyTNOperator
    from summit.ldscore.generalized_gxe_variant import (GeneralizedGxEPlanInputs,
                                                        GlobalVariantProbeSpec,
                                                        generate_global_variant_probes,
                                                        plan_generalized_gxe_variant_work)

    from oracle.oracle import Oracle
    from summit_b200 import bedfile

    n, m = 256, 300
    geno = bedfile.synth_genotypes(n, m, seed=77123)
    rows = bedfile.pack_bed_rows(geno)
    X, _mean, _inv = Oracle().standardize(rows, n, 0, m)
    rng = np.random.default_rng(5150)
    env = rng.normal(size=n)
    cov = rng.normal(size=n)
    store = {"rows": rows, "n": np.array(n), "m": np.array(m)}
    cases = {
        # (Q, K, fixed effects)
        "unprojected": (2, 2, False),
        "projected": (3, 3, True),
    }
    for name, (q, k, projected) in cases.items():
        cols = [np.ones(n), env, 0.3 * env ** 2 + rng.normal(size=n)][:q]
        basis = np.asfortranarray(np.column_stack(cols))
        if projected:
            u, _s, _vt = np.linalg.svd(np.column_stack([np.ones(n), cov]), full_matrices=False)
            fixed = np.asfortranarray(u)
        else:
            fixed = np.empty((n, 0), order="F")
        annot = rng.uniform(0.1, 1.4, size=(m, k))
        annot[rng.random((m, k)) < 0.2] = 0.0
        annot[0] = 0.7  # every column keeps a positive mass
        spec = GlobalVariantProbeSpec(root_seed=9001 + q, probe_offset=7, probe_count=11)
        plan = plan_generalized_gxe_variant_work(GeneralizedGxEPlanInputs(
            num_samples=n, num_variants=m, num_basis=q, num_annotations=k, num_probes=11,
            memory_limit_bytes=512 * 1024 ** 2, genotype_format="bed",
            fixed_effect_rank=fixed.shape[1], preferred_variant_block_width=64,
            preferred_rhs_tile_columns=q * q * 4, rhs_policy="tiled"))
        operator = ArraySequentialGenotypeOperator(np.asfortranarray(X))
        names = tuple(f"annotation_{i}" for i in range(k))
        p1 = GeneralizedGxEPass1Executor(
            genotype_operator=operator, basis=basis, fixed_effect_basis=fixed, annotations=annot,
            annotation_names=names, annotation_masses=np.sum(annot, axis=0), probe_spec=spec,
            work_plan=plan, nn_operator=NumpyNNOperator(threads=1), annotation_tile_width=k,
            probe_tile_width=5, same_person_sample_tile_width=64,
            native_probe_module=False).execute()
        p2 = GeneralizedGxEPass2Executor(
            pass1_result=p1, genotype_operator=operator, basis=basis, fixed_effect_basis=fixed,
            annotations=annot, annotation_names=names, work_plan=plan,
            tn_operator=NumpyTNOperator(threads=1), probe_tile_width=4).execute()
        g = f"{name}/"
        store[g + "basis"] = basis
        store[g + "fixed"] = fixed
        store[g + "annot"] = annot
        store[g + "root_seed"] = np.array(spec.root_seed)
        store[g + "contextual_sources"] = p1.contextual_sources
        for key in ("directional_ldscores", "directed_numerator", "symmetric_numerator",
                    "genetic_gram", "component_kernel_diagonal", "same_person"):
            store[g + key] = np.asarray(getattr(p2, key))
        store[g + "probes"] = generate_global_variant_probes(
            np.arange(m, dtype=np.int64), np.arange(7, 18, dtype=np.int64),
            root_seed=spec.root_seed)
    # a second probe block at large global indices
    store["far_probes"] = generate_global_variant_probes(
        np.arange(10 ** 12, 10 ** 12 + 37, dtype=np.int64),
        np.arange(2 ** 40, 2 ** 40 + 5, dtype=np.int64), root_seed=2 ** 63 + 12345)
    np.savez_compressed(HERE / "generalized_gxe.npz", **store)
    print(f"wrote {HERE / 'generalized_gxe.npz'}")


if __name__ == "__main__":
    main()
