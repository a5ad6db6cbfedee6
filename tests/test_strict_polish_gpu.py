"""Strict FP64 refinements on the device (src/strict_residual_polish.hpp:70-197,
driven from src/pw_core.cpp:1273-1356) on pencils whose reference solve at
tolerance 1e-13 ends in its strict tangent polish (strict_polish.npz records
the reference's polish steps from its own trace).

Bars: converged at 1e-13 with every fresh FP64 residual <= 1e-13, recomputed
by the numpy oracle; S-orthonormal within 1e-12; eigenvalues within 1e-10 Ha
of the reference's; the refinement ran and was accepted. With the reference's
switch SDFT_FRESH_RESIDUAL_POLISH=0 no refinement step runs.
"""
import numpy as np
import pytest

from oracle import sdft_oracle
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

CASES = [("tiny", 1), ("tiny", 3), ("si8", 2026)]


def solve_and_check(context, golden, name, seed, precision):
    g = golden("strict_polish")
    tol = float(g["tolerance"])
    key = f"{name}_{seed}"
    assert int(g[f"{key}_polish_steps"]) > 0  # the reference needed its polish here
    inputs = getattr(synthetic, name)(seed=seed)
    op = PlaneWaveOperator(context, inputs)
    try:
        result = op.davidson(inputs.roots, 256, tol, precision=precision)
    finally:
        op.close()
    assert result["converged"], result["stats"]
    assert np.max(result["residuals"]) <= tol
    assert np.max(np.abs(result["eigenvalues"] - g[f"{key}_eigenvalues"])) < 1e-10
    oracle = sdft_oracle.Operator(inputs)
    vectors = result["eigenvectors"].T
    fresh, metric = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], vectors)
    assert np.max(fresh) <= 1.01 * tol
    gram = vectors.conj().T @ oracle.apply_s(vectors)
    assert np.max(np.abs(gram - np.eye(gram.shape[0]))) <= 1e-12
    return result["stats"]


@pytest.mark.parametrize("name,seed", CASES)
def test_fp64_solve_polishes_to_reference(context, golden, name, seed):
    stats = solve_and_check(context, golden, name, seed, "fp64")
    assert stats["polish_steps"] + stats["manifold_steps"] > 0
    assert stats["polish_accepted"] + stats["manifold_accepted"] > 0


@pytest.mark.parametrize("name,seed", CASES[:2])
def test_mixed_solve_polishes_to_reference(context, golden, name, seed):
    solve_and_check(context, golden, name, seed, "mixed")


def test_polish_switch_off(context, monkeypatch):
    monkeypatch.setenv("SDFT_FRESH_RESIDUAL_POLISH", "0")
    inputs = synthetic.tiny(seed=3)
    op = PlaneWaveOperator(context, inputs)
    try:
        result = op.davidson(inputs.roots, 256, 1e-13, precision="fp64", vectors=False)
    finally:
        op.close()
    assert result["stats"]["polish_steps"] == 0 and result["stats"]["manifold_steps"] == 0
    monkeypatch.setenv("SDFT_FRESH_RESIDUAL_POLISH", "2")
    op = PlaneWaveOperator(context, inputs)
    try:
        from sdft_b200 import _capi as C
        with pytest.raises(C.InvalidArgument, match="must be 0 or 1"):
            op.davidson(inputs.roots, 10, 1e-13, precision="fp64", vectors=False)
    finally:
        op.close()
