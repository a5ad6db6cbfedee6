"""Residual-minimisation trial for SCF warm solves (sdft_b200_rmm_trial).

Warm starts: the reference's converged vectors of an operator, the trial run
on the same operator with V(G) scaled by 1 + eps (the SCF's next iteration).
Against the reference's solve_generalized_hermitian_rmm_trial run on the same
inputs (oracle/_ref): the same outcome (a residual-checked trial manifold,
explicitly not converged, or the Davidson fallback), trial step counts within
one, every pair certified by the numpy oracle at the tolerance with fresh
FP64 residuals, S-orthonormal within 1e-10, and eigenvalues within 1e-8 Ha of
the exact ones (Rayleigh quotients of residual-1e-5 vectors).
"""
import dataclasses

import numpy as np
import pytest

from oracle import ref_oracle, sdft_oracle
from sdft_b200 import _capi as C
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def warm(reference):
    out = {}
    for name in ("tiny", "si8"):
        base = getattr(synthetic, name)()
        out[name] = (base, ref_oracle.ReferenceOperator(reference, base).davidson(base.roots, 256, 1e-10))
    return out


def _check(result, inputs, tolerance):
    oracle = sdft_oracle.Operator(inputs)
    vectors = result["eigenvectors"].T
    fresh, metric = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], vectors)
    assert np.max(fresh) <= 1.01 * tolerance
    gram = vectors.conj().T @ oracle.apply_s(vectors)
    assert np.max(np.abs(gram - np.eye(gram.shape[0]))) <= 1e-10


@pytest.mark.parametrize("name,eps,tolerance", [("tiny", 0.0, 1e-6), ("tiny", 1e-5, 1e-6), ("tiny", 1e-4, 1e-5),
                                                ("si8", 1e-5, 1e-5), ("si8", 1e-4, 1e-6), ("tiny", 1e-3, 1e-6)])
def test_rmm_trial_matches_reference(context, reference, warm, name, eps, tolerance):
    base, solved = warm[name]
    inputs = dataclasses.replace(base, v_values=base.v_values * (1 + eps))
    ref = ref_oracle.ReferenceOperator(reference, inputs).rmm_trial(base.roots, solved["eigenvectors"], 256,
                                                                     tolerance)
    op = PlaneWaveOperator(context, inputs)
    got = op.rmm_trial(base.roots, solved["eigenvectors"], 256, tolerance)
    assert got["trial_manifold"] == ref["trial_manifold"]
    if ref["trial_manifold"]:
        assert not got["converged"]
        assert abs(got["iterations"] - ref["iterations"]) <= 1
    else:
        assert got["converged"] and ref["converged"]
    _check(got, inputs, tolerance)
    exact = op.davidson(base.roots, 256, 1e-12)["eigenvalues"]
    assert np.max(np.abs(got["eigenvalues"] - exact)) < 1e-8
    assert np.max(np.abs(ref["eigenvalues"] - exact)) < 1e-8


def test_rmm_trial_rejects_strict_requests(context, warm):
    base, solved = warm["tiny"]
    op = PlaneWaveOperator(context, base)
    with pytest.raises(C.InvalidArgument, match="coarse explicit SCF warm request"):
        op.rmm_trial(base.roots, solved["eigenvectors"], 256, 1e-10)


def test_rmm_trial_with_one_iteration_budget_falls_back(context, warm):
    """max_iterations 1 leaves no trial step (min(16, 1/2) = 0): the Davidson
    solve runs with the whole budget from the warm block."""
    base, solved = warm["tiny"]
    op = PlaneWaveOperator(context, base)
    got = op.rmm_trial(base.roots, solved["eigenvectors"], 1, 1e-6)
    assert not got["trial_manifold"] and got["iterations"] == 1
