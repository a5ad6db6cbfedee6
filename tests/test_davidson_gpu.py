"""Device Davidson against the reference's solutions (golden fixtures) and the oracle.

Bars: eigenvalues within 1e-10 Ha of the reference; every returned pair
certified by a fresh FP64 residual <= the tolerance (1e-12 Ha), recomputed
independently by the numpy oracle; S-orthonormality within 1e-12
(tests/native/plane_wave_operator_smoke.cpp:224-266).
"""
import numpy as np
import pytest

from oracle import sdft_oracle
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tiny_op(context, tiny_inputs):
    return PlaneWaveOperator(context, tiny_inputs)


@pytest.fixture(scope="module")
def si8_op(context, si8_inputs):
    return PlaneWaveOperator(context, si8_inputs)


def check_solution(result, inputs, golden_values, tol=1e-12):
    assert result["converged"], result["stats"]
    assert np.max(result["residuals"]) <= tol
    assert np.max(np.abs(result["eigenvalues"] - golden_values)) < 1e-10
    oracle = sdft_oracle.Operator(inputs)
    vectors = result["eigenvectors"].T  # columns
    fresh, metric = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], vectors)
    assert np.max(fresh) <= 1.01 * tol
    assert np.max(metric) <= 1e-12
    gram = vectors.conj().T @ oracle.apply_s(vectors)
    assert np.max(np.abs(gram - np.eye(gram.shape[0]))) <= 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tiny_solve(tiny_op, tiny_inputs, golden, precision):
    g = golden("tiny")
    result = tiny_op.davidson(tiny_inputs.roots, 256, 1e-12, precision=precision)
    check_solution(result, tiny_inputs, g["eigenvalues"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_si8_solve(si8_op, si8_inputs, golden, precision):
    g = golden("si8")
    result = si8_op.davidson(si8_inputs.roots, 256, 1e-12, precision=precision)
    check_solution(result, si8_inputs, g["eigenvalues"])
    if precision == "mixed":
        assert result["stats"]["h_columns_search"] > 0 and result["stats"]["fp64_refreshes"] >= 1


def test_iteration_limited_solve_is_not_converged(tiny_op, tiny_inputs):
    result = tiny_op.davidson(tiny_inputs.roots, 1, 1e-12)
    assert not result["converged"]
    oracle = sdft_oracle.Operator(tiny_inputs)
    fresh, metric = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], result["eigenvectors"].T)
    assert np.max(np.abs(fresh - result["residuals"])) < 1e-13
    assert np.max(metric) < 1e-12


def test_repeated_solves_reuse_workspace(tiny_op, tiny_inputs):
    a = tiny_op.davidson(tiny_inputs.roots, 256, 1e-12)
    b = tiny_op.davidson(tiny_inputs.roots, 256, 1e-12)
    assert np.array_equal(a["eigenvalues"], b["eigenvalues"])  # deterministic device path


def test_invalid_davidson_arguments(tiny_op):
    from sdft_b200 import _capi as C
    with pytest.raises(C.InvalidArgument):
        tiny_op.davidson(0)
    with pytest.raises(C.InvalidArgument):
        tiny_op.davidson(4, tolerance=-1.0)
    with pytest.raises(C.InvalidArgument):
        tiny_op.davidson(4, subspace_factor=3)


@pytest.mark.parametrize("steps", [-1, 0, 3])
def test_mixed_correction_steps_converge_to_reference(si8_op, si8_inputs, golden, steps):
    """The mixed form with the reference's single preconditioner step (-1), the
    default Jacobi-Davidson CG steps (0) and three steps: same certified pairs."""
    result = si8_op.davidson(si8_inputs.roots, 256, 1e-12, precision="mixed", correction_steps=steps)
    check_solution(result, si8_inputs, golden("si8")["eigenvalues"])
    assert (result["stats"]["correction_columns"] > 0) == (steps != -1)


def test_correction_steps_cut_outer_iterations(si8_op, si8_inputs):
    plain = si8_op.davidson(si8_inputs.roots, 256, 1e-12, precision="mixed", correction_steps=-1, vectors=False)
    steered = si8_op.davidson(si8_inputs.roots, 256, 1e-12, precision="mixed", correction_steps=6, vectors=False)
    assert plain["converged"] and steered["converged"]
    assert steered["iterations"] < plain["iterations"]
    assert steered["stats"]["rayleigh_ritz_calls"] < plain["stats"]["rayleigh_ritz_calls"]


def test_correction_steps_are_mixed_only(tiny_op, tiny_inputs):
    from sdft_b200 import _capi as C
    with pytest.raises(C.InvalidArgument, match="mixed form only"):
        tiny_op.davidson(tiny_inputs.roots, 50, 1e-10, precision="fp64", correction_steps=3)
    with pytest.raises(C.InvalidArgument):
        tiny_op.davidson(tiny_inputs.roots, 50, 1e-10, precision="mixed", correction_steps=-2)
