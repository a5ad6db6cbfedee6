"""Band-group solve (sdft_b200_band_groups) against the reference's
solve_generalized_hermitian_band_groups run on the same inputs (oracle/_ref).

Both solves converge to the tolerance (1e-10 Ha) in the default two-sweep
mode and in the swept mode (SDFT_BAND_GROUP_SWEEP=1), with group sizes 8 and
4; the eigenvalues agree within 1e-10 Ha, every pair is certified by the
numpy oracle with fresh FP64 residuals and the block is S-orthonormal within
1e-10. Iteration counts are not compared: the local solves' restarts follow
each implementation's own Rayleigh-Ritz rounding.
"""
import os

import numpy as np
import pytest

from oracle import ref_oracle, sdft_oracle
from sdft_b200 import _capi as C
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture
def environment():
    saved = {k: os.environ.get(k) for k in ("SDFT_BAND_GROUP_SWEEP", "SDFT_BAND_GROUP_SIZE",
                                            "SDFT_BAND_GROUP_LOCAL_STEPS")}
    yield os.environ
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def _certify(result, inputs):
    oracle = sdft_oracle.Operator(inputs)
    vectors = result["eigenvectors"].T
    fresh, _ = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], vectors)
    assert np.max(fresh) <= 1.01 * TOL
    gram = vectors.conj().T @ oracle.apply_s(vectors)
    assert np.max(np.abs(gram - np.eye(gram.shape[0]))) <= 1e-10


@pytest.mark.parametrize("name", ["tiny", "si8"])
@pytest.mark.parametrize("sweep,size", [("0", "8"), ("0", "4"), ("1", "8")])
def test_band_groups_match_reference(context, reference, environment, name, sweep, size):
    inputs = getattr(synthetic, name)()
    environment["SDFT_BAND_GROUP_SWEEP"] = sweep
    environment["SDFT_BAND_GROUP_SIZE"] = size
    ref = ref_oracle.ReferenceOperator(reference, inputs).band_groups(inputs.roots, 256, TOL)
    got = PlaneWaveOperator(context, inputs).band_groups(inputs.roots, 256, TOL)
    assert ref["converged"] and got["converged"], got["stats"]
    assert np.max(np.abs(got["eigenvalues"] - ref["eigenvalues"])) < 1e-10
    _certify(got, inputs)


def test_band_groups_warm_start(context, reference, environment):
    inputs = synthetic.si8()
    warm = ref_oracle.ReferenceOperator(reference, inputs).davidson(inputs.roots, 256, 1e-12)
    got = PlaneWaveOperator(context, inputs).band_groups(inputs.roots, 256, TOL, initial=warm["eigenvectors"])
    assert got["converged"]
    assert np.max(np.abs(got["eigenvalues"] - warm["eigenvalues"])) < 1e-10
    _certify(got, inputs)


def test_band_group_controls_are_checked(context, environment):
    inputs = synthetic.tiny()
    op = PlaneWaveOperator(context, inputs)
    environment["SDFT_BAND_GROUP_SIZE"] = "0"
    with pytest.raises(C.InvalidArgument, match="SDFT_BAND_GROUP_SIZE"):
        op.band_groups(inputs.roots)
    environment.pop("SDFT_BAND_GROUP_SIZE")
    environment["SDFT_BAND_GROUP_LOCAL_STEPS"] = "2"
    with pytest.raises(C.InvalidArgument, match="fixed local-step experiment"):
        op.band_groups(inputs.roots)
