"""S~ signature on the device against the oracle (the reference's overlap()
signature block, src/plane_wave_operator.cpp:702-717, pinned in
tests/test_oracle_pins.py), and the solve routing it drives: a numerically
singular S~ is the reference's runtime_error, an indefinite one (which the
reference hands to its indefinite-metric Davidson, src/pw_core.cpp:556-557)
is UNSUPPORTED. Pencils: the generator's (lambda_min(S~) = 0.3) and the same
pencil with Q scaled to a singular and to an indefinite S~.
"""
import numpy as np
import pytest

from oracle import sdft_oracle
from sdft_b200 import _capi as C
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu


def variants(inputs):
    minimum, _, _ = sdft_oracle.metric_signature(sdft_oracle.Operator(inputs))
    factor = synthetic.singular_overlap_factor(minimum, inputs.regularization)
    return {"definite": inputs, "singular": synthetic.scaled_overlap(inputs, factor),
            "indefinite": synthetic.scaled_overlap(inputs, 1.5)}


@pytest.mark.parametrize("name", ["tiny", "si8"])
def test_signature_matches_oracle(context, name):
    for kind, inputs in variants(getattr(synthetic, name)()).items():
        expected, indefinite, singular = sdft_oracle.metric_signature(sdft_oracle.Operator(inputs))
        op = PlaneWaveOperator(context, inputs)
        try:
            if kind == "singular":
                assert singular
                with pytest.raises(C.SdftError, match="original PAW overlap is numerically singular") as info:
                    op.metric_signature()
                assert info.value.status == C.RUNTIME_ERROR
            else:
                sig = op.metric_signature()
                assert abs(sig["minimum"] - expected) < 1e-12
                assert sig["indefinite"] == indefinite == (kind == "indefinite")
        finally:
            op.close()


def test_solves_refuse_singular_and_indefinite_metrics(context, tiny_inputs):
    cases = variants(tiny_inputs)
    op = PlaneWaveOperator(context, cases["singular"])
    try:
        with pytest.raises(C.SdftError, match="numerically singular") as info:
            op.davidson(tiny_inputs.roots, 50, 1e-10)
        assert info.value.status == C.RUNTIME_ERROR
        with pytest.raises(C.SdftError, match="numerically singular"):
            op.band_groups(tiny_inputs.roots, 50, 1e-10)
    finally:
        op.close()
    op = PlaneWaveOperator(context, cases["indefinite"])
    try:
        with pytest.raises(C.Unsupported, match="indefinite"):
            op.davidson(tiny_inputs.roots, 50, 1e-10)
        warm = np.eye(op.npw, tiny_inputs.roots, dtype=np.complex128).T
        with pytest.raises(C.Unsupported):
            op.rmm_trial(tiny_inputs.roots, warm)
    finally:
        op.close()


def test_signature_follows_an_update(context, si8_inputs):
    """update() replaces Q, so the signature is computed again."""
    cases = variants(si8_inputs)
    op = PlaneWaveOperator(context, si8_inputs)
    try:
        assert abs(op.metric_signature()["minimum"] - 0.3) < 1e-12
        bad = cases["indefinite"]
        op.update(bad.v_hkl, bad.v_values, bad.d, bad.q)
        expected, _, _ = sdft_oracle.metric_signature(sdft_oracle.Operator(bad))
        sig = op.metric_signature()
        assert sig["indefinite"] and abs(sig["minimum"] - expected) < 1e-12
        with pytest.raises(C.Unsupported):
            op.davidson(si8_inputs.roots, 10, 1e-10)
        op.update(si8_inputs.v_hkl, si8_inputs.v_values, si8_inputs.d, si8_inputs.q)
        result = op.davidson(si8_inputs.roots, 256, 1e-12)
        assert result["converged"]
    finally:
        op.close()
