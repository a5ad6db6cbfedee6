"""SCF refresh of a live operator (sdft_b200_operator_update).

The reference's SCF builds a new PlaneWaveOperator every iteration with the
new V(G) and D and the same projectors, kept resident through an immutable
projector identity (src/scf_core.cpp:2312-2313). The device operator is
updated in place instead. Along an SCF-like sequence of potentials and D
blocks (synthetic.scf_step), each step checks that the updated operator
- holds the arrays of an operator created from the same inputs and applies
  H~ and S~ like it, bit for bit, in FP64 and in the mixed form;
- applies H~ and S~ like the reference's operator built with a shared
  projector identity, within 1e-12 relative in FP64 (the reference's own
  application limit, tests/native/plane_wave_operator_smoke.cpp:60);
- gives, warm-started from the previous step's vectors as an SCF does, the
  eigenvalues of a solve on the new operator bit for bit, the reference's
  within 1e-10 Ha, and pairs certified by the numpy oracle at 1e-12 Ha.
"""
import ctypes

import numpy as np
import pytest

from conftest import probe_block, relative_error
from oracle import sdft_oracle
from sdft_b200 import _capi as C
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _same_operator(updated, fresh):
    a, b = updated.arrays(), fresh.arrays()
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    x = probe_block(updated.npw, 5, 17)
    for precision in ("fp64", "mixed"):
        for overlap in (False, True):
            assert np.array_equal(updated.apply(x, overlap=overlap, precision=precision),
                                  fresh.apply(x, overlap=overlap, precision=precision)), (precision, overlap)


@pytest.mark.parametrize("name,steps", [("tiny", 3), ("si8", 2)])
def test_scf_sequence(context, reference, request, name, steps):
    from oracle import ref_oracle
    base = request.getfixturevalue(f"{name}_inputs")
    live = PlaneWaveOperator(context, base)
    identity = 0x5CF0 + steps  # one immutable projector identity for the whole sequence, as the SCF keeps
    warm = None
    for step in range(1, steps + 1):
        inputs = synthetic.scf_step(base, step, keep=0.5 if step == 2 else 1.0)
        live.update(inputs.v_hkl, inputs.v_values, inputs.d, inputs.q)
        fresh = PlaneWaveOperator(context, inputs)
        _same_operator(live, fresh)
        ref = ref_oracle.ReferenceOperator(reference, inputs, projector_identity=identity)
        x = probe_block(live.npw, 4, 100 + step)
        assert relative_error(live.apply(x, overlap=False), ref.apply(x, overlap=False)) < FP64_TOL
        assert relative_error(live.apply(x, overlap=True), ref.apply(x, overlap=True)) < FP64_TOL

        roots = inputs.roots
        solved = live.davidson(roots, 256, 1e-12, initial=warm)
        again = fresh.davidson(roots, 256, 1e-12, initial=warm)
        assert solved["converged"], solved["stats"]
        assert np.array_equal(solved["eigenvalues"], again["eigenvalues"])
        expected = ref.davidson(roots, 256, 1e-12, initial=warm)
        assert np.max(np.abs(solved["eigenvalues"] - expected["eigenvalues"])) < 1e-10
        oracle = sdft_oracle.Operator(inputs)
        fresh_res, metric = sdft_oracle.certified_residuals(oracle, solved["eigenvalues"], solved["eigenvectors"].T)
        assert np.max(fresh_res) <= 1.01e-12
        assert np.max(metric) <= 1e-12
        warm = solved["eigenvectors"]
        fresh.close()


def test_mixed_solve_after_update(context, si8_inputs):
    live = PlaneWaveOperator(context, si8_inputs)
    inputs = synthetic.scf_step(si8_inputs, 1)
    live.update(inputs.v_hkl, inputs.v_values, inputs.d, inputs.q)
    fresh = PlaneWaveOperator(context, inputs)
    a = live.davidson(inputs.roots, 256, 1e-12, precision="mixed")
    b = fresh.davidson(inputs.roots, 256, 1e-12, precision="mixed")
    assert a["converged"] and np.array_equal(a["eigenvalues"], b["eigenvalues"])


def _hermitian_break(values, keys):
    """V(G) with one nonzero key's partner left out of step."""
    bad = values.copy()
    for i, k in enumerate(keys):
        if any(k) and abs(bad[i]) > 0:
            bad[i] = bad[i] + 0.5
            return bad
    raise AssertionError("no nonzero key")


def test_rejected_update_leaves_operator_unchanged(context, tiny_inputs):
    live = PlaneWaveOperator(context, tiny_inputs)
    before = live.arrays()
    x = probe_block(live.npw, 3, 5)
    hx = live.apply(x)
    step = synthetic.scf_step(tiny_inputs, 1)
    with pytest.raises(C.InvalidArgument, match="not Hermitian"):
        live.update(step.v_hkl, _hermitian_break(step.v_values, step.v_hkl), step.d, step.q)
    bad_d = step.d.copy()
    bad_d[0, 0, 1] += 0.3
    with pytest.raises(C.InvalidArgument, match="Hermitian PAW blocks"):
        live.update(step.v_hkl, step.v_values, bad_d, step.q)
    nonfinite = step.v_values.copy()
    nonfinite[0] = np.nan
    with pytest.raises(C.InvalidArgument, match="nonfinite local potential"):
        live.update(step.v_hkl, nonfinite, step.d, step.q)
    with pytest.raises(ValueError):
        live.update(step.v_hkl, step.v_values, step.d[:-1], step.q)
    after = live.arrays()
    for key in before:
        assert np.array_equal(before[key], after[key]), key
    assert np.array_equal(live.apply(x), hx)


def test_snapshot_operator_is_not_updatable(context, tiny_inputs):
    import pathlib
    path = pathlib.Path(__file__).parent / "golden" / "tiny_cold.pwo3"
    op, _ = PlaneWaveOperator.from_snapshot(context, path)
    with pytest.raises(ValueError):
        op.update(tiny_inputs.v_hkl, tiny_inputs.v_values, tiny_inputs.d, tiny_inputs.q)
    vh = np.ascontiguousarray(tiny_inputs.v_hkl, dtype=np.int32)
    vv = np.ascontiguousarray(tiny_inputs.v_values, dtype=np.complex128)
    d = np.ascontiguousarray(tiny_inputs.d, dtype=np.complex128)
    q = np.ascontiguousarray(tiny_inputs.q, dtype=np.complex128)
    status = C.library().sdft_b200_operator_update(op.handle, vh.shape[0], vh.ctypes.data_as(C.I32),
                                                   vv.ctypes.data_as(C.D), d.ctypes.data_as(C.D),
                                                   q.ctypes.data_as(C.D))
    assert status == C.INVALID_ARGUMENT
    assert "snapshot" in C.last_error()
