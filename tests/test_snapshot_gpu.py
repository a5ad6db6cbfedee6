"""Solver snapshots (the reference's SDFTPWO3 files) served on the device:
the operator built from a snapshot the reference wrote has the reference's
arrays bit for bit, applies like the operator built from the same inputs, and
its Davidson solves (cold and warm) give the reference's eigenvalues for the
same snapshot within 1e-10 Ha, every pair certified at the snapshot's
tolerance (tests/golden/make_golden.py --snapshots)."""
import pathlib

import numpy as np
import pytest

from conftest import probe_block, relative_error
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def inputs_op(context, tiny_inputs):
    op = PlaneWaveOperator(context, tiny_inputs)
    yield op
    op.close()


@pytest.mark.parametrize("name", ["tiny_cold", "tiny_warm"])
def test_snapshot_operator_matches_reference_arrays(context, golden, inputs_op, name):
    op, settings = PlaneWaveOperator.from_snapshot(context, GOLDEN / f"{name}.pwo3")
    try:
        g = golden("tiny")
        assert op.shape == tuple(int(v) for v in g["shape"])
        arrays = op.arrays()
        for key, ref in (("indices", g["indices"]), ("kinetic", g["kinetic"]), ("h_diagonal", g["h_diagonal"]),
                         ("s_diagonal", g["s_diagonal"]), ("local_potential", g["local_real"])):
            assert np.array_equal(arrays[key], ref), key
        x = probe_block(op.npw, 4, 23)
        for overlap in (False, True):
            assert relative_error(op.apply(x, overlap=overlap), inputs_op.apply(x, overlap=overlap)) < 1e-13
        assert (settings["initial"] is not None) == (name == "tiny_warm")
    finally:
        op.close()


@pytest.mark.parametrize("name", ["tiny_cold", "tiny_warm"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_snapshot_solve_matches_reference(context, golden, name, precision):
    op, s = PlaneWaveOperator.from_snapshot(context, GOLDEN / f"{name}.pwo3")
    try:
        result = op.davidson(s["roots"], s["iterations"], s["tolerance"], precision=precision, initial=s["initial"])
        assert result["converged"], result["stats"]
        assert np.max(result["residuals"]) <= s["tolerance"]
        expected = golden("snapshots")[f"{name}_eigenvalues"]
        assert np.max(np.abs(result["eigenvalues"] - expected)) < 1e-10
    finally:
        op.close()
