"""CUDA operator applications against the reference's outputs (golden fixtures).

Tolerances: FP64 plain form 1e-12 relative (the reference's own application
limit, tests/native/plane_wave_operator_smoke.cpp:60); mixed search form
(FP32 FFT + FP32-accumulated projector GEMMs) 2e-5 relative.
"""
import numpy as np
import pytest

from conftest import probe_block, relative_error
from oracle import sdft_oracle
from sdft_b200 import _capi as C
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 2e-5


@pytest.fixture(scope="module")
def tiny_op(context, tiny_inputs):
    return PlaneWaveOperator(context, tiny_inputs)


@pytest.fixture(scope="module")
def si8_op(context, si8_inputs):
    return PlaneWaveOperator(context, si8_inputs)


@pytest.mark.parametrize("name", ["tiny", "si8"])
def test_operator_arrays_match_reference(request, golden, name):
    op = request.getfixturevalue(f"{name}_op")
    g = golden(name)
    assert op.shape == tuple(int(v) for v in g["shape"])
    arrays = op.arrays()
    assert np.array_equal(arrays["indices"], g["indices"])          # integer map bit-exact
    assert np.array_equal(arrays["kinetic"], g["kinetic"])          # same division as the reference
    assert relative_error(arrays["local_potential"], g["local_real"]) < 1e-13
    assert relative_error(arrays["h_diagonal"], g["h_diagonal"]) < 1e-13
    assert relative_error(arrays["s_diagonal"], g["s_diagonal"]) < 1e-13


@pytest.mark.parametrize("name", ["tiny", "si8"])
@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_apply_matches_reference(request, golden, name, precision, tol):
    op = request.getfixturevalue(f"{name}_op")
    g = golden(name)
    x = probe_block(op.npw, 4, int(g["probe_seed"]))
    assert relative_error(op.apply(x, overlap=False, precision=precision), g["hx"]) < tol
    assert relative_error(op.apply(x, overlap=True, precision=precision), g["sx"]) < tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair_equals_separate_applications(si8_op, precision):
    x = probe_block(si8_op.npw, 7, 3)
    hy, sy = si8_op.apply_pair(x, precision=precision)
    assert np.array_equal(hy, si8_op.apply(x, overlap=False, precision=precision))
    assert np.array_equal(sy, si8_op.apply(x, overlap=True, precision=precision))


def test_projection_matches_oracle(si8_op, si8_inputs):
    x = probe_block(si8_op.npw, 5, 9)
    ref = sdft_oracle.Operator(si8_inputs).project(x)
    assert relative_error(si8_op.project(x, precision="fp64"), ref) < 1e-13
    assert relative_error(si8_op.project(x, precision="mixed"), ref) < 1e-5


def test_single_column_and_wide_block_agree(si8_op):
    x = probe_block(si8_op.npw, 33, 5)
    wide = si8_op.apply(x)
    cols = np.stack([si8_op.apply(x[:, j])[:, 0] for j in (0, 17, 32)], axis=1)
    assert relative_error(cols, wide[:, [0, 17, 32]]) < 1e-15


def test_device_pointers_match_host(si8_op):
    torch = pytest.importorskip("torch")
    x = probe_block(si8_op.npw, 6, 21)
    host = si8_op.apply(x, precision="fp64")
    dx = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T  # column-major view
    torch.cuda.synchronize()  # the context runs on its own stream
    dy = si8_op.apply(dx, precision="fp64")
    si8_op.context.synchronize()
    assert np.array_equal(dy.T.cpu().numpy().T, host)


def test_alias_and_argument_errors(si8_op, context):
    lib = C.library()
    x = probe_block(si8_op.npw, 2, 1)
    import ctypes
    ptr = ctypes.c_void_p(x.ctypes.data)
    assert lib.sdft_b200_apply(si8_op.handle, C.HAMILTONIAN, ptr, 2, ptr, C.FP64, C.HOST) == C.INVALID_ARGUMENT
    assert "invalid" in C.last_error()
    with pytest.raises(ValueError):
        si8_op.apply(x, precision="fp16")


def test_construction_rejects_invalid_inputs(context):
    base = synthetic.tiny()
    bad = synthetic.tiny()
    i = int(np.nonzero(np.any(bad.v_hkl != 0, axis=1))[0][0])
    bad.v_values = bad.v_values.copy()
    bad.v_values[i] += 0.5j  # breaks V(-G) = conj V(G)
    with pytest.raises(C.InvalidArgument, match="not Hermitian"):
        PlaneWaveOperator(context, bad)
    dup = synthetic.tiny()
    dup.hkl = dup.hkl.copy()
    dup.hkl[1] = dup.hkl[0]
    with pytest.raises(C.InvalidArgument, match="duplicate"):
        PlaneWaveOperator(context, dup)
    asym = synthetic.tiny()
    asym.d = asym.d.copy()
    asym.d[0, 0, 1] += 0.3
    with pytest.raises(C.InvalidArgument, match="Hermitian PAW"):
        PlaneWaveOperator(context, asym)
    nan = synthetic.tiny()
    nan.amplitudes = nan.amplitudes.copy()
    nan.amplitudes[0, 0] = np.nan
    with pytest.raises(C.InvalidArgument, match="nonfinite"):
        PlaneWaveOperator(context, nan)
    PlaneWaveOperator(context, base)  # the context stays usable after rejected inputs


def test_release_memory_hands_pooled_memory_back():
    """Operator arrays and working buffers are stream-ordered pool memory:
    after the operator closes they stay reserved in the library's pool (the
    next operator reuses them without synchronising the device), and
    Context.release_memory hands them back to the device."""
    import torch
    from sdft_b200 import synthetic
    from sdft_b200.operator import Context
    ctx = Context(0)
    op = PlaneWaveOperator(ctx, synthetic.si8())
    columns = 2000
    x = torch.from_numpy(np.ascontiguousarray(probe_block(op.npw, columns, 11).T)).cuda().T
    y = torch.empty((columns, op.npw), dtype=torch.complex128, device="cuda").T
    op.local_apply(x, out=y, precision="fp64")  # cuBLAS and other lazy set-up happen here
    ctx.release_memory()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    op.local_apply(x, out=y, precision="fp64")  # the FP64 slab: slots x n1 x n2 x 2000 x 16 B
    ctx.synchronize()
    op.close()
    held = free_before - torch.cuda.mem_get_info()[0]
    ctx.release_memory()
    returned = torch.cuda.mem_get_info()[0] - (free_before - held)
    try:
        assert held > 256 * 2**20  # the slab stayed in the pool after close
        assert returned >= held - 64 * 2**20
    finally:
        ctx.close()
