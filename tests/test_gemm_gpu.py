"""Complex GEMM boundary (the reference's complex_gemm): FP64 and tcgen05 mixed.

Oracle: numpy complex128 products. Bars: FP64 1e-13 relative (Frobenius);
mixed (BF16 split products, FP32 tensor-memory accumulation) 2e-5 relative,
the same bar as the mixed operator applications.
"""
import numpy as np
import pytest

from conftest import relative_error
from sdft_b200.operator import complex_gemm

pytestmark = pytest.mark.gpu

SHAPES = [(512, 160, 3001, False), (300, 17, 130, True), (64, 1, 64, False), (1, 9, 5000, True),
          (700, 40, 512, True), (129, 129, 257, False)]


def random(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("m,n,k,adjoint", SHAPES)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_complex_gemm_matches_numpy(context, m, n, k, adjoint, precision, tol):
    rng = np.random.default_rng(m * 7919 + n * 31 + k)
    a = random(rng, (k, m) if adjoint else (m, k))
    b = random(rng, (k, n))
    ref = (a.conj().T if adjoint else a) @ b
    out = complex_gemm(context, a, b, adjoint_a=adjoint, precision=precision)
    assert relative_error(out, ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_complex_gemm_accumulates(context, precision, tol):
    rng = np.random.default_rng(5)
    a, b, c = random(rng, (96, 400)), random(rng, (400, 33)), random(rng, (96, 33))
    out = complex_gemm(context, a, b, precision=precision, c=c)
    assert relative_error(out, a @ b + c) < tol


def test_mixed_gemm_is_deterministic(context):
    rng = np.random.default_rng(9)
    a, b = random(rng, (256, 6000)), random(rng, (6000, 48))
    first = complex_gemm(context, a, b, precision="mixed")
    second = complex_gemm(context, a, b, precision="mixed")
    assert np.array_equal(first, second)


@pytest.mark.parametrize("add", [0, 1])
def test_host_gemm_on_submatrix_leaves_other_rows(context, add):
    """C is a row block of a taller host matrix (ldc > m), as in the reference's
    per-atom products into a shared projection array: only the block changes."""
    import ctypes
    from sdft_b200 import _capi as C
    rng = np.random.Generator(np.random.PCG64(17))
    m, n, k, ldc, offset = 8, 13, 8, 40, 16
    a = np.asfortranarray(rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k)))
    b = np.asfortranarray(rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n)))
    full = np.asfortranarray(rng.standard_normal((ldc, n)) + 1j * rng.standard_normal((ldc, n)))
    expected = full.copy(order="F")
    expected[offset:offset + m] = a @ b + (expected[offset:offset + m] if add else 0)
    base = full.ctypes.data + 16 * offset
    C.check(C.library().sdft_b200_complex_gemm(context.handle, 0, 0, m, n, k, ctypes.c_void_p(a.ctypes.data), m,
                                               ctypes.c_void_p(b.ctypes.data), k, ctypes.c_void_p(base), ldc, C.FP64,
                                               add, C.HOST))
    assert np.array_equal(full[:offset], expected[:offset])
    assert np.array_equal(full[offset + m:], expected[offset + m:])
    assert relative_error(full[offset:offset + m], expected[offset:offset + m]) < 1e-14


@pytest.mark.parametrize("adjoint", [False, True])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_immutable_left_is_cached_per_identity(context, adjoint, precision, tol):
    """The reference's complex_gemm_immutable_left contract
    (src/compute_backend.hpp:32-41): the left operand is read once per
    identity; a new identity picks up new contents of the same host array."""
    from sdft_b200.operator import complex_gemm_immutable_left
    rng = np.random.default_rng(17 + adjoint)
    a = np.asfortranarray(random(rng, (300, 120) if adjoint else (120, 300)))
    original = a.copy()
    op_a = (lambda x: x.conj().T) if adjoint else (lambda x: x)
    identity = 900 + 2 * adjoint + (precision == "mixed") * 10
    for call in range(3):
        b = random(rng, (300, 7 + call))
        out = complex_gemm_immutable_left(context, identity, a, b, adjoint_a=adjoint, precision=precision)
        assert relative_error(out, op_a(original) @ b) < tol
        a[:] = random(rng, a.shape)  # same identity: the cached operand stays the original one
    out = complex_gemm_immutable_left(context, identity + 1, a, b, adjoint_a=adjoint, precision=precision)
    assert relative_error(out, op_a(a) @ b) < tol
    if precision == "fp64":
        plain = complex_gemm(context, a, b, adjoint_a=adjoint, precision="fp64")
        assert np.array_equal(out, plain)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_triple_right_equals_three_products(context, precision, tol):
    from sdft_b200.operator import complex_gemm_triple_right
    rng = np.random.default_rng(23)
    lefts = [random(rng, (2000, 96)) for _ in range(3)]
    b = random(rng, (96, 40))
    outs = complex_gemm_triple_right(context, lefts, b, precision=precision)
    for a, out in zip(lefts, outs):
        assert relative_error(out, a @ b) < tol
        assert np.array_equal(out, complex_gemm(context, a, b, precision=precision))


def test_triple_right_rejects_aliased_outputs(context):
    import ctypes
    from sdft_b200 import _capi as C
    rng = np.random.default_rng(2)
    a = [np.asfortranarray(random(rng, (10, 4))) for _ in range(3)]
    b = np.asfortranarray(random(rng, (4, 3)))
    out = np.zeros((10, 3), np.complex128, order="F")
    lib = C.library()
    a_ptrs = (ctypes.c_void_p * 3)(*[x.ctypes.data for x in a])
    same = (ctypes.c_void_p * 3)(*([out.ctypes.data] * 3))
    assert lib.sdft_b200_complex_gemm_triple_right(context.handle, 10, 3, 4, a_ptrs, 10, ctypes.c_void_p(b.ctypes.data),
                                                   4, same, 10, C.FP64, C.HOST) == C.INVALID_ARGUMENT
    into_b = (ctypes.c_void_p * 3)(b.ctypes.data, out.ctypes.data, a[0].ctypes.data)
    assert lib.sdft_b200_complex_gemm_triple_right(context.handle, 4, 3, 4, a_ptrs, 10, ctypes.c_void_p(b.ctypes.data),
                                                   4, into_b, 4, C.FP64, C.HOST) == C.INVALID_ARGUMENT


def test_mixed_gemm_with_adjoint_right_operand(context):
    """The tensor-core path forms B^H on the device for an adjoint right operand."""
    import ctypes
    from sdft_b200 import _capi as C
    rng = np.random.default_rng(4)
    a = np.asfortranarray(random(rng, (64, 200)))
    b = np.asfortranarray(random(rng, (48, 200)))  # op(B) = B^H is 200 x 48
    out = np.zeros((64, 48), np.complex128, order="F")
    C.check(C.library().sdft_b200_complex_gemm(context.handle, 0, 1, 64, 48, 200, ctypes.c_void_p(a.ctypes.data), 64,
                                               ctypes.c_void_p(b.ctypes.data), 48, ctypes.c_void_p(out.ctypes.data), 64,
                                               C.MIXED, 0, C.HOST))
    assert relative_error(out, a @ b.conj().T) < 2e-5


def test_autotuner_records_each_shape_class_once(context):
    """The tile autotuner keeps one (width, split) choice per shape class, and a
    repeated product of that class gives the same bits."""
    from sdft_b200 import _capi as C
    rng = np.random.default_rng(31)
    a, b = random(rng, (200, 3000)), random(rng, (3000, 24))
    first = complex_gemm(context, a, b, precision="mixed")
    table = C.gemm_tuned_classes()
    assert table, "no tuned shape class recorded"
    for rows, cols, kblocks, width, splits in table:
        assert rows % 128 == 0 and cols % 32 == 0 and kblocks > 0
        assert width in (128, 160, 256) and 1 <= splits <= 128
    again = complex_gemm(context, a, b, precision="mixed")
    assert np.array_equal(first, again)
    assert len(C.gemm_tuned_classes()) == len(table)
