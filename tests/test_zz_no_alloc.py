"""sdft_b200_apply_local_noalloc: the fused local H~psi with its slab and
twiddle tables in the library's static device array. Collected last (file
name), and self-contained so that it also passes alone in a fresh process.

Checks: the same results as sdft_b200_apply_local on two calls in a row in
each precision, no change in free device memory across calls after the
first (set-up) call, a clear rejection of a block beyond the array (the
largest accepted block is exactly the column limit the rejection names),
calls for two operators with different grids interleaved on one stream (each
rewrites the shared tables), the rejection of host pointers before any
launch, and a call captured into a CUDA graph after the set-up call, replayed
on new inputs, equal to the regular entry point."""
import numpy as np
import pytest

from conftest import probe_block

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def operators():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdft_b200 import synthetic
    from sdft_b200.operator import Context, PlaneWaveOperator
    ctx = Context(0)
    ops = {"si8": PlaneWaveOperator(ctx, synthetic.si8()), "tiny": PlaneWaveOperator(ctx, synthetic.tiny())}
    yield ops
    for op in ops.values():
        op.close()
    ctx.close()


@pytest.fixture(scope="module")
def si8_operator(operators):
    return operators["si8"]


def _device_block(npw, columns, seed):
    import torch
    x = probe_block(npw, columns, seed)
    block = torch.from_numpy(x.T.copy()).cuda().T  # column-major, ld npw
    torch.cuda.synchronize()  # the context runs on its own stream
    return block


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_regular_entry_point(si8_operator, precision):
    import torch
    op = si8_operator
    for call, seed in enumerate((3, 4)):
        x = _device_block(op.npw, 24, seed)
        regular = op.local_apply(x, out=torch.empty((24, op.npw), dtype=torch.complex128, device="cuda").T,
                                 precision=precision)
        static = op.local_apply_noalloc(x, torch.empty((24, op.npw), dtype=torch.complex128, device="cuda").T,
                                        precision=precision)
        torch.cuda.synchronize()
        assert torch.equal(static, regular), f"call {call}: results differ from sdft_b200_apply_local"


def test_noalloc_calls_leave_free_memory_unchanged(si8_operator):
    import torch
    op = si8_operator
    x = _device_block(op.npw, 16, 5)
    y = torch.empty((16, op.npw), dtype=torch.complex128, device="cuda").T
    op.local_apply_noalloc(x, y, precision="mixed")  # set-up call
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for precision in ("mixed", "fp64", "mixed"):
        op.local_apply_noalloc(x, y, precision=precision)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_rejects_blocks_beyond_the_static_array(si8_operator):
    import torch
    from sdft_b200 import _capi
    op = si8_operator
    columns = 1000  # ~1 GB of FP64 slab for Si8, far above 32 MiB
    x = torch.zeros((columns, op.npw), dtype=torch.complex128, device="cuda").T
    y = torch.empty_like(x.T).T
    torch.cuda.synchronize()
    with pytest.raises(_capi.InvalidArgument, match="static scratch; at most [0-9]+ columns"):
        op.local_apply_noalloc(x, y, precision="fp64")
    small = _device_block(op.npw, 2, 6)
    out = op.local_apply_noalloc(small, torch.empty((2, op.npw), dtype=torch.complex128, device="cuda").T)
    assert torch.isfinite(torch.view_as_real(out)).all()


def _pair(op, columns, seed, precision):
    import torch
    x = _device_block(op.npw, columns, seed)
    regular = op.local_apply(x, out=torch.empty((columns, op.npw), dtype=torch.complex128, device="cuda").T,
                             precision=precision)
    static = op.local_apply_noalloc(x, torch.empty((columns, op.npw), dtype=torch.complex128, device="cuda").T,
                                    precision=precision)
    op.context.synchronize()
    return static, regular


def test_noalloc_column_limit_is_exact(si8_operator):
    import re
    import torch
    from sdft_b200 import _capi
    op = si8_operator
    x = torch.zeros((4000, op.npw), dtype=torch.complex128, device="cuda").T
    y = torch.empty_like(x.T).T
    torch.cuda.synchronize()
    with pytest.raises(_capi.InvalidArgument) as info:
        op.local_apply_noalloc(x, y, precision="fp64")
    limit = int(re.search(r"at most ([0-9]+) columns", str(info.value)).group(1))
    assert 1 <= limit < 4000
    static, regular = _pair(op, limit, 7, "fp64")
    assert torch.equal(static, regular)
    over = _device_block(op.npw, limit + 1, 8)
    with pytest.raises(_capi.InvalidArgument, match=f"at most {limit} columns"):
        op.local_apply_noalloc(over, torch.empty_like(over.T).T, precision="fp64")


def test_noalloc_interleaved_operators_with_different_grids(operators):
    import torch
    si8, tiny = operators["si8"], operators["tiny"]
    assert si8.shape != tiny.shape
    for round_, precision in enumerate(("fp64", "mixed", "fp64")):
        for op in (si8, tiny, si8):
            static, regular = _pair(op, 5, 20 + round_, precision)
            assert torch.equal(static, regular), f"{op.shape} {precision}: results differ after the other grid's call"


def test_noalloc_rejects_host_pointers_before_launch(si8_operator):
    import ctypes
    import torch
    from sdft_b200 import _capi
    op = si8_operator
    launches = _capi.library().sdft_b200_kernel_launches()
    host = np.zeros((op.npw, 2), dtype=np.complex128, order="F")
    device = _device_block(op.npw, 2, 9)
    lib = _capi.library()
    status = lib.sdft_b200_apply_local_noalloc(op.handle, ctypes.c_void_p(host.ctypes.data), 2,
                                               ctypes.c_void_p(device.data_ptr()), _capi.FP64)
    assert status == _capi.INVALID_ARGUMENT and "device memory" in _capi.last_error()
    status = lib.sdft_b200_apply_local_noalloc(op.handle, ctypes.c_void_p(device.data_ptr()), 2,
                                               ctypes.c_void_p(host.ctypes.data), _capi.FP64)
    assert status == _capi.INVALID_ARGUMENT
    assert _capi.library().sdft_b200_kernel_launches() == launches
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_call_replays_from_a_cuda_graph(precision):
    import torch
    from sdft_b200 import synthetic
    from sdft_b200.operator import Context, PlaneWaveOperator
    stream = torch.cuda.Stream()
    ctx = Context(0, stream.cuda_stream)
    op = PlaneWaveOperator(ctx, synthetic.si8())
    try:
        x = _device_block(op.npw, 6, 31)
        y = torch.empty((6, op.npw), dtype=torch.complex128, device="cuda").T
        op.local_apply_noalloc(x, y, precision=precision)  # set-up call, outside the capture
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream, capture_error_mode="thread_local"):
            op.local_apply_noalloc(x, y, precision=precision)
        x.copy_(_device_block(op.npw, 6, 32))  # new inputs in the captured buffer
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        regular = op.local_apply(x, out=torch.empty((6, op.npw), dtype=torch.complex128, device="cuda").T,
                                 precision=precision)
        ctx.synchronize()
        assert torch.equal(y, regular)
        del graph
    finally:
        op.close()
        ctx.close()
