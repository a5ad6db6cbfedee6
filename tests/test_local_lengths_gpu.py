"""The fused local H~psi at every grid length its register-resident kernels
are compiled for (the one-thread pencil up to 72 points, the pair-split
pencil above, the pair-split plane passes for even lengths, and the plane
passes through the slab in global memory where two shared-memory planes do
not fit), on small cubic cells whose alias-free grid rule
(src/plane_wave_operator.cpp:445-457) lands on that length; a k-point of
(k, k, k) makes the span odd where needed.

Bars: the FP32 local apply (mixed form) within 2e-5 relative of the FP64
one (the mixed bar of tests/native/plane_wave_operator_smoke.cpp), per column
and for the block; the FP64 apply within 1e-12 of the numpy oracle's local
term; the mixed full H~x / S~x pair bit-identical to separate applies.
"""
import numpy as np
import pytest

from conftest import probe_block, relative_error
from oracle import sdft_oracle
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

# grid length -> (Ecut in Ha, k) for synthetic.tiny (a = 7 bohr, diamond Si8-like sites).
CELLS = {35: (26.0, 0.0), 40: (33.0, 0.0), 42: (40.5, 0.0), 45: (45.0, 0.5), 48: (53.5, 0.5), 49: (58.5, 0.0),
         54: (63.5, 0.5), 56: (74.0, 0.5), 60: (79.0, 0.0), 63: (91.0, 0.0), 70: (103.5, 0.0), 72: (124.0, 0.5),
         75: (131.0, 0.0), 80: (145.5, 0.0), 81: (161.5, 0.0), 84: (169.5, 0.5), 90: (178.0, 0.0),
         96: (204.5, 0.5), 98: (232.5, 0.0), 100: (242.5, 0.5), 112: (294.0, 0.0), 120: (316.0, 0.0),
         128: (400.0, 0.5)}
# Lengths checked against the numpy oracle as well: small ones, and ones whose
# plane passes run through the slab in global memory because two shared-memory
# planes do not fit (the FP64 form from 98 points on, FP32 from 120).
ORACLE_LENGTHS = {35, 40, 45, 49, 98, 112, 120, 128}
COLUMNS = 6


@pytest.mark.parametrize("n", sorted(CELLS))
def test_local_apply_mixed_matches_fp64_at_grid_length(context, n):
    import torch
    ecut, k = CELLS[n]
    inputs = synthetic.tiny(ecut_ha=ecut, kpoint=(k, k, k), roots=4)
    op = PlaneWaveOperator(context, inputs)
    try:
        assert op.shape == (n, n, n)
        x = probe_block(op.npw, COLUMNS, 100 + n)
        xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T
        y64 = op.local_apply(xd, precision="fp64")
        y32 = op.local_apply(xd, precision="mixed")
        context.synchronize()
        a64 = y64.T.cpu().numpy().T
        a32 = y32.T.cpu().numpy().T
        assert relative_error(a32, a64) < 2e-5
        for c in range(COLUMNS):
            assert relative_error(a32[:, c], a64[:, c]) < 2e-5
        if n in ORACLE_LENGTHS:  # the numpy oracle's local term (FFTs of the full grid)
            oracle = sdft_oracle.Operator(inputs)
            assert relative_error(a64, oracle.local(x)) < 1e-12
        hy, sy = op.apply_pair(xd, precision="mixed")
        h = op.apply(xd, overlap=False, precision="mixed")
        s = op.apply(xd, overlap=True, precision="mixed")
        context.synchronize()
        assert torch.equal(hy, h) and torch.equal(sy, s)
    finally:
        op.close()


def test_operator_above_65535_plane_waves(context):
    """An operator whose plane-wave count exceeds the CUDA grid's y limit
    (65 535): the tensor-core packing of B^H (one packed row per plane wave)
    and the mixed applies stride past it."""
    import torch
    inputs = synthetic.build_operator("large", 10.26, 1, 122.0, 8)
    assert inputs.hkl.shape[0] > 65535
    op = PlaneWaveOperator(context, inputs)
    try:
        x = probe_block(op.npw, 4, 65536)
        xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T
        for overlap in (False, True):
            y64 = op.apply(xd, overlap=overlap, precision="fp64")
            y32 = op.apply(xd, overlap=overlap, precision="mixed")
            context.synchronize()
            assert relative_error(y32.T.cpu().numpy(), y64.T.cpu().numpy()) < 2e-5
    finally:
        op.close()
