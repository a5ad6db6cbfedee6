"""The k-point batch workload's cell: GaAs-shaped zincblende 2x2x2 supercell
(a = 21.36 bohr, 64 atoms, depths -2.2 / -1.8 Ha), Ecut 18 Ha, 192 bands, at
two k-points of the 3x3x3 Monkhorst-Pack mesh, against the reference
(gaas64_k*.npz, tests/golden/make_golden.py --gaas64).

Bars: the sphere/grid index map and the kinetic energies bit-exact; H~x and
S~x of a seeded 16-column probe through their norms and probe-vector inner
products (FP64 1e-12 relative, mixed 2e-5); the solve (mixed form, the
library default) converged with every fresh FP64 residual <= 1e-12 Ha and
eigenvalues within 1e-10 Ha of the reference's; at one k-point the residuals
are recomputed by the numpy oracle.
"""
import numpy as np
import pytest

from conftest import probe_block
from oracle import sdft_oracle
from sdft_b200 import synthetic
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

KPOINTS = (26, 5)


@pytest.fixture(scope="module", params=KPOINTS)
def kpoint_case(request, context):
    index = request.param
    inputs = synthetic.gaas_kpoint(index)
    op = PlaneWaveOperator(context, inputs)
    yield index, inputs, op
    op.close()


def test_gaas64_operator_matches_reference(kpoint_case, golden):
    index, inputs, op = kpoint_case
    g = golden(f"gaas64_k{index}")
    assert np.array_equal(inputs.kpoint, g["kpoint"])
    assert op.shape == tuple(int(v) for v in g["shape"])
    arrays = op.arrays()
    assert np.array_equal(arrays["indices"], g["indices"].astype(np.uint64))
    assert np.array_equal(arrays["kinetic"], g["kinetic"])
    x = probe_block(op.npw, 16, int(g["probe_seed"]))
    u = probe_block(op.npw, 1, int(g["checksum_seed"]))[:, 0]
    for precision, tol in (("fp64", 1e-12), ("mixed", 2e-5)):
        for overlap, key in ((False, "hx"), (True, "sx")):
            y = op.apply(x, overlap=overlap, precision=precision)
            norms = np.linalg.norm(y, axis=0)
            assert np.max(np.abs(norms - g[f"{key}_norms"]) / g[f"{key}_norms"]) < tol
            dots = u.conj() @ y
            assert np.max(np.abs(dots - g[f"{key}_dots"]) / (np.linalg.norm(u) * g[f"{key}_norms"])) < tol


def test_gaas64_solve_matches_reference(kpoint_case, golden):
    index, inputs, op = kpoint_case
    g = golden(f"gaas64_k{index}")
    assert bool(g["converged"])
    check_vectors = index == KPOINTS[0]
    result = op.davidson(inputs.roots, 256, 1e-12, precision="mixed", vectors=check_vectors)
    assert result["converged"], result["stats"]
    assert np.all(result["residuals"] <= 1e-12)
    assert np.max(np.abs(result["eigenvalues"] - g["eigenvalues"])) < 1e-10
    if check_vectors:
        oracle = sdft_oracle.Operator(inputs)
        vectors = result["eigenvectors"].T
        fresh, metric = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], vectors)
        assert np.max(fresh) <= 1.01e-12 and np.max(metric) <= 1e-12
