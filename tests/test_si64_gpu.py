"""The headline pencil (Si64-shaped cell, a = 20.52 bohr, 64 atoms, Ecut 15 Ha,
NPW 23 847, grid 70^3, 512 projectors, 160 bands) against the reference.

The benchmark quotes its metric on this pencil, so its operator and its solve
are pinned here at full size:
- the operator's integer index map and kinetic energies bit-exact, the H/S
  diagonals and V(r) within 1e-13 relative (si64_apply.npz, written by the
  reference's snapshot, tests/golden/make_golden.py --si64-apply);
- H~x and S~x of a seeded 160-column block in ONE call through the C ABI (the
  launch size the roofline is measured on): two columns in full, every column
  through its norm and its inner product with a seeded probe vector; FP64 plain
  form 1e-12 relative (tests/native/plane_wave_operator_smoke.cpp:60), mixed
  form 2e-5;
- the Davidson solve in both forms: all 160 pairs converged, fresh FP64
  residuals <= 1e-12 Ha on the device and recomputed by the numpy oracle,
  S-orthonormal, eigenvalues within 1e-10 Ha of the reference's own solve
  (si64_solution.npz; src/pw_core.cpp:1125-1149).
"""
import numpy as np
import pytest

from conftest import probe_block
from oracle import sdft_oracle
from sdft_b200.operator import PlaneWaveOperator

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 2e-5
EIGENVALUE_TOL = 1e-10
RESIDUAL_TOL = 1e-12


@pytest.fixture(scope="module")
def si64_inputs():
    from sdft_b200 import synthetic
    return synthetic.si64()


@pytest.fixture(scope="module")
def si64_op(context, si64_inputs):
    op = PlaneWaveOperator(context, si64_inputs)
    yield op
    op.close()


def test_si64_operator_arrays_match_reference(si64_op, golden):
    g = golden("si64_apply")
    assert si64_op.shape == tuple(int(v) for v in g["shape"])
    arrays = si64_op.arrays()
    assert np.array_equal(arrays["indices"], g["indices"])  # integer sphere/grid map bit-exact
    assert np.array_equal(arrays["kinetic"], g["kinetic"])
    for name in ("h_diagonal", "s_diagonal"):
        assert np.max(np.abs(arrays[name] - g[name])) <= 1e-13 * np.max(np.abs(g[name]))
    local = arrays["local_potential"]
    scale = np.max(np.abs(g["local_values"]))
    assert np.max(np.abs(local[g["local_points"]] - g["local_values"])) <= 1e-13 * scale
    assert abs(local.sum() - float(g["local_sum"])) <= 1e-13 * scale * local.size
    assert abs(np.dot(local, local) - float(g["local_sum2"])) <= 1e-12 * float(g["local_sum2"])


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_si64_apply_160_columns_matches_reference(si64_op, golden, precision, tol):
    torch = pytest.importorskip("torch")
    g = golden("si64_apply")
    x = probe_block(si64_op.npw, 160, int(g["probe_seed"]))
    u = probe_block(si64_op.npw, 1, int(g["checksum_seed"]))[:, 0]
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T  # column-major device block
    for overlap, key in ((False, "hx"), (True, "sx")):
        yd = si64_op.apply(xd, overlap=overlap, precision=precision)
        si64_op.context.synchronize()
        y = yd.T.cpu().numpy().T
        full = y[:, g["columns"]]
        assert np.linalg.norm(full - g[key]) / np.linalg.norm(g[key]) < tol
        norms = np.linalg.norm(y, axis=0)
        assert np.max(np.abs(norms - g[f"{key}_norms"]) / g[f"{key}_norms"]) < tol
        dots = u.conj() @ y
        assert np.max(np.abs(dots - g[f"{key}_dots"]) / (np.linalg.norm(u) * g[f"{key}_norms"])) < tol


def test_si64_pair_equals_separate_at_160_columns(si64_op):
    torch = pytest.importorskip("torch")
    x = probe_block(si64_op.npw, 160, 5)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T
    for precision in ("fp64", "mixed"):
        hy, sy = si64_op.apply_pair(xd, precision=precision)
        h = si64_op.apply(xd, overlap=False, precision=precision)
        s = si64_op.apply(xd, overlap=True, precision=precision)
        si64_op.context.synchronize()
        assert torch.equal(hy, h) and torch.equal(sy, s)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_si64_solve_matches_reference(si64_op, si64_inputs, golden, precision):
    g = golden("si64_solution")
    result = si64_op.davidson(si64_inputs.roots, 256, RESIDUAL_TOL, precision=precision)
    assert result["converged"], result["stats"]
    assert np.all(result["residuals"] <= RESIDUAL_TOL)
    assert np.max(np.abs(result["eigenvalues"] - g["eigenvalues"])) < EIGENVALUE_TOL
    oracle = sdft_oracle.Operator(si64_inputs)
    vectors = result["eigenvectors"].T
    fresh, metric = sdft_oracle.certified_residuals(oracle, result["eigenvalues"], vectors)
    assert np.max(fresh) <= 1.01 * RESIDUAL_TOL
    assert np.max(metric) <= 1e-12
    gram = vectors.conj().T @ oracle.apply_s(vectors)
    assert np.max(np.abs(gram - np.eye(gram.shape[0]))) <= 1e-10
