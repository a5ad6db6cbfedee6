"""C ABI checks that need no GPU: the library loads, exports its header, host logic is exact."""
import ctypes
import pathlib
import subprocess

import numpy as np
import pytest

from conftest import gpu_available
from sdft_b200 import _capi as C
from sdft_b200 import operator as sop
from sdft_b200 import synthetic


def test_library_loads():
    assert C.LIBRARY.exists(), "libsdft_b200.so must be built in-tree"
    lib = C.library()
    assert b"sm_100a" in lib.sdft_b200_version()


def test_every_declared_symbol_is_exported():
    declared = C.declared_symbols()
    assert len(declared) >= 13
    exported = subprocess.run(["nm", "-D", "--defined-only", str(C.LIBRARY)], capture_output=True, text=True,
                              check=True).stdout
    names = {line.split()[-1] for line in exported.splitlines() if line.strip()}
    missing = [s for s in declared if s not in names]
    assert not missing, missing
    lib = C.library()
    for s in declared:
        assert hasattr(lib, s)


def test_library_is_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", str(C.LIBRARY)], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


@pytest.mark.parametrize("factory", [synthetic.tiny, synthetic.si8])
def test_enumeration_bit_exact(golden, factory):
    x = factory()
    hkl, cart, kin = sop.enumerate_g_vectors(x.reciprocal, x.ecut_ha * synthetic.HARTREE_TO_EV)
    g = golden(x.name)
    assert np.array_equal(hkl, g["hkl"]) and np.array_equal(kin, g["kinetic_ev"])
    assert np.array_equal(cart, x.cartesian)


def test_enumeration_kpoint_and_errors():
    x = synthetic.tiny()
    for k in ((1 / 3, 0.0, -1 / 3), (0.25, 0.5, 0.0)):
        a = sop.enumerate_g_vectors(x.reciprocal, 4.0 * synthetic.HARTREE_TO_EV, k)
        b = synthetic.enumerate_g_vectors(x.reciprocal, 4.0 * synthetic.HARTREE_TO_EV, k)
        assert all(np.array_equal(u, v) for u, v in zip(a, b))
    with pytest.raises(C.InvalidArgument):
        sop.enumerate_g_vectors(x.reciprocal, -1.0)
    with pytest.raises(C.InvalidArgument):
        sop.enumerate_g_vectors(np.zeros((3, 3)), 10.0)
    assert "cutoff" in C.last_error() or "singular" in C.last_error()


def test_context_without_gpu_reports_cuda_error():
    if gpu_available():
        pytest.skip("a GPU is present")
    lib = C.library()
    handle = ctypes.c_void_p()
    status = lib.sdft_b200_context_create(0, None, ctypes.byref(handle))
    assert status == C.CUDA_ERROR
    assert "CUDA" in C.last_error()


def test_solve_footprint_is_host_arithmetic():
    """The server's admission budget needs no device: it grows with the roots
    and the subspace factor and covers at least the three basis blocks."""
    from sdft_b200 import synthetic
    from sdft_b200.serving import solve_footprint
    x = synthetic.si8()
    small = solve_footprint(x, 8)
    large = solve_footprint(x, 16)
    wide = solve_footprint(x, 16, subspace_factor=16)
    assert 0 < small < large < wide
    capacity = min(x.npw, max(8 * 16, 64))
    assert large > 3 * 16 * x.npw * capacity


def test_server_without_gpu_reports_cuda_error():
    if gpu_available():
        pytest.skip("a GPU is present")
    lib = C.library()
    handle = ctypes.c_void_p()
    assert lib.sdft_b200_server_create(0, 1 << 30, 2, ctypes.byref(handle)) == C.CUDA_ERROR
    assert "CUDA" in C.last_error()
    assert lib.sdft_b200_server_create(0, 1 << 30, 0, ctypes.byref(handle)) == C.INVALID_ARGUMENT


def test_operator_update_null_operator_is_invalid_argument():
    """The SCF refresh checks its handle before any device work."""
    lib = C.library()
    assert lib.sdft_b200_operator_update(None, 0, None, None, None, None) == C.INVALID_ARGUMENT
    assert "null operator" in C.last_error()


def test_scf_step_keeps_potential_and_blocks_hermitian():
    """The seeded SCF sequence (test input of the operator refresh) keeps V(G)
    Hermitian on its keys, G = 0 present, and every D block Hermitian."""
    from sdft_b200 import synthetic
    x = synthetic.tiny()
    for step, keep in ((1, 1.0), (2, 0.5)):
        y = synthetic.scf_step(x, step, keep=keep)
        values = {tuple(k): v for k, v in zip(y.v_hkl.tolist(), y.v_values)}
        assert (0, 0, 0) in values
        assert max(abs(v - np.conj(values.get((-k[0], -k[1], -k[2]), 0.0))) for k, v in values.items()) == 0.0
        assert np.array_equal(y.d, np.conj(np.transpose(y.d, (0, 2, 1))))
        assert np.array_equal(y.amplitudes, x.amplitudes) and np.array_equal(y.q, x.q)
        assert (y.v_hkl.shape[0] == x.v_hkl.shape[0]) == (keep == 1.0)


def test_snapshot_header_matches_reference_file():
    """The snapshot reader's header (host only) agrees with the file the
    reference wrote (tests/golden/tiny_*.pwo3); non-snapshots are refused."""
    import struct
    from sdft_b200.operator import snapshot_info
    golden = pathlib.Path(__file__).resolve().parent / "golden"
    for name, warm in (("tiny_cold", False), ("tiny_warm", True)):
        raw = (golden / f"{name}.pwo3").read_bytes()
        n, count, s0, s1, s2, nproj, roots, iters, ninit = struct.unpack_from("<9Q", raw, 8)
        reg, tol = struct.unpack_from("<2d", raw, 80)
        info = snapshot_info(golden / f"{name}.pwo3")
        assert (info["npw"], info["grid_points"], info["projectors"], info["roots"], info["iterations"]) == (
            n, count, nproj, roots, iters)
        assert info["shape"] == (s0, s1, s2) and info["atoms"] == struct.unpack_from("<Q", raw, 96)[0]
        assert info["regularization"] == reg and info["tolerance"] == tol
        assert (info["initial_values"] == n * roots) == warm and (info["initial_values"] == 0) != warm
    with pytest.raises(C.SdftError, match="unsupported solver snapshot format"):
        snapshot_info(golden / "tiny.npz")
    with pytest.raises(C.SdftError, match="cannot open solver snapshot"):
        snapshot_info(golden / "no_such_snapshot.pwo3")


def test_functional_support_query_and_checks_are_host_only(golden):
    """The functional's support query (capacity 0) runs on the host with no
    context, and the reference's input checks fail before any device work."""
    from sdft_b200 import density
    case = synthetic.functional_case("triclinic")
    lib = C.library()
    lat = np.ascontiguousarray(case["lattice"], dtype=np.float64).reshape(9)
    keys = np.ascontiguousarray(case["keys"], dtype=np.int32)
    values = np.ascontiguousarray(case["values"], dtype=np.complex128)
    core_keys = np.ascontiguousarray(case["core_keys"], dtype=np.int32)
    core = np.ascontiguousarray(case["core_values"], dtype=np.complex128)
    count = ctypes.c_size_t()
    assert lib.sdft_b200_density_functionals(None, lat.ctypes.data_as(C.D), keys.shape[0], keys.ctypes.data_as(C.I32),
                                             values.ctypes.data_as(C.D), core_keys.shape[0],
                                             core_keys.ctypes.data_as(C.I32), core.ctypes.data_as(C.D), 0, None,
                                             None, None, 0, ctypes.byref(count), None) == C.OK
    assert count.value == golden("functional_triclinic")["core_hkl"].shape[0]

    def fails(match, lattice=case["lattice"], k=case["keys"], v=case["values"], ck=None, cv=None, padding=0):
        with pytest.raises(C.InvalidArgument, match=match):
            density.density_functionals(None, lattice, k, v, ck, cv, padding, support_only=True)

    fails("singular", lattice=np.zeros((3, 3)))
    fails("empty", k=np.zeros((0, 3)), v=np.zeros(0))
    fails("duplicate", k=np.concatenate([keys, keys[:1]]), v=np.concatenate([values, values[:1]]))
    bad = values.copy()
    bad[3] = np.nan
    fails("non-finite valence density", v=bad)
    bad_core = core.copy()
    bad_core[0] = np.inf
    fails("pseudo-core", ck=core_keys, cv=bad_core)
    fails("quadrature", padding=9)
    fails("above 512", k=np.array([[300, 0, 0], [0, 0, 0]]), v=np.array([0.1, 1.0]))


def test_solver_routes_check_handles_without_a_gpu():
    """The RMM trial and the band-group solve reject a null operator before
    any device work."""
    lib = C.library()
    opts = C.DavidsonOptions(roots=4, max_iterations=8, tolerance=1e-6, precision=C.FP64, subspace_factor=8,
                             handoff=1e-8)
    values = np.zeros(4)
    residuals = np.zeros(4)
    assert lib.sdft_b200_rmm_trial(None, ctypes.byref(opts), None, values.ctypes.data_as(C.D), None,
                                   residuals.ctypes.data_as(C.D), None, None, C.HOST) == C.INVALID_ARGUMENT
    assert "RMM" in C.last_error()
    assert lib.sdft_b200_band_groups(None, ctypes.byref(opts), None, values.ctypes.data_as(C.D), None,
                                     residuals.ctypes.data_as(C.D), None, C.HOST) == C.INVALID_ARGUMENT
    assert "band-group" in C.last_error()


def test_collinear_support_query_and_checks_are_host_only(golden):
    """The collinear form's support query runs on the host with no context and
    equals the reference's support; its input checks fail before device work."""
    from sdft_b200 import density
    case = synthetic.collinear_case("triclinic")
    args = (case["lattice"], case["up_keys"], case["up"], case["down_keys"], case["down"], case["core_keys"],
            case["core_values"])
    keys = density.collinear_functionals(None, *args, support_only=True)
    assert np.array_equal(keys, golden("collinear_triclinic")["core_hkl"])
    with pytest.raises(C.InvalidArgument, match="invalid collinear density/lattice"):
        density.collinear_functionals(None, np.zeros((3, 3)), *args[1:], support_only=True)
    with pytest.raises(C.InvalidArgument, match="invalid collinear density/lattice"):
        density.collinear_functionals(None, case["lattice"], case["up_keys"], case["up"], np.zeros((0, 3)),
                                      np.zeros(0), support_only=True)
    with pytest.raises(C.InvalidArgument, match="invalid collinear XC padding"):
        density.collinear_functionals(None, *args, padding=9, support_only=True)
