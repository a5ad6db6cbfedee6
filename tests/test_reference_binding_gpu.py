"""The reference's own tests, linked against libsdft_b200 through
sparse-dft_b200/reference_binding/compute_b200.cpp (SDFT_COMPUTE_BACKEND=cuda).

compute_backend_smoke checks complex_gemm in every operation pair, with
padded strides and beta 0/1, and complex_gemm_immutable_left with identity
changes against direct sums (2e-11), all routed through the accelerator;
fft_backend_smoke checks the accelerated local H against a direct
convolution oracle (2e-11) and, with --require-gpu, that the GPU path really
ran; sdft_b200_solver_replay (the device-resident solve route of
reference_binding/b200_solver.cpp behind the reference's replay CLI, checked
by the reference's own CPU operator) must pass its report and agree with the
reference's replay eigenvalues; plane_wave_operator_smoke checks the exact=false search applications
(local FFT + PAW chain on the GPU) against dense H/S (1e-10) and the Davidson
eigenvalues against a dense generalized eigensolver (1e-11).
"""
import json
import os
import pathlib
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BINDING = pathlib.Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "binding"


def run(binary, args, env_extra, tmp_path):
    path = BINDING / binary
    if not path.exists():
        pytest.skip("reference binding not built (make -C sparse-dft_b200/reference_binding)")
    env = dict(os.environ, OMP_NUM_THREADS="4", OPENBLAS_NUM_THREADS="1", **env_extra)
    return subprocess.run([str(path), *args], cwd=tmp_path, env=env, capture_output=True, text=True, timeout=900)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reference_fft_backend_smoke_runs_on_b200(tmp_path, precision):
    out = run("fft_backend_smoke", ["--require-gpu"],
              {"SDFT_COMPUTE_BACKEND": "cuda", "SDFT_GPU_FFT": "1", "SDFT_GPU_FFT_MIN_POINTS": "0",
               "SDFT_B200_ACCELERATOR_PRECISION": precision}, tmp_path)
    report = json.loads(out.stdout.strip().splitlines()[-1])
    assert all(case["accelerated"] for case in report["cases"]), report
    if precision == "fp64":
        assert out.returncode == 0 and report["passed"], out.stdout + out.stderr
    else:
        # FP32 FFTs: the 2e-11 limit is an FP64 bar; the mixed form stays near FP32 rounding.
        assert report["maximum_scaled_error"] < 1e-6, report


def test_reference_plane_wave_operator_smoke_runs_on_b200(tmp_path):
    out = run("plane_wave_operator_smoke", [],
              {"SDFT_COMPUTE_BACKEND": "cuda", "SDFT_GPU_FFT": "1", "SDFT_GPU_FFT_MIN_POINTS": "0",
               "SDFT_GPU_PAW_CHAIN": "1", "SDFT_GPU_MIN_WORK": "0"}, tmp_path)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "plane_wave_operator PASS" in out.stdout


def test_reference_pbe_backend_smoke_runs_on_b200(tmp_path):
    out = run("pbe_backend_smoke", [], {"SDFT_COMPUTE_BACKEND": "cuda", "SDFT_GPU_PBE": "1"}, tmp_path)
    report = json.loads(out.stdout.strip().splitlines()[-1])
    assert report["accelerated"], report
    assert out.returncode == 0 and report["passed"], out.stdout + out.stderr


def test_reference_compute_backend_smoke_runs_on_b200(tmp_path):
    out = run("compute_backend_smoke", [], {"SDFT_COMPUTE_BACKEND": "cuda", "SDFT_GPU_MIN_WORK": "0"}, tmp_path)
    assert out.returncode == 0, out.stdout + out.stderr
    report = json.loads(out.stdout.strip().splitlines()[-1])
    assert report["backend"] == "cuda", report
    assert report["independent_reference_scaled_error"] < 2e-11, report


GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("snapshot", ["tiny_cold", "tiny_warm"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_solve_route_replays_reference_snapshots(tmp_path, golden, snapshot, precision):
    report_path = tmp_path / "report.json"
    out = run("sdft_b200_solver_replay", [str(GOLDEN / f"{snapshot}.pwo3"), str(report_path), "256", precision], {},
              tmp_path)
    assert out.returncode == 0, out.stdout + out.stderr
    report = json.loads(report_path.read_text())
    assert report["passed"] and report["solver"] == "b200" and report["solver_converged"], report
    assert report["fresh_max_residual"] <= report["tolerance"] and report["s_normalization_error"] <= 1e-12
    import numpy as np
    expected = golden("snapshots")[f"{snapshot}_eigenvalues"]
    assert np.max(np.abs(np.array(report["eigenvalues_hartree"]) - expected)) < 1e-10
