#!/usr/bin/env python
"""Benchmark: certified eigenpairs/s of the generalized Davidson solve on one B200.

Workload: the Si64-shaped Gamma-point pencil (a = 20.52 bohr, 64 atoms, Ecut 15 Ha,
NPW 23847, FFT grid 70^3, 512 projectors, 160 bands, tolerance 1e-12 Ha, cold
start), seeded synthetic inputs. One step = one full Davidson solve of that
pencil in the mixed-precision form (FP32 FFT/V_loc, FP32-accumulated search
GEMMs, FP64 Rayleigh-Ritz, refresh and certification), inputs resident in HBM.
The FP64 plain form is timed on the same GPU beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs N independent replicas (one per rank, launched by torchrun); the
solve itself does not shard. --impl reference times the reference's own CPU
implementation (oracle/_ref) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sparse-dft_b200"))

METRIC = "certified eigenpairs/s at <=1e-12 Ha, mixed vs FP64 on 1 B200; p50/p99 solve ms"
UNIT = "certified eigenpairs/s"
TOLERANCE = 1e-12
WORKLOAD = "si64_gamma_davidson"


def config(args, extra=None):
    cfg = {"workload": WORKLOAD, "cell": "Si64 diamond 2x2x2, a=20.52 bohr", "npw": 23847, "fft_grid": [70, 70, 70],
           "projectors": 512, "bands": 160, "ecut_ha": 15.0, "tolerance_ha": TOLERANCE, "start": "cold",
           "l2": "inputs larger than L2 (basis + images 1.5 GB, slab 220 MB per 160-column apply)"}
    if extra:
        cfg.update(extra)
    return cfg


def load_inputs():
    """Synthetic Si64 pencil; cached as .npz in the temp dir (seeded, deterministic)."""
    import numpy as np
    from sdft_b200 import synthetic
    cache = pathlib.Path(tempfile.gettempdir()) / "sdft_b200_si64_seed2026.npz"
    if cache.exists():
        data = dict(np.load(cache))
        return synthetic.OperatorInputs(
            name="si64", lattice=data["lattice"], reciprocal=data["reciprocal"], volume=float(data["volume"]),
            positions=data["positions"], species=data["species"], kpoint=data["kpoint"], ecut_ha=15.0,
            hkl=data["hkl"], cartesian=data["cartesian"], kinetic_ev=data["kinetic_ev"], v_hkl=data["v_hkl"],
            v_values=data["v_values"], projectors=data["projectors"], amplitudes=data["amplitudes"], d=data["d"],
            q=data["q"], roots=160, q_scale=float(data["q_scale"]))
    x = synthetic.si64()
    try:
        np.savez(cache, lattice=x.lattice, reciprocal=x.reciprocal, volume=x.volume, positions=x.positions,
                 species=x.species, kpoint=x.kpoint, hkl=x.hkl, cartesian=x.cartesian, kinetic_ev=x.kinetic_ev,
                 v_hkl=x.v_hkl, v_values=x.v_values, projectors=x.projectors, amplitudes=x.amplitudes, d=x.d,
                 q=x.q, q_scale=x.q_scale)
    except OSError:
        pass
    return x


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.path = pathlib.Path(tempfile.mkstemp(prefix="sdft_clocks_", suffix=".csv")[1])
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        loaded = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit() and float(r[3] or 0) > 200.0] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def distributed():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reference_cpu_sample(inputs, iterations: int):
    """The reference's own Davidson (oracle/_ref) for `iterations` iterations on the host cores."""
    from oracle import ref_oracle
    lib = ref_oracle.ReferenceLibrary()
    op = ref_oracle.ReferenceOperator(lib, inputs)
    t0 = time.perf_counter()
    result = op.davidson(inputs.roots, iterations, TOLERANCE)
    seconds = time.perf_counter() - t0
    return seconds, result


CALIBRATION = ROOT / "tests" / "golden" / "si64_reference_timing.json"
SAMPLE_ITERATIONS = 2


def reference_calibration():
    """Full-solve time over the time of its first SAMPLE_ITERATIONS
    iterations, both measured for the reference on one host by
    `bench.py --calibrate-reference` (the first iterations apply the
    operator to all 2*roots guard columns and so cost more than the average
    one; the ratio carries that shape to another host's sample)."""
    data = json.loads(CALIBRATION.read_text())
    return data


def calibrate_reference(args):
    """One full reference solve of the pencil and three SAMPLE_ITERATIONS
    samples on all host threads; writes the ratio to tests/golden."""
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    inputs = load_inputs()
    samples = [reference_cpu_sample(inputs, SAMPLE_ITERATIONS)[0] for _ in range(3)]
    full, result = reference_cpu_sample(inputs, 256)
    data = {"workload": WORKLOAD, "threads": threads, "full_solve_seconds": full,
            "full_solve_iterations": int(result["iterations"]), "converged": bool(result["converged"]),
            "sample_iterations": SAMPLE_ITERATIONS, "sample_seconds": samples,
            "ratio": full / statistics.median(samples), "host": os.uname().nodename,
            "how": "python bench.py --calibrate-reference (oracle/_ref, unmodified reference sources)"}
    text = json.dumps(data, indent=1)
    print(text, flush=True)
    if args.write_calibration:
        CALIBRATION.write_text(text + "\n")


def run_reference(args):
    world, rank, _ = distributed()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    inputs = load_inputs()
    calibration = reference_calibration()
    for _ in range(args.warmup):
        pass  # the reference has no device state to warm; its setup is outside the timed region
    times = []
    for _ in range(args.steps):
        seconds, _ = reference_cpu_sample(inputs, SAMPLE_ITERATIONS)
        times.append(seconds)
    solve = statistics.median(times) * calibration["ratio"]
    value = inputs.roots / solve
    sample = (f"reference Davidson (oracle/_ref, unmodified src/ + FFTW-API shim): its first {SAMPLE_ITERATIONS} "
              f"iterations per step, scaled to its full {calibration['full_solve_iterations']}-iteration solve by "
              f"the measured full/sample time ratio {calibration['ratio']:.2f} "
              f"({calibration['full_solve_seconds']:.0f} s full solve on {calibration['threads']} threads)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.median(times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": config(args, {"parallelism": "cpu", "threads": threads}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "extrapolated_solve_ms": solve * 1e3}), flush=True)


def run_b200(args):
    import numpy as np
    import torch
    world, rank, local = distributed()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(local)
    from sdft_b200 import _capi as C
    from sdft_b200.operator import Context, PlaneWaveOperator

    inputs = load_inputs()
    stream = torch.cuda.Stream()  # library kernels and the CUDA events share this stream
    torch.cuda.set_stream(stream)
    ctx = Context(local, stream.cuda_stream)
    op = PlaneWaveOperator(ctx, inputs)
    roots = inputs.roots
    lib = C.library()

    def solve(precision):
        return op.davidson(roots, 256, TOLERANCE, precision=precision, vectors=False)

    def certified(result):
        return int(np.sum(result["residuals"] <= TOLERANCE))

    reference_values = reference_eigenvalues()

    def eigenvalue_error(result):
        return float(np.max(np.abs(result["eigenvalues"] - reference_values)))

    for _ in range(max(args.warmup, 0)):
        solve("mixed")
    torch.cuda.synchronize()
    barrier(world)
    launches0 = lib.sdft_b200_kernel_launches()
    step_ms, pairs, iters, stats, errors = [], 0, [], None, []
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        start_all = torch.cuda.Event(enable_timing=True)
        end_all = torch.cuda.Event(enable_timing=True)
        start_all.record(stream)
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            result = solve("mixed")
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            pairs += certified(result)
            iters.append(result["iterations"])
            errors.append(eigenvalue_error(result))
            stats = result["stats"]
        end_all.record(stream)
        torch.cuda.synchronize()
    launches = lib.sdft_b200_kernel_launches() - launches0
    barrier(world)
    total_ms = max_over_ranks(start_all.elapsed_time(end_all), world)
    value = pairs * world / (total_ms / 1e3)

    # FP64 plain form on the same GPU (after the timed region).
    fp64_ms, fp64_pairs, fp64_errors = [], 0, []
    for _ in range(max(1, min(args.steps, 2))):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r64 = solve("fp64")
        e1.record(stream)
        torch.cuda.synchronize()
        fp64_ms.append(e0.elapsed_time(e1))
        fp64_pairs += certified(r64)
        fp64_errors.append(eigenvalue_error(r64))
    fp64_value = fp64_pairs / (sum(fp64_ms) / 1e3)

    # Roofline of the fused local H~psi (FP32 slab FFT) on a 160-column block.
    roofline = fused_local_roofline(op, inputs, stream)
    apply_errors = operator_apply_errors(op, stream)

    # End to end through the public API with host buffers: operator upload from
    # host arrays, solve, eigenvectors read back, every step.
    e2e = end_to_end(ctx, inputs, stream, steps=max(1, min(args.steps, 3)))

    density_rows = None
    if rank == 0 and world == 1 and not args.no_density:
        density_rows = density_side(ctx, inputs, stream, roofline["peak"])

    serving_rows = None
    if rank == 0 and world == 1 and not args.no_serving:
        serving_rows = serving_stream(local, requests=args.serving_requests,
                                      forms=("mixed",) if args.serving_mixed_only else ("mixed", "fp64"),
                                      log=args.serving_log)

    kpoint_rows = None
    if rank == 0 and world == 1 and not args.no_kpoints:
        kpoint_rows = kpoint_batch(local, range(27) if args.all_kpoints else KPOINT_SAMPLE)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(inputs)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 (mixed search, FP64 certificate)",
            "data": "synthetic (seeded)",
            "config": config(args, {"parallelism": f"replicas{world}", "precision": "mixed"}),
            "p50_solve_ms": statistics.median(step_ms), "p99_solve_ms": float(np.percentile(step_ms, 99)),
            "iterations": iters, "certified_pairs_per_solve": pairs / args.steps,
            "max_eigenvalue_error_vs_reference": max(errors),
            "eigenvalue_error_per_solve": errors,
            "max_apply_error_fp64": max(apply_errors["fp64"].values()),
            "max_apply_error_mixed": max(apply_errors["mixed"].values()),
            "apply_errors": apply_errors,
            "fp64_plain": {"value": fp64_value, "unit": UNIT, "p50_solve_ms": statistics.median(fp64_ms),
                           "certified_pairs_per_solve": fp64_pairs / len(fp64_ms),
                           "max_eigenvalue_error_vs_reference": max(fp64_errors)},
            "mixed_over_fp64": statistics.median(fp64_ms) / statistics.median(step_ms),
            "solver_stats": stats, "clocks": clocks.summary(), "gpu_launches": int(launches),
            "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "density_side": density_rows,
            "serving": serving_rows, "kpoint_batch": kpoint_rows,
        }
        print(json.dumps(line), flush=True)
    op.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def reference_eigenvalues():
    """The reference's own 160 eigenvalues of this pencil (its FP64 solve)."""
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "si64_solution.npz")["eigenvalues"]


def operator_apply_errors(op, stream):
    """Relative error of H~x and S~x against the reference's on a seeded
    160-column block (one call each, device pointers): the two columns the
    reference fixture holds in full, and every column through its norm and
    its inner product with a seeded probe vector. Per precision and operator."""
    import numpy as np
    import torch
    g = np.load(ROOT / "tests" / "golden" / "si64_apply.npz")

    def probe(columns, seed):
        rng = np.random.Generator(np.random.PCG64(seed))
        return rng.standard_normal((op.npw, columns)) + 1j * rng.standard_normal((op.npw, columns))

    x = probe(160, int(g["probe_seed"]))
    u = probe(1, int(g["checksum_seed"]))[:, 0]
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T
    out = {}
    for precision in ("fp64", "mixed"):
        out[precision] = {}
        for overlap, key in ((False, "hx"), (True, "sx")):
            y = op.apply(xd, overlap=overlap, precision=precision)
            torch.cuda.synchronize()
            y = y.T.cpu().numpy().T
            full = np.linalg.norm(y[:, g["columns"]] - g[key]) / np.linalg.norm(g[key])
            norms = np.max(np.abs(np.linalg.norm(y, axis=0) - g[f"{key}_norms"]) / g[f"{key}_norms"])
            dots = np.max(np.abs(u.conj() @ y - g[f"{key}_dots"]) / (np.linalg.norm(u) * g[f"{key}_norms"]))
            out[precision]["H" if key == "hx" else "S"] = float(max(full, norms, dots))
    return out


def fused_local_roofline(op, inputs, stream):
    import torch
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    cols = inputs.roots
    x = torch.randn(cols, op.npw, dtype=torch.complex128, device="cuda").T
    y = torch.empty((cols, op.npw), dtype=torch.complex128, device="cuda").T
    for _ in range(3):
        op.local_apply(x, y, precision="mixed")
    torch.cuda.synchronize()
    reps = 20
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        op.local_apply(x, y, precision="mixed")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    n0, n1, n2 = op.shape
    grid = n0 * n1 * n2
    # Algorithmic bytes per column: read psi and write H~psi (FP64 complex,
    # 16 B) plus one full-grid FP32 write+read for each of the two transform
    # halves; V(r) (FP32) once per launch. The pruned slab moves fewer grid
    # bytes than this (active i0 rows only).
    per_column = 2 * 16 * op.npw + 2 * (2 * 8 * grid)
    algorithmic = per_column * cols + 4 * grid
    achieved = algorithmic / (ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of plane_in + pencil + plane_out for one
    # 160-column launch, from one ncu capture of `bench.py --case local
    # --columns 160` (profiles/fused_local_h_si64_160cols.md).
    traffic = 956_765_952 if cols == 160 and (n0, n1, n2) == (70, 70, 70) else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": "fused local H~psi (plane_in + pencil + plane_out), FP32, 160 columns",
            "ms_per_launch": ms, "algorithmic_bytes": algorithmic,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}


def density_side(ctx, inputs, stream, peak):
    """Config-3 density-side rows on the Si64 cell, device-resident inputs, one
    timed call each after a warm-up call (CUDA events on the library's stream):
    band density of 128 occupied bands (f_n = 2) on the supports f = 4, 8, 16;
    the compensation charge of 64 atoms on the f = 16 support from the one-centre
    occupations of 128 bands; PBE on every point of the f = 16 density grid;
    the Hartree + PBE functionals (spin-unpolarised and collinear) of the
    f = 4 densities, wall clock. GB/s use the scope table's algorithmic bytes."""
    import numpy as np
    import torch
    from sdft_b200 import density, synthetic
    from sdft_b200.density import fast_length

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    bands = 128
    psi = torch.from_numpy(synthetic.band_coefficients(inputs, bands)).cuda()
    occ = np.full(bands, 2.0)
    out = {"bands": bands, "band_density": {}}
    grid16 = None
    densities = {}
    for factor in (4.0, 8.0, 16.0):
        support = synthetic.density_support(inputs, factor)
        ms, values = timed(lambda: density.band_density(ctx, inputs.hkl, psi, occ, inputs.volume, support))
        densities[factor] = (support, values.cpu().numpy())
        span = [int(2 * max(np.abs(support[:, a]).max(), inputs.hkl[:, a].max() - min(inputs.hkl[:, a].min(), 0)) + 1)
                for a in range(3)]
        n = [fast_length(max(3, v)) for v in span]
        points = n[0] * n[1] * n[2]
        grid16 = n
        algorithmic = bands * (16 * inputs.npw + 2 * 2 * 16 * points) + 2 * 8 * points
        gbs = algorithmic / (ms * 1e-3) / 1e9
        out["band_density"][f"f{int(factor)}"] = {"grid": n, "support": int(support.shape[0]), "ms": ms,
                                                  "achieved_gbs": gbs, "frac_of_hbm": gbs / peak}
    # Error of the f = 4 and f = 8 densities against the f = 16 one on their
    # keys (all of which the f = 16 support holds), relative to max |n_16(G)|.
    support16, values16 = densities[16.0]
    where16 = {tuple(key): i for i, key in enumerate(support16.tolist())}
    scale16 = float(np.max(np.abs(values16)))
    for factor in (4.0, 8.0):
        support, values = densities[factor]
        index = np.array([where16[tuple(key)] for key in support.tolist()])
        out["band_density"][f"f{int(factor)}"]["max_error_vs_f16"] = float(
            np.max(np.abs(values - values16[index])) / scale16)
    # Compensation charge on the f = 16 support.
    aug = synthetic.augmentation()
    rows = int(np.sum(2 * aug["channel_l"] + 1))
    atoms = inputs.positions.shape[0]
    amplitudes = synthetic.projected_amplitudes(atoms, rows, bands)
    onsite = density.onsite_density(ctx, amplitudes, rows, occ)
    keys = synthetic.density_support(inputs, 16.0)
    charge = density.CompensationCharge(ctx, inputs.lattice, inputs.positions, keys, aug, synthetic.lm_transform(aug))
    rho = torch.from_numpy(onsite).cuda()
    ms, _ = timed(lambda: charge.density(rho))
    lms = (int(aug["max_l"]) + 1) ** 2
    algorithmic = keys.shape[0] * (16 + 8 * lms)
    out["compensation"] = {"keys": int(keys.shape[0]), "atoms": atoms, "ms": ms,
                           "achieved_gbs": algorithmic / (ms * 1e-3) / 1e9,
                           "atom_terms_per_s": keys.shape[0] * atoms / (ms * 1e-3)}
    charge.close()
    # PBE on every point of the f = 16 density grid.
    points = grid16[0] * grid16[1] * grid16[2]
    nval = torch.exp(torch.linspace(-20.0, 1.0, points, dtype=torch.float64, device="cuda"))
    gval = 0.3 * nval
    ms, _ = timed(lambda: density.pbe_points(ctx, nval, gval))
    out["pbe"] = {"points": points, "ms": ms, "points_per_s": points / (ms * 1e-3),
                  "achieved_gbs": points * 64 / (ms * 1e-3) / 1e9}
    # Hartree + PBE functional, spin-unpolarised and collinear, of the Si64
    # f = 4 Gaussian densities with a frozen core (142^3 grid, prime-71 axes):
    # wall time of the host call, the host key sort and union included.
    case = synthetic.functional_case("si64")
    args = (case["lattice"], case["keys"], case["values"], case["core_keys"], case["core_values"])
    spin = synthetic.collinear_case("si64")
    spin_args = (spin["lattice"], spin["up_keys"], spin["up"], spin["down_keys"], spin["down"], spin["core_keys"],
                 spin["core_values"])
    density.density_functionals(ctx, *args)
    density.collinear_functionals(ctx, *spin_args)
    start = time.perf_counter()
    result = density.density_functionals(ctx, *args)
    middle = time.perf_counter()
    density.collinear_functionals(ctx, *spin_args)
    end = time.perf_counter()
    out["functional"] = {"grid": list(result["grid"]), "keys": int(result["hkl"].shape[0]),
                         "ms": (middle - start) * 1e3, "collinear_ms": (end - middle) * 1e3,
                         "timing": "wall clock of the host call (host key sort and union included)"}
    return out


def _serving_request(index, seed):
    """One request of the seeded serving stream (run in a spawned host process)."""
    from sdft_b200 import synthetic
    return synthetic.serving_request(index, seed=seed)


def serving_stream(device, requests=8, slots=4, rate_hz=1.0, cap=150e9, seed=4242, forms=("mixed", "fp64"),
                   generators=8, log=None):
    """A sample of the seeded serving stream through the solve server: the
    first `requests` requests of the config-4 stream (cubic cells of 2-128
    atoms drawn log-uniformly, Ecut U(10, 25) Ha, bands 1.25x occupied within
    [8, 320], 1-8 k-points, one solve per k-point), Poisson arrivals at
    rate_hz, admitted by device footprint under `cap` with `slots` concurrent
    solves; the same stream in each form. `generators` spawned host processes
    build the requests ahead of their arrival (the clock starts once the
    first 2 x `generators` are built); a request submitted after its
    arrival time because its inputs were not ready yet counts as
    generation-paced (its latency is measured from its submission).
    Latency = finish of a request's last k-point - submission of its first.
    log: a path that receives one JSON line per request as its last k-point
    finishes (a long sample leaves its partial results there)."""
    import concurrent.futures
    import multiprocessing
    import numpy as np
    from sdft_b200.serving import SolveServer

    arrivals = np.cumsum(np.random.Generator(np.random.PCG64(seed)).exponential(1.0 / rate_hz, size=requests))
    context = multiprocessing.get_context("spawn")

    def run(precision):
        with concurrent.futures.ProcessPoolExecutor(max_workers=generators, mp_context=context) as pool, \
                SolveServer(device, cap, slots) as server:
            pending = [pool.submit(_serving_request, i, seed) for i in range(min(requests, 2 * generators))]
            concurrent.futures.wait([f for f in pending])  # the clock starts with the look-ahead window built
            tickets, paced, atoms, kpoints = [], 0, [], []
            t0 = None
            for i in range(requests):
                ops = pending[i].result()
                pending[i] = None
                if len(pending) < requests:
                    pending.append(pool.submit(_serving_request, len(pending), seed))
                if t0 is None:
                    t0 = time.perf_counter() - arrivals[0]
                delay = arrivals[i] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                else:
                    paced += 1
                atoms.append(int(ops[0].positions.shape[0]))
                kpoints.append(len(ops))
                tickets.append([server.submit(x, precision=precision) for x in ops])
                del ops
            results = []
            for i, group in enumerate(tickets):
                results.append([server.wait(t) for t in group])
                if log:
                    with open(log, "a") as f:
                        done = results[-1]
                        f.write(json.dumps({"form": precision, "request": i, "atoms": atoms[i],
                                            "kpoints": kpoints[i],
                                            "latency_ms": 1e3 * (max(r["timing"]["finished"] for r in done) -
                                                                 min(r["timing"]["submitted"] for r in done)),
                                            "certified": int(sum(np.sum(r["residuals"] <= TOLERANCE) for r in done)),
                                            "converged": all(r["converged"] for r in done)}) + "\n")
            makespan = time.perf_counter() - t0 - arrivals[0]
            memory = server.memory()
        latency = [1e3 * (max(r["timing"]["finished"] for r in group) - min(r["timing"]["submitted"] for r in group))
                   for group in results]
        flat = [r for group in results for r in group]
        pairs = sum(int(np.sum(r["residuals"] <= TOLERANCE)) for r in flat)
        spans = sorted((r["timing"]["started"], r["timing"]["finished"]) for r in flat)
        events = sorted([(a, 1) for a, _ in spans] + [(b, -1) for _, b in spans])
        depth = peak_depth = 0
        for _, step in events:
            depth += step
            peak_depth = max(peak_depth, depth)
        return {"p50_ms": float(np.percentile(latency, 50)), "p99_ms": float(np.percentile(latency, 99)),
                "certified_pairs_per_s": pairs / makespan, "certified_pairs": pairs,
                "solves": len(flat), "all_converged": all(r["converged"] for r in flat),
                "makespan_s": makespan, "peak_concurrent_solves": peak_depth,
                "peak_budget_gb": memory["peak"] / 1e9, "generation_paced_requests": paced,
                "atoms_range": [min(atoms), max(atoms)], "kpoints_total": int(sum(kpoints))}

    out = {"requests": requests, "slots": slots, "arrival_rate_hz": rate_hz, "memory_cap_gb": cap / 1e9,
           "sample": f"the first {requests} requests of the seeded config-4 stream: 2-128 atoms (log-uniform), "
                     "Ecut U(10, 25) Ha, 1-8 k-points, bands 1.25x occupied in [8, 320]"}
    for form in forms:
        out["mixed" if form == "mixed" else "fp64_plain"] = run(form)
    return out


KPOINT_SAMPLE = (26, 5, 13, 0)


def kpoint_batch(device, indices, slots=4, cap=150e9):
    """The k-point batch workload: the GaAs-shaped 2x2x2 zincblende cell
    (a = 21.36 bohr, 64 atoms, Ecut 18 Ha, 192 bands) at k-points of the 3x3x3
    Monkhorst-Pack mesh (uneven plane-wave counts), each a mixed-form solve,
    all submitted at once to the solve server (admission by device footprint,
    `slots` concurrent solves). The host builds every operator's inputs before
    the first submission; the makespan runs from the first submission to the
    last result. Eigenvalue errors against the reference where a fixture of
    that k-point exists."""
    import numpy as np
    from sdft_b200 import _capi as C
    from sdft_b200 import synthetic
    from sdft_b200.serving import SolveServer

    inputs = [synthetic.gaas_kpoint(k) for k in indices]
    with SolveServer(device, cap, slots) as server:
        t0 = time.perf_counter()
        tickets = [server.submit(x, precision="mixed") for x in inputs]
        results = [server.wait(t) for t in tickets]
        makespan = time.perf_counter() - t0
        memory = server.memory()
    rows, pairs, latency = [], 0, []
    for k, x, r in zip(indices, inputs, results):
        row = {"k": int(k), "kpoint": [float(v) for v in x.kpoint], "npw": int(x.npw), "iterations": r["iterations"],
               "converged": r["converged"], "certified": int(np.sum(r["residuals"] <= TOLERANCE)),
               "solve_ms": 1e3 * (r["timing"]["finished"] - r["timing"]["started"])}
        fixture = ROOT / "tests" / "golden" / f"gaas64_k{k}.npz"
        if fixture.exists():
            row["eigenvalue_error_vs_reference"] = float(np.max(np.abs(r["eigenvalues"] -
                                                                       np.load(fixture)["eigenvalues"])))
        rows.append(row)
        pairs += row["certified"]
        latency.append(row["solve_ms"])
    return {"cell": "GaAs zincblende 2x2x2, a=21.36 bohr, 64 atoms, Ecut 18 Ha, 192 bands",
            "kpoints": len(indices), "slots": slots, "precision": "mixed", "makespan_s": makespan,
            "certified_pairs_per_s": pairs / makespan, "certified_pairs": pairs,
            "p50_solve_ms": float(np.percentile(latency, 50)), "p99_solve_ms": float(np.percentile(latency, 99)),
            "peak_budget_gb": memory["peak"] / 1e9, "per_kpoint": rows,
            "gemm_autotuned_classes": len(C.gemm_tuned_classes())}


def pinned_inputs(inputs):
    """A copy of the operator inputs whose arrays live in pinned host memory."""
    import dataclasses
    import torch

    def pin(array):
        t = torch.from_numpy(array.copy())
        return t.pin_memory().numpy()

    fields = {f: pin(getattr(inputs, f)) for f in ("hkl", "kinetic_ev", "v_hkl", "v_values", "projectors",
                                                    "amplitudes", "d", "q")}
    return dataclasses.replace(inputs, **fields)


def end_to_end(ctx, inputs, stream, steps):
    import numpy as np
    import torch
    from sdft_b200.operator import PlaneWaveOperator
    h2d = (inputs.amplitudes.nbytes + inputs.v_values.nbytes + inputs.v_hkl.nbytes + inputs.hkl.nbytes +
           inputs.kinetic_ev.nbytes + inputs.d.nbytes + inputs.q.nbytes)
    d2h = inputs.roots * inputs.npw * 16 + 2 * inputs.roots * 8
    inputs = pinned_inputs(inputs)
    pairs, seconds = 0, 0.0
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        op = PlaneWaveOperator(ctx, inputs)
        result = op.davidson(inputs.roots, 256, TOLERANCE, precision="mixed", vectors=True)
        torch.cuda.synchronize()
        seconds += time.perf_counter() - t0
        pairs += int(np.sum(result["residuals"] <= TOLERANCE))
        op.close()
    return {"value": pairs / seconds, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "path": "sdft_b200_operator_create (pinned host arrays) + sdft_b200_davidson (host eigenvectors)"}


def cpu_baseline(inputs):
    from oracle import ref_oracle
    if not ref_oracle.available():
        return None
    threads = os.cpu_count() or 1
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    calibration = reference_calibration()
    seconds, _ = reference_cpu_sample(inputs, SAMPLE_ITERATIONS)
    solve = seconds * calibration["ratio"]
    return {"value": inputs.roots / solve, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"reference Davidson, its first {SAMPLE_ITERATIONS} iterations on the host cores "
                      f"({seconds:.1f} s), scaled to its full {calibration['full_solve_iterations']}-iteration solve "
                      f"by the measured full/sample ratio {calibration['ratio']:.2f}"}


def run_case(args):
    """A few launches of one kernel family on the bench workload, for profiling
    captures (no JSON): local, pair, project, density, pbe, compensation;
    local, pair, project and compensation print each call's CUDA-event time."""
    import numpy as np
    import torch
    from sdft_b200 import density, synthetic
    from sdft_b200.operator import Context, PlaneWaveOperator
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = Context(0, stream.cuda_stream)
    inputs = load_inputs()
    cols = args.columns
    if args.case in ("local", "pair", "project"):
        op = PlaneWaveOperator(ctx, inputs)
        x = torch.randn(cols, op.npw, dtype=torch.complex128, device="cuda").T
        for _ in range(args.repeat):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if args.case == "local":
                op.local_apply(x, precision=args.precision)
            elif args.case == "pair":
                op.apply_pair(x, precision=args.precision)
            else:
                op.project(x, precision=args.precision)
            e1.record(stream)
            torch.cuda.synchronize()
            print(f"{args.case} {args.precision} {cols} columns: {e0.elapsed_time(e1):.3f} ms")
        op.close()
    elif args.case == "density":
        support = synthetic.density_support(inputs, args.factor)
        psi = torch.from_numpy(synthetic.band_coefficients(inputs, cols)).cuda()
        for _ in range(args.repeat):
            density.band_density(ctx, inputs.hkl, psi, np.full(cols, 2.0), inputs.volume, support)
        torch.cuda.synchronize()
    elif args.case == "pbe":
        n = np.exp(np.linspace(-20, 1, cols * 65536))
        for _ in range(args.repeat):
            density.pbe_points(ctx, n, 0.3 * n)
    elif args.case == "compensation":
        aug = synthetic.augmentation()
        rows = int(np.sum(2 * aug["channel_l"] + 1))
        atoms = inputs.positions.shape[0]
        onsite = density.onsite_density(ctx, synthetic.projected_amplitudes(atoms, rows, cols), rows,
                                        np.full(cols, 2.0))
        keys = synthetic.density_support(inputs, args.factor)
        charge = density.CompensationCharge(ctx, inputs.lattice, inputs.positions, keys, aug,
                                            synthetic.lm_transform(aug))
        rho = torch.from_numpy(onsite).cuda()
        for _ in range(args.repeat):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            charge.density(rho)
            e1.record(stream)
            torch.cuda.synchronize()
            print(f"compensation keys {keys.shape[0]} atoms {atoms}: {e0.elapsed_time(e1):.3f} ms")
        charge.close()
    ctx.close()
    print("case", args.case, "done")


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["b200", "reference"], default="b200")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU reference sample")
    parser.add_argument("--no-density", action="store_true", help="skip the density-side measurements")
    parser.add_argument("--no-serving", action="store_true", help="skip the serving-stream sample")
    parser.add_argument("--no-kpoints", action="store_true", help="skip the GaAs64 k-point batch")
    parser.add_argument("--serving-requests", type=int, default=8,
                        help="requests of the serving-stream sample (the stream has 2000)")
    parser.add_argument("--serving-mixed-only", action="store_true",
                        help="run the serving sample in the mixed form only")
    parser.add_argument("--serving-log", help="file that receives one JSON line per finished serving request")
    parser.add_argument("--all-kpoints", action="store_true", help="all 27 k-points of the GaAs64 batch (default: 4)")
    parser.add_argument("--case", choices=["local", "pair", "project", "density", "pbe", "compensation"],
                        help="run a few launches of one kernel family for a profiler capture and exit")
    parser.add_argument("--columns", type=int, default=32, help="columns (bands) for --case")
    parser.add_argument("--repeat", type=int, default=2, help="repetitions for --case")
    parser.add_argument("--precision", choices=["fp64", "mixed"], default="mixed", help="precision for --case")
    parser.add_argument("--factor", type=float, default=16.0, help="density support factor f for --case density")
    parser.add_argument("--calibrate-reference", action="store_true",
                        help="time one full reference solve and its first-iterations sample on the host cores")
    parser.add_argument("--write-calibration", action="store_true",
                        help="with --calibrate-reference: write tests/golden/si64_reference_timing.json")
    args = parser.parse_args()
    if args.calibrate_reference:
        calibrate_reference(args)
    elif args.case:
        run_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
