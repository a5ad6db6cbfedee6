"""Generates tests/golden/*.npz from the reference's own CPU implementation.

Run in a container that has the reference built into oracle/_ref:

    make -C oracle/ref && python tests/golden/make_golden.py [--si64]

Inputs are the seeded synthetic pencils of sdft_b200.synthetic (regenerated
from their seeds by the tests, so only reference OUTPUTS are stored). Values
come from the unmodified reference: the PWO3 solver snapshot it writes
(src/plane_wave_operator.cpp:542-569) for its internal arrays, its
apply_block_into / apply_pair_into callbacks for H~x, S~x, and
solve_generalized_hermitian_davidson for eigenpairs; the density side from
plane_wave_density_fft, pbe_unpolarized, onsite_density_from_amplitudes, the
PawCompensationOperator (density and project_potential_batch) and
evaluate_density_functionals / evaluate_collinear_density_functionals
(functional_*.npz, collinear_*.npz, on synthetic.functional_case /
collinear_case). Single groups: --kpoints, --snapshots, --projection,
--functional, --collinear, --si64-apply (si64_apply.npz: the
headline pencil's operator arrays and a 160-column H~x/S~x probe), --polish
(strict_polish.npz: solves at tolerance 1e-13 that end in the reference's
strict polish), --gaas64 [k ...] (gaas64_k*.npz: the 64-atom GaAs cell at
Ecut 18 Ha, 192 bands, two k-points of the 3x3x3 mesh; long).
"""
from __future__ import annotations

import argparse
import pathlib
import struct
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sparse-dft_b200"))

from sdft_b200 import synthetic  # noqa: E402
from oracle import ref_oracle  # noqa: E402

HERE = pathlib.Path(__file__).resolve().parent


def read_pwo3(path):
    """Parse a PWO3 snapshot (little-endian; layout of src/plane_wave_operator.cpp:553-567)."""
    raw = pathlib.Path(path).read_bytes()
    if raw[:8] != b"SDFTPWO3":
        raise ValueError("not a PWO3 snapshot")
    n, count, s0, s1, s2, nproj, roots, iters, ninit = struct.unpack_from("<9Q", raw, 8)
    reg, tol = struct.unpack_from("<2d", raw, 80)
    off = 96
    (atoms,) = struct.unpack_from("<Q", raw, off)
    off += 8
    channels = np.frombuffer(raw, dtype="<u8", count=atoms, offset=off)
    off += 8 * atoms
    out = {"shape": (s0, s1, s2), "count": count, "regularization": reg, "tolerance": tol, "roots": roots,
           "iterations": iters, "channels": channels.copy()}
    out["indices"] = np.frombuffer(raw, dtype="<u8", count=n, offset=off).copy()
    off += 8 * n
    for name, length in (("kinetic", n), ("h_diagonal", n), ("s_diagonal", n), ("local_real", count)):
        out[name] = np.frombuffer(raw, dtype="<f8", count=length, offset=off).copy()
        off += 8 * length
    out["all_b"] = np.frombuffer(raw, dtype="<c16", count=nproj * n, offset=off).reshape((nproj, n), order="F").copy()
    off += 16 * nproj * n
    d, q = [], []
    for c in channels:
        c = int(c)
        d.append(np.frombuffer(raw, dtype="<c16", count=c * c, offset=off).reshape((c, c), order="F").copy())
        off += 16 * c * c
        q.append(np.frombuffer(raw, dtype="<c16", count=c * c, offset=off).reshape((c, c), order="F").copy())
        off += 16 * c * c
    out["d"], out["q"] = d, q
    out["initial"] = np.frombuffer(raw, dtype="<c16", count=ninit, offset=off).copy()
    return out


def probe_block(npw: int, columns: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.asfortranarray(rng.standard_normal((npw, columns)) + 1j * rng.standard_normal((npw, columns)))


def operator_fixture(lib, inputs, name, columns=4, seed=11, solve=True):
    op = ref_oracle.ReferenceOperator(lib, inputs)
    with tempfile.TemporaryDirectory() as tmp:
        path = pathlib.Path(tmp) / "op.pwop"
        op.save_snapshot(path, inputs.roots, inputs.max_iterations, inputs.tolerance)
        snap = read_pwo3(path)
    x = probe_block(inputs.npw, columns, seed)
    hx = op.apply(x, overlap=False, exact=True)
    sx = op.apply(x, overlap=True, exact=True)
    fields = dict(shape=np.array(snap["shape"]), indices=snap["indices"], kinetic=snap["kinetic"],
                  h_diagonal=snap["h_diagonal"], s_diagonal=snap["s_diagonal"], local_real=snap["local_real"],
                  hkl=inputs.hkl, kinetic_ev=inputs.kinetic_ev, probe_seed=np.array(seed), hx=hx, sx=sx)
    if solve:
        t = time.time()
        result = op.davidson(inputs.roots, inputs.max_iterations, inputs.tolerance)
        fields.update(eigenvalues=result["eigenvalues"], residuals=result["residuals"],
                      converged=np.array(result["converged"]), iterations=np.array(result["iterations"]),
                      seconds=np.array(time.time() - t))
    np.savez_compressed(HERE / f"{name}.npz", **fields)
    print(name, "npw", inputs.npw, "grid", snap["shape"], {k: v for k, v in fields.items() if k in ("iterations",)})


def pbe_sampling(count: int = 131072):
    """The density/gradient sweep of the reference's tests/native/pbe_backend_smoke.cpp:15-16."""
    i = np.arange(count, dtype=np.float64)
    n = np.exp(-23.025850929940457 + 27.630 * np.mod(i, 10007) / 10006.0)
    g = np.where(np.mod(i, 7) == 0, 10.0 ** (-9.0 + 11.0 * np.mod(i, 31) / 30.0), n * np.mod(i, 101) / 3.0)
    return n, g


def pbe_fixture(lib, stride: int = 16):
    """Reference PBE points (src/pbe_xc.cpp:119) on every stride-th point of the sweep."""
    n, g = pbe_sampling()
    n, g = n[::stride].copy(), g[::stride].copy()
    np.savez_compressed(HERE / "pbe.npz", density=n, gradient=g, points=lib.pbe(n, g))
    print("pbe", n.size, "points")


def density_occupations(bands: int) -> np.ndarray:
    """Mostly f = 2, one fractional and one empty band (the empty one is skipped)."""
    occ = np.full(bands, 2.0)
    occ[3] = 1.25
    occ[bands // 2 - 1] = 0.0
    return occ


def density_fixture(lib, inputs, name, factor, bands):
    """Reference plane_wave_density_fft (src/density_functionals.cpp:407) on seeded bands."""
    support = synthetic.density_support(inputs, factor)
    coefficients = synthetic.band_coefficients(inputs, bands)
    occ = density_occupations(bands)
    density = lib.density(inputs.hkl, coefficients, occ, inputs.volume, support)
    np.savez_compressed(HERE / f"density_{name}.npz", support=support, occupations=occ, factor=np.array(factor),
                        bands=np.array(bands), density=density)
    print("density", name, "support", support.shape[0])


def compensation_fixture(lib, inputs, name, factor, bands):
    """Reference onsite_density_from_amplitudes (src/onsite_density.hpp:13), the (L,M)
    transform and PawCompensationOperator::density_sum (src/paw_compensation.cpp:465)."""
    aug = synthetic.augmentation()
    atoms = inputs.positions.shape[0]
    rows = int(np.sum(2 * aug["channel_l"] + 1))
    amplitudes = synthetic.projected_amplitudes(atoms, rows, bands)
    occ = density_occupations(bands)
    onsite = np.stack([lib.onsite_density(amplitudes[a * rows:(a + 1) * rows], occ) for a in range(atoms)])
    transform = lib.lm_transform(aug)
    keys = synthetic.density_support(inputs, factor)
    charge = lib.compensation_density(inputs.lattice, inputs.positions, keys, aug, onsite)
    np.savez_compressed(HERE / f"compensation_{name}.npz", occupations=occ, onsite=onsite, transform=transform,
                        factor=np.array(factor), bands=np.array(bands), charge=charge)
    print("compensation", name, "keys", keys.shape[0])


def compensation_project_fixture(lib, inputs, name, factor):
    """Reference project_potential_batch (src/paw_compensation.cpp:552) of a
    seeded potential given on the support minus a few modes plus keys
    outside it (those never enter)."""
    aug = synthetic.augmentation()
    keys = synthetic.density_support(inputs, factor)
    rng = np.random.Generator(np.random.PCG64(71))
    keep = rng.uniform(size=keys.shape[0]) > 0.02
    extra = keys[:5] * 0 + np.array([[40, 0, 0], [0, 41, 0], [0, 0, 42], [43, 1, 0], [-44, 0, 2]])
    pkeys = np.concatenate([keys[keep], extra]).astype(np.int32)
    potential = rng.standard_normal(pkeys.shape[0]) + 1j * rng.standard_normal(pkeys.shape[0])
    out = lib.compensation_project(inputs.lattice, inputs.positions, keys, aug, pkeys, potential)
    np.savez_compressed(HERE / f"compensation_project_{name}.npz", factor=np.array(factor), potential_keys=pkeys,
                        potential=potential, projection=out)
    print("compensation projection", name, "keys", keys.shape[0], "potential keys", pkeys.shape[0])


def snapshot_fixtures(lib):
    """Solver snapshots written by the reference (save_solver_snapshot) for
    the tiny pencil, cold and warm (the reference's eigenvectors with seeded
    1e-3 perturbations), and the reference's solves of each snapshot as
    loaded by its own load_solver_snapshot."""
    inputs = synthetic.tiny()
    op = ref_oracle.ReferenceOperator(lib, inputs)
    base = op.davidson(inputs.roots, inputs.max_iterations, inputs.tolerance)
    rng = np.random.Generator(np.random.PCG64(17))
    warm = base["eigenvectors"] + 1e-3 * (rng.standard_normal(base["eigenvectors"].shape) +
                                         1j * rng.standard_normal(base["eigenvectors"].shape))
    results = {}
    for name, initial in (("tiny_cold", None), ("tiny_warm", warm)):
        path = HERE / f"{name}.pwo3"
        if path.exists():
            path.unlink()
        op.save_snapshot(path, inputs.roots, inputs.max_iterations, inputs.tolerance, initial)
        loaded = ref_oracle.ReferenceOperator.from_snapshot(lib, path)
        r = loaded["operator"].davidson(loaded["roots"], loaded["iterations"], loaded["tolerance"],
                                        initial=loaded["initial"])
        results[f"{name}_eigenvalues"] = r["eigenvalues"]
        results[f"{name}_iterations"] = np.array(r["iterations"])
    np.savez_compressed(HERE / "snapshots.npz", **results)
    print("snapshots", {k: v for k, v in results.items() if "iterations" in k})


def functional_fixtures(lib):
    """Reference evaluate_density_functionals (src/density_functionals.cpp:696-729)
    of the seeded Gaussian densities of synthetic.functional_case, without and
    with the frozen core: support keys, potential, xc_potential and scalars."""
    for name in ("si8", "triclinic"):
        case = synthetic.functional_case(name)
        fields = {}
        for label, core in (("plain", False), ("core", True)):
            kw = {"core_keys": case["core_keys"], "core_values": case["core_values"]} if core else {}
            out = lib.density_functionals(case["lattice"], case["keys"], case["values"], **kw)
            for key, value in out.items():
                fields[f"{label}_{key}"] = np.asarray(value)
        np.savez_compressed(HERE / f"functional_{name}.npz", **fields)
        print("functional", name, "support", fields["core_hkl"].shape[0], "grid points", int(fields["plain_grid_points"]))


def collinear_fixtures(lib):
    """Reference evaluate_collinear_density_functionals (src/density_functionals.cpp:732-806)
    of synthetic.collinear_case, without and with the frozen core: support keys
    and per channel the potential, xc_potential and scalars."""
    for name in ("si8", "triclinic"):
        case = synthetic.collinear_case(name)
        fields = {}
        for label, core in (("plain", False), ("core", True)):
            kw = {"core_keys": case["core_keys"], "core": case["core_values"]} if core else {}
            out = lib.collinear_functionals(case["lattice"], case["up_keys"], case["up"], case["down_keys"],
                                            case["down"], **kw)
            fields[f"{label}_hkl"] = out["hkl"]
            for channel in ("up", "down"):
                for key, value in out[channel].items():
                    if key != "hkl":
                        fields[f"{label}_{channel}_{key}"] = np.asarray(value)
        np.savez_compressed(HERE / f"collinear_{name}.npz", **fields)
        print("collinear", name, "support", fields["core_hkl"].shape[0])


KPOINT_MESH = {"gaas_k13": (0.0, 1.0 / 3.0, 1.0 / 3.0), "gaas_k26": (1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0)}


SI64_APPLY_COLUMNS = 160
SI64_FULL_COLUMNS = (0, 159)
SI64_SAMPLE_POINTS = 4096


def si64_apply_fixture(lib):
    """The Si64 pencil at the headline size: the reference's H~x and S~x of a
    seeded 160-column probe (two columns in full, and for every column its
    norm and its inner product with a seeded probe vector u), the operator's
    index map, kinetic energies and diagonals in full, and V(r) at seeded grid
    points plus its sum and sum of squares."""
    inputs = synthetic.si64()
    op = ref_oracle.ReferenceOperator(lib, inputs)
    with tempfile.TemporaryDirectory() as tmp:
        path = pathlib.Path(tmp) / "op.pwop"
        op.save_snapshot(path, inputs.roots, inputs.max_iterations, inputs.tolerance)
        snap = read_pwo3(path)
    seed = 11
    x = probe_block(inputs.npw, SI64_APPLY_COLUMNS, seed)
    hx, sx = op.apply(x, overlap=False, exact=True), op.apply(x, overlap=True, exact=True)
    u = probe_block(inputs.npw, 1, 12)[:, 0]
    rng = np.random.Generator(np.random.PCG64(13))
    local = snap["local_real"]
    points = rng.choice(local.size, SI64_SAMPLE_POINTS, replace=False)
    cols = np.array(SI64_FULL_COLUMNS)
    np.savez_compressed(
        HERE / "si64_apply.npz", shape=np.array(snap["shape"]), indices=snap["indices"], kinetic=snap["kinetic"],
        h_diagonal=snap["h_diagonal"], s_diagonal=snap["s_diagonal"], local_points=points,
        local_values=local[points], local_sum=np.array(local.sum()), local_sum2=np.array(np.dot(local, local)),
        probe_seed=np.array(seed), checksum_seed=np.array(12), columns=cols, hx=hx[:, cols], sx=sx[:, cols],
        hx_dots=u.conj() @ hx, sx_dots=u.conj() @ sx, hx_norms=np.linalg.norm(hx, axis=0),
        sx_norms=np.linalg.norm(sx, axis=0))
    print("si64_apply npw", inputs.npw, "grid", snap["shape"])


POLISH_CASES = (("tiny", 1), ("tiny", 3), ("si8", 2026))
POLISH_TOLERANCE = 1e-13


def polish_case(name, seed):
    """One reference solve at POLISH_TOLERANCE with SDFT_TRACE_STRICT_POLISH=1
    (run in a child process so that its stderr trace can be counted)."""
    import json
    import os
    import subprocess
    code = (f"import sys, json; sys.path[:0] = [{str(ROOT)!r}, {str(ROOT / 'sparse-dft_b200')!r}]\n"
            "from oracle import ref_oracle\nfrom sdft_b200 import synthetic\nimport numpy as np\n"
            f"x = synthetic.{name}(seed={seed})\n"
            f"r = ref_oracle.ReferenceOperator(ref_oracle.ReferenceLibrary(), x).davidson(x.roots, 256, {POLISH_TOLERANCE})\n"
            "print(json.dumps({'eigenvalues': list(map(float, r['eigenvalues'])), 'iterations': r['iterations'],"
            " 'converged': r['converged'], 'max_residual': float(np.max(r['residuals']))}))\n")
    env = dict(os.environ, SDFT_TRACE_STRICT_POLISH="1")
    run = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    result = json.loads(run.stdout.strip().splitlines()[-1])
    result["polish_steps"] = sum(1 for line in run.stderr.splitlines() if line.startswith("strict_polish "))
    return result


def polish_fixtures():
    """The reference's solves at tolerance 1e-13, where its strict tangent
    polish (src/strict_residual_polish.hpp:118-197, driven from
    src/pw_core.cpp:1273-1336) takes the last steps: eigenvalues, iterations
    and the number of polish steps its trace reports."""
    fields = {"tolerance": np.array(POLISH_TOLERANCE)}
    for name, seed in POLISH_CASES:
        r = polish_case(name, seed)
        key = f"{name}_{seed}"
        fields[f"{key}_eigenvalues"] = np.array(r["eigenvalues"])
        fields[f"{key}_iterations"] = np.array(r["iterations"])
        fields[f"{key}_polish_steps"] = np.array(r["polish_steps"])
        print("polish", key, {k: r[k] for k in ("iterations", "converged", "max_residual", "polish_steps")})
    np.savez_compressed(HERE / "strict_polish.npz", **fields)


GAAS64_KPOINTS = (26, 5)


def gaas64_fixture(lib, index):
    """Config-2 cell (GaAs 2x2x2, a = 21.36 bohr, 64 atoms, Ecut 18 Ha, 192
    bands) at k-point `index` of the 3x3x3 mesh: the reference's Davidson
    eigenvalues at 1e-12, its index map and kinetic energies in full, and for
    a seeded 16-column probe the norms and probe-vector inner products of its
    H~x and S~x."""
    inputs = synthetic.gaas_kpoint(index)
    op = ref_oracle.ReferenceOperator(lib, inputs)
    with tempfile.TemporaryDirectory() as tmp:
        path = pathlib.Path(tmp) / "op.pwop"
        op.save_snapshot(path, inputs.roots, inputs.max_iterations, inputs.tolerance)
        snap = read_pwo3(path)
    x = probe_block(inputs.npw, 16, 11)
    u = probe_block(inputs.npw, 1, 12)[:, 0]
    hx, sx = op.apply(x, overlap=False, exact=True), op.apply(x, overlap=True, exact=True)
    t = time.time()
    result = op.davidson(inputs.roots, inputs.max_iterations, inputs.tolerance)
    np.savez_compressed(
        HERE / f"gaas64_k{index}.npz", kpoint=np.array(inputs.kpoint), shape=np.array(snap["shape"]),
        indices=snap["indices"].astype(np.uint32), kinetic=snap["kinetic"], probe_seed=np.array(11),
        checksum_seed=np.array(12), hx_norms=np.linalg.norm(hx, axis=0), sx_norms=np.linalg.norm(sx, axis=0),
        hx_dots=u.conj() @ hx, sx_dots=u.conj() @ sx, eigenvalues=result["eigenvalues"],
        residuals=result["residuals"], converged=np.array(result["converged"]),
        iterations=np.array(result["iterations"]), seconds=np.array(time.time() - t))
    print(f"gaas64_k{index} npw", inputs.npw, "grid", snap["shape"], "iterations", result["iterations"],
          "converged", result["converged"], "seconds", round(time.time() - t, 1))


def kpoint_fixtures(lib):
    """Reference operator and solve of the 8-atom GaAs cell at two k-points of
    the 3x3x3 Monkhorst-Pack mesh (complex, off-Gamma pencils, two species)."""
    for name, kpoint in KPOINT_MESH.items():
        operator_fixture(lib, synthetic.gaas_small(kpoint), name)


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--si64", action="store_true", help="also solve the Si64 pencil (long)")
    parser.add_argument("--kpoints", action="store_true", help="only the off-Gamma GaAs fixtures")
    parser.add_argument("--snapshots", action="store_true", help="only the solver snapshot fixtures")
    parser.add_argument("--projection", action="store_true", help="only the compensation projection fixture")
    parser.add_argument("--functional", action="store_true", help="only the Hartree + XC functional fixtures")
    parser.add_argument("--collinear", action="store_true", help="only the collinear spin functional fixtures")
    parser.add_argument("--si64-apply", action="store_true", help="only the Si64 operator and 160-column apply fixture")
    parser.add_argument("--polish", action="store_true", help="only the strict-polish solves at tolerance 1e-13")
    parser.add_argument("--gaas64", type=int, nargs="*", help="only the config-2 GaAs64 k-point solves (long)")
    args = parser.parse_args()
    lib = ref_oracle.ReferenceLibrary()
    if args.kpoints:
        kpoint_fixtures(lib)
        return
    if args.snapshots:
        snapshot_fixtures(lib)
        return
    if args.projection:
        compensation_project_fixture(lib, synthetic.si8(), "si8", 2.0)
        return
    if args.functional:
        functional_fixtures(lib)
        return
    if args.collinear:
        collinear_fixtures(lib)
        return
    if args.si64_apply:
        si64_apply_fixture(lib)
        return
    if args.polish:
        polish_fixtures()
        return
    if args.gaas64 is not None:
        for index in args.gaas64 or GAAS64_KPOINTS:
            gaas64_fixture(lib, index)
        return
    operator_fixture(lib, synthetic.tiny(), "tiny")
    operator_fixture(lib, synthetic.si8(), "si8", solve=True)
    pbe_fixture(lib)
    density_fixture(lib, synthetic.tiny(), "tiny", 4.0, 6)
    density_fixture(lib, synthetic.si8(), "si8", 2.0, 16)
    compensation_fixture(lib, synthetic.si8(), "si8", 2.0, 16)
    kpoint_fixtures(lib)
    snapshot_fixtures(lib)
    compensation_project_fixture(lib, synthetic.si8(), "si8", 2.0)
    functional_fixtures(lib)
    collinear_fixtures(lib)
    if args.si64:
        inputs = synthetic.si64()
        op = ref_oracle.ReferenceOperator(lib, inputs)
        t = time.time()
        result = op.davidson(inputs.roots, inputs.max_iterations, inputs.tolerance)
        np.savez_compressed(HERE / "si64_solution.npz", eigenvalues=result["eigenvalues"],
                            residuals=result["residuals"], converged=np.array(result["converged"]),
                            iterations=np.array(result["iterations"]), seconds=np.array(time.time() - t))


if __name__ == "__main__":
    main()
