"""Seeded synthetic operator inputs for the generalized Davidson hot path.

Every workload the benchmarks and tests use is built here from a fixed seed:
no dataset or pseudopotential file is read. The construction:

* cubic cell a*I (bohr); Si diamond sites (fcc + (1/4,1/4,1/4)), GaAs
  zincblende (Ga on fcc, As on the +(1/4,1/4,1/4) sites), replicated for
  supercells;
* plane-wave basis from ``enumerate_g_vectors`` (kinetic sort, then h,k,l),
  the same rule as the reference (src/pw_core.cpp:140-171);
* V_loc(G) = sum_a exp(-iG.tau_a) depth_a (2 pi w^2)^{3/2}/Omega exp(-|G|^2 w^2/2)
  (a real-space Gaussian well of depth ``depth_a`` Hartree and width w = 1 bohr
  per atom) plus seeded complex noise of standard deviation ``noise`` Hartree
  per Fourier component on 1/2|G|^2 <= noise_cut*Ecut, paired so that
  V(-G) = conj V(G) and V(0) is real;
* 8 projectors per atom: l=0 with sigma in {0.8, 1.2} and l=1 (3 real m) with
  sigma in {0.8, 1.2}; the Fourier transform of r^l exp(-r^2/(2 sigma^2)) Y_lm:
  B_p(G+k) = Omega^{-1/2} (-i)^l (2 pi)^{3/2} sigma^{2l+3} |G+k|^l
             exp(-|G+k|^2 sigma^2/2) Y_lm(G+k) exp(-i (G+k).tau);
  Y_lm are the real harmonics without Condon-Shortley phase used by the
  reference (src/paw_compensation.cpp:122-148);
* D_a: real symmetric 8x8, entries U(-0.5, 0.5) Hartree;
* Q_a: real symmetric 8x8, entries U(-0.5, 0.5), all atoms scaled by the
  largest s in (0, 1] with lambda_min(S) >= 0.3, S evaluated on the
  projector span exactly as the reference's overlap() signature check does
  (src/plane_wave_operator.cpp:702-717).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Sequence

import numpy as np

HARTREE_TO_EV = 27.211386245988
TWO_PI = 6.283185307179586476925286766559


@dataclasses.dataclass
class OperatorInputs:
    """Arrays that define one H~ / S~ pencil, in the reference's conventions."""

    name: str
    lattice: np.ndarray          # (3,3) rows are lattice vectors, bohr
    reciprocal: np.ndarray       # (3,3) rows are reciprocal vectors, 1/bohr
    volume: float
    positions: np.ndarray        # (atoms,3) fractional
    species: np.ndarray          # (atoms,) int
    kpoint: np.ndarray           # (3,) fractional
    ecut_ha: float
    hkl: np.ndarray              # (n,3) int32, basis order
    cartesian: np.ndarray        # (n,3) G (without k), 1/bohr
    kinetic_ev: np.ndarray       # (n,) 1/2|G+k|^2 in eV
    v_hkl: np.ndarray            # (nv,3) int32 potential keys
    v_values: np.ndarray         # (nv,) complex128 Hartree
    projectors: np.ndarray       # (atoms,) int64
    amplitudes: np.ndarray       # (sum np, n) complex128, row-major per atom
    d: np.ndarray                # (atoms, np, np) complex128
    q: np.ndarray                # (atoms, np, np) complex128
    roots: int
    tolerance: float = 1e-12
    max_iterations: int = 256
    regularization: float = 1e-12
    hartree_to_ev: float = HARTREE_TO_EV
    q_scale: float = 1.0

    @property
    def npw(self) -> int:
        return int(self.hkl.shape[0])

    @property
    def total_projectors(self) -> int:
        return int(self.projectors.sum())


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def enumerate_g_vectors(reciprocal: np.ndarray, cutoff_ev: float, kpoint: Sequence[float] = (0.0, 0.0, 0.0),
                        hartree_to_ev: float = HARTREE_TO_EV):
    """Plane-wave sphere 1/2|G+k|^2 <= cutoff, sorted by (kinetic, h, k, l).

    Same arithmetic, operation order and ordering as the reference's
    enumerate_g_vectors (src/pw_core.cpp:140-171), so the integer order is
    bit-identical. Returns (hkl int32 (n,3), cartesian (n,3), kinetic_ev (n,)).
    """
    b0, b1, b2 = (np.asarray(reciprocal[i], dtype=np.float64) for i in range(3))
    if not (cutoff_ev > 0 and math.isfinite(cutoff_ev)):
        raise ValueError("plane-wave cutoff must be finite and positive")
    gmax = math.sqrt(2.0 * cutoff_ev / hartree_to_ev)
    det = float(_dot(b0, _cross(b1, b2)))
    if abs(det) < 1e-12 or not math.isfinite(det):
        raise ValueError("reciprocal lattice is singular")
    d0 = _cross(b1, b2) * (1.0 / det)
    d1 = _cross(b2, b0) * (1.0 / det)
    d2 = _cross(b0, b1) * (1.0 / det)
    kx, ky, kz = (float(v) for v in kpoint)
    hmax = int(math.ceil(gmax * math.sqrt(float(_dot(d0, d0))) + abs(kx))) + 1
    kmax = int(math.ceil(gmax * math.sqrt(float(_dot(d1, d1))) + abs(ky))) + 1
    lmax = int(math.ceil(gmax * math.sqrt(float(_dot(d2, d2))) + abs(kz))) + 1
    shift = (b0 * kx + b1 * ky) + b2 * kz
    h, k, l = np.meshgrid(np.arange(-hmax, hmax + 1), np.arange(-kmax, kmax + 1), np.arange(-lmax, lmax + 1),
                          indexing="ij")
    h = h.ravel().astype(np.float64)
    k = k.ravel().astype(np.float64)
    l = l.ravel().astype(np.float64)
    # g = (b0*h + b1*k) + b2*l, component-wise, as add(add(scale,scale),scale)
    gx = (b0[0] * h + b1[0] * k) + b2[0] * l
    gy = (b0[1] * h + b1[1] * k) + b2[1] * l
    gz = (b0[2] * h + b1[2] * k) + b2[2] * l
    sx, sy, sz = gx + shift[0], gy + shift[1], gz + shift[2]
    g2 = (sx * sx + sy * sy) + sz * sz
    keep = 0.5 * g2 <= cutoff_ev / hartree_to_ev + 1e-12
    kinetic = (0.5 * g2[keep]) * hartree_to_ev
    hi, ki, li = h[keep].astype(np.int32), k[keep].astype(np.int32), l[keep].astype(np.int32)
    order = np.lexsort((li, ki, hi, kinetic))
    hkl = np.stack([hi[order], ki[order], li[order]], axis=1).astype(np.int32)
    cart = np.stack([gx[keep][order], gy[keep][order], gz[keep][order]], axis=1)
    return hkl, cart, kinetic[order]


def real_harmonic(l: int, m: int, q: np.ndarray) -> np.ndarray:
    """Real spherical harmonics Y_lm(q/|q|), no Condon-Shortley phase.

    Restates the associated-Legendre recurrence of the reference's
    paw_real_spherical_harmonic (src/paw_compensation.cpp:122-148), vectorised
    over rows of q. Y_00 = 1/sqrt(4 pi) at q = 0, higher l give 0 there.
    """
    q = np.asarray(q, dtype=np.float64)
    radius = np.sqrt(q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2])
    small = radius < 1e-14
    safe = np.where(small, 1.0, radius)
    z = np.clip(q[:, 2] / safe, -1.0, 1.0)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    order = abs(m)
    pmm = np.ones_like(z)
    for kk in range(1, order + 1):
        pmm = pmm * ((2.0 * kk - 1.0) * s)
    value = pmm
    if l > order:
        previous = pmm
        value = (2.0 * order + 1.0) * z * pmm
        for degree in range(order + 2, l + 1):
            nxt = ((2.0 * degree - 1.0) * z * value - (degree + order - 1.0) * previous) / (degree - order)
            previous, value = value, nxt
    factor = math.sqrt((2.0 * l + 1.0) / (4.0 * math.pi) *
                       math.exp(math.lgamma(l - order + 1.0) - math.lgamma(l + order + 1.0)))
    if order:
        factor *= math.sqrt(2.0)
    angle = order * np.arctan2(q[:, 1], q[:, 0])
    result = factor * value * (np.sin(angle) if m < 0 else np.cos(angle))
    return np.where(small, (1.0 / math.sqrt(4.0 * math.pi)) if l == 0 else 0.0, result)


DIAMOND_FCC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], dtype=np.float64)


def zincblende_sites(reps: int):
    """Fractional positions and species (0 = fcc site, 1 = +1/4 site) of a reps^3 supercell."""
    base = []
    for sub, offset in ((0, 0.0), (1, 0.25)):
        for site in DIAMOND_FCC:
            base.append((sub, site + offset))
    positions, species = [], []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                for sub, site in base:
                    positions.append((site + np.array([i, j, k], dtype=np.float64)) / reps)
                    species.append(sub)
    return np.array(positions), np.array(species, dtype=np.int64)


def _potential_keys(reciprocal: np.ndarray, cut_ha: float):
    """All integer G with 1/2|G|^2 <= cut_ha, lexicographic (h,k,l) order."""
    hkl, cart, _ = enumerate_g_vectors(reciprocal, cut_ha * HARTREE_TO_EV)
    order = np.lexsort((hkl[:, 2], hkl[:, 1], hkl[:, 0]))
    return hkl[order], cart[order]


def local_potential(lattice, reciprocal, positions, depths, ecut_ha, noise, noise_cut, width, rng):
    volume = abs(float(np.linalg.det(lattice)))
    hkl, cart = _potential_keys(reciprocal, noise_cut * ecut_ha)
    tau = positions @ lattice                      # cartesian atom positions
    g2 = np.einsum("ij,ij->i", cart, cart)
    shape = (2.0 * math.pi * width * width) ** 1.5 / volume * np.exp(-0.5 * g2 * width * width)
    phase = np.exp(-1j * (cart @ tau.T))           # (nv, atoms)
    values = shape * (phase @ np.asarray(depths, dtype=np.float64))
    # Hermitian noise: draw on the positive half, mirror to -G.
    positive = (hkl[:, 0] > 0) | ((hkl[:, 0] == 0) & ((hkl[:, 1] > 0) | ((hkl[:, 1] == 0) & (hkl[:, 2] > 0))))
    zero = (hkl[:, 0] == 0) & (hkl[:, 1] == 0) & (hkl[:, 2] == 0)
    draws = rng.standard_normal((hkl.shape[0], 2))
    noise_values = noise * (draws[:, 0] + 1j * draws[:, 1]) / math.sqrt(2.0)
    noise_values[zero] = noise * draws[zero, 0]
    values = values + np.where(positive | zero, noise_values, 0.0)
    negative = np.nonzero(~(positive | zero))[0]
    if np.array_equal(hkl[::-1], -hkl):
        # A key set closed under G -> -G in lexicographic order lists -G at the mirrored position.
        partner = hkl.shape[0] - 1 - negative
    else:
        index = {tuple(key): i for i, key in enumerate(hkl.tolist())}
        partner = np.array([index[(-hkl[i, 0], -hkl[i, 1], -hkl[i, 2])] for i in negative], dtype=np.int64)
    values[negative] = np.conj(values[partner])
    values[zero] = values[zero].real
    return hkl.astype(np.int32), values.astype(np.complex128)


def projector_amplitudes(cartesian, kcart, positions, lattice, volume):
    """(atoms*8, n) complex128 row-major: 2 s-type then 2 x 3 p-type per atom."""
    q = cartesian + kcart[None, :]
    qn = np.sqrt(np.einsum("ij,ij->i", q, q))
    tau = positions @ lattice
    rows = []
    channels = [(0, 0, 0.8), (0, 0, 1.2)] + [(1, m, s) for s in (0.8, 1.2) for m in (-1, 0, 1)]
    ylm = {(l, m): real_harmonic(l, m, q) for l, m, _ in channels}
    for a in range(tau.shape[0]):
        structure = np.exp(-1j * (q @ tau[a]))
        for l, m, sigma in channels:
            radial = (2.0 * math.pi) ** 1.5 * sigma ** (2 * l + 3) * qn ** l * np.exp(-0.5 * qn * qn * sigma * sigma)
            rows.append(((-1j) ** l) / math.sqrt(volume) * radial * ylm[(l, m)] * structure)
    return np.ascontiguousarray(np.array(rows, dtype=np.complex128))


def _block_diag(blocks: np.ndarray) -> np.ndarray:
    atoms, p, _ = blocks.shape
    out = np.zeros((atoms * p, atoms * p), dtype=blocks.dtype)
    for a in range(atoms):
        out[a * p:(a + 1) * p, a * p:(a + 1) * p] = blocks[a]
    return out


def _gram_root(amplitudes: np.ndarray) -> np.ndarray:
    """(B B^H)^(1/2) with the Gram eigenvalues clamped at 0."""
    gram = amplitudes @ amplitudes.conj().T
    w, v = np.linalg.eigh(0.5 * (gram + gram.conj().T))
    return (v * np.sqrt(np.maximum(w, 0.0))) @ v.conj().T


def _root_minimum(root: np.ndarray, q_blocks: np.ndarray, regularization: float) -> float:
    qfull = _block_diag(q_blocks)
    small = (1.0 + regularization) * np.eye(root.shape[0]) + root @ qfull @ root
    lam = np.linalg.eigvalsh(0.5 * (small + small.conj().T))
    return float(min(1.0 + regularization, lam.min()))


def overlap_minimum(amplitudes: np.ndarray, q_blocks: np.ndarray, regularization: float) -> float:
    """lambda_min of S~ on the projector span, as src/plane_wave_operator.cpp:702-717 evaluates it."""
    return _root_minimum(_gram_root(amplitudes), q_blocks, regularization)


def _scale_q_linear(amplitudes, q_raw, regularization, floor=0.3):
    """The scale of _scale_q in closed form: lambda_min((1+reg) I + s R Q R)
    is (1+reg) + s mu for the lowest eigenvalue mu of R Q R, so one
    eigenvalue solve gives the largest s <= 1 that keeps it at the floor."""
    root = _gram_root(amplitudes)
    rqr = root @ _block_diag(q_raw) @ root
    mu = float(np.linalg.eigvalsh(0.5 * (rqr + rqr.conj().T)).min())
    top = 1.0 + regularization
    return 1.0 if top + mu >= floor else (floor - top) / mu


def _scale_q(amplitudes, q_raw, regularization, floor=0.3):
    # The Gram root depends on B alone: formed once, not per bisection step
    # (each step's arithmetic is unchanged).
    root = _gram_root(amplitudes)
    if _root_minimum(root, q_raw, regularization) >= floor:
        return 1.0
    lo, hi = 0.0, 1.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if _root_minimum(root, mid * q_raw, regularization) >= floor:
            lo = mid
        else:
            hi = mid
    return lo


def build_operator(name: str, a: float, reps: int, ecut_ha: float, roots: int, depths=(-2.0, -2.0),
                   kpoint=(0.0, 0.0, 0.0), seed: int = 2026, noise: float = 0.05, noise_cut: float = 4.0,
                   width: float = 1.0, tolerance: float = 1e-12, max_iterations: int = 256,
                   regularization: float = 1e-12, sites=None, potential=None,
                   q_scaling: str = "bisection") -> OperatorInputs:
    """One synthetic H~/S~ pencil on an a*reps cubic zincblende/diamond supercell
    (or on the given (fractional positions, species) sites of an a*reps cube).
    potential: the (v_hkl, v_values) this call would draw (same cell, seed and
    noise arguments), reused instead of recomputed; q_scaling: "bisection"
    (the fixtures' inputs) or "linear" (_scale_q_linear, the same floor in
    one eigenvalue solve)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cell = a * reps
    lattice = np.eye(3) * cell
    reciprocal = np.eye(3) * (TWO_PI / cell)
    volume = cell ** 3
    positions, species = zincblende_sites(reps) if sites is None else (np.asarray(sites[0], dtype=np.float64),
                                                                        np.asarray(sites[1], dtype=np.int64))
    atom_depths = np.array([depths[s] for s in species], dtype=np.float64)
    hkl, cart, kinetic = enumerate_g_vectors(reciprocal, ecut_ha * HARTREE_TO_EV, kpoint)
    if potential is None:
        v_hkl, v_values = local_potential(lattice, reciprocal, positions, atom_depths, ecut_ha, noise, noise_cut,
                                          width, rng)
    else:
        v_hkl, v_values = potential
        rng.standard_normal((v_hkl.shape[0], 2))  # the noise draws local_potential takes, so d and Q repeat
    kcart = np.asarray(kpoint, dtype=np.float64) @ reciprocal
    amplitudes = projector_amplitudes(cart, kcart, positions, lattice, volume)
    atoms = positions.shape[0]
    d = rng.uniform(-0.5, 0.5, size=(atoms, 8, 8))
    d = 0.5 * (d + np.transpose(d, (0, 2, 1)))
    q_raw = rng.uniform(-0.5, 0.5, size=(atoms, 8, 8))
    q_raw = 0.5 * (q_raw + np.transpose(q_raw, (0, 2, 1)))
    scale = (_scale_q_linear if q_scaling == "linear" else _scale_q)(amplitudes, q_raw.astype(np.complex128),
                                                                     regularization)
    return OperatorInputs(name=name, lattice=lattice, reciprocal=reciprocal, volume=volume, positions=positions,
                          species=species, kpoint=np.asarray(kpoint, dtype=np.float64), ecut_ha=ecut_ha, hkl=hkl,
                          cartesian=cart, kinetic_ev=kinetic, v_hkl=v_hkl, v_values=v_values,
                          projectors=np.full(atoms, 8, dtype=np.int64), amplitudes=amplitudes,
                          d=d.astype(np.complex128), q=(scale * q_raw).astype(np.complex128), roots=roots,
                          tolerance=tolerance, max_iterations=max_iterations, regularization=regularization,
                          q_scale=scale)


def scaled_overlap(inputs: OperatorInputs, factor: float) -> OperatorInputs:
    """The same pencil with every Q_a multiplied by factor. The lowest
    eigenvalue of (1+reg) I + R Q R moves linearly, from its value m at
    factor 1 to (1+reg) + factor (m - (1+reg)): zero (a singular S~) at
    factor (1+reg) / (1+reg-m), negative (an indefinite S~) beyond."""
    import dataclasses
    return dataclasses.replace(inputs, q=np.asarray(inputs.q) * factor, q_scale=inputs.q_scale * factor)


def singular_overlap_factor(minimum: float, regularization: float) -> float:
    """The Q factor of scaled_overlap at which S~'s lowest eigenvalue reaches 0."""
    return (1.0 + regularization) / (1.0 + regularization - minimum)


def si8(seed: int = 2026, **kw) -> OperatorInputs:
    """Diamond-cubic Si8, a = 10.26 bohr, Gamma, Ecut 15 Ha, 16 bands."""
    return build_operator("si8", 10.26, 1, 15.0, 16, seed=seed, **kw)


def si64(seed: int = 2026, **kw) -> OperatorInputs:
    """Si64 supercell, a = 20.52 bohr (2x2x2 of 10.26), Gamma, Ecut 15 Ha, 160 bands, 512 projectors."""
    return build_operator("si64", 10.26, 2, 15.0, 160, seed=seed, **kw)


def gaas_kpoint(index: int, seed: int = 2026, **kw) -> OperatorInputs:
    """GaAs 2x2x2 zincblende (a = 21.36), Ecut 18 Ha, 192 bands, k of a 3x3x3 Monkhorst-Pack mesh."""
    i, j, k = index // 9, (index // 3) % 3, index % 3
    kpoint = tuple((2 * v - 2) / 6.0 for v in (i, j, k))  # ((2n - q - 1)/2q) for q = 3, n = 1..3
    return build_operator(f"gaas_k{index}", 10.68, 2, 18.0, 192, depths=(-2.2, -1.8), kpoint=kpoint, seed=seed,
                          **kw)


def gaas_small(kpoint=(1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0), seed: int = 2027, ecut_ha: float = 6.0, roots: int = 12,
               **kw) -> OperatorInputs:
    """GaAs 8-atom zincblende cell (a = 10.68 bohr, depths -2.2 / -1.8 Ha) at one k-point of the 3x3x3 mesh:
    the k-point batch's construction at test size."""
    return build_operator("gaas_small", 10.68, 1, ecut_ha, roots, depths=(-2.2, -1.8), kpoint=kpoint, seed=seed,
                          **kw)


def scf_step(inputs: OperatorInputs, step: int, seed: int = 91, keep: float = 1.0) -> OperatorInputs:
    """Inputs of one SCF-like iteration on the same basis and projectors: V(G)
    scaled by (1 + 0.05 step) plus Hermitian noise of 0.01 Ha on its keys, D
    plus Hermitian noise of 0.02 Ha per atom; B and Q unchanged (the
    reference's SCF rebuilds its operator each iteration with new V and D and
    the same projectors). keep < 1 retains that fraction of the nonzero key
    pairs (k, -k), so the key set changes as well; G = 0 is always kept."""
    rng = np.random.Generator(np.random.PCG64([seed, step]))
    keys = [tuple(int(v) for v in k) for k in inputs.v_hkl]
    where = {k: i for i, k in enumerate(keys)}
    noise = 0.01 * (rng.standard_normal(len(keys)) + 1j * rng.standard_normal(len(keys)))
    values = inputs.v_values * (1.0 + 0.05 * step)
    selected = []
    for i, k in enumerate(keys):
        j = where.get((-k[0], -k[1], -k[2]))
        if j is None:  # an unpaired key must stay as it is (its partner is an implicit zero)
            selected.append(i)
            continue
        if j < i:
            continue
        if i == j:
            values[i] = values[i] + noise[i].real
            selected.append(i)
        elif keep >= 1.0 or rng.uniform() < keep:
            w = 0.5 * (noise[i] + np.conj(noise[j]))
            values[i] = values[i] + w
            values[j] = values[j] + np.conj(w)
            selected += [i, j]
    order = np.sort(np.asarray(selected, dtype=np.int64))
    d = inputs.d.copy()
    for a in range(d.shape[0]):
        e = rng.standard_normal(d.shape[1:]) + 1j * rng.standard_normal(d.shape[1:])
        d[a] = d[a] + 0.01 * (e + e.conj().T)
    return dataclasses.replace(inputs, name=f"{inputs.name}_scf{step}", v_hkl=np.ascontiguousarray(inputs.v_hkl[order]),
                               v_values=np.ascontiguousarray(values[order]), d=d)


SI_VOLUME_PER_ATOM = 10.26 ** 3 / 8.0  # bohr^3, diamond Si


def serving_request(index: int, seed: int = 4242, atoms=(2, 128), ecut_ha=(10.0, 25.0), kpoints=(1, 8)):
    """One request of the seeded serving stream: a cubic cell with a
    log-uniform atom count (random sites, two species), Ecut uniform in the
    range, bands = 1.25 x the occupied count (2 per atom) within [8, 320], and
    1..8 k-points; returns one OperatorInputs per k-point (Q scaled in
    closed form, V(G) drawn once per cell)."""
    rng = np.random.Generator(np.random.PCG64([seed, index]))
    count = int(round(math.exp(rng.uniform(math.log(atoms[0]), math.log(atoms[1])))))
    a = (count * SI_VOLUME_PER_ATOM) ** (1.0 / 3.0)
    positions = rng.uniform(0.0, 1.0, size=(count, 3))
    species = rng.integers(0, 2, size=count)
    ecut = float(rng.uniform(ecut_ha[0], ecut_ha[1]))
    bands = int(min(320, max(8, round(1.25 * 2 * count))))
    nk = int(rng.integers(kpoints[0], kpoints[1] + 1))
    out = []
    for j in range(nk):
        kpoint = tuple(float(v) for v in rng.uniform(-0.5, 0.5, size=3)) if j else (0.0, 0.0, 0.0)
        potential = (out[0].v_hkl, out[0].v_values) if out else None  # V(G) is the cell's, not the k-point's
        out.append(build_operator(f"request{index}_k{j}", a, 1, ecut, bands, depths=(-2.2, -1.8), kpoint=kpoint,
                                  seed=seed * 1000 + index, sites=(positions, species), potential=potential,
                                  q_scaling="linear"))
    return out


def tiny(seed: int = 7, ecut_ha: float = 4.0, roots: int = 6, a: float = 7.0, **kw) -> OperatorInputs:
    """A small diamond cell for fast parity tests (a few hundred plane waves)."""
    return build_operator("tiny", a, 1, ecut_ha, roots, seed=seed, **kw)


def density_support(inputs: OperatorInputs, factor: float) -> np.ndarray:
    """Density Fourier support {1/2 |G|^2 <= factor * Ecut} of the cell, (m, 3) int32 keys."""
    hkl, _, _ = enumerate_g_vectors(inputs.reciprocal, factor * inputs.ecut_ha * inputs.hartree_to_ev)
    return np.ascontiguousarray(hkl, dtype=np.int32)


def gaussian_density(lattice, positions, keys, charge: float = 4.0, width: float = 1.2) -> np.ndarray:
    """n_G = sum_sites (charge / Omega) exp(-|G|^2 width^2 / 4) exp(-i G.tau) on the keys: normalised
    Gaussian charges at the fractional positions (a smooth stand-in for a valence or pseudo-core
    density; the truncated support leaves small negative regions, as real densities have)."""
    a = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
    volume = abs(float(np.dot(a[0], np.cross(a[1], a[2]))))
    b = 2.0 * math.pi * np.linalg.inv(a).T
    k = np.asarray(keys, dtype=np.float64).reshape(-1, 3)
    q = k @ b
    g2 = (q * q).sum(axis=1)
    taus = np.asarray(positions, dtype=np.float64).reshape(-1, 3) @ a
    phases = np.exp(-1j * (q @ taus.T)).sum(axis=1)
    return (charge / volume) * np.exp(-g2 * width * width / 4.0) * phases


def functional_case(name: str) -> dict:
    """Seeded inputs of the Hartree + XC functional: lattice (rows, bohr), density keys and values
    (Gaussian valence charges on {1/2|G|^2 <= f Ecut}) and a frozen core (narrower Gaussians on a
    smaller support). si8: diamond Si8 (a = 10.26), f Ecut = 15 Ha, grid 34^3 (2 x 17);
    triclinic: a skewed 2-site cell on a box of keys, grid 18 x 22 x 14 (2 x 11, 2 x 7), with the
    core on a box that reaches past it (22 x 22 x 18 with the core);
    si64: Si64 (a = 20.52), f Ecut = 60 Ha (f = 4 of the 15 Ha basis), grid 142^3 (2 x 71)."""
    if name == "triclinic":
        lattice = np.array([[6.0, 0.0, 0.0], [0.3, 6.0, 0.0], [0.1, 0.2, 6.6]])
        positions = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.3]])
        keys = np.array([(h, k, l) for h in range(-4, 5) for k in range(-5, 6) for l in range(-3, 4)], dtype=np.int32)
        core_keys = np.array([(h, k, l) for h in range(-5, 6) for k in range(-3, 4) for l in range(-4, 5)],
                             dtype=np.int32)  # reaches past the density box: core-only keys
    else:
        reps, cut_ha = {"si8": (1, 15.0), "si64": (2, 60.0)}[name]
        lattice = np.eye(3) * 10.26 * reps
        positions, _ = zincblende_sites(reps)
        reciprocal = 2.0 * math.pi * np.linalg.inv(lattice).T
        keys, _, _ = enumerate_g_vectors(reciprocal, cut_ha * HARTREE_TO_EV)
        core_keys, _, _ = enumerate_g_vectors(reciprocal, 0.5 * cut_ha * HARTREE_TO_EV)
    keys = np.ascontiguousarray(keys, dtype=np.int32)
    core_keys = np.ascontiguousarray(core_keys, dtype=np.int32)
    return {"lattice": lattice, "keys": keys, "values": gaussian_density(lattice, positions, keys, 4.0, 1.2),
            "core_keys": core_keys, "core_values": gaussian_density(lattice, positions, core_keys, 2.0, 0.8)}


def collinear_case(name: str) -> dict:
    """Spin-polarised inputs of the collinear functional on functional_case's cells: the up
    channel carries 2.4 electrons per site (width 1.2), the down channel 1.6 on keys one
    shell narrower in h (width 1.4), the frozen core as in functional_case."""
    case = functional_case(name)
    lattice, keys = case["lattice"], case["keys"]
    if name == "triclinic":
        positions = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.3]])
    else:
        positions, _ = zincblende_sites({"si8": 1, "si64": 2}[name])
    down_keys = np.ascontiguousarray(keys[np.abs(keys[:, 0]) < np.abs(keys[:, 0]).max()], dtype=np.int32)
    return {"lattice": lattice, "up_keys": keys, "up": gaussian_density(lattice, positions, keys, 2.4, 1.2),
            "down_keys": down_keys, "down": gaussian_density(lattice, positions, down_keys, 1.6, 1.4),
            "core_keys": case["core_keys"], "core_values": case["core_values"]}


def band_coefficients(inputs: OperatorInputs, bands: int, seed: int = 31) -> np.ndarray:
    """Seeded normalised band-major plane-wave coefficients, (bands, npw) complex128,
    with a kinetic decay so that the bands look like smooth valence states."""
    rng = np.random.Generator(np.random.PCG64(seed))
    decay = np.exp(-0.5 * inputs.kinetic_ev / inputs.hartree_to_ev)
    c = (rng.standard_normal((bands, inputs.npw)) + 1j * rng.standard_normal((bands, inputs.npw))) * decay
    return c / np.linalg.norm(c, axis=1, keepdims=True)


def augmentation(channel_l=(0, 0, 1, 1), max_l: int = 2, radial: int = 401, r0: float = 1e-4, rmax: float = 1.6,
                 width: float = 0.45, seed: int = 41) -> dict:
    """Synthetic one-centre augmentation data in the reference's PawAugmentationData
    layout (radial arrays in Angstrom): a logarithmic radial mesh, Gaussian compensation
    shapes g_L(r) r^2 ~ r^L exp(-r^2/width^2) r^2 with unit continuous L-moment, and
    seeded aug_moment(i, j, L) symmetric in (i, j) on the Gaunt-allowed L."""
    rng = np.random.Generator(np.random.PCG64(seed))
    channel_l = np.asarray(channel_l, dtype=np.int32)
    n = channel_l.size
    step = math.log(rmax / r0) / (radial - 1)
    r = r0 * np.exp(step * np.arange(radial))
    r2 = np.zeros((max_l + 1, radial))
    for L in range(max_l + 1):
        norm = 0.5 * math.gamma(L + 1.5) * width ** (2 * L + 3)
        r2[L] = r ** L * np.exp(-(r / width) ** 2) * r * r / norm
    moment = np.zeros((n, n, max_l + 1))
    for i in range(n):
        for j in range(i, n):
            lo, hi = abs(int(channel_l[i] - channel_l[j])), min(max_l, int(channel_l[i] + channel_l[j]))
            for L in range(lo, hi + 1, 2):
                moment[i, j, L] = moment[j, i, L] = rng.uniform(-0.5, 0.5)
    return {"channel_l": channel_l, "max_l": max_l, "radial_grid": r, "aug_moment": moment.ravel(),
            "compensation_r2": r2}


def projected_amplitudes(atoms: int, dim: int, bands: int, seed: int = 43) -> np.ndarray:
    """Seeded projector amplitudes P = B psi, (atoms*dim, bands) complex128 column-major."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = rng.standard_normal((atoms * dim, bands)) + 1j * rng.standard_normal((atoms * dim, bands))
    return np.asfortranarray(0.3 * p)


def real_gaunt(l1: int, m1: int, l2: int, m2: int, L: int, M: int) -> float:
    """int Y_l1m1 Y_l2m2 Y_LM dOmega over the sphere by Gauss-Legendre (16) x uniform-phi (32)
    quadrature, exact for the polynomial degrees of L <= 6 products."""
    x, wx = np.polynomial.legendre.leggauss(16)
    phi = np.arange(32) * (2 * math.pi / 32)
    theta = np.arccos(x)
    q = np.stack([np.outer(np.sin(theta), np.cos(phi)).ravel(), np.outer(np.sin(theta), np.sin(phi)).ravel(),
                  np.repeat(np.cos(theta), phi.size)], axis=1)
    weight = np.repeat(wx, phi.size) * (2 * math.pi / 32)
    return float(np.sum(weight * real_harmonic(l1, m1, q) * real_harmonic(l2, m2, q) * real_harmonic(L, M, q)))


def lm_transform(aug: dict) -> np.ndarray:
    """(L,M) moments of each unit one-centre occupation, [LM, ii*dim+jj] =
    aug_moment(i, j, L) G(l_i m, l_j m' | L M): the compensation transform the
    reference builds from paw_lm_moments_from_density (src/paw_augmentation.cpp:490-525,
    src/paw_compensation.cpp:228-236), here from the real Gaunt coefficients by quadrature."""
    ch = [int(v) for v in aug["channel_l"]]
    max_l = int(aug["max_l"])
    moment = np.asarray(aug["aug_moment"], dtype=np.float64).reshape(len(ch), len(ch), max_l + 1)
    offset = np.concatenate([[0], np.cumsum([2 * l + 1 for l in ch])])
    dim = int(offset[-1])
    out = np.zeros(((max_l + 1) ** 2, dim * dim), dtype=np.complex128)
    for i, li in enumerate(ch):
        for j, lj in enumerate(ch):
            for m in range(-li, li + 1):
                for mp in range(-lj, lj + 1):
                    e = (offset[i] + m + li) * dim + offset[j] + mp + lj
                    for L in range(abs(li - lj), min(max_l, li + lj) + 1):
                        for M in range(-L, L + 1):
                            g = real_gaunt(li, m, lj, mp, L, M)
                            if abs(g) > 1e-12:
                                out[L * L + M + L, e] += moment[i, j, L] * g
    return out
