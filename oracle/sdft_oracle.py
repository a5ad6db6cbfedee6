"""CPU restatement (numpy) of the reference's hot-path arithmetic.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library. Only tests/, the
smoke check in __graft_entry__ and bench.py's CPU-baseline leg may import it;
the product never does. It is pinned against the reference itself (the
unmodified C++ built into oracle/_ref by oracle/ref/Makefile) by
tests/test_oracle_pins.py, and against committed fixtures in tests/golden/.

Each function cites the reference lines it restates (paths relative to the
Sparse-DFT source tree).
"""
from __future__ import annotations

import math

import numpy as np

HARTREE_TO_EV = 27.211386245988


def fast_fft_length(minimum: int) -> int:
    """Smallest 2/3/5/7-smooth n >= minimum (src/fft_planning.hpp:16-23)."""
    n = minimum
    while True:
        r = n
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


def grid_shape(hkl: np.ndarray, v_hkl: np.ndarray, minimal: bool = False):
    """Alias-free FFT grid of the operator (src/plane_wave_operator.cpp:400-457)."""
    low = hkl.min(axis=0)
    high = hkl.max(axis=0)
    width = high - low
    retained = np.all(np.abs(v_hkl) <= width[None, :], axis=1)
    radius = np.abs(v_hkl[retained]).max(axis=0) if retained.any() else np.zeros(3, dtype=int)
    shape = []
    for a in range(3):
        minimum = max(3, 2 * max(int(radius[a]), int(width[a])) + 1)
        shape.append(minimum if minimal else fast_fft_length(minimum))
    return tuple(shape), retained


def index_map(hkl: np.ndarray, shape) -> np.ndarray:
    """Row-major wrapped grid index ((h mod n0)*n1 + k mod n1)*n2 + l mod n2 (src/plane_wave_operator.cpp:94-97)."""
    n0, n1, n2 = shape
    h = np.mod(hkl[:, 0], n0).astype(np.int64)
    k = np.mod(hkl[:, 1], n1).astype(np.int64)
    l = np.mod(hkl[:, 2], n2).astype(np.int64)
    return ((h * n1 + k) * n2 + l).astype(np.uint64)


def backward_fft(grid: np.ndarray) -> np.ndarray:
    """Unnormalised sum_G c_G exp(+iG.r), FFTW_BACKWARD convention."""
    return np.fft.ifftn(grid) * grid.size


def forward_fft(grid: np.ndarray) -> np.ndarray:
    """Unnormalised sum_r f(r) exp(-iG.r), FFTW_FORWARD convention."""
    return np.fft.fftn(grid)


def kinetic_preconditioner(kinetic: float, wavefunction_kinetic: float) -> float:
    """Bounded rational preconditioner (src/pw_core.cpp:33-47)."""
    if not (math.isfinite(kinetic) and kinetic >= 0 and math.isfinite(wavefunction_kinetic) and wavefunction_kinetic >= 0):
        raise ValueError("kinetic preconditioner requires nonnegative Hartree energies")
    scale = 1.5 * max(wavefunction_kinetic, 2.0 / 27.211386245988)
    x = kinetic / scale
    if x > 1.0:
        inv = 1.0 / x
        p = inv * (8.0 + inv * (12.0 + inv * (18.0 + 27.0 * inv)))
        return (2.0 / scale) * p / (p + 16.0)
    p = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
    return (2.0 / scale) * p / (p + 16.0 * x * x * x * x)


class Operator:
    """H~ and S~ of the reference's PlaneWaveOperator (src/plane_wave_operator.cpp:218-374, 393-516)."""

    def __init__(self, x, minimal: bool = False):
        self.n = x.hkl.shape[0]
        self.shape, retained = grid_shape(x.hkl, x.v_hkl, minimal)
        self.count = int(np.prod(self.shape))
        grid = np.zeros(self.shape, dtype=np.complex128)
        keys = x.v_hkl[retained]
        vals = x.v_values[retained]
        grid[np.mod(keys[:, 0], self.shape[0]), np.mod(keys[:, 1], self.shape[1]),
             np.mod(keys[:, 2], self.shape[2])] = vals
        real = backward_fft(grid)
        if np.any(np.abs(real.imag) > 1e-9 * np.maximum(1.0, np.abs(real.real))):
            raise RuntimeError("complex real-space local potential")
        self.local_real = real.real.reshape(-1).copy()
        self.indices = index_map(x.hkl, self.shape)
        self.kinetic = x.kinetic_ev / x.hartree_to_ev
        self.regularization = x.regularization
        self.b = np.asarray(x.amplitudes, dtype=np.complex128)  # (np, n)
        self.atom_offsets = np.concatenate([[0], np.cumsum(x.projectors)]).astype(int)
        self.d = [0.5 * (m + m.conj().T) for m in x.d]
        self.q = [0.5 * (m + m.conj().T) for m in x.q]
        zero = np.all(x.v_hkl == 0, axis=1)
        v0 = float(x.v_values[zero][0].real) if zero.any() else 0.0
        self.h_diagonal = self.kinetic + v0
        self.s_diagonal = np.full(self.n, 1.0 + self.regularization)
        for a, (lo, hi) in enumerate(zip(self.atom_offsets[:-1], self.atom_offsets[1:])):
            b = self.b[lo:hi]
            self.h_diagonal = self.h_diagonal + np.real(np.sum(b.conj() * (self.d[a] @ b), axis=0))
            self.s_diagonal = self.s_diagonal + np.real(np.sum(b.conj() * (self.q[a] @ b), axis=0))

    def local(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.complex128).reshape(self.n, -1, order="F")
        out = np.empty_like(x)
        flat_index = self.indices.astype(np.int64)
        for c in range(x.shape[1]):
            grid = np.zeros(self.count, dtype=np.complex128)
            grid[flat_index] = x[:, c]
            field = backward_fft(grid.reshape(self.shape)) * self.local_real.reshape(self.shape)
            back = forward_fft(field).reshape(-1)
            out[:, c] = self.kinetic * x[:, c] + back[flat_index] / float(self.count)
        return out

    def _onsite(self, p: np.ndarray, blocks) -> np.ndarray:
        out = np.zeros_like(p)
        for a, (lo, hi) in enumerate(zip(self.atom_offsets[:-1], self.atom_offsets[1:])):
            out[lo:hi] = blocks[a] @ p[lo:hi]
        return out

    def project(self, x):
        return self.b @ np.asarray(x, dtype=np.complex128).reshape(self.n, -1, order="F")

    def apply_h(self, x):
        x = np.asarray(x, dtype=np.complex128).reshape(self.n, -1, order="F")
        y = self.local(x)
        if self.b.shape[0]:
            y = y + self.b.conj().T @ self._onsite(self.b @ x, self.d)
        return y

    def apply_s(self, x):
        x = np.asarray(x, dtype=np.complex128).reshape(self.n, -1, order="F")
        y = (1.0 + self.regularization) * x
        if self.b.shape[0]:
            y = y + self.b.conj().T @ self._onsite(self.b @ x, self.q)
        return y

    def dense(self):
        """Dense H~ and S~ (small cases only), column by column."""
        eye = np.eye(self.n, dtype=np.complex128)
        return self.apply_h(eye), self.apply_s(eye)


def metric_signature(op: Operator):
    """Lowest eigenvalue of S~'s nontrivial block, capped at 1+reg, as the
    reference's overlap() computes it (src/plane_wave_operator.cpp:702-717):
    R = (B B^H)^(1/2) with the Gram eigenvalues clamped at 0, then
    (1+reg) I + R Q R. Returns (minimum, indefinite, singular)."""
    reg = op.regularization
    if op.b.shape[0] == 0:
        minimum = 1.0 + reg
    else:
        gram = op.b @ op.b.conj().T
        w, u = np.linalg.eigh(0.5 * (gram + gram.conj().T))
        root = (u * np.sqrt(np.maximum(w, 0.0))) @ u.conj().T
        q = op._onsite(np.eye(op.b.shape[0], dtype=np.complex128), op.q)
        small = (1.0 + reg) * np.eye(op.b.shape[0]) + root @ q @ root
        minimum = min(1.0 + reg, float(np.linalg.eigvalsh(0.5 * (small + small.conj().T))[0]))
    return minimum, minimum < -1e-10, abs(minimum) <= 1e-10


def generalized_eigenvalues(h: np.ndarray, s: np.ndarray, roots: int) -> np.ndarray:
    """Lowest roots of H v = e S v by Cholesky reduction (dense oracle, small n)."""
    hh = 0.5 * (h + h.conj().T)
    ss = 0.5 * (s + s.conj().T)
    lower = np.linalg.cholesky(ss)
    inv = np.linalg.inv(lower)
    a = inv @ hh @ inv.conj().T
    return np.linalg.eigvalsh(0.5 * (a + a.conj().T))[:roots]


def certified_residuals(op: Operator, eigenvalues: np.ndarray, vectors: np.ndarray):
    """Fresh FP64 ||H x - e S x|| and |x^H S x - 1| per root (src/solver_replay_cli.cpp:30-45)."""
    hx = op.apply_h(vectors)
    sx = op.apply_s(vectors)
    res = np.linalg.norm(hx - sx * eigenvalues[None, :], axis=0)
    metric = np.real(np.sum(vectors.conj() * sx, axis=0))
    return res, np.abs(metric - 1.0)


# --- PBE exchange-correlation (src/pbe_xc.cpp) -------------------------------

_PBE_GAMMA = 0.031090690869654895
_PBE_BETA = 0.06672455060314922
_PBE_MU = 0.2195149727645171
_PBE_KAPPA = 0.804


class _Dual:
    """Forward-mode value with d/dn and d/d|grad n|^2 over numpy arrays (src/pbe_xc.cpp:18-60)."""

    __slots__ = ("v", "dn", "dg")

    def __init__(self, v, dn, dg):
        self.v, self.dn, self.dg = v, dn, dg

    @staticmethod
    def lift(x):
        return x if isinstance(x, _Dual) else _Dual(x, 0.0, 0.0)

    def __add__(self, o):
        o = _Dual.lift(o)
        return _Dual(self.v + o.v, self.dn + o.dn, self.dg + o.dg)

    __radd__ = __add__

    def __sub__(self, o):
        o = _Dual.lift(o)
        return _Dual(self.v - o.v, self.dn - o.dn, self.dg - o.dg)

    def __rsub__(self, o):
        return _Dual.lift(o) - self

    def __neg__(self):
        return _Dual(-self.v, -self.dn, -self.dg)

    def __mul__(self, o):
        if not isinstance(o, _Dual):
            return _Dual(self.v * o, self.dn * o, self.dg * o)
        return _Dual(self.v * o.v, self.dn * o.v + self.v * o.dn, self.dg * o.v + self.v * o.dg)

    __rmul__ = __mul__

    def __truediv__(self, o):
        if not isinstance(o, _Dual):
            return self * (1.0 / o)
        inv = 1.0 / o.v
        inv2 = inv * inv
        return _Dual(self.v * inv, (self.dn * o.v - self.v * o.dn) * inv2, (self.dg * o.v - self.v * o.dg) * inv2)

    def __rtruediv__(self, o):
        return _Dual.lift(o) / self

    def pow(self, p):
        value = np.sqrt(self.v) if p == 0.5 else np.power(self.v, p)
        d = p * value / self.v
        return _Dual(value, d * self.dn, d * self.dg)

    def log1p(self):
        return _Dual(np.log1p(self.v), self.dn / (1.0 + self.v), self.dg / (1.0 + self.v))

    def expm1(self):
        value = np.expm1(self.v)
        return _Dual(value, (1.0 + value) * self.dn, (1.0 + value) * self.dg)


def _pw92(rs: _Dual) -> _Dual:
    """PW92 unpolarised correlation energy per particle (src/pbe_xc.cpp:62-72)."""
    a, alpha1, b1, b2, b3, b4 = 0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    root = rs.pow(0.5)
    poly = b1 * root + b2 * rs + b3 * rs * root + b4 * rs * rs
    return -2.0 * a * (1.0 + alpha1 * rs) * (1.0 / (2.0 * a * poly)).log1p()


def pbe_unpolarized(density, gradient_magnitude) -> np.ndarray:
    """(count, 7) PbeXcPoint rows (src/pbe_xc.cpp:74-140): energy density, energy per
    particle, exchange and correlation energy densities, their d/dn potentials and the
    |grad n|^2 coefficient with the cancellation-free sigma response."""
    nv = np.asarray(density, dtype=np.float64).ravel()
    gv = np.asarray(gradient_magnitude, dtype=np.float64).ravel()
    if (not np.all(nv > 0.0)) or (not np.all(np.isfinite(nv))) or np.any(gv < 0.0) or not np.all(np.isfinite(gv)):
        raise ValueError("PBE density must be positive and gradient finite")
    zero = np.zeros_like(nv)
    n = _Dual(nv, np.ones_like(nv), zero)
    g2 = _Dual(gv * gv, zero, np.ones_like(nv))
    pi = math.pi
    root_n = n.pow(1.0 / 3.0)
    rs = np.cbrt(3.0 / (4.0 * pi)) / root_n
    kf = np.cbrt(3.0 * pi * pi) * root_n
    eps_x = (-0.75 * np.cbrt(3.0 / pi)) * root_n
    s2 = g2 / (4.0 * kf * kf * n * n)
    fx = (1.0 + _PBE_KAPPA) - _PBE_KAPPA / (1.0 + (_PBE_MU / _PBE_KAPPA) * s2)
    exchange = n * eps_x * fx
    eps_c = _pw92(rs)
    ks2 = 4.0 * kf / pi
    t2 = g2 / (4.0 * ks2 * n * n)
    em1 = (-eps_c / _PBE_GAMMA).expm1()
    a = (_PBE_BETA / _PBE_GAMMA) / em1
    at2 = a * t2
    t4a2 = at2 * at2
    h = _PBE_GAMMA * ((_PBE_BETA / _PBE_GAMMA) * t2 * (1.0 + at2) / (1.0 + at2 + t4a2)).log1p()
    correlation = n * (eps_c + h)
    u = (_PBE_MU / _PBE_KAPPA) * s2.v
    x = at2.v
    den = 1.0 + x + x * x
    bt = (_PBE_BETA / _PBE_GAMMA) * t2.v * (1.0 + x)
    with np.errstate(all="ignore"):
        far = (1.0 + 2.0 * x) / (den * (den + bt)) - 1.0 / ((1.0 + u) * (1.0 + u))
        near = u * (2.0 + u) / ((1.0 + u) * (1.0 + u)) - (x * x * (3.0 + x * (2.0 + x)) + bt * den) / (den * (den + bt))
    difference = np.where((u > 0.25) | (x > 0.25), far, near)
    total = exchange.v + correlation.v
    return np.stack([total, total / nv, exchange.v, correlation.v, exchange.dn, correlation.dn,
                     _PBE_BETA / (2.0 * ks2.v * nv) * difference], axis=1)


# --- Band density (src/density_functionals.cpp:407-460) -----------------------

def density_grid_shape(hkl, support, fast: bool = False):
    """Alias-free density grid max(3, 2m+1) per axis, m = max(max|support|, max_g - min_g)
    with min/max seeded at 0 (src/density_functionals.cpp:415-428); `fast` rounds each axis
    up to a 2/3/5/7-smooth length (SDFT_FAST_DENSITY_GRID=1, :355-365)."""
    hkl = np.asarray(hkl).reshape(-1, 3)
    support = np.asarray(support).reshape(-1, 3)
    m = np.abs(support).max(axis=0)
    span = np.maximum(hkl.max(axis=0), 0) - np.minimum(hkl.min(axis=0), 0)
    n = [max(3, 2 * int(max(a, b)) + 1) for a, b in zip(m, span)]
    return tuple(fast_fft_length(v) for v in n) if fast else tuple(n)


def plane_wave_density(hkl, coefficients, occupations, volume, support, fast: bool = False) -> np.ndarray:
    """n(G) at the support keys: (1/N) FFT_fwd(sum_b f_b/volume |FFT_bwd(scatter psi_b)|^2)
    (src/density_functionals.cpp:407-460 with :71-77 and :269-284). coefficients: (bands, npw)."""
    hkl = np.asarray(hkl).reshape(-1, 3)
    support = np.asarray(support).reshape(-1, 3)
    coefficients = np.asarray(coefficients, dtype=np.complex128).reshape(len(occupations), hkl.shape[0])
    if hkl.size == 0 or support.size == 0 or not np.isfinite(volume) or volume <= 0:
        raise ValueError("invalid plane-wave FFT density dimensions")
    shape = density_grid_shape(hkl, support, fast)
    flat = index_map(hkl, shape)
    count = int(np.prod(shape))
    density = np.zeros(count)
    for band, f in enumerate(occupations):
        if not np.isfinite(f) or f < 0 or f > 2:
            raise ValueError("invalid FFT spin-summed occupation")
        if f == 0:
            continue
        if not np.all(np.isfinite(coefficients[band].view(np.float64))):
            raise ValueError("nonfinite wavefunction coefficient")
        grid = np.zeros(count, dtype=np.complex128)
        grid[flat] = coefficients[band]
        field = backward_fft(grid.reshape(shape)).ravel()
        density += f / volume * (field.real * field.real + field.imag * field.imag)
    transformed = forward_fft(density.reshape(shape).astype(np.complex128)).ravel()
    return transformed[index_map(support, shape)] / count


# --- One-centre occupations and compensation charge ---------------------------
# src/onsite_density.hpp:10-36, src/paw_compensation.cpp:51-139,185-342,465-524,
# src/paw_augmentation.cpp:490-525.

BOHR_PER_ANGSTROM = 1.8897261254578281  # CODATA convention (src/atomic_units.hpp:10-14)


def onsite_density(amplitudes, occupations) -> np.ndarray:
    """rho_ij = sum_n f_n P_in conj(P_jn) for one atom's rows (src/onsite_density.hpp:13-36)."""
    p = np.asarray(amplitudes, dtype=np.complex128)
    f = np.asarray(occupations, dtype=np.float64)
    if np.any(~np.isfinite(f)) or np.any(f < 0) or np.any(f > 2):
        raise ValueError("invalid projected onsite occupation")
    if not (np.all(np.isfinite(p.real)) and np.all(np.isfinite(p.imag))):
        raise ValueError("nonfinite onsite projection")
    return (p * f[None, :]) @ p.conj().T


def radial_weights(r) -> np.ndarray:
    """Simpson panels from the outer end on a logarithmic mesh, else trapezoids (src/paw_compensation.cpp:51-74)."""
    r = np.asarray(r, dtype=np.float64)
    h = math.log(r[1] / r[0])
    logarithmic = np.isfinite(h) and h > 0 and np.all(np.abs(np.log(r[1:] / r[:-1]) - h) < 2e-7)
    w = np.zeros(r.size)
    if logarithmic:
        k = r.size
        while k >= 3:
            w[k - 1] += r[k - 1] * h / 3.0
            w[k - 2] = 4.0 * r[k - 2] * h / 3.0
            w[k - 3] = r[k - 3] * h / 3.0
            if k == 3:
                break
            k -= 2
    else:
        d = np.diff(r) / 2.0
        w[:-1] += d
        w[1:] += d
    return w


def real_harmonic(l: int, m: int, q: np.ndarray) -> np.ndarray:
    """Real harmonics without the Condon-Shortley phase (src/paw_compensation.cpp:116-139); q (n,3)."""
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3)
    radius = np.sqrt(np.sum(q * q, axis=1))
    small = radius < 1e-14
    safe = np.where(small, 1.0, radius)
    z = np.clip(q[:, 2] / safe, -1.0, 1.0)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    order = abs(m)
    pmm = np.ones_like(z)
    for k in range(1, order + 1):
        pmm = pmm * ((2.0 * k - 1.0) * s)
    value = pmm
    if l > order:
        previous = pmm
        value = (2.0 * order + 1.0) * z * pmm
        for degree in range(order + 2, l + 1):
            nxt = ((2.0 * degree - 1.0) * z * value - (degree + order - 1.0) * previous) / (degree - order)
            previous, value = value, nxt
    factor = math.sqrt((2 * l + 1) / (4 * math.pi) * math.exp(math.lgamma(l - order + 1) - math.lgamma(l + order + 1)))
    factor *= math.sqrt(2.0) if order else 1.0
    angle = order * np.arctan2(q[:, 1], q[:, 0])
    out = factor * value * (np.sin(angle) if m < 0 else np.cos(angle))
    return np.where(small, (1.0 / math.sqrt(4 * math.pi)) if l == 0 else 0.0, out)


def _reciprocal(lattice):
    a = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
    volume = float(np.dot(a[0], np.cross(a[1], a[2])))
    b = 2 * math.pi / volume * np.array([np.cross(a[1], a[2]), np.cross(a[2], a[0]), np.cross(a[0], a[1])])
    return a, b, abs(volume)


def compensation_form(lattice, keys, augmentation) -> np.ndarray:
    """Compact F_LM(G) = nonzero part of 4 pi (-i)^L Y_LM(G^) int g_L r^2 j_L(|G| r) dr, shape (lms, count)
    (src/paw_compensation.cpp:254-301)."""
    from scipy.special import spherical_jn
    _, b, _ = _reciprocal(lattice)
    keys = np.asarray(keys).reshape(-1, 3).astype(np.float64)
    q = keys @ b
    radius = np.sqrt(np.sum(q * q, axis=1)) * BOHR_PER_ANGSTROM
    r = np.asarray(augmentation["radial_grid"], dtype=np.float64)
    r2 = np.asarray(augmentation["compensation_r2"], dtype=np.float64)
    w = radial_weights(r)
    shells, inverse = np.unique(radius, return_inverse=True)
    max_l = int(augmentation["max_l"])
    form = np.zeros(((max_l + 1) ** 2, keys.shape[0]))
    for L in range(max_l + 1):
        integral = (spherical_jn(L, np.outer(shells, r)) * (w * r2[L])[None, :]).sum(axis=1)
        if L == 0:
            integral = np.where(shells < 1e-14, 1.0, integral)
        sign = 1.0 if L % 4 in (0, 3) else -1.0
        for M in range(-L, L + 1):
            form[L * L + M + L] = sign * 4 * math.pi * real_harmonic(L, M, q) * integral[inverse]
    return form


def compensation_density(lattice, fractional, keys, augmentation, transform, onsite) -> np.ndarray:
    """sum_a exp(-i G.tau_a)/Omega sum_LM F_LM(G) M_a,LM with M_a = transform . rho_a (src/paw_compensation.cpp:465-524)."""
    a, b, volume = _reciprocal(lattice)
    keys = np.asarray(keys).reshape(-1, 3)
    q = keys.astype(np.float64) @ b
    form = compensation_form(lattice, keys, augmentation)
    max_l = int(augmentation["max_l"])
    imaginary = np.array([L % 2 for L in range(max_l + 1) for _ in range(2 * L + 1)], dtype=bool)
    complex_form = np.where(imaginary[:, None], 1j * form, form)
    rho = np.asarray(onsite, dtype=np.complex128).reshape(len(fractional), -1)
    moments = rho @ np.asarray(transform).T  # (atoms, lms)
    positions = np.asarray(fractional, dtype=np.float64).reshape(-1, 3) @ a
    total = np.zeros(keys.shape[0], dtype=np.complex128)
    for atom in range(positions.shape[0]):
        phase = np.exp(-1j * (q @ positions[atom]))
        total += phase * (moments[atom] @ complex_form) / volume
    return total


def compensation_project(lattice, fractional, keys, augmentation, transform, potential) -> np.ndarray:
    """The adjoint of compensation_density: out_a = sum_LM [sum_G V(-G) exp(-i G.tau_a) F_LM(G)] T_LM,
    with V given on the support keys (0 for an absent mode); shape (atoms, dim, dim)
    (src/paw_compensation.cpp:552-629)."""
    a, b, _ = _reciprocal(lattice)
    keys = np.asarray(keys).reshape(-1, 3)
    q = keys.astype(np.float64) @ b
    form = compensation_form(lattice, keys, augmentation)
    max_l = int(augmentation["max_l"])
    imaginary = np.array([L % 2 for L in range(max_l + 1) for _ in range(2 * L + 1)], dtype=bool)
    complex_form = np.where(imaginary[:, None], 1j * form, form)
    where = {tuple(k): i for i, k in enumerate(keys.tolist())}
    v = np.asarray(potential, dtype=np.complex128)
    opposite = np.array([v[where[(-k[0], -k[1], -k[2])]] if (-k[0], -k[1], -k[2]) in where else 0.0
                         for k in keys.tolist()], dtype=np.complex128)
    positions = np.asarray(fractional, dtype=np.float64).reshape(-1, 3) @ a
    t = np.asarray(transform, dtype=np.complex128)
    dim = int(round(math.sqrt(t.shape[1])))
    out = np.zeros((positions.shape[0], dim, dim), dtype=np.complex128)
    for atom in range(positions.shape[0]):
        phase = np.exp(-1j * (q @ positions[atom]))
        responses = complex_form @ (opposite * phase)
        out[atom] = (responses @ t).reshape(dim, dim)
    return out



# --- Hartree + PBE functional (src/density_functionals.cpp:462-729) ----------

def density_functionals(lattice, keys, values, core_keys=None, core_values=None, padding: int = 2,
                        fast: bool = False) -> dict:
    """The reference's evaluate_density_functionals with its default packing, in
    numpy. The support (density keys, plus frozen-core keys for XC) is taken in
    map order (lexicographic h, k, l). Hartree per density key (:476-497):
    V_H = 4 pi n / q^2 and E_H = sum 2 pi Omega |n|^2 / q^2 for q^2 > 1e-12,
    stress 4 pi |n|^2 q_a q_c / q^4 minus E_H / Omega on the diagonal (:693).
    XC on the grid padding * max(3, 2m+1) per axis (:498-519; `fast` rounds
    each axis up to a 2/3/5/7-smooth length): n, grad n by backward FFTs of n_G
    and i q n_G (valence and core transformed separately and summed, :527-559),
    PBE at max(1e-10, n) per point, tile sums of electrons, energy and stress
    (:600-641, summed exactly here), forward FFTs of the local potential and
    the gradient responses, v_xc(G) = l(G) - i q.d(G) (:665-683), and
    <n, v_xc> = Omega sum Re n(G) v_xc(-G) (:684-691)."""
    a = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
    det = float(np.dot(a[0], np.cross(a[1], a[2])))
    volume = abs(det)
    if volume < 1e-12 or not math.isfinite(volume):
        raise ValueError("singular density-grid lattice")
    b = 2.0 * math.pi / det * np.array([np.cross(a[1], a[2]), np.cross(a[2], a[0]), np.cross(a[0], a[1])])
    density = {tuple(int(v) for v in k): complex(x) for k, x in zip(np.asarray(keys).reshape(-1, 3), np.asarray(values).ravel())}
    if not density:
        raise ValueError("density Fourier support is empty")
    core = {}
    if core_keys is not None:
        core = {tuple(int(v) for v in k): complex(x)
                for k, x in zip(np.asarray(core_keys).reshape(-1, 3), np.asarray(core_values).ravel())}
    support = sorted(set(density) | set(core))
    sk = np.array(support, dtype=np.int64).reshape(-1, 3)
    q = sk[:, 0:1] * b[0] + sk[:, 1:2] * b[1] + sk[:, 2:3] * b[2]
    q2 = (q * q).sum(axis=1)
    in_density = np.array([k in density for k in support])
    rho = np.array([density.get(k, 0.0) for k in support], dtype=np.complex128)
    rho_core = np.array([core.get(k, 0.0) for k in support], dtype=np.complex128)
    # Hartree (density keys only).
    coulomb = in_density & (q2 > 1e-12)
    norm = (rho.real ** 2 + rho.imag ** 2)
    hartree = np.where(coulomb, 4.0 * math.pi * rho / np.where(coulomb, q2, 1.0), 0.0)
    e_h = math.fsum((2.0 * math.pi * volume * norm[coulomb] / q2[coulomb]).tolist())
    stress_h = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            stress_h[i, j] = math.fsum((4.0 * math.pi * norm[coulomb] * q[coulomb, i] * q[coulomb, j]
                                        / (q2[coulomb] * q2[coulomb])).tolist())
    # XC grid.
    m = np.abs(sk).max(axis=0)
    shape = tuple(padding * max(3, 2 * int(v) + 1) for v in m)
    if fast:
        shape = tuple(fast_fft_length(v) for v in shape)
    if max(shape) > 512:
        raise ValueError("XC grid axis above 512 points")
    idx = tuple(np.mod(sk[:, a_], shape[a_]) for a_ in range(3))

    def fields(coefficients):
        grids = np.zeros((4,) + shape, dtype=np.complex128)
        grids[0][idx] = coefficients
        for axis in range(3):
            grids[axis + 1][idx] = 1j * q[:, axis] * coefficients
        return [backward_fft(g).real for g in grids]

    if core:
        valence_fields = fields(np.where(in_density, rho, 0.0))
        core_fields = fields(rho_core)
        total = [v + c for v, c in zip(valence_fields, core_fields)]
        valence = valence_fields[0]
    else:
        total = fields(rho)
        valence = total[0]
    raw, gx, gy, gz = total
    n = np.maximum(1e-10, raw)
    grad = np.sqrt(gx * gx + gy * gy + gz * gz)
    xc = pbe_unpolarized(n.ravel(), grad.ravel())
    energy = xc[:, 0].reshape(shape)
    local = (xc[:, 4] + xc[:, 5]).reshape(shape)
    coefficient = xc[:, 6].reshape(shape)
    d = [coefficient * gx, coefficient * gy, coefficient * gz]
    g = [gx, gy, gz]
    points = int(np.prod(shape))
    weight = volume / points
    pressure = energy - local * raw - d[0] * gx - d[1] * gy - d[2] * gz
    stress_xc = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            term = (pressure if i == j else 0.0) - d[i] * g[j]
            stress_xc[i, j] = math.fsum(np.ravel(term).tolist()) / points
    # Forward transforms and v_xc on the support.
    transforms = [forward_fft(f)[idx] / points for f in (local, d[0], d[1], d[2])]
    vxc = transforms[0] - 1j * (q[:, 0] * transforms[1] + q[:, 1] * transforms[2] + q[:, 2] * transforms[3])
    where = {k: i for i, k in enumerate(support)}
    vxc_density = math.fsum(volume * (rho[i] * vxc[where[(-k[0], -k[1], -k[2])]]).real
                            for i, k in enumerate(support) if in_density[i] and (-k[0], -k[1], -k[2]) in where)
    stress_h -= np.eye(3) * (e_h / volume)
    return {"hkl": sk.astype(np.int32), "potential": np.where(in_density, hartree, 0.0) + vxc, "xc_potential": vxc,
            "hartree_energy": e_h, "xc_energy": math.fsum(energy.ravel().tolist()) * weight,
            "vxc_density": vxc_density, "hartree_stress": stress_h, "xc_stress": stress_xc,
            "sampled_electrons": math.fsum(valence.ravel().tolist()) * weight,
            "minimum_density": float(raw.min()), "clipped_density_points": int((raw < 1e-10).sum()),
            "grid_points": points, "grid": shape}


# --- Collinear spin PBE and functional (src/spin_pbe_xc.cpp:54-107,
#     src/density_functionals.cpp:732-806) ------------------------------------

class _D5:
    """Value and derivatives in five variables (n_up, n_down, sigma_uu, sigma_ud, sigma_dd), per point."""

    def __init__(self, v, g=None):
        self.v = np.asarray(v, dtype=np.float64)
        self.g = np.zeros(self.v.shape + (5,)) if g is None else g

    @staticmethod
    def variable(x, k):
        d = _D5(x)
        d.g[..., k] = 1.0
        return d

    @staticmethod
    def lift(x):
        return x if isinstance(x, _D5) else _D5(np.broadcast_to(np.asarray(x, dtype=np.float64), ()).copy())

    def __add__(self, o):
        o = _D5.lift(o)
        return _D5(self.v + o.v, self.g + o.g)

    __radd__ = __add__

    def __sub__(self, o):
        o = _D5.lift(o)
        return _D5(self.v - o.v, self.g - o.g)

    def __rsub__(self, o):
        return _D5.lift(o) - self

    def __neg__(self):
        return _D5(0.0) - self

    def __mul__(self, o):
        o = _D5.lift(o)
        return _D5(self.v * o.v, self.g * o.v[..., None] + self.v[..., None] * o.g)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = _D5.lift(o)
        r = self.v / o.v
        return _D5(r, (self.g - r[..., None] * o.g) / o.v[..., None])

    def __rtruediv__(self, o):
        return _D5.lift(o) / self

    def pow(self, p):
        r = np.power(self.v, p)
        return _D5(r, (p * r / self.v)[..., None] * self.g)

    def log1p(self):
        return _D5(np.log1p(self.v), self.g / (1.0 + self.v)[..., None])

    def expm1(self):
        r = np.expm1(self.v)
        return _D5(r, (1.0 + r)[..., None] * self.g)


def _pw_spin(rs, a, alpha, b1, b2, b3, b4):
    root = rs.pow(0.5)
    poly = b1 * root + b2 * rs + b3 * rs * root + b4 * rs * rs
    return -2 * a * (1 + alpha * rs) * (1 / (2 * a * poly)).log1p()


def _spin_exchange(n, sigma):
    doubled = 2 * n
    root = doubled.pow(1.0 / 3.0)
    kf = np.cbrt(3 * math.pi * math.pi) * root
    denominator = 4 * kf * kf * doubled * doubled
    numerator = 4 * (_PBE_MU / _PBE_KAPPA) * sigma
    fx = 1 + _PBE_KAPPA * numerator / (denominator + numerator)
    return -.375 * np.cbrt(3 / math.pi) * doubled * root * fx


def pbe_collinear(up, down, gu, gd):
    """(energy density, (v_up, v_down), gradient responses (2, N, 3)) of collinear PBE with
    PW92 spin interpolation for densities up, down > 0 and gradients gu, gd (N, 3)
    (src/spin_pbe_xc.cpp:54-107)."""
    up = np.asarray(up, dtype=np.float64)
    down = np.asarray(down, dtype=np.float64)
    uu = gu[:, 0] * gu[:, 0] + gu[:, 1] * gu[:, 1] + gu[:, 2] * gu[:, 2]
    ud = gu[:, 0] * gd[:, 0] + gu[:, 1] * gd[:, 1] + gu[:, 2] * gd[:, 2]
    dd = gd[:, 0] * gd[:, 0] + gd[:, 1] * gd[:, 1] + gd[:, 2] * gd[:, 2]
    nu, nd = _D5.variable(np.maximum(up, 1e-99), 0), _D5.variable(np.maximum(down, 1e-99), 1)
    su, sud, sd = _D5.variable(uu, 2), _D5.variable(ud, 3), _D5.variable(dd, 4)
    n = nu + nd
    root = n.pow(1.0 / 3.0)
    rs = np.cbrt(3 / (4 * math.pi)) / root
    z = (nu - nd) / n
    z.v = np.clip(z.v, -.9999999999999, .9999999999999)
    z2 = z * z
    z4 = z2 * z2
    pu, pd = 1 + z, 1 - z
    denominator = 0.5198420997897463295
    fzz = 8 / (9 * denominator)
    f = (pu.pow(4.0 / 3.0) + pd.pow(4.0 / 3.0) - 2) / denominator
    eu = _pw_spin(rs, .0310907, .21370, 7.5957, 3.5876, 1.6382, .49294)
    ep = _pw_spin(rs, .01554535, .20548, 14.1189, 6.1977, 3.3662, .62517)
    alpha = -_pw_spin(rs, .0168869, .11125, 10.357, 3.6231, .88026, .49671)
    ec = eu + alpha * f / fzz * (1 - z4) + (ep - eu) * f * z4
    phi = .5 * (pu.pow(2.0 / 3.0) + pd.pow(2.0 / 3.0))
    eta = 1e-12
    gz = (np.power(pu.v * pu.v + eta, -1.0 / 6.0) - np.power(pd.v * pd.v + eta, -1.0 / 6.0)) / 3.0
    phi.g = gz[..., None] * z.g
    phi3 = phi * phi * phi
    sigma = su + 2 * sud + sd
    kf = np.cbrt(3 * math.pi * math.pi) * root
    ks2 = 4 * kf / math.pi
    t2 = sigma / (4 * phi * phi * ks2 * n * n)
    a = (_PBE_BETA / _PBE_GAMMA) / (-ec / (_PBE_GAMMA * phi3)).expm1()
    at = a * t2
    h = _PBE_GAMMA * phi3 * ((_PBE_BETA / _PBE_GAMMA) * t2 * (1 + at) / (1 + at + at * at)).log1p()
    ex = _spin_exchange(nu, su) + _spin_exchange(nd, sd)
    total = ex + n * (ec + h)
    g = total.g
    response = np.stack([2 * g[:, 2:3] * gu + g[:, 3:4] * gd, 2 * g[:, 4:5] * gd + g[:, 3:4] * gu])
    return total.v, (g[:, 0], g[:, 1]), response


def collinear_functionals(lattice, up_keys, up_values, down_keys, down_values, core_keys=None, core_values=None,
                          padding: int = 2, fast: bool = False) -> dict:
    """The reference's evaluate_collinear_density_functionals in numpy: Hartree of the total
    density split equally, per channel the XC fields of n_s + core/2 on the padded grid,
    collinear PBE with the floors max(5e-11, n_s) (both raised to 5e-11 when n_up + n_down
    < 1e-10), tile sums summed exactly, per channel v_xc,s = l_s - i q.d_s on the union
    support and <n_s, v_xc,s>; returns {"hkl", "up": {...}, "down": {...}}."""
    a = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
    det = float(np.dot(a[0], np.cross(a[1], a[2])))
    volume = abs(det)
    if not math.isfinite(volume) or volume < 1e-12 or len(up_keys) == 0 or len(down_keys) == 0:
        raise ValueError("invalid collinear density/lattice")
    b = 2.0 * math.pi / det * np.array([np.cross(a[1], a[2]), np.cross(a[2], a[0]), np.cross(a[0], a[1])])

    def as_map(keys, values):
        return {tuple(int(v) for v in k): complex(x) for k, x in zip(np.asarray(keys).reshape(-1, 3),
                                                                      np.asarray(values).ravel())}

    channels = [as_map(up_keys, up_values), as_map(down_keys, down_values)]
    core = as_map(core_keys, core_values) if core_keys is not None else {}
    total = dict(channels[0])
    for k, v in channels[1].items():
        total[k] = total.get(k, 0.0) + v
    support = sorted(set(channels[0]) | set(channels[1]) | set(core))
    sk = np.array(support, dtype=np.int64).reshape(-1, 3)
    q = sk[:, 0:1] * b[0] + sk[:, 1:2] * b[1] + sk[:, 2:3] * b[2]
    q2 = (q * q).sum(axis=1)
    in_total = np.array([k in total for k in support])
    rho_total = np.array([total.get(k, 0.0) for k in support], dtype=np.complex128)
    coulomb = in_total & ~(q2 < 1e-12)
    norm = rho_total.real ** 2 + rho_total.imag ** 2
    hartree = np.where(coulomb, 4 * math.pi * rho_total / np.where(coulomb, q2, 1.0), 0.0)
    eh = math.fsum((2 * math.pi * volume * norm[coulomb] / q2[coulomb]).tolist())
    sh = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            sh[i, j] = math.fsum((4 * math.pi * norm[coulomb] * q[coulomb, i] * q[coulomb, j]
                                  / (q2[coulomb] * q2[coulomb])).tolist())
    sh -= np.eye(3) * (eh / volume)
    m = np.abs(sk).max(axis=0)
    shape = tuple(padding * max(3, 2 * int(v) + 1) for v in m)
    if fast:
        shape = tuple(fast_fft_length(v) for v in shape)
    idx = tuple(np.mod(sk[:, a_], shape[a_]) for a_ in range(3))
    fields = []
    for s in range(2):
        xc = np.array([channels[s].get(k, 0.0) + (0.5 * core[k] if k in core else 0.0) for k in support],
                      dtype=np.complex128)
        grids = np.zeros((4,) + shape, dtype=np.complex128)
        grids[0][idx] = xc
        for axis in range(3):
            grids[axis + 1][idx] = 1j * q[:, axis] * xc
        fields.append([backward_fft(g).real for g in grids])
    raw = [fields[s][0].ravel() for s in range(2)]
    grad = [np.stack([fields[s][1].ravel(), fields[s][2].ravel(), fields[s][3].ravel()], axis=1) for s in range(2)]
    n = [raw[0].copy(), raw[1].copy()]
    low = n[0] + n[1] < 1e-10
    n[0] = np.where(low, np.maximum(n[0], 5e-11), n[0])
    n[1] = np.where(low, np.maximum(n[1], 5e-11), n[1])
    energy, potentials, response = pbe_collinear(np.maximum(5e-11, n[0]), np.maximum(5e-11, n[1]), grad[0], grad[1])
    points = int(np.prod(shape))
    pressure = energy.copy()
    for s in range(2):
        pressure = pressure - potentials[s] * raw[s]
        for ax in range(3):
            pressure = pressure - response[s][:, ax] * grad[s][:, ax]
    stress = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            term = (pressure if i == j else 0.0) - response[0][:, i] * grad[0][:, j] - response[1][:, i] * grad[1][:, j]
            stress[i, j] = math.fsum(np.ravel(term).tolist())
    e_sum = math.fsum(energy.tolist())
    where = {k: i for i, k in enumerate(support)}
    out = {"hkl": sk.astype(np.int32)}
    for s, name in enumerate(("up", "down")):
        transforms = [forward_fft(f.reshape(shape))[idx] / points
                      for f in (potentials[s], response[s][:, 0], response[s][:, 1], response[s][:, 2])]
        vxc = transforms[0] - 1j * (q[:, 0] * transforms[1] + q[:, 1] * transforms[2] + q[:, 2] * transforms[3])
        rho = channels[s]
        vxc_density = math.fsum(volume * (rho[k] * vxc[where[(-k[0], -k[1], -k[2])]]).real
                                for k in support if k in rho and (-k[0], -k[1], -k[2]) in where)
        out[name] = {"hkl": sk.astype(np.int32), "potential": hartree + vxc, "xc_potential": vxc,
                     "hartree_energy": .5 * eh, "hartree_stress": .5 * sh, "xc_energy": .5 * e_sum * volume / points,
                     "xc_stress": .5 * stress / points, "vxc_density": vxc_density,
                     "sampled_electrons": volume * rho[(0, 0, 0)].real if (0, 0, 0) in rho else 0.0,
                     "minimum_density": float(raw[s].min()), "clipped_density_points": int((raw[s] < 0).sum()),
                     "grid_points": points, "grid": shape}
    return out
