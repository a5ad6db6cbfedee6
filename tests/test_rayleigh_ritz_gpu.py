"""Device Rayleigh-Ritz eigensolver (the reference's rayleigh_ritz,
src/pw_core.cpp:56-136) against the dense FP64 oracle: eigenvalues, residuals
||H y - e S y|| and S-orthonormality, on the paths the Davidson solve takes
(S = I exactly, S within 1e-6 of I, S far from I), with degenerate spectra and
at the largest Davidson subspace (160 roots: 1280)."""
import numpy as np
import pytest

from oracle import sdft_oracle

pytestmark = pytest.mark.gpu


def random_unitary(n, rng):
    q, r = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def pencil(n, rng, spectrum=None, overlap=0.0):
    u = random_unitary(n, rng)
    lam = np.sort(rng.uniform(-2.0, 30.0, n)) if spectrum is None else spectrum
    h = (u * lam) @ u.conj().T
    h = 0.5 * (h + h.conj().T)
    e = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = np.eye(n) + overlap * 0.5 * (e + e.conj().T) / np.sqrt(n)
    return h, s


def check(context, h, s, requested, eig_tol=1e-11, res_tol=1e-11):
    from sdft_b200.operator import rayleigh_ritz
    values, vectors = rayleigh_ritz(context, np.tril(h), np.tril(s), requested)
    count = requested or h.shape[0]
    expected = sdft_oracle.generalized_eigenvalues(h, s, count)
    scale = max(1.0, np.max(np.abs(expected)))
    assert np.max(np.abs(values - expected)) < eig_tol * scale
    residual = h @ vectors - (s @ vectors) * values[None, :]
    assert np.max(np.linalg.norm(residual, axis=0)) < res_tol * scale
    gram = vectors.conj().T @ s @ vectors
    assert np.max(np.abs(gram - np.eye(count))) < 1e-11


@pytest.mark.parametrize("n,requested", [(2, 0), (37, 10), (320, 0), (800, 320), (7, 3), (9, 0), (31, 15), (65, 0),
                                         (129, 0)])
def test_identity_overlap(context, n, requested):
    """Odd orders with an odd number of wanted pairs included: the workspace
    keeps its complex arrays 16-byte aligned whatever m * wanted is."""
    rng = np.random.Generator(np.random.PCG64(n))
    h, s = pencil(n, rng)
    check(context, h, s, requested)


@pytest.mark.parametrize("overlap", [1e-9, 5e-7, 3e-6])
def test_near_identity_overlap_uses_loewdin(context, overlap):
    rng = np.random.Generator(np.random.PCG64(11))
    h, s = pencil(500, rng, overlap=overlap)
    check(context, h, s, 160)


def test_far_from_identity_overlap_falls_back(context):
    rng = np.random.Generator(np.random.PCG64(12))
    h, s = pencil(300, rng, overlap=0.2)
    check(context, h, s, 100)


def test_degenerate_and_clustered_spectrum(context):
    rng = np.random.Generator(np.random.PCG64(13))
    n = 640
    lam = np.sort(np.concatenate([np.repeat([-1.0, 0.5, 2.0], [3, 6, 2]), [3.0, 3.0 + 1e-13, 3.0 + 4e-12],
                                  rng.uniform(4.0, 40.0, n - 14)]))
    h, s = pencil(n, rng, spectrum=lam)
    check(context, h, s, 320)


def test_largest_davidson_subspace(context):
    rng = np.random.Generator(np.random.PCG64(14))
    h, s = pencil(1280, rng, overlap=1e-10)
    check(context, h, s, 320)


def test_davidson_shaped_pencil(context):
    """Thick-restart shape: a diagonal block of Ritz values coupled to a new block."""
    rng = np.random.Generator(np.random.PCG64(15))
    k0, n = 320, 480
    h = np.zeros((n, n), dtype=complex)
    h[:k0, :k0] = np.diag(np.sort(rng.uniform(-0.5, 2.0, k0)))
    c = 1e-3 * (rng.standard_normal((k0, n - k0)) + 1j * rng.standard_normal((k0, n - k0)))
    h[:k0, k0:] = c
    h[k0:, :k0] = c.conj().T
    d = rng.standard_normal((n - k0, n - k0)) + 1j * rng.standard_normal((n - k0, n - k0))
    h[k0:, k0:] = 0.5 * (d + d.conj().T) + 5.0 * np.eye(n - k0)
    check(context, h, np.eye(n), 320)
