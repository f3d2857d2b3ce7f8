"""Seeded synthetic inputs for the twisted-mass solver workloads.

Gauge recipe: every link is U = exp(i*eps*H) with H a Gaussian traceless
Hermitian 3x3 matrix laid out as the reference's herm_put_to_gauss builds it
(base/random.hpp:311-341 with sigma=1: eight Gaussians r of standard
deviation 1/sqrt2 as rnd_get_gauss_complex draws them, random.hpp:183-199;
diagonal r2+r7/sqrt3,
-r2+r7/sqrt3, -2r7/sqrt3, off-diagonal (r0,r1), (r3,r4), (r5,r6)).  The
random numbers come from numpy's Philox generator (not the reference's ran2),
so a given seed defines the configuration for this package only; the same
arrays are handed to every implementation that is compared.  After the
exponential the link is projected back onto SU(3) (Gram-Schmidt of rows 0-1,
row 2 = conj(row0 x row1)) so that it is special-unitary to rounding.

Sources: point (one spin-colour at one site) and Z2 noise with entries
(+-1 +- i)/sqrt(2).  All arrays are float64 in the reference's CPU layout:
conf (V, 4, 3, 3, 2), spinor (V, 4, 3, 2), lx site order t,x,y,z (z fastest).
"""
from __future__ import annotations

import numpy as np

SQRT3_INV = 1.0 / np.sqrt(3.0)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


def hermitian_gauss(n: int, rng: np.random.Generator) -> np.ndarray:
    """n Gaussian traceless Hermitian matrices, complex128 (n, 3, 3)."""
    r = rng.standard_normal((8, n)) * np.sqrt(0.5)
    H = np.zeros((n, 3, 3), np.complex128)
    H[:, 0, 0] = r[2] + SQRT3_INV * r[7]
    H[:, 1, 1] = -r[2] + SQRT3_INV * r[7]
    H[:, 2, 2] = -2 * SQRT3_INV * r[7]
    H[:, 1, 0] = r[0] + 1j * r[1]
    H[:, 0, 1] = r[0] - 1j * r[1]
    H[:, 2, 0] = r[3] + 1j * r[4]
    H[:, 0, 2] = r[3] - 1j * r[4]
    H[:, 2, 1] = r[5] + 1j * r[6]
    H[:, 1, 2] = r[5] - 1j * r[6]
    return H


def project_su3(U: np.ndarray) -> np.ndarray:
    """Rows 0,1 orthonormalised, row 2 = conj(row0 x row1): exactly SU(3) to rounding."""
    a = U[..., 0, :]
    a = a / np.sqrt(np.sum(np.abs(a) ** 2, axis=-1, keepdims=True))
    b = U[..., 1, :]
    b = b - np.sum(a.conj() * b, axis=-1, keepdims=True) * a
    b = b / np.sqrt(np.sum(np.abs(b) ** 2, axis=-1, keepdims=True))
    c = np.conj(np.cross(a, b))
    return np.stack([a, b, c], axis=-2)


def expi_hermitian(H: np.ndarray, eps: float, chunk: int = 1 << 20) -> np.ndarray:
    """exp(i*eps*H) by the spectral decomposition of the Hermitian H, in chunks."""
    out = np.empty_like(H)
    for s in range(0, H.shape[0], chunk):
        w, v = np.linalg.eigh(H[s:s + chunk])
        out[s:s + chunk] = (v * np.exp(1j * eps * w)[:, None, :]) @ v.conj().transpose(0, 2, 1)
    return out


def _expi_project_torch(H: np.ndarray, eps: float, device: str, chunk: int = 1 << 21) -> np.ndarray:
    """exp(i*eps*H) by scaling and squaring of its Taylor series (2^-4 scaling,
    order 14: truncation far below rounding for |eps*H| < 4) and the SU(3)
    projection, on a CUDA device.  Agrees with expi_hermitian to rounding."""
    import torch
    out = np.empty_like(H)
    eye = torch.eye(3, dtype=torch.complex128, device=device)
    for s in range(0, H.shape[0], chunk):
        a = torch.from_numpy(H[s:s + chunk]).to(device) * (1j * eps / 16.0)
        term = eye.expand_as(a).clone()
        u = term.clone()
        for k in range(1, 15):
            term = term @ a / k
            u = u + term
        for _ in range(4):
            u = u @ u
        r0 = u[:, 0, :]
        r0 = r0 / torch.sqrt(torch.sum(torch.abs(r0) ** 2, dim=-1, keepdim=True))
        r1 = u[:, 1, :]
        r1 = r1 - torch.sum(r0.conj() * r1, dim=-1, keepdim=True) * r0
        r1 = r1 / torch.sqrt(torch.sum(torch.abs(r1) ** 2, dim=-1, keepdim=True))
        r2 = torch.conj(torch.linalg.cross(r0, r1, dim=-1))
        out[s:s + chunk] = torch.stack([r0, r1, r2], dim=-2).cpu().numpy()
    return out


def gauge_conf(T: int, L: int, eps: float, seed: int, device: str | None = None) -> np.ndarray:
    """Periodic (no boundary sign) SU(3) links, float64 (V, 4, 3, 3, 2).

    With device='cuda' the exponentials are taken on the GPU (torch), which
    is much faster for large lattices; the Gaussian draws are the same."""
    V = T * L ** 3
    rng = _rng(seed)
    H = hermitian_gauss(V * 4, rng)
    if device is not None and str(device).startswith("cuda"):
        U = _expi_project_torch(H, eps, device)
    else:
        U = project_su3(expi_hermitian(H, eps))
    return np.ascontiguousarray(U.view(np.float64).reshape(V, 4, 3, 3, 2))


def apply_time_bc(conf: np.ndarray, T: int, L: int, sign: float = -1.0) -> np.ndarray:
    """Fold a time boundary sign into the t=T-1 time links (the form in which the
    reference's operators, which read links as given, see antiperiodic time)."""
    c = conf.reshape(T, L ** 3, 4, 3, 3, 2).copy()
    c[T - 1, :, 0] *= sign
    return c.reshape(conf.shape)


def point_source(T: int, L: int, site: int = 0, spin: int = 0, col: int = 0) -> np.ndarray:
    s = np.zeros((T * L ** 3, 4, 3, 2))
    s[site, spin, col, 0] = 1.0
    return s


def z2_source(T: int, L: int, seed: int, spin: int | None = None, col: int | None = None) -> np.ndarray:
    """Z2 noise (+-1 +- i)/sqrt2 on every site; restricted to one spin and/or colour if given."""
    V = T * L ** 3
    rng = _rng(seed)
    bits = rng.integers(0, 2, size=(V, 4, 3, 2)).astype(np.float64)
    s = (2 * bits - 1) / np.sqrt(2.0)
    if spin is not None:
        mask = np.zeros((1, 4, 1, 1))
        mask[0, spin] = 1
        s = s * mask
    if col is not None:
        mask = np.zeros((1, 1, 3, 1))
        mask[0, :, col] = 1
        s = s * mask
    return np.ascontiguousarray(s)


def random_spinor(n_sites: int, seed: int) -> np.ndarray:
    return np.ascontiguousarray(_rng(seed).standard_normal((n_sites, 4, 3, 2)))
