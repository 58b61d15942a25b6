"""Poisson negative log-likelihood of ROI images and its gradient: the float64 oracle (test infrastructure only).

The reference has no gradient (its nearest relative is DescribePsfCramerRao's central-difference PSF derivatives,
adapter/inSiliScope/Simulation/PsfGeneratorBridge.cpp:1554-1669), so this model is the contract the GPU adjoint is
checked against, pinned by float64 central differences (tests/test_oracle.py). Its PSF physics is the reference's
Gibson-Lanni/Zernike pupil (ZernikePsf.cpp:188-248) at matched immersion/sample indices and depth 0, evaluated at a
continuous defocus and position:

- pupil grid: k_i = (i - M/2) dk, i < M, dk = 2 kMax / (M - 4), kMax = 2 pi NA / lambda (ZernikePsf.cpp:192-193);
  aperture a = 1 where kx^2 + ky^2 <= kMax^2;
- phase: phi = z kz + 2 pi sum_j c_j Z_j(rho, theta) - p (kx x + ky y), with kz = sqrt((2 pi n / lambda)^2 - k^2)
  (the Gibson-Lanni defocus term k0 ni dt cos(theta_i) at depth 0), rho = k / kMax, Z_j Noll's orthonormal
  Zernike polynomials (j = 4..24: coefficients in waves rms), p the pixel size (nm), (x, y) the emitter in ROI
  pixels, z its defocus (nm);
- field at sub-pixel sample (u_s, v_t) = ((s + 0.5) / os, (t + 0.5) / os) px: E = A U A^T with
  A[s][m] = exp(i k_m p u_s), U = a exp(i phi) (the separable DFT the chirp-Z evaluates);
- expected counts mu[i][j] = N kappa sum over the os x os samples of pixel (i, j) of |E|^2 + b_frame, with
  kappa = (p / os)^2 / (L^2 sum a), L = 2 pi / dk the field's period (Parseval: a PSF integrates to 1 per period);
- NLL = sum over every ROI pixel of mu - k log mu.

Gradient (adjoint): w = 1 - k / mu; G = w N kappa per sample; U_bar = A^H (G o E) conj(A); dNLL/dphi = -2 Im(conj(U_bar)
U); then dphi/dz = kz, dphi/dx = -p kx, dphi/dy = -p ky, dphi/dc_j = 2 pi Z_j; dNLL/dN = sum w PSF; dNLL/db = sum w.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from math import factorial

import numpy as np


@dataclass
class NllSpec:
    wavelength_nm: float = 670.0
    na: float = 1.45
    n_imm: float = 1.518
    pixel_nm: float = 108.0
    roi: int = 32
    os: int = 2
    pupil: int = 32
    noll: tuple = tuple(range(4, 25))


def noll_nm(j: int):
    """Noll's index j >= 1 -> (n, m), m < 0 for the sine modes."""
    n, j1 = 0, j - 1
    while j1 > n:
        n += 1
        j1 -= n
    m = (-1) ** j * ((n % 2) + 2 * ((j1 + ((n + 1) % 2)) // 2))
    return n, m


def zernike_noll(j: int, rho: np.ndarray, theta: np.ndarray) -> np.ndarray:
    """Noll's orthonormal Z_j on the unit disc: sqrt(2 (n + 1)) R_n^|m| cos / sin(|m| theta), sqrt(n + 1) R_n^0."""
    n, m = noll_nm(j)
    am = abs(m)
    r = np.zeros_like(rho)
    for s in range((n - am) // 2 + 1):
        c = (-1) ** s * factorial(n - s) / (factorial(s) * factorial((n + am) // 2 - s) * factorial((n - am) // 2 - s))
        r = r + c * rho ** (n - 2 * s)
    if m == 0:
        return np.sqrt(n + 1.0) * r
    return np.sqrt(2.0 * (n + 1)) * r * (np.cos(am * theta) if m > 0 else np.sin(am * theta))


@dataclass
class NllTables:
    kx: np.ndarray      # (M, M) rad/nm
    ky: np.ndarray
    kz: np.ndarray      # rad/nm, 0 outside the aperture
    a: np.ndarray       # aperture (M, M)
    Z: np.ndarray       # (J, M, M) Noll basis, 0 outside
    A: np.ndarray       # (P, M) complex128
    kappa: float


def tables(spec: NllSpec) -> NllTables:
    M, P = spec.pupil, spec.roi * spec.os
    kmax = 2.0 * np.pi * spec.na / spec.wavelength_nm
    dk = 2.0 * kmax / (M - 4)
    k = (np.arange(M) - M // 2) * dk
    ky, kx = np.meshgrid(k, k, indexing="ij")
    kr2 = kx * kx + ky * ky
    a = (kr2 <= kmax * kmax).astype(np.float64)
    k0n = 2.0 * np.pi * spec.n_imm / spec.wavelength_nm
    kz = np.where(a > 0, np.sqrt(np.maximum(0.0, k0n * k0n - kr2)), 0.0)
    rho = np.sqrt(kr2) / kmax
    theta = np.arctan2(ky, kx)
    Z = np.stack([np.where(a > 0, zernike_noll(j, rho, theta), 0.0) for j in spec.noll])
    u = (np.arange(P) + 0.5) / spec.os
    A = np.exp(1j * np.outer(u * spec.pixel_nm, k))
    L = 2.0 * np.pi / dk
    kappa = (spec.pixel_nm / spec.os) ** 2 / (L * L * a.sum())
    return NllTables(kx, ky, kz, a, Z, A, kappa)


def _fields(t: NllTables, spec: NllSpec, params: np.ndarray, zern: np.ndarray):
    """U (n, M, M) and E (n, P, P) of each emitter."""
    x, y, z = params[:, 0], params[:, 1], params[:, 2]
    zp = 2.0 * np.pi * np.tensordot(zern, t.Z, axes=(0, 0))
    phi = (z[:, None, None] * t.kz + zp[None] - spec.pixel_nm * (t.kx[None] * x[:, None, None] +
                                                                   t.ky[None] * y[:, None, None]))
    U = t.a[None] * np.exp(1j * phi)
    E = np.matmul(np.matmul(t.A, U), t.A.T)
    return U, E


def _pixels(q: np.ndarray, spec: NllSpec) -> np.ndarray:
    n, R, os_ = q.shape[0], spec.roi, spec.os
    return q.reshape(n, R, os_, R, os_).sum(axis=(2, 4))


def expected(spec: NllSpec, params, frame, bg, zern, t: NllTables | None = None):
    """mu (n, R, R): N PSF + b of each emitter's ROI."""
    t = t or tables(spec)
    params = np.asarray(params, np.float64)
    _, E = _fields(t, spec, params, np.asarray(zern, np.float64))
    psf = t.kappa * _pixels(np.abs(E) ** 2, spec)
    return params[:, 3, None, None] * psf + np.asarray(bg, np.float64)[np.asarray(frame)][:, None, None]


def nll(spec: NllSpec, params, frame, bg, zern, counts, t: NllTables | None = None) -> float:
    mu = expected(spec, params, frame, bg, zern, t)
    k = np.asarray(counts, np.float64)
    return float(np.sum(mu - k * np.log(mu)))


def gradient(spec: NllSpec, params, frame, bg, zern, counts, t: NllTables | None = None):
    """(nll, d/dparams (n, 4), d/dbg (F,), d/dzern (J,)) by the adjoint, float64."""
    t = t or tables(spec)
    params = np.asarray(params, np.float64)
    frame = np.asarray(frame)
    bg = np.asarray(bg, np.float64)
    zern = np.asarray(zern, np.float64)
    k = np.asarray(counts, np.float64)
    U, E = _fields(t, spec, params, zern)
    I = np.abs(E) ** 2
    psf = t.kappa * _pixels(I, spec)
    N = params[:, 3]
    mu = N[:, None, None] * psf + bg[frame][:, None, None]
    w = 1.0 - k / mu
    value = float(np.sum(mu - k * np.log(mu)))
    g = np.zeros_like(params)
    g[:, 3] = np.sum(w * psf, axis=(1, 2))
    gb = np.zeros_like(bg)
    np.add.at(gb, frame, np.sum(w, axis=(1, 2)))
    G = np.repeat(np.repeat(w, spec.os, axis=1), spec.os, axis=2) * (N * t.kappa)[:, None, None]
    Ubar = np.matmul(np.matmul(np.conj(t.A).T, G * E), np.conj(t.A))
    dphi = -2.0 * np.imag(np.conj(Ubar) * U)
    g[:, 0] = -spec.pixel_nm * np.sum(dphi * t.kx[None], axis=(1, 2))
    g[:, 1] = -spec.pixel_nm * np.sum(dphi * t.ky[None], axis=(1, 2))
    g[:, 2] = np.sum(dphi * t.kz[None], axis=(1, 2))
    gz = 2.0 * np.pi * np.tensordot(dphi.sum(axis=0), t.Z, axes=([0, 1], [1, 2]))
    return value, g, gb, gz
