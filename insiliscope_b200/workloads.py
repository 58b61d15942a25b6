"""Seeded synthetic workloads with the shapes of the engine's benchmark configurations.

Every random property is a pure function of (seed, address) through the engine's own pcg4d hash
(core/src/rng.h:37-41 HashUnit): static site properties at pcg4d(seed ^ salt, site, 0, purpose), per-frame properties
at pcg4d(seed, site, frame, purpose) -- the DYE_CH-style channel scheme of the reference's world core
(core/src/dyes.h:33-57). Camera maps come from std::mt19937_64(seed) in the order offset, gain, read noise and the
noise stream from seed ^ 0x9E3779B9, as the reference's movie setup does (ScopeMovie.cpp:980-988).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .engine import BLINK_EVENT_DTYPE, EMITTER_DTYPE, FRAME_DTYPE, INTERP_CUBIC, CameraParams, PsfParams

SITE_SALT = 0x5157E5
M32 = np.uint64(0xFFFFFFFF)


def pcg4d(a, b, c, d):
    """Vectorized pcg4d (SMLMCounterRng.h:37-56) on uint32 arrays."""
    a, b, c, d = (np.asarray(x, dtype=np.uint64) & M32 for x in np.broadcast_arrays(a, b, c, d))
    mul, inc = np.uint64(1664525), np.uint64(1013904223)
    a = (a * mul + inc) & M32
    b = (b * mul + inc) & M32
    c = (c * mul + inc) & M32
    d = (d * mul + inc) & M32
    for rnd in range(2):
        a = (a + b * d) & M32
        b = (b + c * a) & M32
        c = (c + a * b) & M32
        d = (d + b * c) & M32
        if rnd == 0:
            a ^= a >> np.uint64(16)
            b ^= b >> np.uint64(16)
            c ^= c >> np.uint64(16)
            d ^= d >> np.uint64(16)
    return a, b, c, d


def hash_unit(seed, cx, cy, k):
    """HashUnit (core/src/rng.h:37-41): ((pcg4d(...).a >> 9) + 0.5) * 2^-23."""
    a = pcg4d(seed, cx, cy, k)[0]
    return ((a >> np.uint64(9)).astype(np.float64) + 0.5) * 1.1920928955078125e-7


def hash_normal(seed, cx, cy, k0):
    u1 = hash_unit(seed, cx, cy, k0)
    u2 = hash_unit(seed, cx, cy, k0 + 1)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


@dataclass
class SmlmMovie:
    """A blink movie: events in frame order with per-frame buckets, and what renders it."""
    width: int
    height: int
    frames: int
    pixel_nm: float
    photons_per_blink: float
    background: float
    events: np.ndarray          # BLINK_EVENT_DTYPE, frame-major
    bucket_start: np.ndarray    # frames + 1 offsets into events
    psf: PsfParams
    camera: CameraParams
    map_seed: int
    offset_mean: float
    offset_std: float
    gain_nominal: float
    gain_std_fraction: float
    read_noise_nominal: float
    read_noise_std_fraction: float
    noise_seed: int

    @property
    def n_events(self) -> int:
        return len(self.events)


def smlm_dstorm(seed: int = 42, sites: int = 4000, frames: int = 200, size: int = 128, pixel_nm: float = 108.0,
                p_on: float = 0.04, median_photons: float = 2000.0, sigma_log: float = 0.5, z_half_nm: float = 600.0,
                frame0: int = 0) -> SmlmMovie:
    """The plain dSTORM movie: 128 x 128 px sCMOS at 108 nm, 200 frames, 4,000 sites uniform over the field with
    z uniform in [-600, 600] nm, each ON in a frame with probability 0.04 (about 160 per frame), photons lognormal
    (median 2000, sigma_log 0.5); background 20 photons/px; Gibson-Lanni PSF, NA 1.45 oil, 670 nm, 64 x 64 pupil,
    chirp-Z to a 4x-oversampled 32 x 32 px kernel (129^2 samples), 49 planes 25 nm apart, Catmull-Rom splat; offset
    N(100, 2) ADU, gain N(2.2, 0.1) e-/ADU, read noise N(1.5, 0.3) e-; QE 1."""
    s = np.arange(sites, dtype=np.uint64)
    st = np.uint64((seed ^ SITE_SALT) & 0xFFFFFFFF)
    x_px = size * hash_unit(st, s, 0, 0)
    y_px = size * hash_unit(st, s, 0, 1)
    z_nm = -z_half_nm + 2.0 * z_half_nm * hash_unit(st, s, 0, 2)
    f = np.arange(frame0, frame0 + frames, dtype=np.uint64)
    F, S = np.meshgrid(f, s, indexing="ij")
    on = hash_unit(seed, S, F, 0) < p_on
    photons = median_photons * np.exp(sigma_log * hash_normal(seed, S, F, 1))
    fi, si = np.nonzero(on)                     # frame-major, site order within a frame
    ev = np.zeros(len(fi), BLINK_EVENT_DTYPE)
    ev["x_um"] = x_px[si] * (pixel_nm / 1000.0)
    ev["y_um"] = y_px[si] * (pixel_nm / 1000.0)
    ev["z_nm"] = z_nm[si]
    ev["t_start"] = (frame0 + fi).astype(np.float64)
    ev["t_end"] = ev["t_start"] + 1.0
    ev["brightness"] = photons[fi, si] / median_photons
    ev["excite"] = 1.0
    counts = np.bincount(fi, minlength=frames)
    bucket = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    psf = PsfParams(wavelength_nm=670.0, na=1.45, immersion_index=1.518, sample_index=1.518,
                    working_distance_um=150.0, sample_depth_nm=0.0, pixel_size_nm=pixel_nm, oversampling=4,
                    kernel_half_width_px=16, nz=49, z_step_nm=25.0, pupil_samples=64, interp=INTERP_CUBIC)
    cam = CameraParams(quantum_efficiency=1.0, dark_electrons=0.0, gain=2.2, read_noise_e=1.5, emccd=False)
    return SmlmMovie(size, size, frames, pixel_nm, median_photons, 20.0, ev, bucket, psf, cam, seed, 100.0, 2.0, 2.2,
                     0.1 / 2.2, 1.5, 0.2, (seed ^ 0x9E3779B9) & 0xFFFFFFFF)


@dataclass
class BinnedMovie:
    """Frames of the binned blink regime: each frame's emitters as CollectFrameEmitters leaves them (position in
    pixels, detected photons, z plane), frame-major."""
    width: int
    height: int
    n_frames: int
    pixel_nm: float
    upscale: int
    psf: PsfParams
    camera: CameraParams
    emitters: np.ndarray        # EMITTER_DTYPE
    frames: np.ndarray          # FRAME_DTYPE
    noise_seed: int


def binned_dense(seed: int = 42, sites: int = 60000, frames: int = 200, size: int = 128, pixel_nm: float = 108.0,
                 p_on: float = 0.04, median_photons: float = 2000.0, sigma_log: float = 0.5, z_half_nm: float = 600.0,
                 upscale: int = 2) -> BinnedMovie:
    """Dense blink frames for the binned regime: 128 x 128 px at 108 nm, 60,000 sites uniform over the field (z
    uniform in [-600, 600] nm), each ON in a frame with probability 0.04 -- about 2,400 per frame, 12.7 per um^2, just
    above the density at which the reference switches to binned (12.5 per um^2) -- photons lognormal (median 2000,
    sigma_log 0.5); the SMLM movie's PSF kernel (oversampling 4, 49 planes 25 nm apart, plane = the nearest, as
    NearestZIndex rounds), u = 2 cells per pixel; EMCCD camera (gain 300, read noise 50 e-, CIC 0.002)."""
    s = np.arange(sites, dtype=np.uint64)
    st = np.uint64((seed ^ SITE_SALT) & 0xFFFFFFFF)
    x_px = size * hash_unit(st, s, 0, 0)
    y_px = size * hash_unit(st, s, 0, 1)
    z_nm = -z_half_nm + 2.0 * z_half_nm * hash_unit(st, s, 0, 2)
    plane = np.clip(np.floor(z_nm / 25.0 + 24.0 + 0.5), 0, 48).astype(np.int32)
    f = np.arange(frames, dtype=np.uint64)
    F, S = np.meshgrid(f, s, indexing="ij")
    on = hash_unit(seed, S, F, 0) < p_on
    fi, si = np.nonzero(on)
    em = np.zeros(len(fi), EMITTER_DTYPE)
    em["x_px"] = x_px[si] - 0.5   # pixel centres at integers: the camera's pixel x spans [x - 0.5, x + 0.5)
    em["y_px"] = y_px[si] - 0.5
    em["photons"] = median_photons * np.exp(sigma_log * hash_normal(seed, S[fi, si], F[fi, si], 1))
    em["plane"] = plane[si]
    counts = np.bincount(fi, minlength=frames)
    fr = np.zeros(frames, FRAME_DTYPE)
    fr["em_start"] = np.concatenate([[0], np.cumsum(counts)[:-1]])
    fr["em_count"] = counts
    fr["frame"] = np.arange(frames)
    fr["bg_scale"] = 1.0
    psf = PsfParams(wavelength_nm=670.0, na=1.45, immersion_index=1.518, sample_index=1.518,
                    working_distance_um=150.0, sample_depth_nm=0.0, pixel_size_nm=pixel_nm, oversampling=4,
                    kernel_half_width_px=16, nz=49, z_step_nm=25.0, pupil_samples=64, interp=INTERP_CUBIC)
    cam = CameraParams(quantum_efficiency=1.0, gain=1.0, read_noise_e=50.0, emccd=True, em_gain=300.0,
                       cic_electrons=0.002, bit_depth=16)
    return BinnedMovie(size, size, frames, pixel_nm, upscale, psf, cam, em, fr, (seed ^ 0x9E3779B9) & 0xFFFFFFFF)


@dataclass
class TwoColourMovie(SmlmMovie):
    """A blink movie of several dye groups: an event's `slot` is its group, each group with its own PSF kernel;
    within a frame's bucket the groups come one after the other, as the engine renders them."""
    psfs: list = None           # PsfParams per group (psf is psfs[0])
    frame_mean: np.ndarray = None   # each frame's Poisson mean


def two_colour_uneven(seed: int = 42, frames: int = 1024, size: int = 256, pixel_nm: float = 108.0,
                      median_mean: float = 300.0, sigma_log_mean: float = 1.0, mean_clip=(10.0, 8000.0),
                      median_photons: float = 2000.0, sigma_log: float = 0.5, z_half_nm: float = 600.0,
                      frame0: int = 0) -> TwoColourMovie:
    """The uneven two-colour movie: 256 x 256 px sCMOS at 108 nm, 1,024 frames. Frame f carries Poisson(mu_f) ON
    emitters, mu_f lognormal (median 300, sigma_log 1) clipped to [10, 8000]; each emitter uniform over the field,
    z uniform in [-600, 600] nm, in channel 0 or 1 with probability 1/2, photons lognormal (median 2000, sigma_log
    0.5). Channel 0: 670 nm with the double-helix phase mask; channel 1: 580 nm astigmatic (Noll 5 = 0.1 lambda rms).
    Both NA 1.45 oil, 64 x 64 pupil, 4x-oversampled 32 x 32 px kernels of 49 planes 25 nm apart, Catmull-Rom; the
    camera as the plain dSTORM movie's. Counts and properties come from numpy's PCG64 seeded with `seed`."""
    rng = np.random.default_rng(seed)
    mu = np.clip(median_mean * np.exp(sigma_log_mean * rng.standard_normal(frames)), *mean_clip)
    counts = rng.poisson(mu)
    n = int(counts.sum())
    fi = np.repeat(np.arange(frames), counts)
    ch = (rng.random(n) < 0.5).astype(np.int32)
    order = np.lexsort((ch, fi))            # frame-major, channel 0 before channel 1, draw order within
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = size * rng.random(n) * (pixel_nm / 1000.0)
    ev["y_um"] = size * rng.random(n) * (pixel_nm / 1000.0)
    ev["z_nm"] = -z_half_nm + 2.0 * z_half_nm * rng.random(n)
    ev["brightness"] = np.exp(sigma_log * rng.standard_normal(n))
    ev["t_start"] = (frame0 + fi).astype(np.float64)
    ev["t_end"] = ev["t_start"] + 1.0
    ev["excite"] = 1.0
    ev["slot"] = ch
    ev = ev[order]
    bucket = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    common = dict(na=1.45, immersion_index=1.518, sample_index=1.518, working_distance_um=150.0, sample_depth_nm=0.0,
                  pixel_size_nm=pixel_nm, oversampling=4, kernel_half_width_px=16, nz=49, z_step_nm=25.0,
                  pupil_samples=64, interp=INTERP_CUBIC)
    dh = PsfParams(wavelength_nm=670.0, double_helix=True, **common)
    astig = PsfParams(wavelength_nm=580.0, zernike=noll_rms_to_osa_waves({5: 0.1}), **common)
    cam = CameraParams(quantum_efficiency=1.0, dark_electrons=0.0, gain=2.2, read_noise_e=1.5, emccd=False)
    return TwoColourMovie(size, size, frames, pixel_nm, median_photons, 20.0, ev, bucket, dh, cam, seed, 100.0, 2.0,
                          2.2, 0.1 / 2.2, 1.5, 0.2, (seed ^ 0x9E3779B9) & 0xFFFFFFFF, [dh, astig], mu)


@dataclass
class WidefieldVolume:
    """A dye volume and what renders its focus series."""
    density: np.ndarray         # (nz, ny, nx) float32, photons per voxel per frame at focus
    voxel_nm: tuple
    psf: PsfParams              # the 3D PSF's request (planes at voxel z pitch)
    psf_shape: tuple            # (kz, ky, kx)
    psf_defocus_nm: np.ndarray  # the kz planes' defocus
    camera: CameraParams
    background: float
    map_seed: int
    offset_mean: float
    offset_std: float
    noise_seed: int


def widefield_cells(seed: int = 42, nx: int = 512, ny: int = 512, nz: int = 64, voxel_nm=(100.0, 100.0, 200.0),
                    cells: int = 50, filaments: int = 200, steps: int = 60, photons_per_dye: float = 0.4,
                    kernel_shape=None) -> WidefieldVolume:
    """The widefield mean-field volume: nx x ny x nz voxels of 100 x 100 x 200 nm holding `cells` random ellipsoidal
    cells (axes 5-15 um, random orientation) with nuclei (0.4 of the axes, 3x the dye density) and `filaments`
    persistent random walks per cell (4 dyes per voxel step). The PSF: 3D Gibson-Lanni, NA 1.4, 520 nm, oil,
    nx x ny x nz samples at the voxel pitch (pupil samples from the reference's automatic choice). EMCCD: EM gain
    300, 5 photons/px background, CIC 0.002, read noise 50 e-, offset N(100, 2) ADU, 1 photon/ADU, QE 1."""
    rng = np.random.default_rng(seed)
    vx, vy, vz = (v / 1000.0 for v in voxel_nm)
    d = np.zeros((nz, ny, nx), np.float32)
    X, Y, Z = nx * vx, ny * vy, nz * vz
    for _ in range(cells):
        c = np.array([rng.uniform(0, X), rng.uniform(0, Y), rng.uniform(0.3, 0.7) * Z])
        ax = rng.uniform(2.5, 7.5, 3)
        th = rng.uniform(0, 2 * np.pi)
        ct, st = np.cos(th), np.sin(th)
        r = ax.max()
        i0, i1 = max(0, int((c[0] - r) / vx)), min(nx, int((c[0] + r) / vx) + 1)
        j0, j1 = max(0, int((c[1] - r) / vy)), min(ny, int((c[1] + r) / vy) + 1)
        k0, k1 = max(0, int((c[2] - ax[2]) / vz)), min(nz, int((c[2] + ax[2]) / vz) + 1)
        if i0 >= i1 or j0 >= j1 or k0 >= k1:
            continue
        zz, yy, xx = np.meshgrid((np.arange(k0, k1) + 0.5) * vz - c[2], (np.arange(j0, j1) + 0.5) * vy - c[1],
                                 (np.arange(i0, i1) + 0.5) * vx - c[0], indexing="ij")
        u = (xx * ct + yy * st) / ax[0]
        v = (-xx * st + yy * ct) / ax[1]
        w = zz / ax[2]
        q = u * u + v * v + w * w
        d[k0:k1, j0:j1, i0:i1] += (q <= 1.0).astype(np.float32) + 2.0 * (q <= 0.16).astype(np.float32)
        # filaments: persistent walks from inside the cell, ending where they leave it
        start = c + (rng.uniform(-0.7, 0.7, (filaments, 3)) * ax[None, :] *
                     np.array([[1.0, 1.0, 0.5]]))
        phi = rng.uniform(0, 2 * np.pi, filaments)
        tilt = rng.normal(0.0, 0.15, filaments)
        pts = []
        p = start.copy()
        alive = np.ones(filaments, bool)
        for _s in range(steps):
            phi += rng.normal(0.0, 0.3, filaments)
            step = 0.15 * np.stack([np.cos(phi), np.sin(phi), tilt], axis=1)
            p = p + step
            rel = p - c
            uu = (rel[:, 0] * ct + rel[:, 1] * st) / ax[0]
            vv = (-rel[:, 0] * st + rel[:, 1] * ct) / ax[1]
            ww = rel[:, 2] / ax[2]
            alive &= (uu * uu + vv * vv + ww * ww) <= 1.0
            pts.append(p[alive])
        pts = np.concatenate(pts) if pts else np.zeros((0, 3))
        ii = (pts[:, 0] / vx).astype(np.int64)
        jj = (pts[:, 1] / vy).astype(np.int64)
        kk = (pts[:, 2] / vz).astype(np.int64)
        ok = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny) & (kk >= 0) & (kk < nz)
        np.add.at(d, (kk[ok], jj[ok], ii[ok]), 4.0)
    d *= photons_per_dye
    kz, ky, kx = kernel_shape if kernel_shape is not None else (nz, ny, nx)
    psf = PsfParams(wavelength_nm=520.0, na=1.4, immersion_index=1.518, sample_index=1.518,
                    working_distance_um=150.0, pixel_size_nm=voxel_nm[0], oversampling=1,
                    kernel_half_width_px=max(kx, ky) // 2, nz=kz, z_step_nm=voxel_nm[2], pupil_samples=0)
    # Convolution orientation: image plane f gets dye plane k through PSF plane f - k + kz/2, whose defocus is the
    # dye's height above the focal plane, (k - f) dz = (kz/2 - j) dz for PSF plane j.
    defocus = (kz // 2 - np.arange(kz)) * voxel_nm[2]
    cam = CameraParams(quantum_efficiency=1.0, dark_electrons=0.0, gain=1.0, read_noise_e=50.0, emccd=True,
                       bit_depth=16, em_gain=300.0, cic_electrons=0.002)
    return WidefieldVolume(d, tuple(voxel_nm), psf, (kz, ky, kx), defocus, cam, 5.0, seed, 100.0, 2.0,
                           (seed ^ 0x9E3779B9) & 0xFFFFFFFF)


def noll_to_nm(j: int) -> tuple[int, int]:
    """Noll's single index j >= 1 -> (n, m), m < 0 for the sine modes (Noll 1976 ordering)."""
    n, j1 = 0, j - 1
    while j1 > n:
        n += 1
        j1 -= n
    m = (-1) ** j * ((n % 2) + 2 * ((j1 + ((n + 1) % 2)) // 2))
    return n, m


def noll_rms_to_osa_waves(noll: dict) -> list:
    """Noll-indexed rms-normalized coefficients (waves) -> the reference's 28 OSA/ANSI unnormalized coefficients
    (waves; ZernikePsf.cpp:58-78 evaluates R_n^m cos/sin without normalization): x sqrt(2 (n + 1)) for m != 0,
    x sqrt(n + 1) for m = 0; OSA index (n (n + 2) + m) / 2."""
    out = [0.0] * 28
    for j, c in noll.items():
        n, m = noll_to_nm(j)
        osa = (n * (n + 2) + m) // 2
        if osa >= 28:
            raise ValueError(f"Noll {j} (n = {n}) is beyond OSA 27")
        out[osa] += c * (np.sqrt(2.0 * (n + 1)) if m != 0 else np.sqrt(n + 1.0))
    return out


@dataclass
class PsfLibrary:
    """A batched PSF library: request sets and, per PSF, its set and defocus."""
    sets: list
    set_of_psf: np.ndarray
    defocus_nm: np.ndarray
    size: int


def psf_library(seed: int = 42, n_z: int = 64, wavelengths=(520.0, 580.0, 670.0, 750.0), n_aberr: int = 16,
                pupil: int = 128, size: int = 64, z_step_nm: float = 25.0, rms_waves: float = 0.05) -> PsfLibrary:
    """The precision config's library: 64 z-planes x 4 wavelengths x 16 Zernike sets = 4,096 PSFs, each a 128 x 128
    pupil chirp-Z'd to 64 x 64 samples at 4x oversampling of 100 nm pixels; Noll 4-15 ~ N(0, 0.05 lambda rms)
    (converted to the reference's OSA coefficients); NA 1.45, oil (ni = ns = 1.518); planes 25 nm apart."""
    rng = np.random.default_rng(seed)
    aberr = [noll_rms_to_osa_waves({j: rng.normal(0.0, rms_waves) for j in range(4, 16)}) for _ in range(n_aberr)]
    sets = []
    for wl in wavelengths:
        for a in aberr:
            sets.append(PsfParams(wavelength_nm=wl, na=1.45, immersion_index=1.518, sample_index=1.518,
                                  pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8, nz=3,
                                  z_step_nm=z_step_nm, pupil_samples=pupil, zernike=list(a)))
    z = (np.arange(n_z) - n_z // 2) * z_step_nm
    set_of = np.repeat(np.arange(len(sets), dtype=np.uint32), n_z)
    defocus = np.tile(z, len(sets)).astype(np.float64)
    return PsfLibrary(sets, set_of, defocus, size)


@dataclass
class NllProblem:
    """ROIs for the Poisson-likelihood gradient: the truth the data are drawn at, and a perturbed point to
    differentiate at."""
    spec: object                # insiliscope_b200.nll.NllSpec
    frame: np.ndarray           # (n,) int32
    params_true: np.ndarray     # (n, 4) float32: x, y (ROI px), z (nm), N
    bg_true: np.ndarray         # (F,) float32
    zern_true: np.ndarray       # (J,) float64, waves rms
    params: np.ndarray          # the evaluation point
    bg: np.ndarray
    zern: np.ndarray
    noise_seed: int
    frame0: int = 0             # the first frame's number in the whole problem (a rank's share starts there)


def nll_rois(seed: int = 42, frames: int = 256, per_frame: int = 1000, spec=None) -> NllProblem:
    """The gradient config: 256 frames x 1,000 emitters, each in its own 32 x 32 px ROI (108 nm, NA 1.45, 670 nm):
    x, y ~ U(14.5, 17.5) px, z ~ U(-500, 500) nm, N lognormal (median 2000, sigma_log 0.5), one background per frame
    ~ U(5, 20) photons/px, 21 Zernike coefficients (Noll 4-24) ~ N(0, 0.03) waves rms. The evaluation point perturbs
    the truth (x, y by N(0, 0.3) px, z by N(0, 50) nm, N by 10 %, backgrounds by 10 %, Zernike by N(0, 0.01)).
    numpy PCG64 seeded with `seed`."""
    from .nll import NllSpec
    spec = spec or NllSpec()
    rng = np.random.default_rng(seed)
    n = frames * per_frame
    frame = np.repeat(np.arange(frames, dtype=np.int32), per_frame)
    c = spec.roi / 2.0
    pt = np.column_stack([rng.uniform(c - 1.5, c + 1.5, n), rng.uniform(c - 1.5, c + 1.5, n),
                          rng.uniform(-500.0, 500.0, n), 2000.0 * np.exp(0.5 * rng.standard_normal(n))])
    bg = rng.uniform(5.0, 20.0, frames)
    zt = rng.normal(0.0, 0.03, len(spec.noll))
    p = pt + np.column_stack([rng.normal(0, 0.3, n), rng.normal(0, 0.3, n), rng.normal(0, 50.0, n),
                              pt[:, 3] * rng.normal(0, 0.1, n)])
    return NllProblem(spec, frame, pt.astype(np.float32), bg.astype(np.float32), zt, p.astype(np.float32),
                      (bg * rng.uniform(0.9, 1.1, frames)).astype(np.float32), zt + rng.normal(0, 0.01, len(zt)),
                      (seed ^ 0x9E3779B9) & 0xFFFFFFFF)


def nll_counts(engine, model, prob: NllProblem, device="cuda"):
    """The data: the expected counts at the truth (the gradient model's forward pass), then the engine's noise chain
    as a photon counter (sCMOS, QE 1, gain 1 photon/ADU, no read noise, offset 0: ADU = the Poisson draw), keyed by
    (noise seed, frame, pixel) with each frame's ROIs stacked into one roi x (per_frame roi) image."""
    import torch
    from .engine import CameraParams
    pt = torch.from_numpy(prob.params_true).to(device)
    fr = torch.from_numpy(prob.frame).to(device)
    bg = torch.from_numpy(prob.bg_true).to(device)
    counts0 = torch.zeros((len(prob.frame), prob.spec.roi, prob.spec.roi), dtype=torch.float32, device=device)
    _, mu, _ = model.evaluate(pt, fr, bg, prob.zern_true, counts0, want_mu=True)
    F = int(prob.frame.max()) + 1
    per = len(prob.frame) // F
    R = prob.spec.roi
    engine.set_static(R, R * per, flat_bg=0.0)
    cam = CameraParams(quantum_efficiency=1.0, dark_electrons=0.0, gain=1.0, read_noise_e=0.0)
    adu = engine.noise_frames_dev(mu.reshape(F, per * R, R), np.arange(prob.frame0, prob.frame0 + F), cam,
                                  prob.noise_seed)
    return adu.to(torch.float32).reshape(len(prob.frame), R, R)
