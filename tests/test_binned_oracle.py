"""The binned blink regime's float64 oracle (oracle.binned_* : the linear convolution BinnedBlinkRenderer computes)
pinned against the reference's own BinnedBlinkRenderer (BinnedBlinks.cpp, float FFTs), compiled from its sources into
oracle/_ref: the same u and R, and the photon images within the float FFT's rounding (5e-6 of the frame maximum).
CPU only."""
import numpy as np
import pytest

from insiliscope_b200 import EMITTER_DTYPE, FRAME_DTYPE, INTERP_CUBIC, PsfParams
from oracle.oracle import binned_cell_kernels_f64, binned_gauss_kernel_f64, binned_render_f64

W, H = 40, 32
TOL = 5e-6


def _req(nz=9):
    return PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=108.0, oversampling=4, kernel_half_width_px=6,
                     nz=nz, z_step_nm=100.0, pupil_samples=64, interp=INTERP_CUBIC)


def binned_movie(seed, n_frames, per_frame, nz, w=W, h=H):
    """Dense frames with the cases Render distinguishes: emitters inside, at the edges, outside by less and by more
    than the kernel radius, photons <= 0, planes beyond the stack, several in one cell."""
    rng = np.random.default_rng(seed)
    em, fr = [], np.zeros(n_frames, FRAME_DTYPE)
    for k in range(n_frames):
        n = per_frame + int(rng.integers(0, 5))
        e = np.zeros(n, EMITTER_DTYPE)
        e["x_px"] = rng.uniform(-12.0, w + 12.0, n)
        e["y_px"] = rng.uniform(-12.0, h + 12.0, n)
        e["photons"] = rng.lognormal(np.log(1500.0), 0.6, n)
        e["plane"] = rng.integers(-2, nz + 3, n)
        e["photons"][:3] = [0.0, -5.0, 800.0]
        e["x_px"][3:6] = e["x_px"][2]   # one cell, three emitters
        e["y_px"][3:6] = e["y_px"][2]
        fr[k]["em_start"] = sum(len(a) for a in em)
        fr[k]["em_count"] = n
        fr[k]["frame"] = k
        em.append(e)
    return np.concatenate(em), fr


def _rel(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("upscale,halo", [(2, None), (4, 0.002), (1, None), (3, None)])
def test_kernel_regime_matches_reference(reference, upscale, halo):
    k = reference.kernel(req=_req())
    radius2 = None
    if halo is not None:
        k = k.halo(halo)
        radius2 = k.spans()[2]
    size, nz, os_, _ = k.info()
    K, u, R = binned_cell_kernels_f64(k.planes(), os_, upscale, radius2)
    em, fr = binned_movie(7 + upscale, 3, 60, nz)
    want, ru, rR, _ = reference.binned_render(k, 0.0, W, H, upscale, em, fr)
    assert (u, R) == (ru, rR)
    got = binned_render_f64(K, u, R, em, fr, W, H)
    assert _rel(got, want) <= TOL


def test_gauss_regime_matches_reference(reference):
    K, u, R = binned_gauss_kernel_f64(1.3, 3)
    em, fr = binned_movie(3, 2, 40, 1)
    want, ru, rR, _ = reference.binned_render(None, 1.3, W, H, 3, em, fr)
    assert (u, R) == (ru, rR)
    assert _rel(binned_render_f64(K, u, R, em, fr, W, H), want) <= TOL
