"""Frames of a drifting widefield sample (RenderShiftedImages): the float64 restatement (oracle.shifted_frame_f64)
pinned on the reference's own RenderShiftedImages (WidefieldRender.cpp, RealFft2d's float transforms, compiled into
oracle/_ref) -- one and two foci, bleach coefficients, drift with and without a sub-cell pose, windows at 1-3 cells
per pixel -- within its float rounding (2e-5 of the frame maximum). CPU only; the device form is in
tests/test_gpu_shift.py."""
import numpy as np
import pytest

from oracle.oracle import shifted_frame_f64


def shift_case(seed, nx, ny, n_bleach=2):
    """Channels' spectra of smooth non-negative images (a dye scene seen through a band limit), persistent first."""
    rng = np.random.default_rng(seed)
    imgs = []
    for _ in range(1 + n_bleach):
        im = rng.random((ny, nx)) ** 4 * 50
        F = np.fft.rfft2(im)
        fy = np.fft.fftfreq(ny)[:, None]
        fx = np.fft.rfftfreq(nx)[None, :]
        imgs.append((F * np.exp(-(fx ** 2 + fy ** 2) / (2 * 0.08 ** 2))).astype(np.complex64))
    return np.stack(imgs)


def coefs(a, w, two):
    """The coefficient of each channel as RenderShiftedImages forms it: float(w_i), float(a_j) x float(w_i)."""
    f32 = np.float32
    wi = f32(1.0 - w) if two else f32(1.0)
    c = [wi] + [f32(aj) * wi for aj in a]
    if two and w != 0:
        c += [f32(w)] + [f32(aj) * f32(w) for aj in a]
    return np.array(c, np.float32)


@pytest.mark.parametrize("nx,ny,window,up,frac,drift,two", [
    (64, 32, (4, 2, 48, 24), 1, (0.0, 0.0), (0.0, 0.0), False),
    (64, 32, (4, 2, 48, 24), 2, (0.3, -0.2), (1.7, -0.45), False),
    (128, 64, (10, 6, 96, 48), 3, (0.1, 0.4), (-2.25, 3.5), True),
    (128, 128, (0, 0, 128, 128), 2, (0.0, 0.0), (0.5, 0.5), True)])
def test_restatement_equals_reference(reference, nx, ny, window, up, frac, drift, two):
    sp0 = shift_case(nx + ny, nx, ny)
    sp1 = shift_case(nx + ny + 1, nx, ny) if two else None
    a, w = [0.6, 0.0], 0.35
    want = reference.shifted_images(nx, ny, sp0, a, frac, drift, window, up, spec1=sp1, w=w)
    spectra = sp0 if not two else np.concatenate([sp0, sp1])
    got = shifted_frame_f64(spectra, coefs(a, w, two), (frac[0] - drift[0], frac[1] - drift[1]), nx, ny, window, up)
    assert np.abs(got - want).max() <= 2e-5 * np.abs(want).max()
