"""The widefield checker pinned on the reference itself (CPU): the float64 restatement of the widefield scene
(oracle.wf_kernel_volume_f64 + wf_scene_f64: KernelWidefieldPsf's cell kernels, PlanFocus's clamped and blended
planes, the linear convolution over the whole dye grid, the FOV cut, WidefieldImages::Render's max(0, .) and binning)
equals the reference's WidefieldScene::UpdateFromGrid + FocusSeries + Render, compiled from its sources into
oracle/_ref, within its float FFTs' rounding (1e-5 of the frame maximum; measured ~2e-7), on grids with and without
margins, with kernel resampling (oversampling 4 -> 2 cells per pixel), dye planes beyond the kernel stack (clamped
to its last plane), dye planes thinner than the stack's step (blended planes) and a capped kernel radius."""
import numpy as np
import pytest

from insiliscope_b200 import PsfParams
from oracle.oracle import binned_cell_kernels_f64, fft_convolve_same_f64, wf_kernel_volume_f64, wf_scene_f64

CASES = [
    # os, upscale, half width px, kernel planes, step nm, plane nm, FOV w, h, dye planes, margin um, cap um
    (1, 1, 8, 9, 200.0, 200.0, 40, 32, 5, 0.3, 100.0),
    (4, 2, 6, 7, 200.0, 200.0, 24, 20, 6, 0.4, 100.0),
    (2, 2, 10, 5, 200.0, 200.0, 30, 28, 7, 0.0, 100.0),     # dye planes beyond the stack: its last planes, clamped
    (1, 1, 9, 11, 150.0, 100.0, 36, 30, 6, 0.2, 100.0),     # planes thinner than the step: blended kernels
    (2, 1, 12, 7, 200.0, 200.0, 32, 32, 4, 0.5, 0.6),       # the kernel radius capped at 0.6 um
]


def _req(os_, half, nzk, step):
    return PsfParams(wavelength_nm=520.0, na=1.4, immersion_index=1.518, sample_index=1.518, pixel_size_nm=100.0,
                     oversampling=os_, kernel_half_width_px=half, nz=nzk, z_step_nm=step, pupil_samples=0)


def scene_case(reference, case, seed=1):
    """The reference scene's frames for a case, the restatement's, and the case's geometry."""
    os_, up, half, nzk, step, plane, W, H, nzd, margin, cap = case
    k = reference.kernel(req=_req(os_, half, nzk, step))
    gx, gy, fx, fy = k.wf_grid(up, 0.1, W, H, (0.05, 0.05), margin, plane)
    rng = np.random.default_rng(seed)
    counts = ((rng.random((nzd, gy, gx)) < 0.05) * rng.integers(1, 5, (nzd, gy, gx))).astype(np.float32)
    foci = (np.arange(nzd) + 0.5) * plane / 1000.0
    got, info = k.wf_focus_series(counts, foci, up, cap, 0.1, W, H, (0.05, 0.05), margin, plane)
    ck, u, R = binned_cell_kernels_f64(k.planes(), os_, up)
    Rc = max(1, min(int(np.ceil(cap / (0.1 / u) - 1e-9)), R))
    ck = ck[:, R - Rc:R + Rc + 1, R - Rc:R + Rc + 1]
    assert info[2] == Rc
    kv = wf_kernel_volume_f64(ck, step, plane, nzd)
    want = wf_scene_f64(counts, kv, (fx, fy, W * u, H * u), u)
    return k, counts, got, want, (gx, gy, fx, fy, u, Rc, kv)


@pytest.mark.parametrize("case", CASES)
def test_restatement_equals_reference_scene(reference, case):
    _, _, got, want, _ = scene_case(reference, case)
    assert got.shape == want.shape
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-5, err


def test_convolution_oracle_is_the_scene_sum():
    """fft_convolve_same_f64 -- the 3D checker of the device focus series -- is the scene's sum over dye planes of
    each plane's 2D linear convolution with the kernel plane at its offset (a direct sum, no FFT)."""
    rng = np.random.default_rng(4)
    counts = rng.random((4, 9, 11))
    kv = rng.random((7, 5, 3))
    got = fft_convolve_same_f64(counts, kv)
    want = np.zeros_like(counts)
    nz, ny, nx = counts.shape
    for f in range(nz):
        for k in range(nz):
            K = kv[f - k + 3]
            for dy in range(-2, 3):
                for dx in range(-1, 2):
                    src = np.zeros((ny, nx))
                    ys, yd = (slice(0, ny - dy), slice(dy, ny)) if dy >= 0 else (slice(-dy, ny), slice(0, ny + dy))
                    xs, xd = (slice(0, nx - dx), slice(dx, nx)) if dx >= 0 else (slice(-dx, nx), slice(0, nx + dx))
                    src[yd, xd] = counts[k][ys, xs]
                    want[f] += K[dy + 2, dx + 1] * src
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)
