"""The binned blink regime on the B200 (iscu_binned_*) against the float64 oracle (the linear convolution
BinnedBlinkRenderer computes) and the reference's own BinnedBlinkRenderer (float FFTs, oracle/_ref): the cell kernels
bit for bit (KernelWidefieldPsf's float64 block sums), the photon images within 1e-6 of the frame maximum of the
oracle and 5e-6 of the reference's (its float FFT's rounding), added into the caller's images."""
import numpy as np
import pytest

from insiliscope_b200 import BinnedRenderer, INTERP_CUBIC
from oracle.oracle import binned_cell_kernels_f64, binned_gauss_kernel_f64, binned_render_f64
from test_binned_oracle import H, W, _req, binned_movie

pytestmark = pytest.mark.gpu


def _rel(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).cuda()


def _render(r, em, fr, base):
    import torch
    img = torch.from_numpy(base.copy()).cuda()
    alone = torch.zeros_like(img)
    r.render_dev(_dev(em), _dev(fr), len(fr), img, alone)
    return img.cpu().numpy(), alone.cpu().numpy()


@pytest.mark.parametrize("upscale,halo", [(2, None), (4, 0.002), (1, None), (3, None)])
def test_kernel_regime(engine, reference, upscale, halo):
    k = reference.kernel(req=_req())
    size, nz, os_, _ = k.info()
    engine.kernel_set_planes(0, k.planes(), os_, 100.0, INTERP_CUBIC)
    radius2 = None
    if halo is not None:
        engine.kernel_set_halo(0, halo)
        k = k.halo(halo)
        radius2 = k.spans()[2]
    K, u, R = binned_cell_kernels_f64(k.planes(), os_, upscale, radius2)
    r = BinnedRenderer(engine, W, H, upscale, slot=0)
    assert (r.upscale, r.radius, r.planes) == (u, R, nz)
    assert np.array_equal(r.kernels(), K)
    em, fr = binned_movie(7 + upscale, 3, 60, nz)
    base = np.random.default_rng(1).random((len(fr), H, W)).astype(np.float32) * 10
    img, alone = _render(r, em, fr, base)
    want = binned_render_f64(K, u, R, em, fr, W, H)
    assert _rel(alone, want) <= 1e-6
    assert np.array_equal(img, base + alone)
    ref, _, _, _ = reference.binned_render(k, 0.0, W, H, upscale, em, fr)
    assert _rel(alone, ref) <= 5e-6
    r.close()
    if halo is not None:
        engine.kernel_set_halo(0, 0.0)


def test_gauss_regime(engine, reference):
    K, u, R = binned_gauss_kernel_f64(1.3, 3)
    r = BinnedRenderer(engine, W, H, 3, sigma_px=1.3)
    assert (r.upscale, r.radius, r.planes) == (u, R, 1)
    np.testing.assert_allclose(r.kernels(), K, rtol=1e-6, atol=0)
    em, fr = binned_movie(3, 2, 40, 1)
    _, alone = _render(r, em, fr, np.zeros((len(fr), H, W), np.float32))
    ref, _, _, _ = reference.binned_render(None, 1.3, W, H, 3, em, fr)
    assert _rel(alone, ref) <= 5e-6
    assert _rel(alone, binned_render_f64(K, u, R, em, fr, W, H)) <= 1e-6
    r.close()


def test_dense_frames_128(engine, reference):
    """Frames of the dense regime the reference picks binned for (2,000+ ON emitters on a 128 x 128 camera), the
    SMLM kernel geometry (oversampling 4, 49 planes), u = 2."""
    from insiliscope_b200.workloads import binned_dense
    mv = binned_dense(frames=6)
    k = reference.kernel(req=mv.psf)
    engine.kernel_set_planes(1, k.planes(), 4, mv.psf.z_step_nm, INTERP_CUBIC)
    r = BinnedRenderer(engine, mv.width, mv.height, mv.upscale, slot=1)
    K, u, R = binned_cell_kernels_f64(k.planes(), 4, mv.upscale)
    _, alone = _render(r, mv.emitters, mv.frames, np.zeros((len(mv.frames), mv.height, mv.width), np.float32))
    want = binned_render_f64(K, u, R, mv.emitters, mv.frames, mv.width, mv.height)
    assert _rel(alone, want) <= 1e-6
    r.close()
