"""Widefield mean-field focus series on the B200 (3D FFT convolution + max(0, .) + background + EMCCD chain) against
the float64 FFT convolution oracle; at full size (512 x 512 x 64 volume and PSF, the widefield config's shape)
through size-independent properties: the impulse response is the PSF itself, and the convolution is linear.
Tolerance: max |I - I64| <= 1e-5 x max |I64| (the north-star bar for noise-free images)."""
import numpy as np
import pytest

from insiliscope_b200 import CameraParams, PsfParams, WidefieldPlan
from oracle.oracle import fft_convolve_same_f64

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _rel(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("vol_shape,psf_shape", [((10, 24, 30), (7, 9, 11)), ((16, 40, 64), (16, 40, 64)),
                                                 ((5, 33, 20), (2, 4, 6)), ((1, 8, 8), (1, 3, 3))])
def test_convolution_vs_oracle(engine, vol_shape, psf_shape):
    import torch
    rng = np.random.default_rng(sum(vol_shape) + sum(psf_shape))
    vol = rng.random(vol_shape).astype(np.float32)
    vol[vol < 0.6] = 0.0
    psf = rng.random(psf_shape).astype(np.float32)
    psf -= 0.2   # some negative taps, so the max(0, .) clamp is exercised
    plan = WidefieldPlan(engine, vol_shape, psf)
    got = plan.convolve_dev(torch.from_numpy(vol).cuda()).cpu().numpy()
    want = np.maximum(fft_convolve_same_f64(vol, psf), 0.0)
    assert _rel(got, want) <= TOL
    plan.close()


def test_pipelined_renders_equal_blocking(engine):
    """Four focus series through three I/O slots (render_async / render_wait, copies beside the passes of the next
    series) give the blocking render's frames bit for bit, each with its own frame numbers."""
    import torch
    rng = np.random.default_rng(11)
    nz, ny, nx = 8, 40, 48
    psf = rng.random((6, 9, 11)).astype(np.float32)
    psf /= psf.sum()
    vols = [(rng.random((nz, ny, nx)) * 40).astype(np.float32) for _ in range(4)]
    cam = CameraParams(quantum_efficiency=1.0, gain=1.0, read_noise_e=50.0, emccd=True, em_gain=300.0,
                       cic_electrons=0.002, bit_depth=16)
    engine.set_static(nx, ny, offset=np.full(nx * ny, 100.0, np.float32))
    plan = WidefieldPlan(engine, (nz, ny, nx), psf)
    want = [plan.render(v, 5.0, cam, 31, frame0=nz * i)[1] for i, v in enumerate(vols)]
    pinned = [torch.from_numpy(v).pin_memory().numpy() for v in vols]
    outs = [torch.empty((nz, ny, nx), dtype=torch.uint16).pin_memory().numpy() for _ in range(3)]
    got = [None] * 4
    for i in range(4):
        io = i % 3
        if i >= 3:
            plan.render_wait(io)
            got[i - 3] = outs[io].copy()
        plan.render_async(io, pinned[i], 5.0, cam, 31, frame0=nz * i, adu=outs[io])
    for i in range(1, 4):
        plan.render_wait(i % 3)
        got[i] = outs[i % 3].copy()
    for i in range(4):
        assert np.array_equal(got[i], want[i]), i
    with pytest.raises(Exception):
        plan.render_wait(0)   # nothing enqueued in the slot any more
    plan.close()


def test_render_noise_bit_exact_on_image(engine, oracle):
    """The frames' ADU are ApplyNoiseChain (EMCCD) of the expected image, frame = frame0 + plane, with the camera
    offset map: bit for bit the oracle's chain on the GPU's own expected image."""
    rng = np.random.default_rng(4)
    nz, ny, nx = 6, 36, 50
    vol = (rng.random((nz, ny, nx)) * 30).astype(np.float32)
    psf = rng.random((5, 7, 9)).astype(np.float32)
    psf /= psf.sum(axis=(1, 2), keepdims=True)
    off, _, _ = oracle.camera_maps(nx, ny, 42, 100.0, 2.0, 1.0, 0.0, 50.0, 0.0)
    engine.set_static(nx, ny, offset=off)
    cam = CameraParams(quantum_efficiency=1.0, gain=1.0, read_noise_e=50.0, emccd=True, em_gain=300.0,
                       cic_electrons=0.002, bit_depth=16)
    plan = WidefieldPlan(engine, (nz, ny, nx), psf)
    image, adu = plan.render(vol, 5.0, cam, 777, frame0=100, want_image=True)
    want_img = np.maximum(fft_convolve_same_f64(vol, psf), 0.0) + 5.0
    assert _rel(image, want_img) <= TOL
    for f in range(nz):
        want = oracle.noise_chain(image[f], cam, off.reshape(ny, nx), None, None, 777, 100 + f)
        assert np.array_equal(adu[f], want), f
    plan.close()


def _full_plan(engine):
    rng = np.random.default_rng(9)
    psf = rng.random((64, 512, 512)).astype(np.float32) * np.float32(1e-4)
    psf[32, 256, 256] += 1.0
    return psf, WidefieldPlan(engine, (64, 512, 512), psf)


def test_full_size_impulse_response(engine):
    """512 x 512 x 64 on the 1024 x 1024 x 128 grid: a unit dye at (z0, y0, x0) images to the PSF shifted there."""
    import torch
    psf, plan = _full_plan(engine)
    assert plan.grid() == (1024, 1024, 128)
    for (z0, y0, x0) in ((32, 256, 256), (3, 17, 500), (60, 490, 9)):
        vol = torch.zeros((64, 512, 512), dtype=torch.float32, device="cuda")
        vol[z0, y0, x0] = 1.0
        got = plan.convolve_dev(vol).cpu().numpy()
        want = np.zeros((64, 512, 512), np.float32)
        zs, ys, xs = slice(max(0, z0 - 32), min(64, z0 + 32)), slice(max(0, y0 - 256), min(512, y0 + 256)), \
            slice(max(0, x0 - 256), min(512, x0 + 256))
        want[zs, ys, xs] = psf[zs.start - z0 + 32: zs.stop - z0 + 32, ys.start - y0 + 256: ys.stop - y0 + 256,
                               xs.start - x0 + 256: xs.stop - x0 + 256]
        assert _rel(got, want) <= TOL, (z0, y0, x0)
    plan.close()


def test_full_size_linearity(engine):
    import torch
    psf, plan = _full_plan(engine)
    rng = np.random.default_rng(10)
    a = torch.from_numpy(rng.random((64, 512, 512), dtype=np.float32)).cuda()
    b = torch.from_numpy((rng.random((64, 512, 512), dtype=np.float32) < 0.01).astype(np.float32) * 50).cuda()
    ia = plan.convolve_dev(a).double()
    ib = plan.convolve_dev(b).double()
    iab = plan.convolve_dev(2.5 * a + b).double()
    assert float((iab - (2.5 * ia + ib)).abs().max() / iab.abs().max()) <= TOL
    plan.close()


def test_large_pupil_psf_vs_oracle(engine, oracle):
    """The PSF path for pupils beyond shared memory (global-memory products), as the widefield PSF (M = 512) uses,
    checked at M = 256 -> 96 x 96 planes against the float64 oracle."""
    req = PsfParams(wavelength_nm=520.0, na=1.4, pixel_size_nm=100.0, oversampling=1, kernel_half_width_px=48,
                    nz=3, z_step_nm=200.0, pupil_samples=256)
    req.zernike[4] = 0.05
    dz = np.array([-600.0, 0.0, 400.0])
    got = engine.psf_library_dev([req], [0, 0, 0], dz, size=96, normalize=True).cpu().numpy()
    want = oracle.psf_planes(req, dz * 1e-9, size=96, normalize=True)
    for i in range(3):
        assert np.abs(got[i] - want[i]).max() <= TOL * want[i].max(), i


@pytest.mark.parametrize("vol_shape,psf_shape,grid", [((40, 400, 400), (24, 200, 200), (512, 512, 64)),
                                                      ((130, 20, 40), (127, 9, 11), (64, 32, 256))])
def test_codelet_lengths_vs_oracle(engine, vol_shape, psf_shape, grid):
    """Grids whose transform lengths run the compiled-in codelets other than the full-size ones (x half length 256,
    y 512, z 64; z 256) against the float64 oracle."""
    import torch
    rng = np.random.default_rng(sum(vol_shape))
    vol = rng.random(vol_shape).astype(np.float32)
    vol[vol < 0.7] = 0.0
    psf = rng.random(psf_shape).astype(np.float32) - 0.2
    plan = WidefieldPlan(engine, vol_shape, psf)
    assert plan.grid() == grid
    got = plan.convolve_dev(torch.from_numpy(vol).cuda()).cpu().numpy()
    want = np.maximum(fft_convolve_same_f64(vol, psf), 0.0)
    assert _rel(got, want) <= TOL
    plan.close()


def test_codelet_2048_impulse(engine):
    """A 2048 x 2048 grid (x half length 1024, y 2048 codelets): unit dyes image to the PSF shifted there."""
    import torch
    rng = np.random.default_rng(12)
    psf = rng.random((1, 1019, 1019)).astype(np.float32) * np.float32(1e-4)
    psf[0, 509, 509] += 1.0
    plan = WidefieldPlan(engine, (2, 1030, 1030), psf)
    assert plan.grid() == (2048, 2048, 4)
    for (z0, y0, x0) in ((0, 515, 515), (1, 3, 1020)):
        vol = torch.zeros((2, 1030, 1030), dtype=torch.float32, device="cuda")
        vol[z0, y0, x0] = 1.0
        got = plan.convolve_dev(vol).cpu().numpy()
        want = np.zeros((2, 1030, 1030), np.float32)
        ys, xs = slice(max(0, y0 - 509), min(1030, y0 + 510)), slice(max(0, x0 - 509), min(1030, x0 + 510))
        want[z0, ys, xs] = psf[0, ys.start - y0 + 509: ys.stop - y0 + 509, xs.start - x0 + 509: xs.stop - x0 + 509]
        assert _rel(got, want) <= TOL, (z0, y0, x0)
    plan.close()


def test_scene_plan_equals_reference_scene(engine, reference):
    """The widefield scene as a device plan (iscu_wf_plan_from_kernel: KernelWidefieldPsf's cells made on the device
    from a kernel slot, PlanFocus's clamped and blended planes, the grid's linear convolution, the FOV window, binning)
    against the reference's WidefieldScene + FocusSeries + Render compiled from its sources, on the pinned cases of
    tests/test_widefield_oracle.py (margins, resampling, clamped and blended planes, a capped radius)."""
    import torch
    from tests.test_widefield_oracle import CASES, scene_case
    for case in CASES:
        os_, up, half, nzk, step, plane, W, H, nzd, margin, cap = case
        k, counts, want, want64, (gx, gy, fx, fy, u, Rc, _) = scene_case(reference, case)
        engine.kernel_set_planes(1, k.planes(), os_, step, 2)
        plan = WidefieldPlan.from_kernel(engine, 1, up, 0.1, cap, plane, counts.shape, (fx, fy, W, H))
        assert plan.frame_shape == (nzd, H, W) and plan.kernel_radius == Rc
        got = plan.convolve_dev(torch.from_numpy(counts).cuda()).cpu().numpy()
        assert _rel(got, want) <= TOL, case
        assert _rel(got, want64) <= TOL, case
        plan.close()


def test_scene_plan_full_size_against_reference(engine, reference):
    """The widefield config at full size as the reference's scene: a 512 x 512 x 64 dye grid of 100 x 100 x 200 nm
    cells (the FOV, no margin; the reference's extra far-edge cell row and column left empty), the 3D Gibson-Lanni
    kernel stack (NA 1.4, 520 nm, 513 x 513 samples, 65 planes 200 nm apart) built on the device, the radius uncapped
    (256 cells); four foci of the series against the reference's FocusSeries within 1e-5 of the frame maximum."""
    import torch
    from insiliscope_b200 import CZT_FP32
    from insiliscope_b200.workloads import widefield_cells
    wv = widefield_cells(seed=42)
    nz, ny, nx = wv.density.shape
    req = wv.psf
    req.nz = 65
    req.kernel_half_width_px = 256
    engine.kernel_build(2, req, CZT_FP32)
    planes = engine.kernel_planes(2)
    assert planes.shape == (65, 513, 513)
    plan = WidefieldPlan.from_kernel(engine, 2, 1, 0.1, 30.0, 200.0, (nz, ny, nx), (0, 0, nx, ny))
    assert plan.kernel_radius == 256 and plan.grid() == (1024, 1024, 128)
    got = plan.convolve_dev(torch.from_numpy(wv.density).cuda()).cpu().numpy()
    k = reference.kernel(planes=planes, os_=1, z_step_nm=200.0, interp=2)
    gx, gy, fx, fy = k.wf_grid(1, 0.1, nx, ny, (0.05, 0.05), 0.0, 200.0)
    assert (gx, gy, fx, fy) == (nx + 1, ny + 1, 0, 0)
    counts = np.zeros((nz, gy, gx), np.float32)
    counts[:, :ny, :nx] = wv.density
    foci = [0, 21, 42, 63]
    reference.set_threads(0)
    try:
        want, info = k.wf_focus_series(counts, (np.array(foci) + 0.5) * 0.2, 1, 30.0, 0.1, nx, ny, (0.05, 0.05), 0.0,
                                       200.0)
    finally:
        reference.set_threads(1)
    assert info[2] == 256
    errs = [_rel(got[f], want[i]) for i, f in enumerate(foci)]
    print("widefield 512x512x64 vs the reference scene, foci", foci, "max rel error", errs)
    assert max(errs) <= TOL
