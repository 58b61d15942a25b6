"""The splat's Fft placement on the B200 (iscu_fft_place_dev: the shift as a float64 convolution, no transform)
against the reference's own PlanSplat with PsfInterpMode::Fft (its FFT route, oracle/_ref) and the float64
restatement: the same tap origins, the shifted block sums within 1e-6 of their maximum; emitters PlanSplat refuses
marked and left blank."""
import numpy as np
import pytest

from insiliscope_b200 import EMITTER_DTYPE
from oracle.oracle import fft_place_f64
from test_fft_place_oracle import place_positions, place_request

pytestmark = pytest.mark.gpu


def test_device_equals_reference(engine, reference, oracle):
    import torch
    k = reference.kernel(req=place_request())
    planes = k.planes()
    size, nz, os_, bw = k.info()
    engine.kernel_set_planes(2, planes, os_, 100.0)
    xy, z = place_positions(2, 300, nz)
    em = np.zeros(len(z) + 2, EMITTER_DTYPE)
    em["x_px"][:len(z)], em["y_px"][:len(z)], em["plane"][:len(z)] = xy[:, 0], xy[:, 1], z
    em["photons"] = 1000.0
    em[-2]["photons"] = 0.0                     # refused: no photons
    em[-1]["plane"] = nz                        # refused: beyond the stack
    sums, origins = engine.fft_place_dev(2, torch.from_numpy(em.view(np.uint8)).cuda())
    sums, origins = sums.cpu().numpy(), origins.cpu().numpy()
    for i, ((x, y), p) in enumerate(zip(xy, z)):
        want, st = k.plan_splat_fft(x, y, int(p))
        assert tuple(origins[i]) == st
        assert np.abs(sums[i] - want).max() <= 1e-6 * np.abs(want).max(), i
        if i < 40:
            tile, _ = fft_place_f64(planes, os_, x, y, int(p))
            ora = oracle.block_sums(tile[None], os_)[0]
            assert np.abs(sums[i] - ora).max() <= 1e-6 * np.abs(ora).max()
    for i in (-2, -1):
        assert origins[i][0] == np.iinfo(np.int32).min and not sums[i].any()


@pytest.mark.parametrize("halo", [None, 0.002])
def test_fft_frames_equal_reference(engine, reference, halo):
    """Frames in the Fft placement (iscu_render_fft_frames_dev) against the reference's RenderPhotonImage with an Fft
    kernel cache of the same planes: the same emitters (the engine's collection, bit for bit the reference's), the
    background, every emitter at its one tap of its shifted sums in list order, the halo cut's spans; the frames
    within 1e-6 of their maximum (the shifted planes' float rounding may differ in a last place)."""
    import torch
    from insiliscope_b200 import BLINK_EVENT_DTYPE
    W, H, PX, F = 48, 40, 108.0, 5
    k = reference.kernel(req=place_request())
    planes = k.planes()
    size, nz, os_, bw = k.info()
    kf = reference.kernel(planes=planes, os_=os_, z_step_nm=100.0, interp=3)   # PsfInterpMode::Fft
    engine.kernel_set_planes(3, planes, os_, 100.0)
    if halo is not None:
        kf = kf.halo(halo)
        engine.kernel_set_halo(3, halo)
    rng = np.random.default_rng(9)
    n = 240
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(-0.5, W * PX / 1000 + 0.5, n)
    ev["y_um"] = rng.uniform(-0.5, H * PX / 1000 + 0.5, n)
    ev["z_nm"] = rng.uniform(-400, 400, n)
    ev["t_start"] = np.sort(rng.integers(0, F, n)).astype(np.float64)
    ev["t_end"] = ev["t_start"] + 1.0
    ev["brightness"] = rng.lognormal(0.0, 0.5, n)
    ev["excite"] = 1.0
    ev["slot"] = 3
    bs = np.concatenate([[0], np.cumsum(np.bincount(ev["t_start"].astype(int), minlength=F))]).astype(np.uint32)
    engine.set_static(W, H, flat_bg=12.0)
    ems, frames, _ = engine.collect_emitters(3, ev, bs, 0, W, H, PX, 2000.0)
    ph = torch.zeros((F, H, W), dtype=torch.float32, device="cuda")
    engine.render_fft_frames_dev(3, torch.from_numpy(ems.view(np.uint8)).cuda(),
                                 torch.from_numpy(frames.view(np.uint8)).cuda(), F, None, 0, photons_dev=ph)
    got = ph.cpu().numpy()
    for f in range(F):
        want = kf.render_photon_image(ev[bs[f]:bs[f + 1]], f, W, H, PX, 2000.0, 12.0)
        assert np.abs(got[f] - want).max() <= 1e-6 * np.abs(want).max(), f
    if halo is not None:
        engine.kernel_set_halo(3, 0.0)


@pytest.mark.parametrize("n,os_", [(7, 1), (17, 2), (31, 3), (157, 3)])
def test_plane_sizes(engine, oracle, n, os_):
    """Plane sizes beside the SMLM kernel's 129 (odd, the half width a multiple of the oversampling): shorter than one
    eight-step block (7), one past two blocks (17), seven past three (31) and the largest (157), against the float64
    restatement within 1e-6 of the sums' maximum."""
    import torch
    rng = np.random.default_rng(n)
    nz = 3
    planes = (rng.random((nz, n, n)) ** 3).astype(np.float32)
    engine.kernel_set_planes(3, planes, os_, 100.0)
    xy = rng.uniform(5.0, 60.0, (12, 2))
    xy[0] = [20.0, 30.0]
    z = rng.integers(0, nz, len(xy))
    em = np.zeros(len(z), EMITTER_DTYPE)
    em["x_px"], em["y_px"], em["plane"], em["photons"] = xy[:, 0], xy[:, 1], z, 500.0
    sums, origins = engine.fft_place_dev(3, torch.from_numpy(em.view(np.uint8)).cuda())
    sums, origins = sums.cpu().numpy(), origins.cpu().numpy()
    for i, ((x, y), p) in enumerate(zip(xy, z)):
        tile, st = fft_place_f64(planes, os_, x, y, int(p))
        assert tuple(origins[i]) == st
        ora = oracle.block_sums(tile[None], os_)[0]
        assert np.abs(sums[i] - ora).max() <= 1e-6 * np.abs(ora).max(), (n, i)
