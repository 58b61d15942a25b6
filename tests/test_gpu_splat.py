"""Blink splat + noise on the B200 against the reference's CPU renderer (RenderPhotonImage + ApplyNoiseChain, built
here from its sources) and the oracle: noise-free photon images and ADU frames bit for bit."""
import numpy as np
import pytest

from insiliscope_b200 import (BLINK_EVENT_DTYPE, EMITTER_DTYPE, INTERP_CUBIC, INTERP_LINEAR, INTERP_NEAREST,
                              CameraParams, PsfParams, frames_table)

pytestmark = pytest.mark.gpu


def _kernel_req(interp, half=6, nz=9):
    req = PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=108.0, oversampling=4, kernel_half_width_px=half,
                    nz=nz, z_step_nm=60.0, pupil_samples=64, interp=interp)
    req.zernike[3] = 0.11
    req.zernike[8] = -0.04
    return req


def _events(rng, n, W, H, frames, px_nm=108.0):
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(-0.6, W * px_nm / 1000 + 0.6, n)
    ev["y_um"] = rng.uniform(-0.6, H * px_nm / 1000 + 0.6, n)
    ev["z_nm"] = rng.uniform(-350, 350, n)
    ev["t_start"] = rng.uniform(-0.5, frames - 0.2, n)
    ev["t_end"] = ev["t_start"] + rng.uniform(0.05, 2.5, n)
    ev["brightness"] = rng.lognormal(0.0, 0.5, n)
    ev["excite"] = 1.0
    return ev


def _collect(engine, slot, ev, frames, W, H, **kw):
    per = []
    for f in range(frames):
        e, _ = engine.collect_frame_emitters(slot, ev, f, W, H, 108.0, 2000.0, **kw)
        per.append(e)
    return np.concatenate(per) if per else np.zeros(0, EMITTER_DTYPE), [len(p) for p in per]


@pytest.mark.parametrize("interp", [INTERP_NEAREST, INTERP_LINEAR, INTERP_CUBIC])
def test_block_sums_and_render_bit_exact(engine, reference, oracle, interp):
    rng = np.random.default_rng(100 + interp)
    k = reference.kernel(req=_kernel_req(interp))
    planes = k.planes()
    engine.kernel_set_planes(0, planes, 4, 60.0, interp)
    assert np.array_equal(engine.kernel_block_sums(0), k.block_sums())
    W, H, F = 45, 38, 5
    ev = _events(rng, 220, W, H, F)
    off, gain, rn = oracle.camera_maps(W, H, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    engine.set_static(W, H, offset=off, gain=gain, read_noise=rn, flat_bg=20.0)
    ems, counts = _collect(engine, 0, ev, F, W, H)
    for f in range(F):
        want_e = oracle.collect_frame_emitters(ev, f, 108.0, 2000.0, planes.shape[0], 60.0)
        assert np.array_equal(ems[sum(counts[:f]):sum(counts[:f + 1])], want_e)
    cam = CameraParams(quantum_efficiency=1.0, gain=2.2, read_noise_e=1.5)
    seed = 42 ^ 0x9E3779B9
    ph, adu = engine.render_frames(ems, frames_table(counts), cam, seed)
    for f in range(F):
        want = k.render_photon_image(ev, f, W, H, 108.0, 2000.0, 20.0)
        assert np.array_equal(ph[f], want), f
        want_adu = reference.noise_chain(want, cam, off.reshape(H, W), gain.reshape(H, W), rn.reshape(H, W), seed, f)
        assert np.array_equal(adu[f], want_adu), f


def test_render_extras_bit_exact(engine, reference, oracle):
    """Drift, global z, min photons, illumination field, background map and fade, and the halo cut."""
    rng = np.random.default_rng(7)
    k = reference.kernel(req=_kernel_req(INTERP_CUBIC, half=7, nz=11))
    kh = k.halo(2e-4)
    engine.kernel_set_planes(1, k.planes(), 4, 60.0, INTERP_CUBIC)
    engine.kernel_set_halo(1, 2e-4)
    W, H, F = 50, 41, 3
    yy, xx = np.mgrid[0:H, 0:W]
    illum = np.exp(-((xx - 20.0) ** 2 + (yy - 25.0) ** 2) / (2 * 18.0 ** 2)).astype(np.float32)
    bg_map = (12.0 + 6.0 * np.sin(xx / 5.0) * np.cos(yy / 7.0)).astype(np.float32)
    engine.set_static(W, H, background=bg_map, illum=illum, flat_bg=0.0)
    ev = _events(rng, 150, W, H, F)
    all_e, counts = [], []
    for f in range(F):
        e, _ = engine.collect_frame_emitters(1, ev, f, W, H, 108.0, 2000.0, drift_x_px=0.37 * f, drift_y_px=-0.21 * f,
                                             global_z_offset_um=0.04, illum=illum, min_photons=250.0)
        all_e.append(e)
        counts.append(len(e))
    scales = [1.0, 0.83, 0.61]
    ph, _ = engine.render_frames(np.concatenate(all_e), frames_table(counts, bg_scales=scales), None, 0,
                                 want_adu=False)
    for f in range(F):
        want = kh.render_photon_image(ev, f, W, H, 108.0, 2000.0, 0.0, drift_x=0.37 * f, drift_y=-0.21 * f,
                                      global_z=0.04, illum=illum, bg_map=bg_map, bg_scale=scales[f], min_photons=250.0)
        assert np.array_equal(ph[f], want), f


def test_device_path_matches_host_path(engine, reference):
    import torch
    rng = np.random.default_rng(3)
    k = reference.kernel(req=_kernel_req(INTERP_CUBIC))
    engine.kernel_set_planes(0, k.planes(), 4, 60.0, INTERP_CUBIC)
    W, H, F = 64, 64, 4
    engine.set_static(W, H, flat_bg=20.0)
    ev = _events(rng, 300, W, H, F)
    ems, counts = _collect(engine, 0, ev, F, W, H)
    fr = frames_table(counts)
    cam = CameraParams(gain=2.2, read_noise_e=1.5)
    ph_h, adu_h = engine.render_frames(ems, fr, cam, 9)
    d_em = torch.from_numpy(ems.view(np.uint8)).cuda()
    d_fr = torch.from_numpy(fr.view(np.uint8)).cuda()
    d_ph = torch.empty((F, H, W), dtype=torch.float32, device="cuda")
    d_adu = torch.empty((F, H, W), dtype=torch.uint16, device="cuda")
    engine.render_frames_dev(d_em, d_fr, F, cam, 9, d_ph, d_adu)
    engine.synchronize()
    assert np.array_equal(d_ph.cpu().numpy(), ph_h)
    assert np.array_equal(d_adu.cpu().numpy(), adu_h)


@pytest.mark.parametrize("emccd", [False, True])
def test_reference_records_selfcheck(engine, reference, oracle, emccd):
    """The reference's own GPU seam contract (SplatGpuHost::SelfCheck, SplatGpu.cpp:464-540): 400 blinks on 64 x 64
    through CollectGpuEmitters' 64-byte records against RenderPhotonImage + ApplyNoiseChain. The reference accepts
    >= 90 % equal pixels; float weights in the record leave only rounding-level differences here."""
    rng = np.random.default_rng(12345)
    req = PsfParams(wavelength_nm=670.0, na=1.4, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=6,
                    nz=5, z_step_nm=100.0, interp=INTERP_CUBIC)
    k = reference.kernel(req=req)
    engine.kernel_set_planes(2, k.planes(), 4, 100.0, INTERP_CUBIC)
    W = H = 64
    ev = np.zeros(400, BLINK_EVENT_DTYPE)
    ev["x_um"] = 6.4 * rng.uniform(size=400)
    ev["y_um"] = 6.4 * rng.uniform(size=400)
    ev["z_nm"] = 300 * rng.uniform(size=400) - 150
    ev["t_start"] = 0.3 * rng.uniform(size=400) - 0.1
    ev["t_end"] = ev["t_start"] + 0.5 + rng.uniform(size=400)
    ev["brightness"] = 0.5 + rng.uniform(size=400)
    ev["excite"] = 1.0
    off, gain, rn = oracle.camera_maps(W, H, 12345, 100.0, 2.0, 0.25, 0.005 / 0.25, 1.2, 0.2)
    cam = CameraParams(quantum_efficiency=0.85, dark_electrons=0.05, gain=0.25, read_noise_e=1.2, emccd=emccd)
    cpu = k.render_photon_image(ev, 0, W, H, 100.0, 1500.0, 20.0, drift_x=0.3, drift_y=-0.2, global_z=0.05)
    want = reference.noise_chain(cpu, cam, off.reshape(H, W), gain.reshape(H, W), rn.reshape(H, W), 777, 3)
    rec = k.collect_gpu_emitters(ev, 0, W, H, 100.0, 1500.0, drift_x=0.3, drift_y=-0.2, global_z=0.05, kernel=2)
    engine.set_static(W, H, offset=off, gain=gain, read_noise=rn, flat_bg=0.0)
    fr = frames_table([len(rec)], frame_ids=[3])
    got = engine.render_gpu_records(rec, fr, cam, 777, extras=np.full(W * H, 20.0, np.float32))[0]
    same = (got == want).mean()
    assert same >= 0.99, same
    assert np.abs(got.astype(float) - want).sum() <= 0.001 * want.sum()


@pytest.mark.parametrize("interp,half,thr", [(INTERP_CUBIC, 16, 1e-4), (INTERP_CUBIC, 7, 2e-3), (INTERP_LINEAR, 9, 5e-4),
                                             (INTERP_NEAREST, 12, 1e-5), (INTERP_CUBIC, 16, 0.5)])
def test_halo_spans_equal_reference(engine, reference, interp, half, thr):
    """The halo cut computed on the device from the resident block sums equals the reference's WithHaloCut spans
    (PsfHaloSpans lo / hi / radius2) for every plane and row, empty rows and a threshold nothing reaches included."""
    req = _kernel_req(interp, half=half, nz=13)
    k = reference.kernel(req=req)
    engine.kernel_set_planes(2, k.planes(), 4, 60.0, interp)
    engine.kernel_set_halo(2, thr)
    lo, hi, r2 = engine.kernel_halo(2)
    want = k.halo(thr).spans()
    assert want is not None
    assert np.array_equal(lo.ravel(), want[0]) and np.array_equal(hi.ravel(), want[1])
    assert np.array_equal(r2, want[2])
    if thr >= 0.5:
        assert (r2 == -1).all() and (lo > hi).all()
    engine.kernel_set_halo(2, 0.0)
