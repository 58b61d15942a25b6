"""The render kernel's forms on an uneven two-colour movie: every tile shape, grid or persistent, the autotuned form
and the captured CUDA graph give the reference's frames bit for bit (the reference's multi-colour frame loop: each
dye group with its own kernel, the later group splatted onto the earlier one, then the noise chain)."""
import numpy as np
import pytest
import torch

from insiliscope_b200 import BLINK_EVENT_DTYPE, INTERP_CUBIC, CameraParams, PsfParams, RenderGraph
from insiliscope_b200.workloads import noll_rms_to_osa_waves

pytestmark = pytest.mark.gpu

W, H, F, PX = 72, 56, 23, 108.0
PER_BLINK, BG = 1800.0, 15.0


def _requests():
    common = dict(na=1.45, pixel_size_nm=PX, oversampling=4, kernel_half_width_px=8, nz=9, z_step_nm=100.0,
                  pupil_samples=64, interp=INTERP_CUBIC)
    return [PsfParams(wavelength_nm=670.0, double_helix=True, **common),
            PsfParams(wavelength_nm=580.0, zernike=noll_rms_to_osa_waves({5: 0.1}), **common)]


def _movie(rng, frames=F):
    """Frame f: Poisson(mu_f) emitters, mu_f lognormal (median 40, sigma 1.2) clipped to [0.5, 400]; channel 0 then 1
    within each frame."""
    mu = np.clip(40.0 * np.exp(1.2 * rng.standard_normal(frames)), 0.5, 400.0)
    counts = rng.poisson(mu)
    counts[3] = 0                                  # an empty frame
    n = int(counts.sum())
    fi = np.repeat(np.arange(frames), counts)
    ch = (rng.random(n) < 0.5).astype(np.int32)
    order = np.lexsort((ch, fi))
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(-0.5, W * PX / 1000 + 0.5, n)
    ev["y_um"] = rng.uniform(-0.5, H * PX / 1000 + 0.5, n)
    ev["z_nm"] = rng.uniform(-450, 450, n)
    ev["t_start"] = fi.astype(np.float64)
    ev["t_end"] = ev["t_start"] + 1.0
    ev["brightness"] = rng.lognormal(0.0, 0.5, n)
    ev["excite"] = 1.0
    ev["slot"] = ch
    ev = ev[order]
    return ev, np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)


@pytest.fixture(scope="module")
def setup(engine, reference, oracle):
    kernels = [reference.kernel(req=r) for r in _requests()]
    for s, k in enumerate(kernels):
        engine.kernel_set_planes(s, k.planes(), 4, 100.0, INTERP_CUBIC)
    off, gain, rn = oracle.camera_maps(W, H, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    engine.set_static(W, H, offset=off, gain=gain, read_noise=rn, flat_bg=BG)
    cam = CameraParams(gain=2.2, read_noise_e=1.5)
    return kernels, (off, gain, rn), cam


def _batch(engine, ev, bucket):
    ems, frames, _ = engine.collect_emitters(-1, ev, bucket, 0, W, H, PX, PER_BLINK)
    return ems.copy(), frames.copy()


def _dev(engine, ems, frames):
    d_em = torch.from_numpy(np.ascontiguousarray(ems).view(np.uint8)).cuda()
    d_fr = torch.from_numpy(np.ascontiguousarray(frames).view(np.uint8)).cuda()
    n = len(frames)
    d_ph = torch.empty((n, H, W), dtype=torch.float32, device="cuda")
    d_adu = torch.empty((n, H, W), dtype=torch.uint16, device="cuda")
    return d_em, d_fr, d_ph, d_adu


def test_forms_match_reference(engine, reference, setup):
    kernels, (off, gain, rn), cam = setup
    rng = np.random.default_rng(31)
    ev, bucket = _movie(rng)
    ems, frames = _batch(engine, ev, bucket)
    assert ems["plane"].max() >> 16 == 1 and ems["plane"].min() >> 16 == 0
    seed = 1234
    _, want_ph, want_adu = reference.render_movie_groups(kernels, ev, 0, F, W, H, PX, PER_BLINK, BG, cam,
                                                         off, gain, rn, seed, want_photons=True)
    try:
        for config in range(engine.RENDER_CONFIGS):
            engine.set_render_config(config)
            assert engine.render_config()[0] == config
            ph, adu = engine.render_frames(ems, frames, cam, seed)
            assert np.array_equal(ph, want_ph), config
            assert np.array_equal(adu, want_adu), config
            ph2, _ = engine.render_frames(ems, frames, None, 0, want_adu=False)
            assert np.array_equal(ph2, want_ph), config
    finally:
        engine.set_render_config(0)


@pytest.mark.parametrize("emccd", [False, True])
def test_two_pass_noise_without_photons(engine, reference, setup, emccd):
    """The two-pass forms when the caller keeps no photon frames (the tiles' photon values in scratch ahead of the
    pooled noise chain), on an sCMOS and an EMCCD camera: the reference's frames bit for bit."""
    kernels, (off, gain, rn), _ = setup
    cam = CameraParams(quantum_efficiency=0.9, dark_electrons=0.02, gain=2.2 if not emccd else 4.0, read_noise_e=1.5,
                       emccd=emccd, em_gain=150.0, cic_electrons=0.003)
    rng = np.random.default_rng(41)
    ev, bucket = _movie(rng)
    ems, frames = _batch(engine, ev, bucket)
    seed = 99
    _, _, want_adu = reference.render_movie_groups(kernels, ev, 0, F, W, H, PX, PER_BLINK, BG, cam, off, gain, rn,
                                                   seed)
    try:
        for config in range(12, engine.RENDER_CONFIGS):
            engine.set_render_config(config)
            ph, adu = engine.render_frames(ems, frames, cam, seed, want_photons=False)
            assert ph is None
            assert np.array_equal(adu, want_adu), config
    finally:
        engine.set_render_config(0)


def test_autotune_and_graph(engine, reference, setup):
    kernels, (off, gain, rn), cam = setup
    rng = np.random.default_rng(77)
    ev, bucket = _movie(rng)
    ems, frames = _batch(engine, ev, bucket)
    d_em, d_fr, d_ph, d_adu = _dev(engine, ems, frames)
    try:
        ms = engine.render_autotune(d_em, d_fr, F, cam, 5, d_adu)
        assert len(ms) == engine.RENDER_CONFIGS and all(m > 0 for m in ms)
        config = engine.render_config()[0]
        assert ms[config] == min(ms)
        ph_h, adu_h = engine.render_frames(ems, frames, cam, 5)
        for persistent_config in (config, 4, 9, 12, 15):
            engine.set_render_config(persistent_config)
            g = RenderGraph(engine, d_em, d_fr, F, cam, 5, d_ph, d_adu)
            d_ph.zero_()
            d_adu.zero_()
            n0 = engine.launch_count
            g.launch()
            assert engine.launch_count > n0
            assert np.array_equal(d_ph.cpu().numpy(), ph_h)
            assert np.array_equal(d_adu.cpu().numpy(), adu_h)
            # the same buffers refilled in place with another batch of the same size: the replay renders it
            ems2 = ems.copy()
            ems2["photons"] *= 0.5
            d_em.copy_(torch.from_numpy(ems2.view(np.uint8)))
            g.launch()
            ph2, adu2 = engine.render_frames(ems2, frames, cam, 5)
            assert np.array_equal(d_ph.cpu().numpy(), ph2)
            assert np.array_equal(d_adu.cpu().numpy(), adu2)
            d_em.copy_(torch.from_numpy(ems.view(np.uint8)))
            g.close()
        _, _, want_adu = reference.render_movie_groups(kernels, ev, 0, F, W, H, PX, PER_BLINK, BG, cam, off, gain, rn,
                                                       5)
        assert np.array_equal(adu_h, want_adu)
    finally:
        engine.set_render_config(0)


def test_heavy_frame_batch(engine, setup):
    """A batch whose frames run from 0 to 3,000 emitters: the persistent forms equal the grid form."""
    _, _, cam = setup
    rng = np.random.default_rng(5)
    counts = np.array([0, 3000, 2, 900, 40, 1, 2200, 0, 10], np.int64)
    n = int(counts.sum())
    fi = np.repeat(np.arange(len(counts)), counts)
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(0, W * PX / 1000, n)
    ev["y_um"] = rng.uniform(0, H * PX / 1000, n)
    ev["z_nm"] = rng.uniform(-400, 400, n)
    ev["t_start"] = fi
    ev["t_end"] = fi + 1.0
    ev["brightness"] = 1.0
    ev["excite"] = 1.0
    ev["slot"] = (rng.random(n) < 0.3).astype(np.int32)
    ev = ev[np.lexsort((ev["slot"], fi))]
    ems, frames = _batch(engine, ev, np.concatenate([[0], np.cumsum(counts)]))
    try:
        engine.set_render_config(0)
        want = engine.render_frames(ems, frames, cam, 9)
        for config in (3, 4, 5, 6, 9, 11, 12, 13, 14, 15, 16, 17):
            engine.set_render_config(config)
            got = engine.render_frames(ems, frames, cam, 9)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), config
    finally:
        engine.set_render_config(0)


def test_two_pass_over_limit_falls_back(engine, reference, setup):
    """A two-pass form whose contributions pass the limit renders in the one-pass form: the same bits."""
    kernels, (off, gain, rn), cam = setup
    ev, bucket = _movie(np.random.default_rng(8))
    ems, frames = _batch(engine, ev, bucket)
    try:
        engine.set_render_config(15)
        want = engine.render_frames(ems, frames, cam, 3)
        engine.set_contrib_limit(1024)
        got = engine.render_frames(ems, frames, cam, 3)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    finally:
        engine.set_contrib_limit(0)
        engine.set_render_config(0)


def test_bad_config_rejected(engine):
    from insiliscope_b200 import IscuError
    with pytest.raises(IscuError):
        engine.set_render_config(engine.RENDER_CONFIGS)
    assert engine.render_config()[0] in range(engine.RENDER_CONFIGS)
