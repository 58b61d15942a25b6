"""Emitter collection on the device (CollectFrameEmitters for a batch) against the host restatement, and the one-call
event render against the host-collected render and the reference's frame loop: bit for bit."""
import numpy as np
import pytest
import torch

from insiliscope_b200 import (BLINK_EVENT_DTYPE, EMITTER_DTYPE, FRAME_DTYPE, INTERP_CUBIC, CameraParams, PsfParams)

pytestmark = pytest.mark.gpu

W, H, PX = 48, 40, 108.0


def _events(rng, n, frames, slots=(0,)):
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(-0.5, W * PX / 1000 + 0.5, n)
    ev["y_um"] = rng.uniform(-0.5, H * PX / 1000 + 0.5, n)
    ev["z_nm"] = rng.uniform(-500, 500, n)
    ev["t_start"] = rng.uniform(-0.5, frames - 0.2, n)
    ev["t_end"] = ev["t_start"] + rng.uniform(0.05, 2.5, n)
    ev["brightness"] = np.where(rng.random(n) < 0.2, 1.0, rng.lognormal(0.0, 0.5, n))
    ev["excite"] = np.where(rng.random(n) < 0.5, 1.0, rng.uniform(0.3, 1.0, n))
    ev["slot"] = rng.choice(slots, n).astype(np.int32)
    return ev


def _buckets(ev, frames):
    """BucketEventsByFrame's index lists: frame k's candidates are the events overlapping [k, k + 1), in event order."""
    idx, start = [], [0]
    for k in range(frames):
        m = np.nonzero((ev["t_end"] > k) & (ev["t_start"] < k + 1))[0]
        idx.extend(m.tolist())
        start.append(len(idx))
    return np.array(idx, np.uint32), np.array(start, np.uint32)


@pytest.fixture(scope="module")
def kernels(engine, reference):
    reqs = [PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=PX, oversampling=4, kernel_half_width_px=6,
                      nz=11, z_step_nm=80.0, pupil_samples=64, interp=INTERP_CUBIC),
            PsfParams(wavelength_nm=580.0, na=1.45, pixel_size_nm=PX, oversampling=4, kernel_half_width_px=6,
                      nz=7, z_step_nm=120.0, pupil_samples=64, interp=INTERP_CUBIC, double_helix=True)]
    ks = [reference.kernel(req=r) for r in reqs]
    for s, (k, r) in enumerate(zip(ks, reqs)):
        engine.kernel_set_planes(s, k.planes(), 4, r.z_step_nm, INTERP_CUBIC)
    return ks


def _dev_collect(engine, slot, ev, bi, bs, frame0, **kw):
    nf = len(bs) - 1
    t = lambda a, dt=None: None if a is None else torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()
    d_ev = torch.from_numpy(ev.view(np.uint8)).cuda()
    cap = kw.pop("cap", max(1, int(bs[-1] - bs[0])))
    d_out = torch.zeros(cap * EMITTER_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_fr = torch.zeros(nf * FRAME_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    d_cl = torch.zeros(1, dtype=torch.int64, device="cuda")
    d_ix = torch.zeros(cap, dtype=torch.int32, device="cuda")
    per = {k: t(kw.get(k), np.float64) for k in ("drift_x_px", "drift_y_px", "global_z_offset_um", "bg_scale")}
    engine.collect_emitters_dev(slot, d_ev, len(ev), t(bs), nf, frame0, PX, 2000.0, d_out, d_fr, d_n,
                                bucket_index_dev=t(bi), drift_x_px_dev=per["drift_x_px"],
                                drift_y_px_dev=per["drift_y_px"], global_z_offset_um_dev=per["global_z_offset_um"],
                                bg_scale_dev=per["bg_scale"], illum_dev=t(kw.get("illum"), np.float32),
                                min_photons=kw.get("min_photons", 0.0), n_clamped_dev=d_cl, event_index_dev=d_ix)
    n = int(d_n.item())
    out = d_out.cpu().numpy().view(EMITTER_DTYPE)
    _dev_collect.last_index = d_ix.cpu().numpy()[:min(n, cap)]
    return out[:min(n, cap)], d_fr.cpu().numpy().view(FRAME_DTYPE), n, int(d_cl.item())


@pytest.mark.parametrize("slot", [0, -1])
@pytest.mark.parametrize("extras", [False, True])
def test_device_collection_matches_host(engine, kernels, slot, extras):
    rng = np.random.default_rng(11 + slot + 4 * extras)
    F = 9
    ev = _events(rng, 500, F, slots=(0, 1))
    bi, bs = _buckets(ev, F)
    engine.set_static(W, H, flat_bg=10.0)
    kw = {}
    if extras:
        yy, xx = np.mgrid[0:H, 0:W]
        kw = dict(drift_x_px=rng.normal(0, 0.7, F), drift_y_px=rng.normal(0, 0.7, F),
                  global_z_offset_um=rng.normal(0, 0.2, F), bg_scale=rng.uniform(0.5, 1.0, F),
                  illum=np.exp(-((xx - 20.0) ** 2 + (yy - 18.0) ** 2) / 300.0).astype(np.float32), min_photons=400.0)
    want_e, want_f, want_cl = engine.collect_emitters(slot, ev, bs, 5, W, H, PX, 2000.0, bucket_index=bi, **kw)
    got_e, got_f, n, cl = _dev_collect(engine, slot, ev, bi, bs, 5, **kw)
    assert n == len(want_e)
    assert got_e.tobytes() == want_e.tobytes()
    assert got_f.tobytes() == want_f.tobytes()
    assert cl == want_cl
    # the ground-truth list: each emitter's event, in the frame's event order
    ix = _dev_collect.last_index
    for f in range(F):
        lo, hi = got_f["em_start"][f], got_f["em_start"][f] + got_f["em_count"][f]
        cand = bi[bs[f]:bs[f + 1]]
        assert np.all(np.isin(ix[lo:hi], cand)) and np.all(np.diff(np.searchsorted(cand, ix[lo:hi])) > 0)
    if not extras:
        assert np.allclose(got_e["x_px"], ev["x_um"][ix] * 1000.0 / PX)


def test_device_collection_overflow_reports_count(engine, kernels):
    rng = np.random.default_rng(3)
    ev = _events(rng, 300, 4)
    bi, bs = _buckets(ev, 4)
    engine.set_static(W, H, flat_bg=10.0)
    want_e, _, _ = engine.collect_emitters(0, ev, bs, 0, W, H, PX, 2000.0, bucket_index=bi)
    got_e, _, n, _ = _dev_collect(engine, 0, ev, bi, bs, 0, cap=50)
    assert n == len(want_e) > 50
    assert got_e.tobytes() == want_e[:50].tobytes()


def test_render_events_matches(engine, reference, oracle, kernels):
    rng = np.random.default_rng(21)
    F = 12
    ev = _events(rng, 700, F, slots=(0, 1))
    bi, bs = _buckets(ev, F)
    off, gain, rn = oracle.camera_maps(W, H, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    engine.set_static(W, H, offset=off, gain=gain, read_noise=rn, flat_bg=15.0)
    cam = CameraParams(gain=2.2, read_noise_e=1.5)
    ems, frames, _ = engine.collect_emitters(-1, ev, bs, 0, W, H, PX, 2000.0, bucket_index=bi)
    want_ph, want_adu = engine.render_frames(ems, frames, cam, 77)
    for config in (0, 12):
        engine.set_render_config(config)
        try:
            ph, adu, n = engine.render_events(-1, ev, bs, 0, PX, 2000.0, cam, 77, bucket_index=bi,
                                              want_photons=True)
        finally:
            engine.set_render_config(0)
        assert n == len(ems)
        assert np.array_equal(ph, want_ph) and np.array_equal(adu, want_adu), config
    # one dye group against the reference's own frame loop (events in frame order, no index lists)
    ev0 = ev[ev["slot"] == 0].copy()
    ev0 = ev0[np.argsort(ev0["t_start"], kind="stable")]
    ev0["t_start"] = np.floor(ev0["t_start"]).clip(0, F - 1)
    ev0["t_end"] = ev0["t_start"] + 1.0
    counts = np.bincount(ev0["t_start"].astype(int), minlength=F)
    bs0 = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    _, adu, _ = engine.render_events(0, ev0, bs0, 0, PX, 2000.0, cam, 5)
    _, _, want = kernels[0].render_movie(ev0, 0, F, W, H, PX, 2000.0, 15.0, cam, off, gain, rn, 5)
    assert np.array_equal(adu, want)


def test_render_events_async_pipeline(engine, kernels):
    """Batches of one movie enqueued across the I/O slots, up to three in flight, into page-locked host frames: each
    equals the blocking call's frames bit for bit and reports the emitters the host collection keeps; a busy slot
    refuses a second batch and keeps its first, and an idle slot refuses a wait."""
    from insiliscope_b200 import IscuError
    rng = np.random.default_rng(41)
    B, NB = 10, 6
    ev = _events(rng, 2400, B * NB, slots=(0, 1))
    engine.set_static(W, H, flat_bg=12.0)
    cam = CameraParams(gain=2.0, read_noise_e=1.4)
    batches = []
    for b in range(NB):
        bi, bs = _buckets(ev, B * (b + 1))
        batches.append((bi, bs[B * b:]))
    pinned = [torch.empty((B, H, W), dtype=torch.uint16).pin_memory().numpy() for _ in range(3)]
    want = [engine.render_events(-1, ev, bs, B * b, PX, 2000.0, cam, 9, bucket_index=bi)
            for b, (bi, bs) in enumerate(batches)]
    kept = [len(engine.collect_emitters(-1, ev, bs, B * b, W, H, PX, 2000.0, bucket_index=bi)[0])
            for b, (bi, bs) in enumerate(batches)]
    assert [w[2] for w in want] == kept and min(kept) > 0
    got = [None] * NB
    for b, (bi, bs) in enumerate(batches):
        io = b % 3
        if b >= 3:
            _, adu, n = engine.render_events_wait(io)
            got[b - 3] = (adu.copy(), n)
        engine.render_events_async(io, -1, ev, bs, B * b, PX, 2000.0, cam, 9, bucket_index=bi, adu_out=pinned[io])
        if b == 0:
            with pytest.raises(IscuError):
                engine.render_events_async(0, -1, ev, bs, 0, PX, 2000.0, cam, 9, bucket_index=bi,
                                           adu_out=pinned[1])
    for b in range(NB - 3, NB):
        _, adu, n = engine.render_events_wait(b % 3)
        got[b] = (adu.copy(), n)
    for b in range(NB):
        assert got[b][1] == kept[b], b
        assert np.array_equal(got[b][0], want[b][1]), b
    with pytest.raises(IscuError):
        engine.render_events_wait(0)
    with pytest.raises(IscuError):
        engine.render_events_async(engine.EVENT_IO_SLOTS, -1, ev, batches[0][1], 0, PX, 2000.0, cam, 9,
                                   bucket_index=batches[0][0])
