"""Parity at the benchmarked configurations' own sizes, through the C ABI, against the reference compiled from its
sources (oracle/_ref) and the float64 oracle:

- the plain dSTORM movie (128 x 128 px, 200 frames, ~160 ON per frame, 129^2 x 49 Catmull-Rom kernel, sCMOS):
  every frame's photons and ADU equal the reference's RenderPhotonImage + ApplyNoiseChain frame loop, for every
  render form; the mismatched-pixel counts are printed (they must be 0: the noise draws call CUDA's float64
  log/exp/cos where the reference calls glibc's, and over the movie's 3.3 M pixel draws none lands on another count);
- the uneven two-colour movie (256 x 256 px, 1,024 frames, 10 to ~8,000 ON per frame): the whole movie rendered on
  the device -- the two-pass form with its full contribution buffer, and the same form forced onto its one-pass
  fallback by a contribution cap -- and a window of frames that holds the heaviest frame compared with the
  reference's two-group frame loop;
- the 4,096-PSF library (128^2 pupils -> 64^2, TF32 x 3 on the tensor cores): every PSF within 1e-5 of the float64
  oracle (max |I - I64| / max I64), worst and median printed;
- the NLL gradient over 256 frames x 1,000 ROIs: frame subsets against the float64 adjoint (<= 1e-4 relative).
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

from insiliscope_b200 import CZT_F16X3, CZT_TF32X3, PsfPlan

pytestmark = pytest.mark.gpu


def _mismatch(a, b):
    return int(np.count_nonzero(a != b))


@pytest.fixture(scope="module")
def c0(engine, reference):
    from insiliscope_b200.workloads import smlm_dstorm
    mv = smlm_dstorm(seed=42)
    k = reference.kernel(req=mv.psf)
    maps = reference.camera_maps(mv.width, mv.height, mv.map_seed, mv.offset_mean, mv.offset_std, mv.gain_nominal,
                                 mv.gain_std_fraction, mv.read_noise_nominal, mv.read_noise_std_fraction)
    reference.set_threads(0)
    try:
        _, ph, adu = k.render_movie(mv.events, 0, mv.frames, mv.width, mv.height, mv.pixel_nm, mv.photons_per_blink,
                                    mv.background, mv.camera, *maps, mv.noise_seed, want_photons=True)
    finally:
        reference.set_threads(1)
    return mv, k, maps, ph, adu


def test_c0_full_movie_every_form_bit_exact(engine, c0):
    mv, k, maps, want_ph, want_adu = c0
    assert mv.frames == 200 and mv.width == mv.height == 128 and len(mv.events) / mv.frames > 140
    planes = k.planes()
    assert planes.shape == (49, 129, 129)
    engine.kernel_set_planes(0, planes, mv.psf.oversampling, mv.psf.z_step_nm, mv.psf.interp)
    engine.set_static(mv.width, mv.height, offset=maps[0], gain=maps[1], read_noise=maps[2], flat_bg=mv.background)
    counts = []
    try:
        for form in range(engine.RENDER_CONFIGS):
            engine.set_render_config(form)
            ph, adu, n = engine.render_events(0, mv.events, mv.bucket_start, 0, mv.pixel_nm, mv.photons_per_blink,
                                              mv.camera, mv.noise_seed, want_photons=True)
            counts.append((form, n, _mismatch(ph, want_ph), _mismatch(adu, want_adu)))
    finally:
        engine.set_render_config(0)
    print("C0 128x128x200: (form, emitters, photon pixels differing, ADU pixels differing):", counts)
    assert all(c[1] == len(mv.events) for c in counts)
    assert all(c[2] == 0 and c[3] == 0 for c in counts), counts


def test_c0_kernel_built_on_device_within_1e5(engine, c0, oracle):
    """The C0 kernel stack (49 planes, 64^2 pupil -> 129^2) built on the device equals the float64 oracle's within
    1e-5 of each plane's maximum and the reference's own planes within the same bar."""
    from insiliscope_b200 import CZT_FP32
    mv, k, _, _, _ = c0
    engine.kernel_build(3, mv.psf, CZT_FP32)
    got = engine.kernel_planes(3)
    want = oracle.psf_planes(mv.psf, oracle.stack_defocus_m(mv.psf), normalize=True)
    ref = k.planes()
    e64 = max(float(np.abs(got[z] - want[z]).max() / want[z].max()) for z in range(len(want)))
    eref = max(float(np.abs(got[z] - ref[z]).max() / ref[z].max()) for z in range(len(ref)))
    print(f"C0 kernel: max rel error vs float64 oracle {e64:.3e}, vs the reference's planes {eref:.3e}")
    assert e64 <= 1e-5 and eref <= 1e-5


@pytest.fixture(scope="module")
def c3(engine, reference):
    from insiliscope_b200.workloads import two_colour_uneven
    mv = two_colour_uneven(seed=42)
    ks = [reference.kernel(req=p) for p in mv.psfs]
    maps = reference.camera_maps(mv.width, mv.height, mv.map_seed, mv.offset_mean, mv.offset_std, mv.gain_nominal,
                                 mv.gain_std_fraction, mv.read_noise_nominal, mv.read_noise_std_fraction)
    counts = np.diff(mv.bucket_start.astype(np.int64))
    heavy = int(np.argmax(counts))
    lo = max(0, min(heavy - 12, mv.frames - 24))
    reference.set_threads(0)
    try:
        _, ph, adu = reference.render_movie_groups(ks, mv.events, lo, 24, mv.width, mv.height, mv.pixel_nm,
                                                   mv.photons_per_blink, mv.background, mv.camera, *maps,
                                                   mv.noise_seed, want_photons=True)
    finally:
        reference.set_threads(1)
    return mv, ks, maps, counts, heavy, lo, ph, adu


@pytest.mark.parametrize("cap", [0, 64 << 20])
def test_c3_whole_movie_two_pass_and_fallback(engine, c3, cap):
    """The two-pass form over the whole 1,024-frame movie (cap 0: the contribution buffer at its full ~2 GB), and the
    same form with a 64 MB cap, which sends it to its one-pass fallback; the window around the heaviest frame equals
    the reference bit for bit, and the two runs equal each other on every frame."""
    mv, ks, maps, counts, heavy, lo, want_ph, want_adu = c3
    assert counts.max() > 6000 and counts.min() < 60 and mv.frames == 1024
    for s, k in enumerate(ks):
        engine.kernel_set_planes(s, k.planes(), mv.psfs[s].oversampling, mv.psfs[s].z_step_nm, mv.psfs[s].interp)
    engine.set_static(mv.width, mv.height, offset=maps[0], gain=maps[1], read_noise=maps[2], flat_bg=mv.background)
    two_pass = [c for c in range(engine.RENDER_CONFIGS) if _passes(engine, c) == 2]
    assert two_pass
    engine.set_contrib_limit(cap)
    engine.set_render_config(two_pass[0])
    try:
        ph, adu, n = engine.render_events(-1, mv.events, mv.bucket_start, 0, mv.pixel_nm, mv.photons_per_blink,
                                          mv.camera, mv.noise_seed, want_photons=True)
    finally:
        engine.set_render_config(0)
        engine.set_contrib_limit(0)
    assert n == len(mv.events)
    w = slice(lo, lo + 24)
    d_ph, d_adu = _mismatch(ph[w], want_ph), _mismatch(adu[w], want_adu)
    print(f"C3 cap {cap}: frames {lo}..{lo + 23} (heaviest {heavy}: {counts[heavy]} emitters): photon pixels "
          f"differing {d_ph}, ADU pixels differing {d_adu}")
    assert d_ph == 0 and d_adu == 0
    key = "movie"
    if key in _c3_runs:
        a_ph, a_adu = _c3_runs[key]
        assert np.array_equal(a_ph, ph) and np.array_equal(a_adu, adu)
    else:
        _c3_runs[key] = (ph, adu)


_c3_runs = {}


def _passes(engine, config):
    engine.set_render_config(config)
    try:
        return engine.render_config()[4]
    finally:
        engine.set_render_config(0)


@pytest.mark.parametrize("method", [CZT_TF32X3, CZT_F16X3])
def test_c2_whole_library_within_1e5(engine, oracle, method):
    """Every PSF of the 4,096-PSF library from the split-precision tensor-core chirp-Z (TF32 x 3, FP16 x 3) within 1e-5
    of the float64 oracle."""
    from insiliscope_b200.workloads import psf_library
    L = psf_library(seed=42)
    plan = PsfPlan(engine, L.sets, size=L.size, method=method)
    got = plan.run(L.set_of_psf, L.defocus_nm)
    assert got.shape == (4096, 64, 64)
    err, l2 = library_errors(oracle, L, got)
    print(f"C2 4096 PSFs, method {method}: max |I - I64| / max I64 worst {err.max():.3e}, median {np.median(err):.3e}; "
          f"rel L2 worst {l2.max():.3e}")
    assert err.max() <= 1e-5


def library_errors(oracle, L, got, threads=16):
    """Per PSF: max |I - I64| / max I64 and ||I - I64|| / ||I64|| against the float64 oracle (sets in parallel)."""
    n = len(L.set_of_psf)
    err, l2 = np.zeros(n), np.zeros(n)

    def one(s):
        idx = np.nonzero(L.set_of_psf == s)[0]
        want = oracle.psf_planes(L.sets[s], L.defocus_nm[idx] * 1e-9, size=L.size, normalize=True)
        d = got[idx].astype(np.float64) - want
        err[idx] = np.abs(d).max(axis=(1, 2)) / want.max(axis=(1, 2))
        l2[idx] = np.sqrt((d ** 2).sum(axis=(1, 2)) / (want ** 2).sum(axis=(1, 2)))

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, range(len(L.sets))))
    return err, l2


def test_c4_full_problem_frame_subsets(engine):
    """The gradient config at full size (256 frames x 1,000 ROIs): a 16-frame subproblem (frames 0-7 and 248-255)
    against the float64 adjoint -- every ROI's x, y, z, N gradient, the frames' background gradients, the 21 Zernike
    gradients and the NLL -- and the full problem's per-ROI gradients on those frames equal the subproblem's."""
    from insiliscope_b200.nll import NllModel, NllSpec
    from insiliscope_b200.workloads import nll_counts, nll_rois
    from oracle.nll_oracle import NllSpec as OSpec, gradient, tables
    spec = NllSpec()
    model = NllModel(engine, spec)
    P = nll_rois(seed=42, spec=spec)
    assert len(P.bg) == 256 and len(P.frame) == 256_000
    counts = nll_counts(engine, model, P)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    _, _, (gp_all, gb_all, _) = model.evaluate(dev(P.params), dev(P.frame), dev(P.bg), P.zern, counts, grad=True)
    gp_all = gp_all.cpu().numpy()
    gb_all = gb_all.cpu().numpy()
    frames = np.r_[0:8, 248:256]
    sel = np.isin(P.frame, frames)
    remap = np.full(256, -1, np.int32)
    remap[frames] = np.arange(len(frames))
    sp, sf, sb = P.params[sel], remap[P.frame[sel]], P.bg[frames]
    sk = counts[torch.from_numpy(np.nonzero(sel)[0]).cuda()]
    value, _, (gp, gb, gz) = model.evaluate(dev(sp), dev(sf), dev(sb), P.zern, sk, grad=True)
    gp, gb, gz = gp.cpu().numpy().astype(np.float64), gb.cpu().numpy(), gz.cpu().numpy()
    ospec = OSpec()
    want_nll, wp, wb, wz = gradient(ospec, sp.astype(np.float64), sf, sb.astype(np.float64), P.zern,
                                    sk.cpu().numpy().astype(np.float64), tables(ospec))
    errs = [float(np.max(np.abs(gp[:, c] - wp[:, c])) / np.max(np.abs(wp[:, c]))) for c in range(4)]
    eb = float(np.max(np.abs(gb - wb)) / np.max(np.abs(wb)))
    ez = float(np.max(np.abs(gz - wz)) / np.max(np.abs(wz)))
    en = abs(value - want_nll) / abs(want_nll)
    print(f"C4 16 of 256 frames (16,000 ROIs): rel error x/y/z/N {errs}, background {eb:.2e}, Zernike {ez:.2e}, "
          f"NLL {en:.2e}")
    assert max(errs) <= 1e-4 and eb <= 1e-4 and ez <= 1e-4 and en <= 1e-5
    # each ROI's gradient depends only on its ROI: the full problem's equal the subproblem's
    assert np.allclose(gp_all[sel], gp, rtol=1e-6, atol=0)
    assert np.allclose(gb_all[frames], gb, rtol=1e-6, atol=0)
