"""The oracle pinned before it is trusted: against the reference's golden vectors (spec/golden rng/stream lines), its
PSF fixture (tests/psf/zernike_ref.bin), the committed outputs of the reference's own functions, and -- where the
reference harness is built -- the reference's functions themselves on fresh seeded inputs. CPU only."""
import json
import os

import numpy as np
import pytest

from insiliscope_b200.engine import BLINK_EVENT_DTYPE, EMITTER_DTYPE, INTERP_CUBIC, INTERP_LINEAR, INTERP_NEAREST, \
    CameraParams, PsfParams


def test_pcg4d_golden(oracle, golden_dir):
    g = json.load(open(os.path.join(golden_dir, "pcg4d_golden.json")))
    assert len(g["rng"]) == 8 and len(g["stream"]) == 2
    for r in g["rng"]:
        a, b, c, d = r["in_u32"]
        assert list(oracle.pcg4d(a, b, c, d)) == r["words"]
        cx = np.int32(np.uint32(b)).item()
        cy = np.int32(np.uint32(c)).item()
        assert repr(oracle.hash_unit(a, cx, cy, d)) == repr(float(r["unit"])) or \
            oracle.hash_unit(a, cx, cy, d) == float(r["unit"])
    for s in g["stream"]:
        seed, cx, cy, base = s["in_u32"]
        got = oracle.hash_stream(seed, np.int32(np.uint32(cx)).item(), np.int32(np.uint32(cy)).item(), base,
                                 len(s["values"]))
        assert np.array_equal(got, np.array([float(v) for v in s["values"]]))


def test_counter_stream_layout(oracle):
    # Four uniforms per hash, consumed a, b, c, d; the counter is the hash's fourth input (SMLMCounterRng.h:75-88).
    u = oracle.counter_uniforms(42, 7, 1000, 3, 9)
    for p in range(3):
        for j in range(9):
            w = oracle.pcg4d(42, 7, 1000 + p, j // 4)[j % 4]
            assert u[p, j] == ((int(w) >> 9) + 0.5) * 2.0 ** -23


def test_zernike_fixture(oracle, golden_dir):
    """The float64 DFT restatement against webSMLM's planes (the fixture the reference matches at rel L2 0)."""
    f = np.load(os.path.join(golden_dir, "zernike_ref.npz"))
    for c in range(4):
        req = PsfParams(wavelength_nm=660.0, na=1.4, immersion_index=1.518, sample_index=float(f["sample_index"][c]),
                        working_distance_um=150.0, sample_depth_nm=float(f["sample_depth_nm"][c]),
                        pixel_size_nm=100.0, zernike=list(f["zernike"][c]), double_helix=bool(f["double_helix"][c]),
                        oversampling=4, kernel_half_width_px=8, nz=3, z_step_nm=100.0, pupil_samples=64)
        got = oracle.psf_planes(req, oracle.stack_defocus_m(req))
        want = f["planes"][c].astype(np.float64)
        for z in range(3):
            rel = np.linalg.norm(got[z] - want[z]) / np.linalg.norm(want[z])
            assert rel < 1e-6, (c, z, rel)
            assert np.argmax(got[z]) == np.argmax(want[z])


def test_ref_outputs_golden(oracle, golden_dir):
    """Absolute noise-chain ADU, camera maps, block sums and a rendered frame: the committed reference outputs."""
    g = np.load(os.path.join(golden_dir, "ref_outputs.npz"))
    W, H = int(g["W"]), int(g["H"])
    off, gain, rn = oracle.camera_maps(W, H, int(g["map_seed"]), 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    assert np.array_equal(off, g["offset"]) and np.array_equal(gain, g["gain"]) and np.array_equal(rn, g["read_noise"])
    sc = CameraParams(quantum_efficiency=0.9, dark_electrons=0.05, gain=2.2, read_noise_e=1.5)
    em = CameraParams(quantum_efficiency=0.9, dark_electrons=0.05, gain=0.05, read_noise_e=40.0, emccd=True,
                      em_gain=300.0, cic_electrons=0.002, bit_depth=16)
    a = oracle.noise_chain(g["photons"], sc, off.reshape(H, W), gain.reshape(H, W), rn.reshape(H, W), 1234, 7)
    assert np.array_equal(a, g["adu_scmos"])
    b = oracle.noise_chain(g["photons"], em, off.reshape(H, W), None, rn.reshape(H, W), 99, 3, pixel_base=480)
    assert np.array_equal(b, g["adu_emccd"])
    sums = oracle.block_sums(g["planes"], 4)
    assert np.array_equal(sums, g["sums"])
    size = g["planes"].shape[1]
    ems = oracle.collect_frame_emitters(g["events"], 1, 108.0, 1500.0, g["planes"].shape[0], 50.0, drift_x=0.3,
                                        drift_y=-0.2, global_z_um=0.02)
    img = oracle.render_frame(sums, 4, size, INTERP_CUBIC, ems, W, H, 20.0)
    assert np.array_equal(img, g["frame1"])


def _small_kernel(reference, interp=INTERP_CUBIC, half=5, nz=7, zernike3=0.1, pupil=64):
    req = PsfParams(wavelength_nm=600.0, na=1.4, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=half,
                    nz=nz, z_step_nm=80.0, pupil_samples=pupil, interp=interp)
    req.zernike[3] = zernike3
    return req, reference.kernel(req=req)


def _events(rng, n, W, H, px_nm=100.0):
    ev = np.zeros(n, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(-0.5, W * px_nm / 1000 + 0.5, n)
    ev["y_um"] = rng.uniform(-0.5, H * px_nm / 1000 + 0.5, n)
    ev["z_nm"] = rng.uniform(-300, 300, n)
    ev["t_start"] = rng.uniform(-0.5, 2.5, n)
    ev["t_end"] = ev["t_start"] + rng.uniform(0.1, 2.0, n)
    ev["brightness"] = rng.uniform(0.2, 2.0, n)
    ev["excite"] = np.where(rng.uniform(size=n) < 0.3, rng.uniform(0.5, 1.0, n), 1.0)
    return ev


@pytest.mark.parametrize("interp", [INTERP_NEAREST, INTERP_LINEAR, INTERP_CUBIC])
def test_render_vs_reference(oracle, reference, interp):
    """Emitter collection, block sums and the splat equal the reference's bit for bit, edges and halo cut included."""
    rng = np.random.default_rng(interp + 11)
    req, k = _small_kernel(reference, interp)
    planes = k.planes()
    sums = oracle.block_sums(planes, 4)
    assert np.array_equal(sums, k.block_sums())
    W, H = 37, 29
    ev = _events(rng, 80, W, H)
    size, nz = planes.shape[1], planes.shape[0]
    for frame in (0, 1, 2):
        want = k.render_photon_image(ev, frame, W, H, 100.0, 1800.0, 15.0, drift_x=-0.4, drift_y=0.7, global_z=-0.03,
                                     min_photons=300.0)
        ems = oracle.collect_frame_emitters(ev, frame, 100.0, 1800.0, nz, 80.0, drift_x=-0.4, drift_y=0.7,
                                            global_z_um=-0.03, min_photons=300.0)
        got = oracle.render_frame(sums, 4, size, interp, ems, W, H, 15.0)
        assert np.array_equal(got, want), frame
    kh = k.halo(1e-3)
    lo, hi, _ = kh.spans()
    want = kh.render_photon_image(ev, 1, W, H, 100.0, 1800.0, 15.0)
    ems = oracle.collect_frame_emitters(ev, 1, 100.0, 1800.0, nz, 80.0)
    got = oracle.render_frame(sums, 4, size, interp, ems, W, H, 15.0, span_lo=lo, span_hi=hi)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("emccd", [False, True])
def test_noise_vs_reference(oracle, reference, emccd):
    rng = np.random.default_rng(3 + emccd)
    W, H = 64, 48
    photons = rng.gamma(1.5, 40.0, size=(H, W)).astype(np.float32)
    photons[::7, ::5] *= 30.0
    # a window: rows [3, 3 + H) of a sensor H + 7 rows tall
    off, gain, rn = reference.camera_maps(W, H + 7, 17, 100.0, 2.0, 2.2, 0.05, 1.5, 0.2, keep_y0=3, keep_rows=H)
    cam = CameraParams(quantum_efficiency=0.85, dark_electrons=0.1, gain=2.2, read_noise_e=1.5, emccd=emccd,
                       em_gain=150.0, bit_depth=14)
    maps = [a.reshape(H, W) for a in (off, gain, rn)]
    want = reference.noise_chain(photons, cam, *maps, 555, 9, pixel_base=3 * W)
    got = oracle.noise_chain(photons, cam, *maps, 555, 9, pixel_base=3 * W)
    assert np.array_equal(got, want)
    assert np.array_equal(reference.noise_chain(photons, cam, None, None, None, 1, 2),
                          oracle.noise_chain(photons, cam, None, None, None, 1, 2))


def test_camera_maps_window_vs_reference(oracle, reference):
    for (y0, rows) in ((0, 0), (5, 7), (20, 100)):
        a = reference.camera_maps(31, 23, 99, 100.0, 2.0, 0.25, 0.3, 1.2, 0.9, y0, rows)
        b = oracle.camera_maps(31, 23, 99, 100.0, 2.0, 0.25, 0.3, 1.2, 0.9, y0, rows)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("dh,depth,ns", [(False, 0.0, 1.518), (True, 0.0, 1.518), (False, 400.0, 1.33)])
def test_psf_vs_reference(oracle, reference, dh, depth, ns):
    """The float64 DFT restatement against ComputeZernikePsfPlanes (Bluestein, float64) on fresh requests."""
    req = PsfParams(wavelength_nm=580.0, na=1.45, sample_index=ns, sample_depth_nm=depth, pixel_size_nm=108.0,
                    oversampling=3, kernel_half_width_px=5, nz=5, z_step_nm=120.0, pupil_samples=96, double_helix=dh)
    req.zernike[3], req.zernike[7], req.zernike[12] = 0.08, -0.05, 0.03
    want = reference.zernike_planes(req).astype(np.float64)
    got = oracle.psf_planes(req, oracle.stack_defocus_m(req))
    for z in range(want.shape[0]):
        assert np.abs(got[z] - want[z]).max() <= 1e-6 * want[z].max(), z


def test_nll_oracle_adjoint_matches_central_differences():
    """The float64 gradient oracle's adjoint against float64 central differences (h = 1e-4 max(1, |theta|))."""
    from oracle.nll_oracle import NllSpec, gradient, nll, tables
    spec = NllSpec(roi=10, os=2, pupil=20)
    rng = np.random.default_rng(5)
    n, F = 4, 2
    t = tables(spec)
    pt = np.column_stack([rng.uniform(4, 6, n), rng.uniform(4, 6, n), rng.uniform(-400, 400, n),
                          rng.uniform(800, 3000, n)])
    frame = rng.integers(0, F, n)
    bg = rng.uniform(5, 15, F)
    zern = rng.normal(0, 0.03, len(spec.noll))
    from oracle.nll_oracle import expected
    counts = rng.poisson(expected(spec, pt, frame, bg, zern, t))
    p = pt + np.column_stack([rng.normal(0, .3, n), rng.normal(0, .3, n), rng.normal(0, 40, n), rng.normal(0, 80, n)])
    b, z = bg * 1.1, zern + 0.01
    _, g, gb, gz = gradient(spec, p, frame, b, z, counts, t)

    def fd(f, x, i):
        h = 1e-4 * max(1.0, abs(x.flat[i]))
        xp, xm = x.copy(), x.copy()
        xp.flat[i] += h
        xm.flat[i] -= h
        return (f(xp) - f(xm)) / (2 * h)

    for i in range(p.size):
        d = fd(lambda P: nll(spec, P, frame, b, z, counts, t), p, i)
        assert abs(d - g.flat[i]) <= 1e-4 * max(abs(d), 1e-2), i
    for i in range(F):
        d = fd(lambda B: nll(spec, p, frame, B, z, counts, t), b, i)
        assert abs(d - gb[i]) <= 1e-4 * max(abs(d), 1e-2)
    for j in range(len(z)):
        d = fd(lambda Z: nll(spec, p, frame, b, Z, counts, t), z, j)
        assert abs(d - gz[j]) <= 1e-4 * max(abs(d), 1.0), j
