"""PSF planes on the B200 (pupil with float64 phases, chirp-Z as DFT matrix products) against the float64 oracle,
the reference's ComputeZernikePsfPlanes / BuildZernikePsfKernelCache, and the reference's PSF fixture.
Tolerance: max |I - I64| <= 1e-5 x max I64 per plane (the north-star bar for the PSF path)."""
import os

import numpy as np
import pytest

from insiliscope_b200 import CZT_F16X3, CZT_FP32, CZT_TF32X3, INTERP_CUBIC, PsfParams

pytestmark = pytest.mark.gpu
TOL = 1e-5
METHODS = [CZT_FP32]


def _max_rel(got, want):
    return max(np.abs(got[z] - want[z]).max() / want[z].max() for z in range(want.shape[0]))


@pytest.mark.parametrize("method", METHODS)
def test_fixture_planes(engine, golden_dir, method):
    f = np.load(os.path.join(golden_dir, "zernike_ref.npz"))
    for c in range(4):
        req = PsfParams(wavelength_nm=660.0, na=1.4, sample_index=float(f["sample_index"][c]),
                        sample_depth_nm=float(f["sample_depth_nm"][c]), pixel_size_nm=100.0,
                        zernike=list(f["zernike"][c]), double_helix=bool(f["double_helix"][c]), oversampling=4,
                        kernel_half_width_px=8, nz=3, z_step_nm=100.0, pupil_samples=64)
        got = engine.psf_library_dev([req], [0, 0, 0], [-100.0, 0.0, 100.0], normalize=False,
                                     method=method).cpu().numpy()
        want = f["planes"][c].astype(np.float64)
        assert _max_rel(got, want) <= TOL, c
        for z in range(3):
            assert np.argmax(got[z]) == np.argmax(want[z])


@pytest.mark.parametrize("method", [CZT_TF32X3, CZT_F16X3])
def test_split_unnormalized_vs_oracle(engine, oracle, method):
    """Unnormalized planes (|E|^2 itself, no sum-1 division) from the tensor-core forms: the FP16 form's operands and
    accumulators carry exact power-of-two scales that only the normalization would otherwise cancel."""
    req = PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8, nz=3,
                    pupil_samples=128)
    dz = np.array([-600.0, 0.0, 450.0])
    got = engine.psf_library_dev([req], [0, 0, 0], dz, size=64, normalize=False, method=method).cpu().numpy()
    want = oracle.psf_planes(req, dz * 1e-9, size=64, normalize=False)
    assert _max_rel(got, want) <= TOL


@pytest.mark.parametrize("method", [CZT_TF32X3, CZT_F16X3])
def test_split_beyond_staged_items(engine, method):
    """More than 96 PSFs per CTA (the tensor-core kernels stage the first 96 items' sets and defocus factors in shared
    memory and read the rest from global memory), three request sets in random order (a set change at most PSFs),
    against the plain FP32 form."""
    rng = np.random.default_rng(11)
    sets = [PsfParams(wavelength_nm=wl, na=1.4, pixel_size_nm=100.0, oversampling=2, kernel_half_width_px=8, nz=3,
                      pupil_samples=64) for wl in (520.0, 600.0, 700.0)]
    n = 15000
    set_of = rng.integers(0, 3, n).astype(np.uint32)
    dz = rng.uniform(-600.0, 600.0, n)
    a = engine.psf_library_dev(sets, set_of, dz, size=33, method=CZT_FP32).cpu().numpy()
    b = engine.psf_library_dev(sets, set_of, dz, size=33, method=method).cpu().numpy()
    err = np.abs(a - b).max(axis=(1, 2)) / a.max(axis=(1, 2))
    assert err.max() <= 2 * TOL, (int(err.argmax()), float(err.max()))


@pytest.mark.parametrize("method", [CZT_FP32, CZT_TF32X3, CZT_F16X3])
def test_library_vs_oracle(engine, oracle, method):
    """The library config's shape (M = 128 pupil -> 64 x 64 at 4x oversampling) with Noll 4-15 aberrations, four
    wavelengths, defocus across +-800 nm, plus a double-helix and a deep, index-mismatched set."""
    rng = np.random.default_rng(5)
    sets = []
    for wl in (520.0, 580.0, 670.0, 750.0):
        z = np.zeros(28)
        z[3:15] = rng.normal(0.0, 0.05 * 2.0, 12)
        sets.append(PsfParams(wavelength_nm=wl, na=1.45, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8,
                              nz=3, z_step_nm=25.0, pupil_samples=128, zernike=list(z)))
    sets.append(PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8,
                          nz=3, z_step_nm=25.0, pupil_samples=128, double_helix=True))
    sets.append(PsfParams(wavelength_nm=580.0, na=1.45, sample_index=1.33, sample_depth_nm=3000.0,
                          pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8, nz=3, z_step_nm=25.0,
                          pupil_samples=128))
    set_of = np.repeat(np.arange(len(sets)), 3)
    dz = np.tile([-800.0, 0.0, 637.5], len(sets))
    got = engine.psf_library_dev(sets, set_of, dz, size=64, normalize=True, method=method).cpu().numpy()
    for i in range(len(set_of)):
        want = oracle.psf_planes(sets[set_of[i]], [dz[i] * 1e-9], size=64, normalize=True)
        assert _max_rel(got[i:i + 1], want) <= TOL, i


@pytest.mark.parametrize("method", METHODS)
def test_kernel_build_vs_reference(engine, reference, method):
    """iscu_kernel_build (planes, sum-1 normalization, block sums) against BuildZernikePsfKernelCache."""
    req = PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=108.0, oversampling=4, kernel_half_width_px=16,
                    nz=49, z_step_nm=25.0, pupil_samples=64, interp=INTERP_CUBIC)
    k = reference.kernel(req=req)
    engine.kernel_build(3, req, method)
    got = engine.kernel_planes(3)
    want = k.planes().astype(np.float64)
    assert got.shape == want.shape == (49, 129, 129)
    assert _max_rel(got, want) <= TOL
    assert np.allclose(got.sum(axis=(1, 2)), 1.0, atol=1e-5)
    sums = engine.kernel_block_sums(3)
    assert np.abs(sums.sum(axis=(1, 2)) - 16.0).max() < 1e-3
    assert np.abs(sums - k.block_sums()).max() <= TOL * k.block_sums().max()


@pytest.mark.parametrize("method", [CZT_TF32X3, CZT_F16X3])
@pytest.mark.parametrize("M,P,nz", [(96, 48, 5), (128, 64, 40), (64, 33, 3), (112, 64, 300)])
def test_split_shapes_vs_oracle(engine, oracle, M, P, nz, method):
    """The tensor-core paths on padded shapes (2P < 128 rows, 2M < 256 K; M = 112 leaves the FP16 form's last K block
    half empty) and more PSFs than SMs (the persistent loop), against the float64 oracle, plane by plane."""
    rng = np.random.default_rng(M + P)
    z = np.zeros(28)
    z[3:15] = rng.normal(0.0, 0.08, 12)
    req = PsfParams(wavelength_nm=600.0, na=1.4, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8,
                    nz=3, z_step_nm=25.0, pupil_samples=M, zernike=list(z))
    dz = rng.uniform(-700.0, 700.0, nz)
    got = engine.psf_library_dev([req], np.zeros(nz, np.uint32), dz, size=P, normalize=True,
                                 method=method).cpu().numpy()
    idx = list(range(0, nz, max(1, nz // 6)))
    want = oracle.psf_planes(req, dz[idx] * 1e-9, size=P, normalize=True)
    for j, i in enumerate(idx):
        assert np.abs(got[i] - want[j]).max() <= TOL * want[j].max(), i


@pytest.mark.parametrize("method", [CZT_TF32X3, CZT_F16X3])
def test_split_matches_fp32(engine, method):
    """The split forms agree with the plain one (all within 1e-5 of float64) on a library of 4 sets, two of them double
    helix, in random order (a set change at most PSFs: the FP16 form reloads its resident DFT operand there)."""
    rng = np.random.default_rng(77)
    sets = [PsfParams(wavelength_nm=wl, na=1.45, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8, nz=3,
                      pupil_samples=128, double_helix=dh) for wl, dh in ((520.0, False), (580.0, True),
                                                                           (670.0, False), (750.0, True))]
    set_of = rng.integers(0, 4, 512).astype(np.uint32)
    dz = rng.uniform(-800.0, 800.0, 512)
    a = engine.psf_library_dev(sets, set_of, dz, size=64, method=CZT_FP32).cpu().numpy()
    b = engine.psf_library_dev(sets, set_of, dz, size=64, method=method).cpu().numpy()
    assert np.abs(a - b).max() <= 2 * TOL * a.max()


@pytest.mark.parametrize("method", [CZT_FP32, CZT_TF32X3, CZT_F16X3])
def test_plan_matches_library(engine, method):
    """A PSF plan (per-set work once, device-resident runs) gives the one-shot library call's planes, bit for bit."""
    import torch
    from insiliscope_b200 import PsfPlan
    from insiliscope_b200.workloads import psf_library
    L = psf_library(seed=3, n_z=8, n_aberr=3)
    plan = PsfPlan(engine, L.sets, size=L.size, method=method)
    d_set = torch.from_numpy(L.set_of_psf.view(np.int32)).cuda()
    d_dz = torch.from_numpy(L.defocus_nm).cuda()
    out = torch.empty((len(L.set_of_psf), 64, 64), dtype=torch.float32, device="cuda")
    got = plan.run_dev(d_set, d_dz, out).cpu().numpy()
    want = engine.psf_library_dev(L.sets, L.set_of_psf, L.defocus_nm, size=64, method=method).cpu().numpy()
    assert np.array_equal(got, want)
    assert np.array_equal(plan.run(L.set_of_psf, L.defocus_nm), want)
    bad = L.set_of_psf.copy()
    bad[3] = 999
    from insiliscope_b200 import IscuError
    with pytest.raises(IscuError):
        plan.run(bad, L.defocus_nm)
    plan.close()


@pytest.mark.parametrize("method", [CZT_F16X3, CZT_FP32])
def test_plan_run_in_chunks_matches_device_run(engine, method):
    """A library large enough (2,100 PSFs) that the host-buffer run splits it into launches whose planes are copied
    back while the next launch computes (sizes that do not divide evenly): the planes equal the device run's bit for
    bit, and a bad set index in the last chunk is still reported."""
    import torch
    from insiliscope_b200 import IscuError, PsfPlan
    from insiliscope_b200.workloads import psf_library
    L = psf_library(seed=9, n_z=35, n_aberr=15)
    assert len(L.set_of_psf) == 2100
    plan = PsfPlan(engine, L.sets, size=L.size, method=method)
    d_set = torch.from_numpy(L.set_of_psf.view(np.int32)).cuda()
    d_dz = torch.from_numpy(L.defocus_nm).cuda()
    out = torch.empty((len(L.set_of_psf), L.size, L.size), dtype=torch.float32, device="cuda")
    want = plan.run_dev(d_set, d_dz, out).cpu().numpy()
    got = plan.run(L.set_of_psf, L.defocus_nm)
    assert np.array_equal(got, want)
    bad = L.set_of_psf.copy()
    bad[-1] = 10_000
    with pytest.raises(IscuError):
        plan.run(bad, L.defocus_nm)
    plan.close()
