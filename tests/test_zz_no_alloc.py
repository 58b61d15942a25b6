"""The allocation-free PSF library entry point (iscu_psf_library_noalloc_dev), for callers that cannot allocate GPU
memory -- a host whose device memory is owned by another framework's allocator or a fixed shared budget, or a loop
that cannot take a cudaFree's device-wide synchronization. Its temporaries sit in the library's static device array
instead of per-call cudaMalloc buffers; its planes must equal the allocating entry point's (iscu_psf_library_dev),
within the PSF tests' tolerance, on two calls in a row (the second reusing the array the first left behind).

Kept in the file pytest collects last, so a run that stops at the first failure has run every other test first."""
import numpy as np
import pytest

from insiliscope_b200 import CZT_FP32, IscuError, PsfParams
from insiliscope_b200 import _abi

pytestmark = pytest.mark.gpu
TOL = 1e-5   # max |difference| per plane relative to the plane maximum, as tests/test_gpu_psf.py


def _sets(rng, wavelengths):
    out = []
    for wl in wavelengths:
        z = np.zeros(28)
        z[3:15] = rng.normal(0.0, 0.1, 12)
        out.append(PsfParams(wavelength_nm=wl, na=1.45, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8,
                             nz=3, z_step_nm=25.0, pupil_samples=128, zernike=list(z)))
    return out


def _max_rel(a, b):
    return max(float(np.abs(a[i] - b[i]).max() / np.abs(b[i]).max()) for i in range(len(b)))


def test_noalloc_matches_allocating_entry_twice(engine):
    import torch
    rng = np.random.default_rng(2024)
    calls = [
        (_sets(rng, (520.0, 670.0, 750.0)), 48),
        (_sets(rng, (580.0, 670.0)) + [PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=100.0, oversampling=4,
                                                 kernel_half_width_px=8, nz=3, z_step_nm=25.0, pupil_samples=128,
                                                 double_helix=True)], 70),
    ]
    for sets, n in calls:
        set_of = rng.integers(0, len(sets), n).astype(np.uint32)
        dz = rng.uniform(-800.0, 800.0, n)
        want = engine.psf_library_dev(sets, set_of, dz, size=64, normalize=True, method=CZT_FP32)
        out = torch.full((n, 64, 64), float("nan"), dtype=torch.float32, device="cuda")
        got = engine.psf_library_noalloc_dev(sets, set_of, dz, out, size=64, normalize=True)
        torch.cuda.synchronize()
        g, w = got.cpu().numpy(), want.cpu().numpy()
        assert np.isfinite(g).all()
        assert _max_rel(g, w) <= TOL


def test_noalloc_rejects_sizes_beyond_its_array(engine):
    import torch
    sets = _sets(np.random.default_rng(1), (600.0,))
    out = torch.empty((1, 64, 64), dtype=torch.float32, device="cuda")
    too_many = [sets[0]] * 5
    with pytest.raises(IscuError) as e:
        engine.psf_library_noalloc_dev(too_many, [0], [0.0], out, size=64)
    assert e.value.code == _abi.ISCU_ERR_LIMIT
    big = PsfParams(wavelength_nm=600.0, na=1.45, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=8,
                    nz=3, pupil_samples=256)
    with pytest.raises(IscuError) as e:
        engine.psf_library_noalloc_dev([big], [0], [0.0], out, size=64)
    assert e.value.code == _abi.ISCU_ERR_LIMIT and "pupil samples" in str(e.value)


def test_noalloc_checks_its_output_and_shared_memory(engine):
    """An output too small, of the wrong type or on the host is refused before the call; a pupil and plane whose
    chirp-Z does not fit one CTA's shared memory (M = 128, P = 100) is refused with ISCU_ERR_LIMIT before any copy
    or launch; the largest plane that fits at M = 128 beside the kernel's static shared memory (P = 98) equals the
    allocating entry point."""
    import torch
    rng = np.random.default_rng(5)
    sets = _sets(rng, (600.0,))
    for bad in (torch.empty((1, 63, 64), dtype=torch.float32, device="cuda"),
                torch.empty((1, 64, 64), dtype=torch.float64, device="cuda"),
                torch.empty((1, 64, 64), dtype=torch.float32)):
        with pytest.raises(ValueError):
            engine.psf_library_noalloc_dev(sets, [0], [0.0], bad, size=64)
    out = torch.empty((2, 100, 100), dtype=torch.float32, device="cuda")
    with pytest.raises(IscuError) as e:
        engine.psf_library_noalloc_dev(sets, [0, 0], [0.0, 100.0], out, size=100)
    assert e.value.code == _abi.ISCU_ERR_LIMIT and "shared memory" in str(e.value)
    dz = rng.uniform(-500.0, 500.0, 3)
    want = engine.psf_library_dev(sets, [0, 0, 0], dz, size=98, normalize=True, method=CZT_FP32)
    out = torch.full((3, 98, 98), float("nan"), dtype=torch.float32, device="cuda")
    got = engine.psf_library_noalloc_dev(sets, [0, 0, 0], dz, out, size=98, normalize=True)
    torch.cuda.synchronize()
    g, w = got.cpu().numpy(), want.cpu().numpy()
    assert np.isfinite(g).all() and _max_rel(g, w) <= TOL
