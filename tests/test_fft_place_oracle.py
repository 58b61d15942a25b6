"""The splat's Fft placement: the float64 restatement (oracle.fft_place_f64: FftShiftKernelTile's zero-padded row and
column shifts, then BuildBlockSums) pinned on the reference's own PlanSplat with PsfInterpMode::Fft, compiled into
oracle/_ref -- the same tap origins and the same shifted block sums, on the SMLM kernel geometry (129 x 129 samples,
oversampling 4). CPU only; the device form is in tests/test_gpu_fft_place.py."""
import numpy as np

from insiliscope_b200 import PsfParams
from oracle.oracle import fft_place_f64


def place_request(nz=9):
    return PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=108.0, oversampling=4, kernel_half_width_px=16,
                     nz=nz, z_step_nm=100.0, pupil_samples=64)


def place_positions(seed, n, nz):
    """Positions over a frame (sub-cell offsets of every kind, the half-way ties included) and planes."""
    rng = np.random.default_rng(seed)
    xy = rng.uniform(-2.0, 130.0, (n, 2))
    xy[:4] = [[10.0, 20.0], [10.125, 20.375], [10.5, 20.5], [10.625, 19.875]]   # shifts 0 and +-1/2 exactly
    return xy, rng.integers(0, nz, n)


def test_restatement_equals_reference(oracle, reference):
    k = reference.kernel(req=place_request())
    planes = k.planes()
    size, nz, os_, bw = k.info()
    xy, z = place_positions(1, 60, nz)
    for (x, y), p in zip(xy, z):
        want, st = k.plan_splat_fft(x, y, int(p))
        tile, st2 = fft_place_f64(planes, os_, x, y, int(p))
        assert st == st2
        got = oracle.block_sums(tile[None], os_)[0]
        assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
