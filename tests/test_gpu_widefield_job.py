"""The focus-job engine (iscu_wf_job_*, the GPU side of a widefield scene's WidefieldAccelerator) against a numpy
model of what WidefieldScene computes on the CPU (ChannelImageStep / ChannelImageFinish, WidefieldRender.cpp:1724-1878):
per channel the sum over its deps of plane spectrum x (w0 K[p0] + w1 K[p1]), the sub-cell ramp (ApplyShiftRamp,
DriftShift.cpp:24-48: Nyquist terms their cosine only), the normalized inverse and the FOV window. numpy's rfft2
layout is RealFft2d's ((ny, nx/2 + 1), ky natural). Grids with odd and even dye-grid sides, transforms whose inputs
fill less than half of them (the half-length first stages) and more, square and oblong transforms; a second job on
the same geometry from resident spectra; a new geometry dropping them. Tolerance 1e-5 of the image maximum."""
import numpy as np
import pytest

from insiliscope_b200 import WidefieldJob

pytestmark = pytest.mark.gpu


def _ramp(NX, NY, fx, fy):
    kx = np.arange(NX // 2 + 1)
    ky = np.arange(NY)
    kys = np.where(ky <= NY // 2, ky, ky - NY)
    ax, ay = 2 * np.pi * kx * fx / NX, 2 * np.pi * kys * fy / NY
    px = np.where(kx == NX // 2, np.cos(ax), np.exp(1j * ax))
    py = np.where(ky == NY // 2, np.cos(ay), np.exp(1j * ay))
    return py[:, None] * px[None, :]


def _model(NX, NY, grid, fov, frac, kernels, planes, channels):
    nx, ny = grid
    x0, y0, cw, ch = fov
    P = {}
    for key, (cells, values) in planes.items():
        img = np.zeros((NY, NX))
        img[cells // nx, cells % nx] = values
        P[key] = np.fft.rfft2(img)
    out = []
    for deps in channels:
        S = np.zeros((NY, NX // 2 + 1), complex)
        for key, p0, p1, w0, w1 in deps:
            k = w0 * kernels[p0].astype(complex) + (w1 * kernels[p1].astype(complex) if p1 is not None else 0)
            S += P[key] * k
        img = np.fft.irfft2(S * _ramp(NX, NY, *frac), s=(NY, NX))
        out.append(img[y0:y0 + ch, x0:x0 + cw])
    return np.array(out)


def _case(rng, NX, NY, nx, ny, n_planes, n_kernels):
    kernels = {}
    for p in range(n_kernels):
        R = 6
        k = np.zeros((NY, NX))
        yy, xx = np.mgrid[-R:R + 1, -R:R + 1]
        k[yy % NY, xx % NX] = np.exp(-(xx ** 2 + yy ** 2) / (2.0 * (1.5 + 0.3 * p) ** 2)) * (1 + 0.1 * p)
        kernels[p] = np.fft.rfft2(k).astype(np.complex64)
    planes = {}
    for q in range(n_planes):
        cells = np.nonzero(rng.random(nx * ny) < 0.05)[0].astype(np.uint32)
        planes[1000 + 7 * q] = (cells, rng.integers(1, 5, len(cells)).astype(np.float32))
    keys = list(planes)
    channels = [[(keys[q], q % n_kernels, (q + 1) % n_kernels if q % 2 else None, 0.7 if q % 2 else 1.0,
                  0.3 if q % 2 else 0.0) for q in range(n_planes)],
                [(keys[q], (q + 2) % n_kernels, None, 1.0, 0.0) for q in range(0, n_planes, 2)]]
    return kernels, planes, channels


@pytest.mark.parametrize("NX,NY,nx,ny,fov,frac", [
    (64, 64, 46, 38, (3, 3, 40, 32), (0.0, 0.0)),          # inputs past half the transform, even sides
    (128, 128, 61, 57, (0, 0, 60, 56), (0.0, 0.0)),        # odd sides within half of it (half-length first stages)
    (128, 128, 65, 57, (8, 8, 48, 40), (0.26, 0.42)),      # x past half, y within it, a sub-cell ramp
    (64, 64, 41, 34, (2, 3, 36, 28), (0.5, 0.1)),          # odd x, Nyquist of the ramp at 0.5
    (256, 128, 200, 57, (10, 4, 180, 50), (0.13, 0.77)),   # oblong
])
def test_job_images_match_numpy_model(engine, NX, NY, nx, ny, fov, frac):
    rng = np.random.default_rng(NX + NY + nx + ny)
    kernels, planes, channels = _case(rng, NX, NY, nx, ny, 6, 4)
    job = WidefieldJob(engine)
    try:
        got = job.images(NX, NY, (nx, ny), fov, frac, 17, kernels, planes, channels)
        want = _model(NX, NY, (nx, ny), fov, frac, kernels, planes, channels)
        assert np.abs(want).max() > 1.0
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= 1e-5, err
        # the same geometry again: the planes are resident, the job names them without their cells
        assert all(job.has_plane(17, k) for k in planes)
        again = job.images(NX, NY, (nx, ny), fov, frac, 17, kernels, {}, channels)
        assert np.array_equal(again, got)
        # a new geometry drops them
        assert not job.has_plane(18, next(iter(planes)))
        other = job.images(NX, NY, (nx, ny), fov, frac, 18, kernels, planes, channels[:1])
        assert np.abs(other[0] - want[0]).max() <= 1e-5 * np.abs(want).max()
    finally:
        job.close()


def test_one_engine_across_transform_sizes(engine):
    """One engine serving scenes of different transform sizes in turn (64, 128, 256 x 128, 64): each job's images
    equal the model's -- the resident spectra's slots are remade for each size."""
    job = WidefieldJob(engine)
    try:
        for g, (NX, NY, nx, ny) in enumerate([(64, 64, 46, 38), (128, 128, 61, 57), (256, 128, 200, 57),
                                              (64, 64, 41, 34)]):
            rng = np.random.default_rng(g)
            kernels, planes, channels = _case(rng, NX, NY, nx, ny, 6, 4)
            fov, frac = (1, 2, nx - 3, ny - 4), (0.3, 0.6)
            got = job.images(NX, NY, (nx, ny), fov, frac, 100 + g, kernels, planes, channels)
            want = _model(NX, NY, (nx, ny), fov, frac, kernels, planes, channels)
            assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max(), (NX, NY)
    finally:
        job.close()
