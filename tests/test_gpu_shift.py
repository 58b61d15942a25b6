"""Frames of a drifting widefield sample on the B200 (iscu_wf_shifted_frames_dev) against the float64 restatement and
the reference's own RenderShiftedImages (oracle/_ref): several frames per call, each with its own channel coefficients
(one or two foci, bleach) and its own drift, on grids whose transforms take one, two and three register groups;
within 2e-5 of the frame maximum (the reference's float transforms round differently), added onto the caller's
frames."""
import numpy as np
import pytest

from insiliscope_b200 import WidefieldShift
from oracle.oracle import shifted_frame_f64
from test_shift_oracle import coefs, shift_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny,window,up", [(64, 32, (4, 2, 48, 24), 2), (256, 128, (16, 8, 192, 96), 3),
                                             (4096, 64, (100, 4, 3000, 48), 2)])
def test_device_frames(engine, reference, nx, ny, window, up):
    import torch
    sp0, sp1 = shift_case(nx + ny, nx, ny), shift_case(nx + ny + 1, nx, ny)
    spectra = np.concatenate([sp0, sp1])
    rng = np.random.default_rng(nx)
    frames = [((0.0, 0.0), (0.0, 0.0), [1.0, 0.0], 0.0, False),
              ((0.3, -0.2), (1.7, -0.45), [0.6, 0.25], 0.0, False),
              ((0.1, 0.4), (-2.25, 3.5), [0.8, 0.1], 0.35, True),
              ((0.0, 0.0), tuple(rng.uniform(-4, 4, 2)), [0.5, 0.5], 0.7, True)]
    n_ch = spectra.shape[0]
    coef = np.zeros((len(frames), n_ch), np.float32)
    shift = np.zeros((len(frames), 2), np.float64)
    for f, (frac, drift, a, w, two) in enumerate(frames):
        c = coefs(a, w, two)
        coef[f, :len(c)] = c
        shift[f] = (frac[0] - drift[0], frac[1] - drift[1])
    camH, camW = window[3] // up, window[2] // up
    base = rng.random((len(frames), camH, camW)).astype(np.float32)
    cam = torch.from_numpy(base.copy()).cuda()
    s = WidefieldShift(engine, nx, ny)
    s.frames_dev(torch.from_numpy(spectra).cuda(), torch.from_numpy(coef).cuda(), torch.from_numpy(shift).cuda(),
                 window, up, cam)
    got = cam.cpu().numpy() - base
    for f, (frac, drift, a, w, two) in enumerate(frames):
        want = reference.shifted_images(nx, ny, sp0, a, frac, drift, window, up, spec1=sp1 if two else None, w=w)
        assert np.abs(got[f] - want).max() <= 2e-5 * np.abs(want).max(), f
        ora = shifted_frame_f64(spectra, coef[f], shift[f], nx, ny, window, up)
        assert np.abs(got[f] - ora).max() <= 2e-5 * np.abs(ora).max(), f
    s.close()
