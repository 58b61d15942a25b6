"""The splat's Fft placement on the B200 (iscu_fft_place_dev: the shift as a float64 convolution, no transform)
against the reference's own PlanSplat with PsfInterpMode::Fft (its FFT route, oracle/_ref) and the float64
restatement: the same tap origins, the shifted block sums within 1e-6 of their maximum; emitters PlanSplat refuses
marked and left blank."""
import numpy as np
import pytest

from insiliscope_b200 import EMITTER_DTYPE
from oracle.oracle import fft_place_f64
from test_fft_place_oracle import place_positions, place_request

pytestmark = pytest.mark.gpu


def test_device_equals_reference(engine, reference, oracle):
    import torch
    k = reference.kernel(req=place_request())
    planes = k.planes()
    size, nz, os_, bw = k.info()
    engine.kernel_set_planes(2, planes, os_, 100.0)
    xy, z = place_positions(2, 300, nz)
    em = np.zeros(len(z) + 2, EMITTER_DTYPE)
    em["x_px"][:len(z)], em["y_px"][:len(z)], em["plane"][:len(z)] = xy[:, 0], xy[:, 1], z
    em["photons"] = 1000.0
    em[-2]["photons"] = 0.0                     # refused: no photons
    em[-1]["plane"] = nz                        # refused: beyond the stack
    sums, origins = engine.fft_place_dev(2, torch.from_numpy(em.view(np.uint8)).cuda())
    sums, origins = sums.cpu().numpy(), origins.cpu().numpy()
    for i, ((x, y), p) in enumerate(zip(xy, z)):
        want, st = k.plan_splat_fft(x, y, int(p))
        assert tuple(origins[i]) == st
        assert np.abs(sums[i] - want).max() <= 1e-6 * np.abs(want).max(), i
        if i < 40:
            tile, _ = fft_place_f64(planes, os_, x, y, int(p))
            ora = oracle.block_sums(tile[None], os_)[0]
            assert np.abs(sums[i] - ora).max() <= 1e-6 * np.abs(ora).max()
    for i in (-2, -1):
        assert origins[i][0] == np.iinfo(np.int32).min and not sums[i].any()
