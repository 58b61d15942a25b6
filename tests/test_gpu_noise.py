"""Counter RNG and camera noise chain on the B200 against the reference's golden vectors and the oracle: integer
(pcg4d words, uniforms, ADU) bit for bit."""
import json
import os

import numpy as np
import pytest

from insiliscope_b200 import CameraParams

pytestmark = pytest.mark.gpu


def test_pcg4d_golden(engine, golden_dir):
    import torch
    g = json.load(open(os.path.join(golden_dir, "pcg4d_golden.json")))
    words = np.array([r["in_u32"] for r in g["rng"]], dtype=np.uint32)
    t = torch.from_numpy(words.view(np.int32)).cuda()
    out = engine.pcg4d(t).cpu().numpy().view(np.uint32)
    assert out.tolist() == [r["words"] for r in g["rng"]]


def test_pcg4d_random_vs_oracle(engine, oracle):
    import torch
    rng = np.random.default_rng(1)
    words = rng.integers(0, 2**32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    out = engine.pcg4d(torch.from_numpy(words.view(np.int32)).cuda()).cpu().numpy().view(np.uint32)
    for i in range(0, 4096, 37):
        assert np.array_equal(out[i], oracle.pcg4d(*[int(x) for x in words[i]]))


def test_counter_uniforms(engine, oracle):
    got = engine.counter_uniforms(0x9E3779B9 ^ 42, 123, 5000, 257, 11).cpu().numpy()
    want = oracle.counter_uniforms(0x9E3779B9 ^ 42, 123, 5000, 257, 11)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("emccd", [False, True])
def test_noise_chain_bit_exact(engine, oracle, emccd):
    """ADU frames equal the CPU chain's for every pixel: photons spanning both Poisson branches (mean 60 boundary),
    zero, negative, and the saturation clamp; per-pixel maps; a window's pixel base."""
    import torch
    rng = np.random.default_rng(10 + emccd)
    W, H, n = 96, 80, 6
    photons = rng.gamma(1.2, 45.0, size=(n, H, W)).astype(np.float32)
    photons[:, ::9, ::4] *= 40.0
    photons[0, 0, :6] = [0.0, -5.0, 59.999, 60.0, 60.001, 1e6]
    off, gain, rn = oracle.camera_maps(W, H, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    if emccd:
        cam = CameraParams(quantum_efficiency=0.9, dark_electrons=0.02, gain=0.05, read_noise_e=30.0, emccd=True,
                           em_gain=300.0, cic_electrons=0.002, bit_depth=16)
        gain = None
    else:
        cam = CameraParams(quantum_efficiency=1.0, dark_electrons=0.0, gain=2.2, read_noise_e=1.5)
    engine.set_static(W, H, pixel_base=7 * W, offset=off, gain=gain, read_noise=rn, flat_bg=0.0)
    frames = [0, 1, 2, 199, 4096, 2**31 + 5]
    got = engine.noise_frames_dev(torch.from_numpy(photons).cuda(), frames, cam, 42 ^ 0x9E3779B9).cpu().numpy()
    mism = 0
    for k in range(n):
        want = oracle.noise_chain(photons[k], cam, off.reshape(H, W), None if gain is None else gain.reshape(H, W),
                                  rn.reshape(H, W), 42 ^ 0x9E3779B9, frames[k], pixel_base=7 * W)
        mism += int((got[k] != want).sum())
    assert mism == 0
