"""The named-kernel backend (sim::GpuBackend on CUDA): the reference's own GPU hosts run unmodified over it and pass
their self-checks and a movie comparison against the reference's CPU frames (oracle/_ref/gpubackend_check, built
from the reference's sources with the checks); the FFT, Hermitian split and narrowed read-back against numpy; the
dispatch's argument checks."""
import os
import re
import subprocess

import numpy as np
import pytest

from insiliscope_b200 import IscuError
from insiliscope_b200.backend import GpuBackend

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK = os.path.join(ROOT, "oracle", "_ref", "gpubackend_check")


@pytest.fixture(scope="module")
def backend(engine):
    be = GpuBackend(engine)
    yield be
    be.close()


def test_reference_hosts_over_the_backend():
    """SplatGpuHost and WidefieldGpuHost (the reference's code) on our kernels: their self-checks pass, and the splat
    host's frames match the reference's CPU frames (RenderPhotonImage + ApplyNoiseChain) on >= 99 % of the pixels."""
    assert os.path.exists(CHECK), "oracle/_ref/gpubackend_check is built with the reference harness (oracle/Makefile)"
    r = subprocess.run([CHECK], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    lines = dict(l.split(" ", 1) for l in r.stdout.splitlines() if " " in l)
    for name in ("backend", "splat_selfcheck", "splat_movie_scmos", "splat_movie_emccd", "splat_movie_scmos_halo",
                 "splat_movie_emccd_halo", "widefield_selfcheck"):
        assert lines.get(name, "").startswith("ok"), (name, lines.get(name))
    assert r.returncode == 0
    for name in ("splat_movie_scmos", "splat_movie_scmos_halo", "splat_movie_emccd", "splat_movie_emccd_halo"):
        m = re.search(r"equal=([0-9.]+) rel_diff=([0-9.e+-]+) emitters=\d+ kept=([0-9.]+)", lines[name])
        assert float(m.group(1)) >= 0.99 and float(m.group(2)) <= 1e-3, (name, lines[name])
        assert (float(m.group(3)) < 1.0) == name.endswith("_halo"), (name, lines[name])   # the cut is exercised


@pytest.mark.parametrize("logn", [1, 3, 7, 10, 11])
def test_fft_rows_and_columns(backend, logn):
    """wf_fft over the rows then the columns of two planes (the hosts' Fft2) equals numpy's 2-D FFT, forward and
    inverse (no scaling), to float32 accuracy."""
    n = 1 << logn
    NX, NY = n, max(2, n // 2)
    rng = np.random.default_rng(logn)
    grid = (rng.standard_normal((2, NY, NX)) + 1j * rng.standard_normal((2, NY, NX))).astype(np.complex64)
    tw = np.zeros(NX + NY, np.float32)
    for off, m in ((0, NX), (NX // 2, NY)):
        k = np.arange(m // 2)
        tw[2 * (off + k)] = np.cos(-2 * np.pi * k / m)
        tw[2 * (off + k) + 1] = np.sin(-2 * np.pi * k / m)
    PS = NX * NY
    for inverse in (0, 1):
        data = backend.make(grid.nbytes, grid.view(np.float32))
        twb = backend.make(tw.nbytes, tw)
        backend.dispatch("wf_fft", [NX, logn, 1, NX, PS, inverse, 0, 0], [data, twb], NY, 1, 2)
        backend.dispatch("wf_fft", [NY, int(np.log2(NY)), NX, 1, PS, inverse, NX // 2, 0], [data, twb], NX, 1, 2)
        got = backend.read_back(data, grid.nbytes, np.float32).view(np.complex64).reshape(grid.shape)
        want = np.fft.fft2(grid.astype(np.complex128)) if not inverse else \
            np.fft.ifft2(grid.astype(np.complex128)) * (NX * NY)
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 2e-6 * max(1, logn), (inverse, err)
        data.close()
        twb.close()


def test_split_packs_half_spectra(backend):
    """wf_split: Z = F(a + i b) of a pair of real planes -> the half spectra of a and b, scaled, as float16 pairs
    (round to nearest even, as numpy converts)."""
    NX, NY = 64, 32
    W = NX // 2 + 1
    SS, PS = W * NY, NX * NY
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal((2, NY, NX))
    Z = np.fft.fft2(a + 1j * b).astype(np.complex64)
    data = backend.make(Z.nbytes, Z.view(np.float32))
    sa, sb = np.float32(1 / 40.0), np.float32(1 / 25.0)
    slots = np.array([1, 3, sa.view(np.uint32), sb.view(np.uint32)], np.uint32)
    sl = backend.make(slots.nbytes, slots)
    spec = backend.make(4 * SS * 4)
    backend.dispatch("wf_split", [NX, NY, W, SS, PS, 1, 0, 0], [data, sl, spec], (W + 15) // 16, (NY + 15) // 16, 1)
    got = backend.read_back(spec, 4 * SS * 4).reshape(4, SS)
    Zc = Z.astype(np.complex64)
    ky, kx = np.meshgrid(np.arange(NY), np.arange(W), indexing="ij")
    zk = Zc[ky, kx]
    zm = np.conj(Zc[(NY - ky) % NY, (NX - kx) % NX])
    A = (np.float32(0.5) * (zk + zm)).astype(np.complex64)
    D = (np.float32(0.5) * (zk - zm)).astype(np.complex64)
    wantA = np.stack([A.real * sa, A.imag * sa], -1).astype(np.float32).astype(np.float16).view(np.uint32)
    wantB = np.stack([D.imag * sb, -D.real * sb], -1).astype(np.float32).astype(np.float16).view(np.uint32)
    assert np.array_equal(got[1], wantA.reshape(-1)) and np.array_equal(got[3], wantB.reshape(-1))
    assert not got[0].any() and not got[2].any()   # other slots untouched


def test_read_low16_and_copy(backend):
    words = np.arange(70000, dtype=np.uint32) * np.uint32(2654435761)
    src = backend.make(words.nbytes, words)
    dst = backend.make(words.nbytes)
    backend.copy(dst, src, words.nbytes)
    backend.write(dst, 8, np.array([7, 9], np.uint32))
    words[2:4] = [7, 9]
    assert np.array_equal(backend.read_back_low16(dst, len(words)), (words & 0xFFFF).astype(np.uint16))
    assert np.array_equal(backend.read_back(dst, words.nbytes), words)


def test_dispatch_argument_checks(backend):
    d = backend.make(64)
    for args in (("no_such_kernel", [0], [d]), ("wf_clear", [1, 256], [d, d]),
                 ("wf_fft", [12, 3, 1, 12, 12, 0, 0], [d, d]), ("wf_fft", [4096, 12, 1, 1, 1, 0, 0], [d, d]),
                 ("wf_scatter", [1, 0, 4, 16, 256], [d, d])):
        with pytest.raises(IscuError):
            backend.dispatch(*args, 1, 1, 1)
    with pytest.raises(IscuError):
        backend.dispatch("wf_clear", [1, 256], [d], 1, 70000, 1)
    backend.dispatch("wf_clear", [16, 256], [d], 0, 1, 1)   # an empty dispatch
