"""libiscu behind the render engine's own C++ seams (include/iscu_sim_seams.hpp), driven by the reference's code
compiled from its sources (oracle/_ref/seams_check, built with the reference harness):

- ComputePsfKernelCache on the B200 (iscu_sim::ComputePsfKernelCacheGpu): the cache the reference's consumers read --
  geometry fields equal, planes within 1e-5 of each plane's maximum, RenderPhotonImage's frames with it within 1e-5 of
  the frame maximum -- for the dSTORM, double-helix and astigmatic kernels;
- a WidefieldAccelerator on the B200 (iscu_sim::WidefieldAcceleratorCuda) installed in the reference's WidefieldScene:
  every focus of a FocusSeries within 1e-5 of the frame maximum of the CPU scene's, with a margin, a sub-cell FOV
  offset, 2 cells per pixel, dye planes beyond the kernel stack and blended planes, and again from resident spectra."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK = os.path.join(ROOT, "oracle", "_ref", "seams_check")


def test_engine_seams_on_the_b200(engine):
    assert os.path.exists(CHECK), "oracle/_ref/seams_check is built with the reference harness (oracle/Makefile)"
    r = subprocess.run([CHECK], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    lines = dict(l.split(" ", 1) for l in r.stdout.splitlines() if " " in l)
    names = ["psfcache_dstorm", "psfcache_double_helix", "psfcache_astigmatic", "accel_aligned",
             "accel_subcell_upscale2", "accel_clamped_planes", "accel_blended_planes"]
    for name in names:
        assert lines.get(name, "").startswith("ok"), (name, lines.get(name))
    for name in names[3:]:
        assert "accelerated=1" in lines[name], lines[name]
    assert r.returncode == 0


MOVIE = os.path.join(ROOT, "oracle", "_ref", "movie_check")


def test_movie_engine_with_the_splat_host_installed(engine):
    """The reference's whole movie engine (RenderScopeMovie, compiled from its sources) with libiscu installed as its
    blink splat + noise host (SetDefaultBlinkSplatGpu over the CUDA named-kernel backend): the host passes the
    reference's own self-check, every frame is drawn by it, and the frames equal the CPU movie's on >= 99 % of the
    pixels (the engine's float32 contract for its GPU host), with and without the halo cut."""
    assert os.path.exists(MOVIE), "oracle/_ref/movie_check is built with the reference harness (oracle/Makefile)"
    r = subprocess.run([MOVIE], capture_output=True, text=True, timeout=900)
    print(r.stdout, r.stderr)
    lines = dict(l.split(" ", 1) for l in r.stdout.splitlines() if " " in l)
    for name in ("movie_install", "movie_dstorm", "movie_dstorm_halo"):
        assert lines.get(name, "").startswith("ok"), (name, lines.get(name))
    assert r.returncode == 0
