"""The C ABI without a GPU: libiscu.so builds for sm_100a, loads, exports every function include/iscu.h declares, and
its host-side functions (camera maps, PSF geometry, argument checks) agree with the oracle."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "iscu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(iscu_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from insiliscope_b200.build import build_library
    from insiliscope_b200 import _abi
    build_library()
    return _abi.load()


def test_exports_every_declared_symbol(lib):
    from insiliscope_b200 import _abi
    names = declared_functions()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (iscu_\w+)", out))
    for n in names:
        assert n in exported, n
        assert n in _abi.SIGNATURES, n
        getattr(lib, n)


def test_camera_maps_match_oracle(lib, oracle):
    from insiliscope_b200 import generate_camera_maps
    for y0, rows in ((0, 0), (4, 9)):
        a = generate_camera_maps(40, 30, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2, y0, rows)
        b = oracle.camera_maps(40, 30, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2, y0, rows)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_camera_maps_match_reference(lib, reference):
    """The maps equal the reference's PixelOffsetMap / PixelGainMap / PixelReadNoiseMap (SMLMNoise.cpp:89-140,
    compiled from its sources) bit for bit: whole sensors, row windows (first rows, middle, last rows, past the end),
    the gain floor reached (a large spread) and the read-noise clamp at 0."""
    from insiliscope_b200 import generate_camera_maps
    cases = [(128, 128, 42, 0, 0, 0.1 / 2.2, 0.2), (256, 256, 42, 0, 0, 0.1 / 2.2, 0.2), (37, 23, 7, 0, 5, 0.3, 0.4),
             (37, 23, 7, 9, 6, 0.3, 0.4), (37, 23, 7, 20, 10, 0.3, 0.4), (64, 16, 3, 2, 1, 1.5, 1.5),
             (1, 1, 5, 0, 0, 0.1, 0.1)]
    for w, h, seed, y0, rows, gfrac, rfrac in cases:
        a = generate_camera_maps(w, h, seed, 100.0, 2.0, 2.2, gfrac, 1.5, rfrac, y0, rows)
        b = reference.camera_maps(w, h, seed, 100.0, 2.0, 2.2, gfrac, 1.5, rfrac, y0, rows)
        for x, y in zip(a, b):
            assert x.shape == y.shape and np.array_equal(x, y), (w, h, seed, y0, rows)
    g = generate_camera_maps(64, 16, 3, 100.0, 2.0, 2.2, 1.5, 1.5, 1.5)
    assert (g[1] == np.float32(0.04 * 2.2)).any() and (g[2] == 0).any()   # the floor and the clamp were exercised


def test_psf_geometry_matches_oracle(lib, oracle):
    from insiliscope_b200 import PsfParams
    for half, os_, nz, m, wl in ((16, 4, 49, 64, 670.0), (8, 4, 64, 128, 520.0), (70, 4, 71, 0, 660.0),
                                 (6, 4, 5, 0, 670.0), (256, 1, 65, 0, 520.0)):
        r = PsfParams(wavelength_nm=wl, na=1.45, pixel_size_nm=108.0, oversampling=os_, kernel_half_width_px=half,
                      nz=nz, pupil_samples=m)
        assert r.geometry() == oracle.psf_geometry(r)


def test_errors_without_device(lib):
    from insiliscope_b200 import _abi
    h = C.c_void_p()
    rc = lib.iscu_create(0, C.byref(h))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        assert rc == _abi.ISCU_OK
        lib.iscu_destroy(h)
    else:
        assert rc == _abi.ISCU_ERR_NODEV and b"device" in lib.iscu_last_error()
    assert lib.iscu_create(0, None) == _abi.ISCU_ERR_ARG
    bad = _abi.PsfRequest()
    assert lib.iscu_psf_geometry(C.byref(bad), None, None, None) == _abi.ISCU_ERR_ARG
    assert b"must be > 0" in lib.iscu_last_error()
    assert lib.iscu_abi_version() == 1


def test_backend_argument_checks_without_device(lib):
    """The named-kernel backend's calls refuse null contexts and buffers before touching a device."""
    from insiliscope_b200 import _abi
    h = C.c_void_p()
    assert lib.iscu_buffer_create(None, 16, None, C.byref(h)) == _abi.ISCU_ERR_ARG
    assert lib.iscu_buffer_bytes(None) == 0
    assert lib.iscu_buffer_write(None, 0, None, 0) == _abi.ISCU_ERR_ARG
    assert lib.iscu_buffer_read(None, 0, None) == _abi.ISCU_ERR_ARG
    assert lib.iscu_buffer_read_low16(None, 0, None) == _abi.ISCU_ERR_ARG
    assert lib.iscu_buffer_copy(None, None, 0) == _abi.ISCU_ERR_ARG
    assert lib.iscu_dispatch(None, b"wf_clear", None, 0, None, 0, 1, 1, 1) == _abi.ISCU_ERR_ARG
    lib.iscu_buffer_destroy(None)


def test_widefield_pipeline_argument_checks_without_device(lib):
    """The pipelined focus-series calls refuse a null plan, null buffers and slots out of range before any device
    work."""
    from insiliscope_b200 import _abi
    assert lib.iscu_wf_render_async(None, 0, None, 0.0, None, 0, 0, None, None) == _abi.ISCU_ERR_ARG
    assert lib.iscu_wf_render_wait(None, 0) == _abi.ISCU_ERR_ARG
    assert b"null" in lib.iscu_last_error()
