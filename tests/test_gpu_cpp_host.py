"""The C++ host seam: tests/cpp/gpusim_main.cpp drives iscu_sim::GpuSimulator (include/iscu_gpusim.hpp, the
sim::GpuSimulator API over the C ABI) with the reference's 64-byte records; its frame equals the engine's own
record render bit for bit and passes the reference's GPU self-check bar (SplatGpu.cpp:523-531: >= 90 % of pixels equal
to RenderPhotonImage + ApplyNoiseChain) -- here every pixel within one ADU."""
import os
import subprocess

import numpy as np
import pytest

from insiliscope_b200 import BLINK_EVENT_DTYPE, INTERP_CUBIC, CameraParams, PsfParams, frames_table

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp):
    from insiliscope_b200.build import LIB, build_library
    build_library()
    exe = os.path.join(tmp, "gpusim_main")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp",
           "gpusim_main.cpp"), LIB, "-Wl,-rpath," + os.path.dirname(LIB), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_gpusim_mirror_renders_records(engine, reference, oracle, tmp_path):
    tmp = str(tmp_path)
    rng = np.random.default_rng(2024)
    req = PsfParams(wavelength_nm=670.0, na=1.4, pixel_size_nm=100.0, oversampling=4, kernel_half_width_px=6,
                    nz=5, z_step_nm=100.0, interp=INTERP_CUBIC)
    k = reference.kernel(req=req)
    planes = k.planes()
    W = H = 64
    ev = np.zeros(300, BLINK_EVENT_DTYPE)
    ev["x_um"] = 6.4 * rng.uniform(size=300)
    ev["y_um"] = 6.4 * rng.uniform(size=300)
    ev["z_nm"] = 300 * rng.uniform(size=300) - 150
    ev["t_start"] = 0.3 * rng.uniform(size=300) - 0.1
    ev["t_end"] = ev["t_start"] + 0.5 + rng.uniform(size=300)
    ev["brightness"] = 0.5 + rng.uniform(size=300)
    ev["excite"] = 1.0
    off, gain, rn = oracle.camera_maps(W, H, 9, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    cam = CameraParams(quantum_efficiency=0.9, dark_electrons=0.02, gain=2.2, read_noise_e=1.5)
    rec = k.collect_gpu_emitters(ev, 0, W, H, 100.0, 1500.0, kernel=0)
    planes.astype(np.float32).tofile(os.path.join(tmp, "planes.f32"))
    for name, a in (("offset", off), ("gain", gain), ("readnoise", rn)):
        np.asarray(a, np.float32).tofile(os.path.join(tmp, name + ".f32"))
    rec.tofile(os.path.join(tmp, "records.bin"))
    exe = _build(tmp)
    args = [exe, tmp, str(planes.shape[1]), str(planes.shape[0]), "4", str(INTERP_CUBIC), "100.0", str(W), str(H),
            "20.0", "777", "3", "1.0", "0", "0.9", "0.02", "2.2", "1.5", "1.0", "0.0"]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(os.path.join(tmp, "adu.u16"), np.uint16).reshape(H, W)
    # the engine's own record path, the same bits
    engine.kernel_set_planes(0, planes, 4, 100.0, INTERP_CUBIC)
    engine.set_static(W, H, offset=off, gain=gain, read_noise=rn, flat_bg=20.0)
    want = engine.render_gpu_records(rec, frames_table([len(rec)], frame_ids=[3]), cam, 777)[0]
    assert np.array_equal(got, want)
    # the reference's self-check bar against its CPU renderer
    cpu = k.render_photon_image(ev, 0, W, H, 100.0, 1500.0, 20.0)
    ref = reference.noise_chain(cpu, cam, off.reshape(H, W), gain.reshape(H, W), rn.reshape(H, W), 777, 3)
    diff = np.abs(got.astype(np.int32) - ref.astype(np.int32))
    assert np.mean(diff == 0) >= 0.9 and diff.max() <= 1
