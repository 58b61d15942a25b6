"""Generates the committed golden fixtures under tests/golden/ from the reference tree (run where it exists).

  pcg4d_golden.json   the reference's own golden vectors for the counter RNG: the `rng` (pcg4d words + HashUnit) and
                      `stream` (HashStream) lines of spec/golden/ref.txt, with their inputs from spec/golden/cases.txt
                      (tolerance 0, tests/parity/golden.mjs:55). Inputs wrap to uint32 as parity_main.cpp's ToU32 does.
  zernike_ref.npz     the reference's PSF fixture tests/psf/zernike_ref.bin (webSMLM's planes: 4 cases x 3 planes x
                      65^2 float32, header "ZPSF" + 4 int32, cli/zernike_psf_check.cpp:236-252) and its cases
                      (:256-266) and request (:203-221).
  ref_outputs.npz     outputs of the reference's own functions built here (oracle/_ref/libiscref.so) on small seeded
                      inputs: camera maps, noise chain (sCMOS and EMCCD), a kernel stack, its block sums and rendered
                      frames -- the absolute ADU values no committed reference golden pins (glibc version recorded).

Usage: ISC_REFERENCE_TREE=<reference tree> python tests/golden/make_golden.py   (after `make -C oracle ref`)
"""
from __future__ import annotations

import json
import os
import platform
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("ISC_REFERENCE_TREE", "")
sys.path.insert(0, ROOT)


def u32(v: int) -> int:
    return v & 0xFFFFFFFF


def make_pcg4d():
    cases = [l.split() for l in open(os.path.join(REF, "spec/golden/cases.txt")) if l.startswith(("rng", "stream"))]
    refs = [l.split() for l in open(os.path.join(REF, "spec/golden/ref.txt")) if l.startswith(("rng", "stream"))]
    assert len(cases) == len(refs)
    rng, stream = [], []
    for c, r in zip(cases, refs):
        if c[0] == "rng":
            seed, cx, cy, k = (int(x) for x in c[1:5])
            rng.append({"in": [seed, cx, cy, k], "in_u32": [u32(seed), u32(cx), u32(cy), u32(k)],
                        "words": [int(x) for x in r[5:9]], "unit": r[9]})
        else:
            seed, cx, cy, base, count = (int(x) for x in c[1:6])
            vals = r[5:]
            assert len(vals) == count
            stream.append({"in": [seed, cx, cy, base], "in_u32": [u32(seed), u32(cx), u32(cy), u32(base)],
                           "values": vals})
    out = {"source": "spec/golden/cases.txt + spec/golden/ref.txt (rng and stream lines)", "rng": rng,
           "stream": stream}
    with open(os.path.join(HERE, "pcg4d_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


def make_zernike():
    b = open(os.path.join(REF, "tests/psf/zernike_ref.bin"), "rb").read()
    assert b[:4] == b"ZPSF"
    cases, nx, ny, nz = struct.unpack("<4i", b[4:20])
    planes = np.frombuffer(b[20:], dtype="<f4").reshape(cases, nz, ny, nx).copy()
    # cli/zernike_psf_check.cpp:256-266: (name, sample index, depth nm, {OSA index: waves}, double helix).
    case_ns = np.array([1.518, 1.518, 1.518, 1.33])
    case_depth = np.array([0.0, 0.0, 0.0, 500.0])
    zern = np.zeros((4, 28))
    zern[0, 5] = 0.15
    zern[1, 5], zern[1, 13], zern[1, 25] = 1.8, 0.8, 0.3
    case_dh = np.array([0, 0, 1, 0], np.int32)
    np.savez_compressed(os.path.join(HERE, "zernike_ref.npz"), planes=planes, sample_index=case_ns,
                        sample_depth_nm=case_depth, zernike=zern, double_helix=case_dh,
                        names=np.array(["AstigmatismModerate", "ExtendedRangeStrong", "DoubleHelix",
                                        "ns 1.33, 500 nm deep"]))


def make_ref_outputs():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    from oracle.oracle import Reference
    from insiliscope_b200.engine import BLINK_EVENT_DTYPE, CameraParams, PsfParams, INTERP_CUBIC
    ref = Reference()
    ref.set_threads(1)
    W, H = 48, 40
    off, gain, rn = ref.camera_maps(W, H, 4242, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    rng = np.random.default_rng(7)
    photons = rng.gamma(2.0, 30.0, size=(H, W)).astype(np.float32)
    photons[0, :8] = [0.0, 1e-3, 59.9, 60.0, 60.5, 500.0, 4000.0, -3.0]
    sc = CameraParams(quantum_efficiency=0.9, dark_electrons=0.05, gain=2.2, read_noise_e=1.5)
    em = CameraParams(quantum_efficiency=0.9, dark_electrons=0.05, gain=0.05, read_noise_e=40.0, emccd=True,
                      em_gain=300.0, cic_electrons=0.002, bit_depth=16)
    adu_scmos = ref.noise_chain(photons, sc, off.reshape(H, W), gain.reshape(H, W), rn.reshape(H, W), 1234, 7)
    adu_emccd = ref.noise_chain(photons, em, off.reshape(H, W), None, rn.reshape(H, W), 99, 3, pixel_base=480)
    req = PsfParams(wavelength_nm=670.0, na=1.45, pixel_size_nm=108.0, oversampling=4, kernel_half_width_px=6,
                    nz=9, z_step_nm=50.0, pupil_samples=64, interp=INTERP_CUBIC)
    req.zernike[3] = 0.12
    k = ref.kernel(req=req)
    planes = k.planes()
    sums = k.block_sums()
    ev = np.zeros(60, BLINK_EVENT_DTYPE)
    ev["x_um"] = rng.uniform(-0.3, W * 0.108 + 0.3, 60)
    ev["y_um"] = rng.uniform(-0.3, H * 0.108 + 0.3, 60)
    ev["z_nm"] = rng.uniform(-250, 250, 60)
    ev["t_start"] = rng.uniform(-0.2, 1.5, 60)
    ev["t_end"] = ev["t_start"] + rng.uniform(0.2, 1.5, 60)
    ev["brightness"] = rng.uniform(0.5, 1.5, 60)
    ev["excite"] = 1.0
    frame1 = k.render_photon_image(ev, 1, W, H, 108.0, 1500.0, 20.0, drift_x=0.3, drift_y=-0.2, global_z=0.02)
    glibc = " ".join(platform.libc_ver())
    np.savez_compressed(os.path.join(HERE, "ref_outputs.npz"), W=W, H=H, map_seed=4242, offset=off, gain=gain,
                        read_noise=rn, photons=photons, adu_scmos=adu_scmos, adu_emccd=adu_emccd, planes=planes,
                        sums=sums, events=ev, frame1=frame1, glibc=glibc)


if __name__ == "__main__":
    if not os.path.isdir(REF):
        sys.exit("set ISC_REFERENCE_TREE to the reference's source tree")
    make_pcg4d()
    make_zernike()
    make_ref_outputs()
    print("golden fixtures written to", HERE)
