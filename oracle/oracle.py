"""TEST INFRASTRUCTURE -- the oracle's Python face. Used only by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, as the checker; the product never imports it.

Two checkers over the same C ABI types (include/iscu.h):
  Oracle     liboracle.so: the CPU restatement of the reference's algorithms (iscoracle.cpp), always available.
  Reference  _ref/libiscref.so: the reference's own hot-path sources compiled here (Makefile), when built.
Plus the float64 FFT convolution that checks the widefield path (numpy).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libiscref.so")
vp = C.c_void_p


def reference_tree(tree: str | None = None) -> str | None:
    """The reference's source tree: the argument, else $ISC_REFERENCE_TREE; None when neither names a directory."""
    tree = tree or os.environ.get("ISC_REFERENCE_TREE")
    return tree if tree and os.path.isdir(tree) else None


def build(reference: bool = True, tree: str | None = None) -> None:
    """Builds liboracle.so, and _ref/libiscref.so when the reference tree is known (argument or $ISC_REFERENCE_TREE)
    and present; without it an already built _ref/ is kept as it is."""
    src = reference_tree(tree) if reference else None
    targets = ["oracle"] + (["ref", f"REF={src}"] if src else [])
    subprocess.run(["make", "-s", "-C", HERE, "-j8", *targets], check=True)


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def _struct_ptr(s):
    return C.byref(s) if s is not None else None


class Oracle:
    """The CPU restatement (liboracle.so)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build(reference=False)
        L = C.CDLL(ORACLE_SO)
        u32, i32, f64, i64 = C.c_uint32, C.c_int32, C.c_double, C.c_int64
        L.or_pcg4d.argtypes = [u32, u32, u32, u32, vp]
        L.or_hash_unit.argtypes = [u32, i32, i32, u32]
        L.or_hash_unit.restype = f64
        L.or_hash_stream.argtypes = [u32, i32, i32, u32, u32, vp]
        L.or_counter_uniforms.argtypes = [u32, u32, u32, u32, u32, vp]
        L.or_camera_maps.argtypes = [u32, u32, C.c_uint64, f64, f64, f64, f64, f64, f64, u32, u32, vp, vp, vp]
        L.or_noise_chain.argtypes = [vp, u32, u32, vp, vp, vp, vp, u32, u32, u32, vp]
        L.or_psf_geometry.argtypes = [vp, vp, vp, vp]
        L.or_psf_planes.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, vp]
        L.or_block_sums.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp]
        L.or_render_frame.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, u32, u32, u32,
                                      f64, vp, vp, f64, vp]
        L.or_collect_frame_emitters.argtypes = [vp, u32, i64, f64, f64, f64, f64, f64, C.c_int, f64, C.c_int, f64,
                                                vp]
        L.or_collect_frame_emitters.restype = u32
        self.L = L

    def pcg4d(self, a, b, c, d):
        out = np.zeros(4, np.uint32)
        self.L.or_pcg4d(a, b, c, d, _p(out))
        return out

    def hash_unit(self, seed, cx, cy, k):
        return self.L.or_hash_unit(seed, cx, cy, k)

    def hash_stream(self, seed, cx, cy, base, n):
        out = np.zeros(n, np.float64)
        self.L.or_hash_stream(seed, cx, cy, base, n, _p(out))
        return out

    def counter_uniforms(self, seed, frame, pixel0, npix, per):
        out = np.zeros((npix, per), np.float64)
        self.L.or_counter_uniforms(seed, frame, pixel0, npix, per, _p(out))
        return out

    def camera_maps(self, w, h, seed, off_mean, off_std, gain, gain_frac, rn, rn_frac, keep_y0=0, keep_rows=0):
        rows = min(keep_rows, max(0, h - keep_y0)) if keep_rows else h
        o, g, r = (np.zeros(w * rows, np.float32) for _ in range(3))
        self.L.or_camera_maps(w, h, seed, off_mean, off_std, gain, gain_frac, rn, rn_frac, keep_y0, keep_rows, _p(o),
                              _p(g), _p(r))
        return o, g, r

    def noise_chain(self, photons, camera, offset, gain, read_noise, seed, frame, pixel_base=0):
        photons = np.ascontiguousarray(photons, np.float32)
        h, w = photons.shape
        out = np.zeros((h, w), np.uint16)
        cam = camera.c()
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        o, g, r = f(offset), f(gain), f(read_noise)
        self.L.or_noise_chain(_p(photons), w, h, C.byref(cam), _p(o), _p(g), _p(r), seed, frame, pixel_base, _p(out))
        return out

    def psf_geometry(self, req):
        r = req.c()
        s, nz, m = C.c_int(), C.c_int(), C.c_int()
        self.L.or_psf_geometry(C.byref(r), C.byref(s), C.byref(nz), C.byref(m))
        return s.value, nz.value, m.value

    def psf_planes(self, req, defocus_m, size=0, normalize=False):
        r = req.c()
        P = size if size > 0 else self.psf_geometry(req)[0]
        dz = np.ascontiguousarray(defocus_m, np.float64)
        out = np.zeros((len(dz), P, P), np.float64)
        self.L.or_psf_planes(C.byref(r), size, _p(dz), len(dz), int(normalize), _p(out))
        return out

    def stack_defocus_m(self, req):
        """The reference's plane defocus: zStep * 1e-9 * (z - (nz-1)/2)."""
        _, nz, _ = self.psf_geometry(req)
        return np.array([req.z_step_nm * 1e-9 * (z - (nz - 1) / 2.0) for z in range(nz)])

    def block_sums(self, planes, os_):
        planes = np.ascontiguousarray(planes, np.float32)
        nz, n, _ = planes.shape
        bw = n + os_ - 1
        out = np.zeros((nz, bw, bw), np.float32)
        self.L.or_block_sums(_p(planes), n, os_, nz, _p(out))
        return out

    def render_frame(self, sums, os_, size, interp, emitters, w, h, flat_bg, bg_map=None, illum=None, bg_scale=1.0,
                     span_lo=None, span_hi=None):
        sums = np.ascontiguousarray(sums, np.float32)
        nz, bw, _ = sums.shape
        emitters = np.ascontiguousarray(emitters)
        out = np.zeros((h, w), np.float32)
        f = lambda a, t: None if a is None else np.ascontiguousarray(a, t)
        self.L.or_render_frame(_p(sums), nz, bw, os_, size, interp, _p(f(span_lo, np.int16)), _p(f(span_hi, np.int16)),
                               _p(emitters), len(emitters), w, h, flat_bg, _p(f(bg_map, np.float32)),
                               _p(f(illum, np.float32)), bg_scale, _p(out))
        return out

    def collect_frame_emitters(self, events, frame, pixel_nm, per_blink, nz, z_step_nm, drift_x=0.0, drift_y=0.0,
                               global_z_um=0.0, slot=0, min_photons=0.0):
        from insiliscope_b200.engine import EMITTER_DTYPE
        events = np.ascontiguousarray(events)
        out = np.zeros(len(events), EMITTER_DTYPE)
        n = self.L.or_collect_frame_emitters(_p(events), len(events), frame, pixel_nm, per_blink, drift_x, drift_y,
                                             global_z_um, nz, z_step_nm, slot, min_photons, _p(out))
        return out[:n].copy()


class Reference:
    """The reference's own functions, compiled from its sources (oracle/Makefile -> _ref/libiscref.so)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise RuntimeError("the reference harness is not built (oracle/_ref/libiscref.so)")
        L = C.CDLL(REF_SO)
        u32, i32, f64, i64 = C.c_uint32, C.c_int32, C.c_double, C.c_int64
        L.ref_last_error.restype = C.c_char_p
        L.ref_set_threads.argtypes = [C.c_uint]
        L.ref_threads.restype = C.c_uint
        L.ref_pcg4d.argtypes = [u32, u32, u32, u32, vp]
        L.ref_hash_unit.argtypes = [u32, i32, i32, u32]
        L.ref_hash_unit.restype = f64
        L.ref_hash_stream.argtypes = [u32, i32, i32, u32, u32, vp]
        L.ref_counter_uniforms.argtypes = [u32, u32, u32, u32, u32, vp]
        L.ref_counter_poisson.argtypes = [u32, u32, u32, f64]
        L.ref_counter_poisson.restype = f64
        L.ref_counter_gamma.argtypes = [u32, u32, u32, f64]
        L.ref_counter_gamma.restype = f64
        L.ref_camera_maps.argtypes = [u32, u32, C.c_uint64, f64, f64, f64, f64, f64, f64, u32, u32, vp, vp, vp]
        L.ref_noise_chain.argtypes = [vp, u32, u32, vp, vp, vp, vp, u32, u32, u32, C.c_int, vp]
        L.ref_psf_geometry.argtypes = [vp, vp]
        L.ref_dye_blinks.argtypes = [C.c_int, vp, vp, vp, C.c_int, u32, i32, i32, f64, f64, vp, C.c_int]
        L.ref_dye_blinks.restype = C.c_int
        L.ref_dye_blinks_batch.argtypes = [C.c_int, vp, vp, vp, C.c_int, vp, u32, f64, f64, vp]
        L.ref_dye_blinks_batch.restype = f64
        L.ref_dye_h1.argtypes = [u32, i32, i32, C.c_int]
        L.ref_dye_h1.restype = u32
        L.ref_zernike_planes.argtypes = [vp, vp]
        L.ref_kernel_build.argtypes = [vp]
        L.ref_kernel_build.restype = vp
        L.ref_kernel_from_planes.argtypes = [vp, C.c_int, C.c_int, C.c_int, f64, C.c_int]
        L.ref_kernel_from_planes.restype = vp
        L.ref_kernel_halo.argtypes = [vp, f64]
        L.ref_kernel_halo.restype = vp
        L.ref_kernel_free.argtypes = [vp]
        L.ref_kernel_info.argtypes = [vp, vp, vp, vp, vp]
        L.ref_kernel_planes.argtypes = [vp, vp]
        L.ref_kernel_block_sums.argtypes = [vp, vp]
        L.ref_kernel_spans.argtypes = [vp, vp, vp, vp]
        L.ref_nearest_z.argtypes = [vp, f64]
        L.ref_render_photon_image.argtypes = [vp, vp, u32, i64, u32, u32, f64, f64, f64, f64, f64, f64, vp, vp, f64,
                                              f64, C.c_int, C.c_int, vp]
        L.ref_collect_gpu_emitters.argtypes = [vp, vp, u32, i64, u32, u32, f64, f64, f64, f64, f64, C.c_int, f64, vp,
                                               u32]
        L.ref_collect_gpu_emitters.restype = u32
        L.ref_render_movie.argtypes = [vp, vp, u32, u32, u32, u32, u32, f64, f64, f64, vp, vp, vp, vp, u32, vp, vp]
        L.ref_render_movie.restype = f64
        L.ref_render_movie_groups.argtypes = [vp, C.c_int, vp, u32, u32, u32, u32, u32, f64, f64, f64, vp, vp, vp, vp,
                                              u32, vp, vp]
        L.ref_render_movie_groups.restype = f64
        L.ref_drift_trajectory.argtypes = [C.c_long, C.c_long, f64, vp, C.c_int, vp]
        L.ref_illumination_field.argtypes = [C.c_uint, C.c_uint, C.c_int, f64, vp, vp]
        L.ref_illumination_field.restype = C.c_size_t
        L.ref_background_fade_scale.argtypes = [f64, f64]
        L.ref_background_fade_scale.restype = f64
        L.ref_binned_render.argtypes = [vp, f64, C.c_uint, C.c_uint, C.c_int, vp, vp, u32, vp, vp, vp]
        L.ref_binned_render.restype = f64
        u64 = C.c_uint64
        L.ref_tiff_open.argtypes = [C.c_char_p, u64, C.c_int]
        L.ref_tiff_open.restype = vp
        L.ref_tiff_bytes.argtypes = [u64, u64, u64, u64, u64]
        L.ref_tiff_bytes.restype = u64
        L.ref_tiff_page_u16.argtypes = [vp, vp, C.c_size_t, u32, u32, C.c_char_p]
        L.ref_tiff_page_f32.argtypes = [vp, vp, C.c_size_t, u32, u32, C.c_char_p]
        L.ref_tiff_page_rows.argtypes = [vp, vp, u32, u32, u32, C.c_char_p]
        L.ref_tiff_rows.argtypes = [vp, u64, u32, u32, vp]
        L.ref_tiff_big.argtypes = [vp]
        L.ref_tiff_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.ref_tiff_close.argtypes = [vp]
        L.ref_csv_numbers.argtypes = [vp, u32, C.c_char_p, vp, vp]
        L.ref_shifted_images.argtypes = [C.c_uint, C.c_uint, vp, vp, C.c_int, f64, vp, f64, f64, f64, f64, C.c_uint,
                                         C.c_uint, C.c_uint, C.c_uint, C.c_uint, vp]
        L.ref_plan_splat_fft.argtypes = [vp, f64, f64, C.c_int, vp, vp]
        L.ref_wf_grid.argtypes = [C.c_int, f64, C.c_uint, C.c_uint, f64, f64, f64, f64, vp]
        L.ref_wf_scene_create.argtypes = [vp, C.c_int, f64, f64, C.c_uint, C.c_uint, f64, f64, f64, f64, C.c_long,
                                          C.c_uint, vp, f64, C.c_int, vp]
        L.ref_wf_scene_create.restype = vp
        L.ref_wf_scene_series.argtypes = [vp, vp, C.c_uint, vp]
        L.ref_wf_scene_series.restype = f64
        L.ref_wf_scene_destroy.argtypes = [vp]
        L.ref_plan_splat_fft.restype = C.c_int
        L.ref_plan_splat_fft_batch.argtypes = [vp, vp, vp, u32]
        L.ref_plan_splat_fft_batch.restype = f64
        L.ref_csv_table.argtypes = [vp, u32, u32, vp, vp, C.c_size_t]
        L.ref_csv_table.restype = C.c_size_t
        self.L = L

    def set_threads(self, n):
        self.L.ref_set_threads(n)

    def threads(self):
        return self.L.ref_threads()

    def pcg4d(self, a, b, c, d):
        out = np.zeros(4, np.uint32)
        self.L.ref_pcg4d(a, b, c, d, _p(out))
        return out

    def hash_unit(self, seed, cx, cy, k):
        return self.L.ref_hash_unit(seed, cx, cy, k)

    def hash_stream(self, seed, cx, cy, base, n):
        out = np.zeros(n, np.float64)
        self.L.ref_hash_stream(seed, cx, cy, base, n, _p(out))
        return out

    def counter_uniforms(self, seed, frame, pixel0, npix, per):
        out = np.zeros((npix, per), np.float64)
        self.L.ref_counter_uniforms(seed, frame, pixel0, npix, per, _p(out))
        return out

    def camera_maps(self, w, h, seed, off_mean, off_std, gain, gain_frac, rn, rn_frac, keep_y0=0, keep_rows=0):
        rows = min(keep_rows, max(0, h - keep_y0)) if keep_rows else h
        o, g, r = (np.zeros(w * rows, np.float32) for _ in range(3))
        self.L.ref_camera_maps(w, h, seed, off_mean, off_std, gain, gain_frac, rn, rn_frac, keep_y0, keep_rows, _p(o),
                               _p(g), _p(r))
        return o, g, r

    def noise_chain(self, photons, camera, offset, gain, read_noise, seed, frame, pixel_base=0, parallel=False):
        photons = np.ascontiguousarray(photons, np.float32)
        h, w = photons.shape
        out = np.zeros((h, w), np.uint16)
        cam = camera.c()
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        o, g, r = f(offset), f(gain), f(read_noise)
        self.L.ref_noise_chain(_p(photons), w, h, C.byref(cam), _p(o), _p(g), _p(r), seed, frame, pixel_base,
                               int(parallel), _p(out))
        return out

    def zernike_planes(self, req):
        r = req.c()
        size, nz, _ = _geometry(req)
        out = np.zeros((nz, size, size), np.float32)
        if self.L.ref_zernike_planes(C.byref(r), _p(out)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out

    def render_movie_groups(self, kernels, events, frame0, n_frames, w, h, pixel_nm, per_blink, bg, camera, offset,
                            gain, read_noise, seed, want_photons=False, want_adu=True):
        """The reference's multi-colour frame loop: dye group g = the events whose slot is g, splatted with kernels[g]
        onto the frame in group order (the later groups accumulating), then the noise chain; frames in parallel on
        its pool. Returns (seconds, photons, adu)."""
        events = np.ascontiguousarray(events)
        ph = np.zeros((n_frames, h, w), np.float32) if want_photons else None
        adu = np.zeros((n_frames, h, w), np.uint16) if want_adu else None
        cam = camera.c()
        hs = (C.c_void_p * len(kernels))(*[k.h for k in kernels])
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        t = self.L.ref_render_movie_groups(hs, len(kernels), _p(events), len(events), frame0, n_frames, w, h, pixel_nm,
                                           per_blink, bg, C.byref(cam), _p(f(offset)), _p(f(gain)),
                                           _p(f(read_noise)), seed, _p(ph), _p(adu))
        return t, ph, adu

    def drift_trajectory(self, seed, frames, frame_sec, s):
        """sim::DriftTrajectory; s: an insiliscope_b200 DriftSettings. (frames, 3) nm."""
        p = np.array([s.xy_nm_per_sqrt_sec, s.z_nm_per_sqrt_sec, s.xy_speed_nm_per_sec, s.z_speed_nm_per_sec,
                      s.xy_angle_deg, s.angle_wander_deg, s.z_angle_wander_deg, s.speed_wander_pct,
                      s.wander_time_sec], np.float64)
        out = np.zeros((frames, 3), np.float64)
        self.L.ref_drift_trajectory(seed, frames, frame_sec, _p(p), s.z_direction, _p(out))
        return out

    def illumination_field(self, w, h, profile, fwhm_pct):
        out = np.zeros((h, w), np.float32)
        mf = C.c_double(1.0)
        n = self.L.ref_illumination_field(w, h, profile, fwhm_pct, _p(out), C.byref(mf))
        return (out if n else None), mf.value

    def background_fade_scale(self, t, decay):
        return self.L.ref_background_fade_scale(t, decay)

    def kernel(self, req=None, planes=None, os_=4, z_step_nm=25.0, interp=2):
        return RefKernel(self, req, planes, os_, z_step_nm, interp)

    def dye_blinks(self, mode, kin, h1, k, n, t0, t1, history=None):
        """One dye's blinks overlapping [t0, t1) from the world core's own schedules: (m, 3) float64 rows of
        (tOn, tOff, brightness)."""
        kin = np.ascontiguousarray(kin, np.float64)
        st = hk = None
        n_seg = 0
        if history is not None:
            st = np.ascontiguousarray(history[0], np.float64)
            hk = np.ascontiguousarray(history[1], np.float64).reshape(-1, 6)
            n_seg = len(st)
        cap = 64
        while True:
            out = np.zeros((cap, 3), np.float64)
            m = self.L.ref_dye_blinks(int(mode), _p(kin), _p(st), _p(hk), n_seg, int(h1) & 0xFFFFFFFF, int(k),
                                      int(n), float(t0), float(t1), _p(out), cap)
            if m <= cap:
                return out[:m]
            cap = m

    def dye_blinks_batch(self, mode, kin, dyes, t0, t1, history=None):
        """The core's schedules over a DYE_DTYPE array on the reference's thread pool: (per-dye row counts, seconds)."""
        kin = np.ascontiguousarray(kin, np.float64)
        st = hk = None
        n_seg = 0
        if history is not None:
            st = np.ascontiguousarray(history[0], np.float64)
            hk = np.ascontiguousarray(history[1], np.float64).reshape(-1, 6)
            n_seg = len(st)
        dyes = np.ascontiguousarray(dyes)
        counts = np.zeros(len(dyes), np.uint32)
        sec = self.L.ref_dye_blinks_batch(int(mode), _p(kin), _p(st), _p(hk), n_seg, _p(dyes), len(dyes), float(t0),
                                          float(t1), _p(counts))
        return counts, sec

    def csv_numbers(self, values, fmt):
        """sim::AppendCsvNumber of each value (CsvNumber.cpp): a list of str."""
        v = np.ascontiguousarray(values, np.float64)
        fields = np.zeros((len(v), 48), np.uint8)
        lens = np.zeros(len(v), np.uint8)
        self.L.ref_csv_numbers(_p(v), len(v), fmt.encode(), _p(fields), _p(lens))
        return [bytes(fields[i, :lens[i]]).decode() for i in range(len(v))]

    def csv_table(self, columns, fmts):
        """A numeric table (columns: (n_cols, n_rows) float64) as GroundTruth's Rows formats it, on the reference's
        thread pool: (the text as bytes, wall seconds)."""
        import time
        cols = np.ascontiguousarray(columns, np.float64)
        n_cols, n_rows = cols.shape
        f = (C.c_char_p * n_cols)(*[x.encode() for x in fmts])
        t0 = time.perf_counter()
        need = self.L.ref_csv_table(_p(cols), n_rows, n_cols, f, None, 0)
        out = np.zeros(max(1, need), np.uint8)
        t1 = time.perf_counter()
        self.L.ref_csv_table(_p(cols), n_rows, n_cols, f, _p(out), need)
        sec = time.perf_counter() - t1
        return bytes(out[:need]), sec

    def shifted_images(self, nx, ny, spec0, a, frac, drift, window, up, spec1=None, w=0.0, cam=None):
        """RenderShiftedImages of channels' spectra (complex64 (n_ch, ny, nx/2 + 1): persistent, then bleach) at one
        or two foci: the camera frame (ch/up, cw/up) float32 (+= onto cam when given)."""
        x0, y0, cw, ch = window
        s0 = np.ascontiguousarray(spec0, np.complex64)
        s1 = None if spec1 is None else np.ascontiguousarray(spec1, np.complex64)
        av = np.ascontiguousarray(a, np.float64)
        out = np.zeros((ch // up, cw // up), np.float32) if cam is None else np.array(cam, np.float32, copy=True)
        self.L.ref_shifted_images(nx, ny, _p(s0), _p(s1), s0.shape[0], w, _p(av), frac[0], frac[1], drift[0],
                                  drift[1], x0, y0, cw, ch, up, _p(out))
        return out

    def tiff(self, path, expected_bytes=0, big=False):
        """The reference's TiffWriter (cli/tiff_writer.h) on `path`."""
        return RefTiff(self, path, expected_bytes, big)

    def binned_render(self, kernel, sigma_px, w, h, upscale, emitters, frames, img=None):
        """sim::BinnedBlinkRenderer: Setup on `kernel` (a RefKernel; None: the Gaussian of sigma_px), Render of each
        frame's emitters (EMITTER_DTYPE / FRAME_DTYPE records) into img (n, h, w) float32 (+=; zeros when None), frames
        in parallel on the reference's pool. Returns (img, u, R, wall seconds)."""
        em = np.ascontiguousarray(emitters)
        fr = np.ascontiguousarray(frames)
        if img is None:
            img = np.zeros((len(fr), h, w), np.float32)
        u, r = C.c_int(), C.c_int()
        sec = self.L.ref_binned_render(kernel.h if kernel is not None else None, sigma_px, w, h, upscale, _p(em),
                                       _p(fr), len(fr), _p(img), C.byref(u), C.byref(r))
        if sec < 0:
            raise RuntimeError("BinnedBlinkRenderer::Setup refused")
        return img, u.value, r.value, sec

    def dye_h1(self, seed, cx, cy, mt_index):
        return int(self.L.ref_dye_h1(int(seed) & 0xFFFFFFFF, int(cx), int(cy), int(mt_index)))


class RefTiff:
    """A TiffWriter in the reference harness: page / page_rows / rows return the writer's bool, error() its
    message."""

    def __init__(self, ref, path, expected_bytes, big):
        self.L = ref.L
        self.h = self.L.ref_tiff_open(str(path).encode(), int(expected_bytes), int(big))

    @staticmethod
    def _d(desc):
        return None if desc is None else desc.encode()

    def page(self, px, w, h, desc=None):
        px = np.ascontiguousarray(px)
        fn = self.L.ref_tiff_page_f32 if px.dtype == np.float32 else self.L.ref_tiff_page_u16
        return bool(fn(self.h, _p(px), px.size, w, h, self._d(desc)))

    def page_rows(self, px, rows, w, h, desc=None):
        px = np.ascontiguousarray(px, np.uint16)
        return bool(self.L.ref_tiff_page_rows(self.h, _p(px), rows, w, h, self._d(desc)))

    def rows(self, page, y0, rows, px):
        px = np.ascontiguousarray(px, np.uint16)
        return bool(self.L.ref_tiff_rows(self.h, page, y0, rows, _p(px)))

    def big(self):
        return bool(self.L.ref_tiff_big(self.h))

    def error(self):
        buf = C.create_string_buffer(4096)
        self.L.ref_tiff_error(self.h, buf, 4096)
        return buf.value.decode()

    def close(self):
        ok = bool(self.L.ref_tiff_close(self.h))
        self.h = None
        return ok


def _geometry(req):
    return Oracle().psf_geometry(req)


class RefKernel:
    """A sim::PsfKernelCache in the reference harness."""

    def __init__(self, ref: Reference, req=None, planes=None, os_=4, z_step_nm=25.0, interp=2, handle=None):
        self.ref = ref
        L = ref.L
        if handle is not None:
            self.h = handle
        elif req is not None:
            r = req.c()
            self.h = L.ref_kernel_build(C.byref(r))
            if not self.h:
                raise RuntimeError(L.ref_last_error().decode())
        else:
            planes = np.ascontiguousarray(planes, np.float32)
            nz, s, _ = planes.shape
            self.h = L.ref_kernel_from_planes(_p(planes), s, nz, os_, z_step_nm, interp)

    def __del__(self):
        try:
            self.ref.L.ref_kernel_free(self.h)
        except Exception:
            pass

    def info(self):
        v = [C.c_int() for _ in range(4)]
        self.ref.L.ref_kernel_info(self.h, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def planes(self):
        size, nz, _, _ = self.info()
        out = np.zeros((nz, size, size), np.float32)
        self.ref.L.ref_kernel_planes(self.h, _p(out))
        return out

    def block_sums(self):
        _, nz, _, bw = self.info()
        out = np.zeros((nz, bw, bw), np.float32)
        self.ref.L.ref_kernel_block_sums(self.h, _p(out))
        return out

    def plan_splat_fft(self, x, y, z):
        """PlanSplat with the Fft placement: (shifted block sums (bw, bw) float32, (x0, y0, bx, by))."""
        size, nz, os_, bw = self.info()
        sums = np.zeros((bw, bw), np.float32)
        st = np.zeros(4, np.int32)
        if not self.ref.L.ref_plan_splat_fft(self.h, x, y, z, _p(sums), _p(st)):
            raise RuntimeError("PlanSplat refused")
        return sums, tuple(int(v) for v in st)

    def plan_splat_fft_batch(self, xy, z):
        """PlanSplat (Fft) for each emitter on the reference's pool; wall seconds."""
        xy = np.ascontiguousarray(xy, np.float64)
        z = np.ascontiguousarray(z, np.int32)
        return self.ref.L.ref_plan_splat_fft_batch(self.h, _p(xy), _p(z), len(z))

    def halo(self, threshold):
        return RefKernel(self.ref, handle=self.ref.L.ref_kernel_halo(self.h, threshold))

    def wf_grid(self, upscale, pixel_um, width, height, origin_um, margin_um, zplane_nm):
        """WidefieldScene::GridSpecFor of the widefield scene below: (grid nx, grid ny, FOV cell x0, FOV cell y0)."""
        g = np.zeros(4, np.uint32)
        self.ref.L.ref_wf_grid(upscale, pixel_um, width, height, origin_um[0], origin_um[1], margin_um, zplane_nm,
                               _p(g))
        return tuple(int(v) for v in g)

    def wf_scene(self, counts, upscale, cap_um, pixel_um, width, height, origin_um, margin_um, zplane_nm, k0=0,
                 focus0_um=0.0, gpu_mode=True):
        """The reference's widefield scene (WidefieldScene over KernelWidefieldPsf of this kernel) on a dense
        persistent dye grid counts (nzd, gny, gnx), the grid wf_grid gives."""
        return RefWfScene(self, counts, upscale, cap_um, pixel_um, width, height, origin_um, margin_um, zplane_nm,
                          k0, focus0_um, gpu_mode)

    def wf_focus_series(self, counts, foci_um, upscale, cap_um, pixel_um, width, height, origin_um, margin_um,
                        zplane_nm, k0=0, gpu_mode=True):
        """wf_scene(...).series(foci_um): camera frames (n, height, width) float32 and (FFT nx, FFT ny, radius)."""
        sc = self.wf_scene(counts, upscale, cap_um, pixel_um, width, height, origin_um, margin_um, zplane_nm, k0,
                           foci_um[0], gpu_mode)
        try:
            return sc.series(foci_um)[0], sc.info
        finally:
            sc.close()

    def spans(self):
        size, nz, os_, _ = self.info()
        cam = ((size - 1) // 2) // os_
        lo = np.zeros(nz * (2 * cam + 1), np.int16)
        hi = np.zeros_like(lo)
        r2 = np.zeros(nz, np.int32)
        rc = self.ref.L.ref_kernel_spans(self.h, _p(lo), _p(hi), _p(r2))
        return None if rc < 0 else (lo, hi, r2)

    def nearest_z(self, z_um):
        return self.ref.L.ref_nearest_z(self.h, z_um)

    def render_photon_image(self, events, frame, w, h, pixel_nm, per_blink, bg, drift_x=0.0, drift_y=0.0,
                            global_z=0.0, illum=None, bg_map=None, bg_scale=1.0, min_photons=0.0, parallel=False,
                            onto=None):
        """RenderPhotonImage; onto: an earlier dye group's image to splat onto (RenderExtras::accumulate)."""
        events = np.ascontiguousarray(events)
        out = np.zeros((h, w), np.float32) if onto is None else np.array(onto, np.float32, copy=True)
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        self.ref.L.ref_render_photon_image(self.h, _p(events), len(events), frame, w, h, pixel_nm, per_blink, bg,
                                           drift_x, drift_y, global_z, _p(f(illum)), _p(f(bg_map)), bg_scale,
                                           min_photons, int(parallel), int(onto is not None), _p(out))
        return out

    def collect_gpu_emitters(self, events, frame, w, h, pixel_nm, per_blink, drift_x=0.0, drift_y=0.0, global_z=0.0,
                             kernel=0, min_photons=0.0):
        from insiliscope_b200.engine import GPU_SPLAT_EMITTER_DTYPE
        events = np.ascontiguousarray(events)
        out = np.zeros(len(events), GPU_SPLAT_EMITTER_DTYPE)
        n = self.ref.L.ref_collect_gpu_emitters(self.h, _p(events), len(events), frame, w, h, pixel_nm, per_blink,
                                                drift_x, drift_y, global_z, kernel, min_photons, _p(out), len(out))
        return out[:n].copy()

    def render_movie(self, events, frame0, n_frames, w, h, pixel_nm, per_blink, bg, camera, offset, gain,
                     read_noise, seed, want_photons=False, want_adu=True):
        """The reference's frame loop (frames in parallel on its pool). Returns (seconds, photons, adu)."""
        events = np.ascontiguousarray(events)
        ph = np.zeros((n_frames, h, w), np.float32) if want_photons else None
        adu = np.zeros((n_frames, h, w), np.uint16) if want_adu else None
        cam = camera.c()
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        t = self.ref.L.ref_render_movie(self.h, _p(events), len(events), frame0, n_frames, w, h, pixel_nm, per_blink,
                                        bg, C.byref(cam), _p(f(offset)), _p(f(gain)), _p(f(read_noise)), seed,
                                        _p(ph), _p(adu))
        return t, ph, adu


class RefWfScene:
    """A reference WidefieldScene (ref_wf_scene_create): series(foci) -> (frames, wall seconds)."""

    def __init__(self, kernel, counts, upscale, cap_um, pixel_um, width, height, origin_um, margin_um, zplane_nm, k0,
                 focus0_um, gpu_mode):
        self.L = kernel.ref.L
        self.counts = np.ascontiguousarray(counts, np.float32)
        self.shape = (height, width)
        info = np.zeros(3, np.uint32)
        self.h = self.L.ref_wf_scene_create(kernel.h, upscale, cap_um, pixel_um, width, height, origin_um[0],
                                            origin_um[1], margin_um, zplane_nm, k0, self.counts.shape[0],
                                            _p(self.counts), focus0_um, int(gpu_mode), _p(info))
        if not self.h:
            raise RuntimeError(self.L.ref_last_error().decode())
        self.info = tuple(int(v) for v in info)

    def series(self, foci_um):
        foci = np.ascontiguousarray(foci_um, np.float64)
        out = np.zeros((len(foci),) + self.shape, np.float32)
        sec = self.L.ref_wf_scene_series(self.h, _p(foci), len(foci), _p(out))
        if sec < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out, sec

    def close(self):
        if self.h:
            self.L.ref_wf_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def binned_cell_kernels_f64(planes, os_, upscale, radius2=None):
    """The binned renderer's plane kernels at the cell pitch (KernelWidefieldPsf, WidefieldRender.cpp:262-322;
    BinnedBlinkRenderer::Setup, BinnedBlinks.cpp:150-188): u = the largest divisor of os up to upscale, r = os / u
    oversampled samples per cell, s0 = floor((n - 1) / 2 - r / 2 + 1); cell (dx, dy) = the float64 sum over the r x r
    block from (s0 + dx r, s0 + dy r) clipped to the plane, rows then columns, as float32; R = the cells that reach
    the plane, capped by the halo cut at ceil((sqrt(max radius2) + 1) u). Returns (K (nz, 2R+1, 2R+1), u, R)."""
    P = np.asarray(planes, np.float32)
    nz, n, _ = P.shape
    os_ = max(1, int(os_))
    u = 1
    for c in range(max(1, min(int(upscale), os_)), 1, -1):
        if os_ % c == 0:
            u = c
            break
    r = max(1, os_ // u)
    s0 = int(np.floor((n - 1) / 2.0 - r / 2.0 + 1.0))
    d_min = int(np.ceil((-s0 - r + 1) / float(r)))
    d_max = int(np.floor((n - 1 - s0) / float(r)))
    R = max(1, max(-d_min, d_max))
    if radius2 is not None and len(radius2):
        r2 = int(np.max(radius2))
        if r2 >= 0:
            R = min(R, int(np.ceil((np.sqrt(float(r2)) + 1.0) * u)))
    R = max(1, R)
    d = np.arange(-R, R + 1)
    ya = s0 + d * r
    acc = np.zeros((nz, 2 * R + 1, 2 * R + 1), np.float64)
    for iy in range(r):                      # the block's rows, then its columns: the reference's summation order
        y = ya + iy
        for ix in range(r):
            x = ya + ix
            ok = ((y >= 0) & (y < n))[:, None] & ((x >= 0) & (x < n))[None, :]
            v = P[:, np.clip(y, 0, n - 1)][:, :, np.clip(x, 0, n - 1)].astype(np.float64)
            acc += np.where(ok[None], v, 0.0)
    return acc.astype(np.float32), u, R


def binned_gauss_kernel_f64(sigma_px, upscale):
    """The renderer's kernel without a PSF (BinnedBlinks.cpp:190-212): u = upscale clamped to 1..8,
    R = ceil(3 sigma u), exp(-(x^2 + y^2) / (2 (sigma u)^2)) normalized in float64, as float32."""
    u = max(1, min(int(upscale), 8))
    R = max(1, int(np.ceil(3.0 * sigma_px * u)))
    x = np.arange(-R, R + 1, dtype=np.float64)
    sc = sigma_px * u
    k = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (2.0 * sc * sc))
    return (k / k.sum()).astype(np.float32)[None], u, R


def binned_render_f64(K, u, R, emitters, frames, w, h):
    """BinnedBlinkRenderer::Render (BinnedBlinks.cpp:216-246) as the linear convolution it computes, in float64:
    per frame every emitter with photons > 0 at cell floor((x + 0.5) u) (skipped beyond R cells outside the frame),
    plane (plane & 0xFFFF) clamped, adds float32(photons) x K[plane] around its cell; the cells (float32) clamped at
    0 are summed u x u per pixel in float64. Returns (n, h, w) float32."""
    K = np.asarray(K, np.float64)
    nz = K.shape[0]
    cw, ch = w * u, h * u
    out = np.zeros((len(frames), h, w), np.float32)
    for k, fr in enumerate(frames):
        canvas = np.zeros((ch + 4 * R, cw + 4 * R), np.float64)   # cells -2R .. c + 2R
        for e in emitters[int(fr["em_start"]): int(fr["em_start"]) + int(fr["em_count"])]:
            if not (e["photons"] > 0.0):
                continue
            cx = int(np.floor((e["x_px"] + 0.5) * u))
            cy = int(np.floor((e["y_px"] + 0.5) * u))
            if cx < -R or cy < -R or cx >= cw + R or cy >= ch + R:
                continue
            p = min(nz - 1, max(0, int(e["plane"]) & 0xFFFF))
            ph = float(np.float32(e["photons"]))
            canvas[cy + R: cy + 3 * R + 1, cx + R: cx + 3 * R + 1] += ph * K[p]
        cells = canvas[2 * R: 2 * R + ch, 2 * R: 2 * R + cw].astype(np.float32)
        cells = np.maximum(cells, np.float32(0)).astype(np.float64)
        out[k] = cells.reshape(h, u, w, u).sum(axis=(1, 3)).astype(np.float32)
    return out


def fft_shift_tile_f64(plane, shift_x, shift_y):
    """FftShiftKernelTile (PsfGeneratorBridge.cpp:1293-1370) in float64: each row of the n x n plane zero-padded to
    N (the power of two >= 2n), transformed, times exp(2 pi i kk shift / N) with kk the wrapped frequency (k - N from
    N/2 on), transformed back over N, the first n kept (complex); then the same along the columns of that; the real
    part as float32 -- g(i) = f(i + shift), band-limited."""
    P = np.asarray(plane, np.float64)
    n = P.shape[0]
    N = 1
    while N < 2 * n:
        N <<= 1
    kk = np.arange(N)
    kk = np.where(kk < N // 2, kk, kk - N)

    def shift_lines(a, s):   # lines along the last axis
        A = np.fft.fft(a, N, axis=-1) * np.exp(2j * np.pi * kk * s / N)
        return np.fft.ifft(A, axis=-1)[..., :n]

    mid = shift_lines(P, shift_x)
    out = shift_lines(mid.T, shift_y).T
    return out.real.astype(np.float32)


def fft_place_f64(planes, os_, x, y, z):
    """The Fft placement of one emitter (PlanSplat, PsfGeneratorBridge.cpp:1441-1456): the nearest setup's centre
    pixel x0 = floor(x + 0.5) and tap origin t = kc + (x0 - x - 0.5) os + 0.5 (kc = (n - 1) / 2), its rounding half up
    r = floor(t + 0.5), the plane shifted by (tx - rx, ty - ry); returns (the shifted plane, (x0, y0, rx, ry))."""
    P = np.asarray(planes[z])
    n = P.shape[0]
    kc = (n - 1) / 2.0
    x0, y0 = int(np.floor(x + 0.5)), int(np.floor(y + 0.5))
    tx = kc + (x0 - x - 0.5) * os_ + 0.5
    ty = kc + (y0 - y - 0.5) * os_ + 0.5
    rx, ry = np.floor(tx + 0.5), np.floor(ty + 0.5)
    return fft_shift_tile_f64(P, tx - rx, ty - ry), (x0, y0, int(rx), int(ry))


def shifted_frame_f64(spectra, coef, shift, nx, ny, window, up, scale=1.0):
    """RenderShiftedImages (WidefieldRender.cpp:2905-2935; ApplyShiftRamp / ShiftedCamera, DriftShift.cpp:23-71) in
    float64: S = sum of coef[c] x spectra[c] (zero coefficients skipped), times exp(2 pi i (kx sx / nx + ky' sy / ny))
    (Nyquist terms: their cosine), the inverse as RealFft2d's (a complex inverse along y, then along x the packed
    real inverse of the half spectrum: Z[k] = (X[k] + conj X[H-k]) + i conj(w^k) (X[k] - conj X[H-k]), H = nx / 2),
    / (nx ny); the window's cells clamped at 0, summed up x up per pixel, times scale."""
    x0, y0, cw, ch = window
    H, W = nx // 2, nx // 2 + 1
    S = np.zeros((ny, W), np.complex128)
    for c, s in zip(coef, spectra):
        if c != 0:
            S += float(c) * np.asarray(s, np.complex128)
    sx, sy = shift
    if sx != 0 or sy != 0:
        kx = np.arange(W)
        px = np.exp(2j * np.pi * kx * sx / nx)
        px[kx == nx // 2] = np.cos(2 * np.pi * (nx // 2) * sx / nx)
        ky = np.arange(ny)
        kys = np.where(ky <= ny // 2, ky, ky - ny)
        py = np.exp(2j * np.pi * kys * sy / ny)
        py[ky == ny // 2] = np.cos(2 * np.pi * (ny // 2) * sy / ny)
        S = S * py[:, None] * px[None, :]
    X = np.fft.ifft(S, axis=0) * ny                 # unnormalised inverse along y
    k = np.arange(H)
    w = np.exp(-2j * np.pi * k / nx)
    xk, xm = X[:, k], np.conj(X[:, H - k])
    Z = (xk + xm) + 1j * np.conj(w) * (xk - xm)
    z = np.fft.ifft(Z, axis=1) * H
    img = np.empty((ny, nx))
    img[:, 0::2], img[:, 1::2] = z.real, z.imag
    img /= nx * ny
    cells = np.maximum(img[y0:y0 + ch, x0:x0 + cw], 0.0)
    Hc, Wc = ch // up, cw // up
    cam = cells[:Hc * up, :Wc * up].reshape(Hc, up, Wc, up).sum(axis=(1, 3)) * scale
    return cam.astype(np.float32)


def wf_kernel_volume_f64(cell_kernels, zstep_nm, zplane_nm, nzd):
    """The widefield scene's kernel for every dye-plane-to-focus offset of a focus series taken at the dye planes'
    centres, as one (2 nzd - 1)-plane volume: plane j serves a dye plane d = nzd - 1 - j planes above the focus
    (defocus d zplane). PlanFocus (WidefieldRender.cpp:1460-1522) with KernelWidefieldPsf::PlaneCoord (:282-287):
    t = defocus 1000 / zStep + (nz - 1) / 2 clamped to the stack [0, nz - 1], p0 = floor(t) (the last plane: frac 0),
    weights (1 - frac, frac) as float32; the plane w0 K[p0] + w1 K[p0 + 1] in float64."""
    K = np.asarray(cell_kernels, np.float64)
    nzk = K.shape[0]
    out = np.zeros((2 * nzd - 1,) + K.shape[1:], np.float64)
    for j in range(2 * nzd - 1):
        d = nzd - 1 - j
        t = d * zplane_nm / zstep_nm + (nzk - 1) / 2.0 if nzk > 1 and zstep_nm > 0 else 0.0
        t = min(nzk - 1.0, max(0.0, t))
        p0 = int(np.floor(t))
        frac = t - p0
        if p0 >= nzk - 1:
            p0, frac = nzk - 1, 0.0
        out[j] = float(np.float32(1.0 - frac)) * K[p0]
        if frac > 0.0:
            out[j] += float(np.float32(frac)) * K[p0 + 1]
    return out


def wf_scene_f64(counts, kernel_volume, fov, upscale):
    """The widefield scene's camera frames in float64 for foci at the dye planes' centres: per focus f the linear
    convolution sum_k counts[k] (x) kernel_volume[f - k + nzd - 1] over the whole grid (ChannelImageStep /
    ChannelImageFinish, WidefieldRender.cpp:1724-1878), the FOV cells (x0, y0, cw, ch) cut out, then each camera pixel
    the sum of max(0, cell) over its upscale x upscale cells (WidefieldImages::Render, :547-586)."""
    x0, y0, cw, ch = fov
    u = int(upscale)
    full = fft_convolve_same_f64(counts, kernel_volume)
    cells = np.maximum(full[:, y0:y0 + ch, x0:x0 + cw], 0.0)
    n = cells.shape[0]
    return cells.reshape(n, ch // u, u, cw // u, u).sum(axis=(2, 4))


def fft_convolve_same_f64(volume: np.ndarray, psf: np.ndarray) -> np.ndarray:
    """Linear 3D convolution of volume (nz, ny, nx) with psf (kz, ky, kx) centred on (kz//2, ky//2, kx//2), cropped
    to the volume, in float64 (the widefield mean-field focus series' oracle)."""
    v = np.asarray(volume, np.float64)
    k = np.asarray(psf, np.float64)
    shape = [a + b - 1 for a, b in zip(v.shape, k.shape)]
    axes = list(range(v.ndim))
    F = np.fft.rfftn(v, shape, axes=axes) * np.fft.rfftn(k, shape, axes=axes)
    full = np.fft.irfftn(F, shape, axes=axes)
    sl = tuple(slice(kk // 2, kk // 2 + n) for kk, n in zip(k.shape, v.shape))
    return full[sl]
