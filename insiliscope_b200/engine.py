"""Python host side of the engine: the reference's GPU seam (sim::GpuSimulator, GpuSimD3D11.h:61-111) and the PSF
entry (ComputePsfKernelCache, PsfGeneratorBridge.h:317) over the C ABI of libiscu.so.

Host arrays are numpy; device arrays are torch CUDA tensors (torch is the device-memory plumbing, the work runs in
libiscu.so's kernels). Errors raise IscuError with the library's message -- the reference seam's `bool` + `err`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import (CZT_FP32, CZT_TF32X3, CZT_F16X3, INTERP_CUBIC, INTERP_LINEAR, INTERP_NEAREST, Camera, IscuError, PsfRequest,
                   check, load)

EMITTER_DTYPE = np.dtype([("x_px", "<f8"), ("y_px", "<f8"), ("photons", "<f8"), ("plane", "<i4"),
                          ("reserved", "<i4")])
FRAME_DTYPE = np.dtype([("em_start", "<u4"), ("em_count", "<u4"), ("frame", "<u4"), ("reserved", "<u4"),
                        ("bg_scale", "<f8")])
GPU_SPLAT_EMITTER_DTYPE = np.dtype([("x0", "<i4"), ("y0", "<i4"), ("bx", "<i4"), ("by", "<i4"), ("plane", "<i4"),
                                    ("n_taps", "<i4"), ("photons", "<f4"), ("cut_radius2", "<i4"),
                                    ("wx", "<f4", (4,)), ("wy", "<f4", (4,))])
BLINK_EVENT_DTYPE = np.dtype([("x_um", "<f8"), ("y_um", "<f8"), ("z_nm", "<f8"), ("t_start", "<f8"),
                              ("t_end", "<f8"), ("brightness", "<f8"), ("excite", "<f8"), ("slot", "<i4"),
                              ("reserved", "<i4")])
DYE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("h1", "<u4"), ("k", "<i4"), ("n", "<i4"),
                      ("id", "<u4"), ("structure", "<i4"), ("reserved", "<i4")])
EVENT_STRIDE = 10   # isc_events_in_window's row: x, y, z, tOn, tOff, brightness, id, structure, state, aux
LABEL_DSTORM, LABEL_PALM, LABEL_DNA_PAINT, LABEL_WIDEFIELD = 0, 1, 2, 3
assert DYE_DTYPE.itemsize == 48
assert EMITTER_DTYPE.itemsize == C.sizeof(_abi.Emitter) == 32
assert FRAME_DTYPE.itemsize == C.sizeof(_abi.Frame) == 24
assert GPU_SPLAT_EMITTER_DTYPE.itemsize == C.sizeof(_abi.GpuSplatEmitter) == 64
assert BLINK_EVENT_DTYPE.itemsize == C.sizeof(_abi.BlinkEvent) == 64


@dataclass
class CameraParams:
    """sim::CameraNoiseParams (SMLMNoise.h:35-50)."""
    quantum_efficiency: float = 1.0
    dark_electrons: float = 0.0
    gain: float = 1.0
    read_noise_e: float = 1.5
    emccd: bool = False
    bit_depth: int = 16
    em_gain: float = 300.0
    cic_electrons: float = 0.002

    def c(self) -> Camera:
        return Camera(self.quantum_efficiency, self.dark_electrons, self.gain, self.read_noise_e, int(self.emccd),
                      int(self.bit_depth), self.em_gain, self.cic_electrons)


@dataclass
class PsfParams:
    """sim::PsfGeneratorRequest, GibsonLanniZernike (PsfGeneratorBridge.h:91-158); zernike: OSA 0-27, waves."""
    wavelength_nm: float = 660.0
    na: float = 1.4
    immersion_index: float = 1.518
    sample_index: float = 1.518
    working_distance_um: float = 150.0
    sample_depth_nm: float = 0.0
    pixel_size_nm: float = 100.0
    zernike: list = field(default_factory=lambda: [0.0] * 28)
    double_helix: bool = False
    mask_modes: int = 5
    mask_waist: float = 1.0
    oversampling: int = 4
    kernel_half_width_px: int = 8
    nz: int = 1
    pupil_samples: int = 0
    z_step_nm: float = 100.0
    interp: int = INTERP_NEAREST

    def c(self) -> PsfRequest:
        r = PsfRequest()
        r.wavelength_nm = self.wavelength_nm
        r.na = self.na
        r.immersion_index = self.immersion_index
        r.sample_index = self.sample_index
        r.working_distance_um = self.working_distance_um
        r.sample_depth_nm = self.sample_depth_nm
        r.pixel_size_nm = self.pixel_size_nm
        z = list(self.zernike) + [0.0] * (28 - len(self.zernike))
        for j in range(28):
            r.zernike[j] = float(z[j])
        r.mask_double_helix = int(self.double_helix)
        r.mask_modes = int(self.mask_modes)
        r.mask_waist = float(self.mask_waist)
        r.oversampling = int(self.oversampling)
        r.kernel_half_width_px = int(self.kernel_half_width_px)
        r.nz = int(self.nz)
        r.pupil_samples = int(self.pupil_samples)
        r.z_step_nm = float(self.z_step_nm)
        r.interp = int(self.interp)
        return r

    def geometry(self) -> tuple[int, int, int]:
        """(plane size, planes, pupil samples) as the reference derives them (ZernikePsf.cpp:118-158)."""
        s, nz, m = C.c_int32(), C.c_int32(), C.c_int32()
        req = self.c()
        check(load().iscu_psf_geometry(C.byref(req), C.byref(s), C.byref(nz), C.byref(m)))
        return s.value, nz.value, m.value


def _ptr(a) -> C.c_void_p:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())   # torch tensor


def _require_tensor(t, name: str, dtypes, device, min_numel: int):
    """ValueError unless t is a contiguous torch tensor of one of `dtypes` (torch dtypes) with at least min_numel
    elements, on CUDA device `device` (None: in host memory), so the library never writes past a caller's buffer."""
    import torch
    where = f"cuda:{device}" if device is not None else "the host"
    ok = (isinstance(t, torch.Tensor) and t.dtype in dtypes and t.is_contiguous() and t.numel() >= min_numel and
          (t.is_cuda and t.device.index == device if device is not None else not t.is_cuda))
    if not ok:
        names = " or ".join(str(d).replace("torch.", "") for d in dtypes)
        raise ValueError(f"{name} must be a contiguous {names} tensor on {where} with at least {min_numel} elements")


def _require_array(a, name: str, dtype, min_size: int):
    """ValueError unless a is a C-contiguous numpy array of dtype with at least min_size elements."""
    if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous and a.size >= min_size):
        raise ValueError(f"{name} must be a C-contiguous {np.dtype(dtype).name} array with at least {min_size} "
                         "elements")


def _n_records(a) -> int:
    """EMITTER_DTYPE records in a device (torch, any dtype viewed as bytes) or host emitter buffer."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.nbytes // EMITTER_DTYPE.itemsize
    return a.numel() * a.element_size() // EMITTER_DTYPE.itemsize


def _f32(a, n=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def generate_camera_maps(width, height, seed, offset_mean=100.0, offset_std=2.0, gain=1.0, gain_std_fraction=0.0,
                         read_noise=1.5, read_noise_std_fraction=0.0, keep_y0=0, keep_rows=0):
    """PixelOffsetMap/GainMap/ReadNoiseMap::Generate from one mt19937_64(seed), offset then gain then read noise."""
    rows = keep_rows if keep_rows else height
    rows = min(rows, max(0, height - keep_y0)) if keep_rows else height
    off = np.empty(width * rows, np.float32)
    g = np.empty_like(off)
    rn = np.empty_like(off)
    check(load().iscu_generate_camera_maps(width, height, seed, offset_mean, offset_std, gain, gain_std_fraction,
                                            read_noise, read_noise_std_fraction, keep_y0, keep_rows, _ptr(off),
                                            _ptr(g), _ptr(rn)))
    return off, g, rn


class Engine:
    """One libiscu context: a device, a stream, up to four resident kernel stacks and the camera statics.

    The `*_dev` methods take torch CUDA tensors. The library works on its own (non-blocking) stream; by default these
    methods wait for torch's current stream before they enqueue and for the library's stream before they return
    (sync=True). Callers that order the two streams themselves -- e.g. work issued under
    `torch.cuda.stream(engine.torch_stream())` -- pass sync=False."""

    def __init__(self, device: int = 0):
        import weakref
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.iscu_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self.width = self.height = 0
        self._plans = weakref.WeakSet()
        self._pending_io = {}   # I/O slot -> the host arrays of its enqueued event-render batch

    def close(self):
        """Destroys the context, after the plans made on it (a plan must not outlive its context)."""
        if self.h:
            for p in list(self._plans):
                p.close()
            self.lib.iscu_destroy(self.h)   # waits for the copies in flight first
            self.h = None
            self._pending_io = {}

    def _before(self, sync):
        if sync:
            import torch
            torch.cuda.current_stream(self.device).synchronize()

    def _after(self, sync):
        if sync:
            self.synchronize()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------------------------------------- plumbing
    def synchronize(self):
        check(self.lib.iscu_synchronize(self.h))

    @property
    def launch_count(self) -> int:
        return int(self.lib.iscu_launch_count(self.h))

    @property
    def stream_handle(self) -> int:
        return int(self.lib.iscu_stream(self.h) or 0)

    def torch_stream(self):
        import torch
        return torch.cuda.ExternalStream(self.stream_handle, device=f"cuda:{self.device}")

    # -------------------------------------------------------------------------------------------- RNG
    def pcg4d(self, words):
        """pcg4d of each row of an (n, 4) uint32 CUDA tensor (SMLMCounterRng.h:37-56)."""
        import torch
        words = words.contiguous()
        out = torch.empty_like(words)
        self._before(True)
        check(self.lib.iscu_pcg4d_dev(self.h, _ptr(words), _ptr(out), words.shape[0]))
        self.synchronize()
        return out

    def counter_uniforms(self, seed, frame, pixel0, npix, per_pixel):
        """The first per_pixel uniforms of each pixel's CounterRng stream (SMLMCounterRng.h:60-91), float64."""
        import torch
        out = torch.empty((npix, per_pixel), dtype=torch.float64, device=f"cuda:{self.device}")
        check(self.lib.iscu_counter_uniforms_dev(self.h, seed, frame, pixel0, npix, per_pixel, _ptr(out)))
        self.synchronize()
        return out

    # -------------------------------------------------------------------------------------------- camera
    def set_static(self, width, height, pixel_base=0, offset=None, gain=None, read_noise=None, background=None,
                   illum=None, flat_bg=0.0):
        n = width * height
        arrs = [_f32(a, n) for a in (offset, gain, read_noise, background, illum)]
        check(self.lib.iscu_set_static(self.h, width, height, pixel_base, *[_ptr(a) for a in arrs], float(flat_bg)))
        self.width, self.height = width, height

    def noise_frames_dev(self, photons, frames, camera: CameraParams, seed, out=None, sync=True):
        """ApplyNoiseChain on (n, h, w) float32 CUDA photons; frames: the frame index of each (host indices, or an
        int32/uint32 CUDA tensor of them). Returns the uint16 frames (into `out` when given)."""
        import torch
        photons = photons.contiguous()
        if isinstance(frames, torch.Tensor):
            fr = frames
        else:
            fr = torch.as_tensor(np.asarray(frames, dtype=np.int64).astype(np.uint32).view(np.int32),
                                 device=photons.device)
        if out is None:
            out = torch.empty(photons.shape, dtype=torch.uint16, device=photons.device)
        cam = camera.c()
        self._before(sync)
        check(self.lib.iscu_noise_frames_dev(self.h, _ptr(photons), photons.shape[0], _ptr(fr), C.byref(cam), seed,
                                             _ptr(out)))
        self._after(sync)
        return out

    # -------------------------------------------------------------------------------------------- PSF
    def psf_library_dev(self, sets, set_of_psf, defocus_nm, size=0, normalize=True, method=CZT_FP32, out=None):
        """A PSF library (n, P, P) float32 CUDA tensor; see iscu_psf_library_dev. method: CZT_FP32 (any size),
        CZT_F16X3 or CZT_TF32X3 (the tensor-core forms: pupil samples M <= 128, a multiple of 16, planes <= 64 x 64)."""
        import torch
        reqs = (PsfRequest * len(sets))(*[s.c() for s in sets])
        so = np.ascontiguousarray(set_of_psf, dtype=np.uint32)
        dz = np.ascontiguousarray(defocus_nm, dtype=np.float64)
        if len(dz) != len(so):
            raise ValueError(f"defocus_nm has {len(dz)} entries, set_of_psf {len(so)}")
        P = size if size > 0 else sets[0].geometry()[0]
        if out is None:
            out = torch.empty((len(so), P, P), dtype=torch.float32, device=f"cuda:{self.device}")
        _require_tensor(out, "out", (torch.float32,), self.device, len(so) * P * P)
        check(self.lib.iscu_psf_library_dev(self.h, reqs, len(sets), _ptr(so), _ptr(dz), len(so), size,
                                            int(normalize), method, _ptr(out)))
        return out

    def psf_library_noalloc_dev(self, sets, set_of_psf, defocus_nm, out, size=0, normalize=True):
        """iscu_psf_library_noalloc_dev: the FP32 PSF library with no device allocation in the call (its
        temporaries in the library's static device array); out: a caller-owned (n, P, P) float32 CUDA tensor."""
        import torch
        reqs = (PsfRequest * len(sets))(*[s.c() for s in sets])
        so = np.ascontiguousarray(set_of_psf, dtype=np.uint32)
        dz = np.ascontiguousarray(defocus_nm, dtype=np.float64)
        if len(dz) != len(so):
            raise ValueError(f"defocus_nm has {len(dz)} entries, set_of_psf {len(so)}")
        P = size if size > 0 else sets[0].geometry()[0]
        _require_tensor(out, "out", (torch.float32,), self.device, len(so) * P * P)
        check(self.lib.iscu_psf_library_noalloc_dev(self.h, reqs, len(sets), _ptr(so), _ptr(dz), len(so), size,
                                                    int(normalize), _ptr(out)))
        return out

    def fft_place_dev(self, slot, emitters_dev, sync=True):
        """The Fft placement of each emitter (iscu_fft_place_dev; emitters: uint8 view of EMITTER_DTYPE records):
        (shifted block sums (n, bw, bw) float32, origins (n, 4) int32: x0, y0, bx, by) CUDA tensors."""
        import torch
        n = _n_records(emitters_dev)
        size, nz, os_, bw = self.kernel_info(slot)[:4]
        sums = torch.empty((n, bw, bw), dtype=torch.float32, device=emitters_dev.device)
        origins = torch.empty((n, 4), dtype=torch.int32, device=emitters_dev.device)
        self._before(sync)
        check(self.lib.iscu_fft_place_dev(self.h, slot, _ptr(emitters_dev), n, _ptr(sums), _ptr(origins)))
        self._after(sync)
        return sums, origins

    def render_fft_frames_dev(self, slot, emitters_dev, frames_dev, n_frames, camera: CameraParams | None, seed,
                              photons_dev=None, adu_dev=None, sync=True):
        """Frames with the Fft placement (iscu_render_fft_frames_dev) on torch CUDA buffers, as render_frames_dev."""
        cam = camera.c() if camera is not None else None
        self._before(sync)
        check(self.lib.iscu_render_fft_frames_dev(self.h, slot, _ptr(emitters_dev), _n_records(emitters_dev),
                                                  _ptr(frames_dev), n_frames, C.byref(cam) if cam is not None else None,
                                                  seed, _ptr(photons_dev), _ptr(adu_dev)))
        self._after(sync)

    def csv_numbers_dev(self, values_dev, fmt, sync=True):
        """AppendCsvNumber of each float64 CUDA value (iscu_csv_numbers_dev): (fields (n, 48) uint8, lengths (n,)
        uint8) CUDA tensors."""
        import torch
        n = values_dev.numel()
        fields = torch.empty((n, 48), dtype=torch.uint8, device=values_dev.device)
        lens = torch.empty(n, dtype=torch.uint8, device=values_dev.device)
        self._before(sync)
        check(self.lib.iscu_csv_numbers_dev(self.h, _ptr(values_dev.contiguous()), n, fmt.encode(), _ptr(fields),
                                            _ptr(lens)))
        self._after(sync)
        return fields, lens

    def csv_table_dev(self, columns_dev, fmts, out_dev=None):
        """A numeric table's rows (iscu_csv_table_dev; columns_dev (n_cols, n_rows) float64 CUDA): the text as a uint8
        CUDA tensor (a view of out_dev when given, which must hold it)."""
        import torch
        cols = columns_dev.contiguous()
        n_cols, n_rows = cols.shape
        f = (C.c_char_p * n_cols)(*[x.encode() for x in fmts])
        nbytes = C.c_uint64()
        self._before(True)
        if out_dev is None:
            rc = self.lib.iscu_csv_table_dev(self.h, _ptr(cols), n_rows, n_cols, f, None, 0, C.byref(nbytes))
            if rc != _abi.ISCU_ERR_LIMIT:
                check(rc)
            out_dev = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device=cols.device)
        check(self.lib.iscu_csv_table_dev(self.h, _ptr(cols), n_rows, n_cols, f, _ptr(out_dev), out_dev.numel(),
                                          C.byref(nbytes)))
        return out_dev[:nbytes.value]

    def kernel_build(self, slot, req: PsfParams, method=CZT_FP32):
        r = req.c()
        check(self.lib.iscu_kernel_build(self.h, slot, C.byref(r), method))

    def kernel_set_planes(self, slot, planes, oversampling, z_step_nm, interp=INTERP_CUBIC):
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        nz, s, s2 = planes.shape
        assert s == s2
        check(self.lib.iscu_kernel_set_planes(self.h, slot, _ptr(planes), s, nz, oversampling, z_step_nm, interp))

    def kernel_set_halo(self, slot, threshold):
        check(self.lib.iscu_kernel_set_halo(self.h, slot, float(threshold)))

    def kernel_halo(self, slot):
        """A cut slot's spans: (lo, hi) of shape (nz, 2 camRad + 1) int16 and radius2 (nz,) int32."""
        size, nz, os_, _ = self.kernel_info(slot)
        n = 2 * (((size - 1) // 2) // os_) + 1
        lo, hi = np.empty((nz, n), np.int16), np.empty((nz, n), np.int16)
        r2 = np.empty(nz, np.int32)
        check(self.lib.iscu_kernel_get_halo(self.h, slot, _ptr(lo), _ptr(hi), _ptr(r2)))
        return lo, hi, r2

    def kernel_info(self, slot):
        v = [C.c_int32() for _ in range(4)]
        check(self.lib.iscu_kernel_info(self.h, slot, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)   # size, nz, os, bw

    def kernel_planes(self, slot):
        size, nz, _, _ = self.kernel_info(slot)
        out = np.empty((nz, size, size), np.float32)
        check(self.lib.iscu_kernel_get_planes(self.h, slot, _ptr(out)))
        return out

    def kernel_block_sums(self, slot):
        _, nz, _, bw = self.kernel_info(slot)
        out = np.empty((nz, bw, bw), np.float32)
        check(self.lib.iscu_kernel_get_block_sums(self.h, slot, _ptr(out)))
        return out

    # -------------------------------------------------------------------------------------------- splat + noise
    def render_frames(self, emitters, frames, camera: CameraParams | None, seed, want_photons=True, want_adu=True):
        """Host path: emitters (EMITTER_DTYPE), frames (FRAME_DTYPE) -> (photons (n,h,w) f32 | None, adu | None)."""
        emitters = np.ascontiguousarray(emitters, dtype=EMITTER_DTYPE)
        frames = np.ascontiguousarray(frames, dtype=FRAME_DTYPE)
        n = len(frames)
        ph = np.empty((n, self.height, self.width), np.float32) if want_photons else None
        adu = np.empty((n, self.height, self.width), np.uint16) if (want_adu and camera is not None) else None
        cam = camera.c() if camera is not None else None
        check(self.lib.iscu_render_frames(self.h, _ptr(emitters), len(emitters), _ptr(frames), n,
                                          C.byref(cam) if cam is not None else None, seed, _ptr(ph), _ptr(adu)))
        return ph, adu

    def render_frames_dev(self, emitters_dev, frames_dev, n_frames, camera: CameraParams | None, seed,
                          photons_dev=None, adu_dev=None, sync=True):
        """Device path on torch CUDA buffers (emitters: uint8 view of EMITTER_DTYPE records, frames likewise)."""
        cam = camera.c() if camera is not None else None
        self._before(sync)
        check(self.lib.iscu_render_frames_dev(self.h, _ptr(emitters_dev), _n_records(emitters_dev), _ptr(frames_dev),
                                              n_frames,
                                              C.byref(cam) if cam is not None else None, seed, _ptr(photons_dev),
                                              _ptr(adu_dev)))
        self._after(sync)

    def collect_emitters_dev(self, slot, events_dev, n_events, bucket_start_dev, n_frames, frame0, pixel_size_nm,
                             photons_per_blink, out_dev, frames_out_dev, n_out_dev, bucket_index_dev=None,
                             drift_x_px_dev=None, drift_y_px_dev=None, global_z_offset_um_dev=None,
                             bg_scale_dev=None, illum_dev=None, min_photons=0.0, n_clamped_dev=None,
                             event_index_dev=None, sync=True):
        """iscu_collect_emitters_dev on CUDA tensors (events: uint8 view of BLINK_EVENT_DTYPE records; out: of
        EMITTER_DTYPE records, its capacity the record count; frames_out: FRAME_DTYPE records; n_out: 1 uint32/int32)."""
        self._before(sync)
        check(self.lib.iscu_collect_emitters_dev(
            self.h, int(slot), _ptr(events_dev), int(n_events), _ptr(bucket_index_dev), _ptr(bucket_start_dev),
            int(frame0), int(n_frames), float(pixel_size_nm), float(photons_per_blink), _ptr(drift_x_px_dev),
            _ptr(drift_y_px_dev), _ptr(global_z_offset_um_dev), _ptr(bg_scale_dev), _ptr(illum_dev),
            float(min_photons), _ptr(out_dev), _ptr(event_index_dev), _n_records(out_dev), _ptr(frames_out_dev),
            _ptr(n_out_dev),
            _ptr(n_clamped_dev)))
        self._after(sync)

    def _event_batch(self, events, bucket_start, camera, bucket_index, drift_x_px, drift_y_px, global_z_offset_um,
                     bg_scale, want_photons, adu_out, photons_out):
        """The host arrays of one event-render batch (contiguous, the ABI's dtypes) and its outputs."""
        events = np.ascontiguousarray(events, dtype=BLINK_EVENT_DTYPE)
        bs = np.ascontiguousarray(bucket_start, dtype=np.uint32)
        nf = len(bs) - 1
        bi = None if bucket_index is None else np.ascontiguousarray(bucket_index, dtype=np.uint32)
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        per_frame = tuple(f64(a) for a in (drift_x_px, drift_y_px, global_z_offset_um, bg_scale))
        for a in per_frame:
            if a is not None and len(a) < nf:
                raise ValueError("a per-frame array is shorter than the batch's frames")
        shape = (nf, self.height, self.width)
        adu = None
        if camera is not None:
            adu = adu_out if adu_out is not None else np.empty(shape, np.uint16)
        ph = photons_out if photons_out is not None else (np.empty(shape, np.float32) if want_photons else None)
        for a, dt in ((adu, np.uint16), (ph, np.float32)):
            if a is not None and (a.dtype != dt or not a.flags.c_contiguous or a.size < nf * self.height * self.width):
                raise ValueError(f"an output must be a contiguous {np.dtype(dt).name} array of (frames, h, w)")
        cam = camera.c() if camera is not None else None
        return events, bs, nf, bi, per_frame, cam, ph, adu

    def render_events(self, slot, events, bucket_start, frame0, pixel_size_nm, photons_per_blink,
                      camera: CameraParams | None, seed, bucket_index=None, drift_x_px=None, drift_y_px=None,
                      global_z_offset_um=None, bg_scale=None, use_illum=False, min_photons=0.0, want_photons=False,
                      adu_out=None, photons_out=None):
        """Host blink events -> host frames in one C-ABI call (iscu_render_events): collection, render and noise on
        the device. Returns (photons | None, adu | None, n_emitters). Pass page-locked adu_out / photons_out (and
        events) for direct copies."""
        events, bs, nf, bi, pf, cam, ph, adu = self._event_batch(events, bucket_start, camera, bucket_index,
                                                                 drift_x_px, drift_y_px, global_z_offset_um, bg_scale,
                                                                 want_photons, adu_out, photons_out)
        n = C.c_uint32()
        check(self.lib.iscu_render_events(self.h, int(slot), _ptr(events), len(events), _ptr(bi), _ptr(bs),
                                          int(frame0), nf, float(pixel_size_nm), float(photons_per_blink),
                                          *[_ptr(a) for a in pf], int(bool(use_illum)), float(min_photons),
                                          C.byref(cam) if cam is not None else None, int(seed), _ptr(ph), _ptr(adu),
                                          C.byref(n), None))
        return ph, adu, n.value

    EVENT_IO_SLOTS = 4

    def render_events_async(self, io_slot, slot, events, bucket_start, frame0, pixel_size_nm, photons_per_blink,
                            camera: CameraParams | None, seed, bucket_index=None, drift_x_px=None, drift_y_px=None,
                            global_z_offset_um=None, bg_scale=None, use_illum=False, min_photons=0.0,
                            want_photons=False, adu_out=None, photons_out=None):
        """render_events enqueued in I/O slot io_slot (iscu_render_events_async): returns at once; the batch's arrays
        are held until render_events_wait(io_slot), which returns what render_events returns. With page-locked host
        buffers the copies of one slot's batch run beside the render of another's."""
        batch = self._event_batch(events, bucket_start, camera, bucket_index, drift_x_px, drift_y_px,
                                  global_z_offset_um, bg_scale, want_photons, adu_out, photons_out)
        events, bs, nf, bi, pf, cam, ph, adu = batch
        check(self.lib.iscu_render_events_async(self.h, int(io_slot), int(slot), _ptr(events), len(events), _ptr(bi),
                                                _ptr(bs), int(frame0), nf, float(pixel_size_nm),
                                                float(photons_per_blink), *[_ptr(a) for a in pf],
                                                int(bool(use_illum)), float(min_photons),
                                                C.byref(cam) if cam is not None else None, int(seed), _ptr(ph),
                                                _ptr(adu)))
        self._pending_io[int(io_slot)] = batch   # held only once enqueued: a refused call leaves the slot's batch be

    def render_events_wait(self, io_slot):
        """Waits for the batch of I/O slot io_slot: (photons | None, adu | None, n_emitters)."""
        n = C.c_uint32()
        check(self.lib.iscu_render_events_wait(self.h, int(io_slot), C.byref(n), None))
        batch = self._pending_io.pop(int(io_slot), None)
        ph, adu = (batch[6], batch[7]) if batch is not None else (None, None)
        return ph, adu, n.value

    # -------------------------------------------------------------------------------------------- blink schedules
    @staticmethod
    def _kinetics(k) -> _abi.Kinetics:
        """A Kinetics struct from a dict / sequence (activation rate, on, off, bleach probability, photon CV, initial
        on)."""
        names = ("activation_rate_per_sec", "on_sec", "off_sec", "bleach_prob", "photon_cv", "initial_on_sec")
        vals = [k[n] for n in names] if isinstance(k, dict) else list(k)
        return _abi.Kinetics(*[float(v) for v in vals])

    def dye_blinks_dev(self, mode, kinetics, dyes_dev, n_dyes, t0, t1, rows_dev, n_rows_dev, history=None,
                       dye_first_dev=None, sync=True):
        """iscu_dye_blinks_dev: each dye's blinks overlapping [t0, t1) as the world core schedules them. dyes_dev: a
        uint8 CUDA view of DYE_DTYPE records; rows_dev: float64 CUDA (max rows, EVENT_STRIDE); n_rows_dev: 1 int32;
        history: (t_start sequence, kinetics sequence) or None."""
        label = _abi.Label(int(mode), 0, self._kinetics(kinetics))
        starts = kin = None
        n_seg = 0
        if history is not None:
            st, ks = history
            n_seg = len(st)
            starts = np.ascontiguousarray(st, np.float64)
            kin = (_abi.Kinetics * n_seg)(*[self._kinetics(k) for k in ks])
        max_rows = 0 if rows_dev is None else rows_dev.numel() // EVENT_STRIDE
        self._before(sync)
        check(self.lib.iscu_dye_blinks_dev(self.h, C.byref(label), _ptr(starts), kin, n_seg, _ptr(dyes_dev),
                                           int(n_dyes), float(t0), float(t1), _ptr(rows_dev), max_rows,
                                           _ptr(dye_first_dev), _ptr(n_rows_dev)))
        self._after(sync)

    def dye_blinks(self, mode, kinetics, dyes, t0, t1, history=None):
        """Host form: dyes (DYE_DTYPE) -> (rows (m, EVENT_STRIDE) float64, first (n + 1,) per dye's first row)."""
        import torch
        dyes = np.ascontiguousarray(dyes, dtype=DYE_DTYPE)
        dev = f"cuda:{self.device}"
        d_dyes = torch.from_numpy(dyes.view(np.uint8)).to(dev)
        d_n = torch.zeros(1, dtype=torch.int32, device=dev)
        d_first = torch.zeros(len(dyes) + 1, dtype=torch.int32, device=dev)
        self.dye_blinks_dev(mode, kinetics, d_dyes, len(dyes), t0, t1, None, d_n, history, d_first)
        total = int(d_n.item())
        rows = torch.empty((max(total, 1), EVENT_STRIDE), dtype=torch.float64, device=dev)
        self.dye_blinks_dev(mode, kinetics, d_dyes, len(dyes), t0, t1, rows, d_n, history, d_first)
        return rows[:total].cpu().numpy(), d_first.cpu().numpy().astype(np.int64)

    RENDER_CONFIGS = 18

    def render_config(self):
        """(config, tile_w, tile_h, persistent, paired) of the render kernel form in use; paired 0 or 1: one pass with
        one or two emitters per step, 2: two passes."""
        v = [C.c_int32() for _ in range(5)]
        check(self.lib.iscu_render_get_config(self.h, *[C.byref(x) for x in v]))
        return v[0].value, v[1].value, v[2].value, bool(v[3].value), v[4].value

    def set_render_config(self, config):
        check(self.lib.iscu_render_set_config(self.h, int(config)))

    RENDER_PASSES = ("grouping", "contributions", "tiles")

    def set_render_timing(self, on):
        check(self.lib.iscu_render_set_timing(self.h, int(bool(on))))

    def render_pass_times(self):
        """Mean ms per render since set_render_timing(True): {grouping, contributions, tiles}, and the call count."""
        ms = (C.c_float * 3)()
        n = C.c_uint32()
        check(self.lib.iscu_render_pass_times(self.h, ms, C.byref(n)))
        return dict(zip(self.RENDER_PASSES, list(ms))), n.value

    def set_contrib_limit(self, nbytes):
        """The most device bytes the two-pass render forms' contributions may take (0: a quarter of the device)."""
        check(self.lib.iscu_render_set_contrib_limit(self.h, int(nbytes)))

    def render_autotune(self, emitters_dev, frames_dev, n_frames, camera: CameraParams, seed, adu_dev):
        """Times the render forms on this device batch, keeps the fastest; returns ms per render of each form."""
        ms = (C.c_float * self.RENDER_CONFIGS)()
        cam = camera.c()
        self._before(True)
        check(self.lib.iscu_render_autotune(self.h, _ptr(emitters_dev), _n_records(emitters_dev), _ptr(frames_dev),
                                            n_frames, C.byref(cam), seed, _ptr(adu_dev), ms))
        self._after(True)
        return list(ms)

    def render_gpu_records(self, records, frames, camera: CameraParams, seed, extras=None):
        """GpuSimulator::RenderFrames over the reference's 64-byte records (GPU_SPLAT_EMITTER_DTYPE)."""
        records = np.ascontiguousarray(records, dtype=GPU_SPLAT_EMITTER_DTYPE)
        frames = np.ascontiguousarray(frames, dtype=FRAME_DTYPE)
        n = len(frames)
        adu = np.empty((n, self.height, self.width), np.uint16)
        ex = _f32(extras, n * self.width * self.height) if extras is not None else None
        cam = camera.c()
        check(self.lib.iscu_render_gpu_records(self.h, _ptr(records), len(records), _ptr(frames), n, _ptr(ex),
                                               C.byref(cam), seed, _ptr(adu)))
        return adu

    def collect_frame_emitters(self, slot, events, frame, width, height, pixel_size_nm, photons_per_blink,
                               drift_x_px=0.0, drift_y_px=0.0, global_z_offset_um=0.0, illum=None, min_photons=0.0):
        """CollectFrameEmitters (SMLMSimulation.cpp:55-101) -> EMITTER_DTYPE records of one frame."""
        events = np.ascontiguousarray(events, dtype=BLINK_EVENT_DTYPE)
        out = np.empty(len(events), EMITTER_DTYPE)
        n = C.c_uint32()
        clamped = C.c_int64(0)
        il = _f32(illum, width * height) if illum is not None else None
        check(self.lib.iscu_collect_frame_emitters(self.h, slot, _ptr(events), len(events), int(frame), width, height,
                                                   pixel_size_nm, photons_per_blink, drift_x_px, drift_y_px,
                                                   global_z_offset_um, _ptr(il), min_photons, _ptr(out), len(out),
                                                   C.byref(n), C.byref(clamped)))
        return out[: n.value].copy(), clamped.value

    def collect_emitters(self, slot, events, bucket_start, frame0, width, height, pixel_size_nm, photons_per_blink,
                         bucket_index=None, drift_x_px=None, drift_y_px=None, global_z_offset_um=None, bg_scale=None,
                         illum=None, min_photons=0.0, max_out=None, out=None, frames_out=None):
        """A batch's emitters and frame table (iscu_collect_emitters). Returns (emitters, frames, n_clamped)."""
        events = np.ascontiguousarray(events, dtype=BLINK_EVENT_DTYPE)
        bs = np.ascontiguousarray(bucket_start, dtype=np.uint32)
        nf = len(bs) - 1
        bi = None if bucket_index is None else np.ascontiguousarray(bucket_index, dtype=np.uint32)
        if out is None:
            out = np.empty(max_out if max_out is not None else max(1, int(bs[-1] - bs[0])), EMITTER_DTYPE)
        if frames_out is None:
            frames_out = np.empty(nf, FRAME_DTYPE)
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        dx, dy, gz, sc = f64(drift_x_px), f64(drift_y_px), f64(global_z_offset_um), f64(bg_scale)
        il = _f32(illum, width * height) if illum is not None else None
        n = C.c_uint32()
        clamped = C.c_int64(0)
        check(self.lib.iscu_collect_emitters(self.h, slot, _ptr(events), _ptr(bi), _ptr(bs), int(frame0), nf, width,
                                             height, pixel_size_nm, photons_per_blink, _ptr(dx), _ptr(dy), _ptr(gz),
                                             _ptr(sc), _ptr(il), min_photons, _ptr(out), len(out), _ptr(frames_out),
                                             C.byref(n), C.byref(clamped)))
        return out[: n.value], frames_out, clamped.value


class RenderGraph:
    """iscu_render_graph: one device batch's render captured into a CUDA graph; launch() replays it on the engine's
    stream (refill the same device buffers in place between launches)."""

    def __init__(self, engine: Engine, emitters_dev, frames_dev, n_frames, camera: CameraParams | None, seed,
                 photons_dev=None, adu_dev=None):
        self.engine = engine
        self.lib = engine.lib
        self._keep = (emitters_dev, frames_dev, photons_dev, adu_dev)
        cam = camera.c() if camera is not None else None
        h = C.c_void_p()
        engine._before(True)
        check(self.lib.iscu_render_graph_create(engine.h, _ptr(emitters_dev), _n_records(emitters_dev),
                                                _ptr(frames_dev), n_frames,
                                                C.byref(cam) if cam is not None else None, seed, _ptr(photons_dev),
                                                _ptr(adu_dev), C.byref(h)))
        self.h = h
        engine._plans.add(self)

    def launch(self, sync=True):
        self.engine._before(sync)
        check(self.lib.iscu_render_graph_launch(self.h))
        self.engine._after(sync)

    def close(self):
        if self.h:
            if self.engine.h:
                self.lib.iscu_render_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PsfPlan:
    """iscu_psf_plan: the per-set PSF work done once; runs over (set index, defocus nm) lists. method as for
    Engine.psf_library_dev."""

    def __init__(self, engine: Engine, sets, size=0, method=CZT_FP32):
        self.engine = engine
        self.lib = engine.lib
        reqs = (PsfRequest * len(sets))(*[s.c() for s in sets])
        h = C.c_void_p()
        check(self.lib.iscu_psf_plan_create(engine.h, reqs, len(sets), size, method, C.byref(h)))
        self.h = h
        P, M = C.c_int32(), C.c_int32()
        check(self.lib.iscu_psf_plan_info(h, C.byref(P), C.byref(M)))
        self.P, self.M = P.value, M.value
        engine._plans.add(self)

    def close(self):
        if self.h:
            if self.engine.h:
                self.lib.iscu_psf_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_dev(self, set_of_dev, defocus_nm_dev, out_dev, normalize=True, sync=True):
        """set_of_dev: int32/uint32 CUDA tensor, defocus_nm_dev: float64 CUDA tensor, out_dev: (n, P, P) float32."""
        import torch
        n = int(set_of_dev.numel())
        dev = self.engine.device
        _require_tensor(set_of_dev, "set_of_dev", (torch.int32, torch.uint32), dev, n)
        _require_tensor(defocus_nm_dev, "defocus_nm_dev", (torch.float64,), dev, n)
        _require_tensor(out_dev, "out_dev", (torch.float32,), dev, n * self.P * self.P)
        self.engine._before(sync)
        check(self.lib.iscu_psf_plan_run_dev(self.h, _ptr(set_of_dev), _ptr(defocus_nm_dev), n, int(normalize),
                                             _ptr(out_dev)))
        if sync:
            check(self.lib.iscu_psf_plan_check(self.h))
        return out_dev

    def check(self):
        check(self.lib.iscu_psf_plan_check(self.h))

    def run(self, set_of, defocus_nm, normalize=True, out=None):
        so = np.ascontiguousarray(set_of, dtype=np.uint32)
        dz = np.ascontiguousarray(defocus_nm, dtype=np.float64)
        if len(dz) != len(so):
            raise ValueError(f"defocus_nm has {len(dz)} entries, set_of {len(so)}")
        if out is None:
            out = np.empty((len(so), self.P, self.P), np.float32)
        _require_array(out, "out", np.float32, len(so) * self.P * self.P)
        check(self.lib.iscu_psf_plan_run(self.h, _ptr(so), _ptr(dz), len(so), int(normalize), _ptr(out)))
        return out


class WidefieldPlan:
    """iscu_wf_plan: the focus series of a dye volume (nz, ny, nx) under a 3D PSF (kz, ky, kx), PSF spectrum resident."""

    def __init__(self, engine: Engine, shape, psf, _handle=None):
        self.engine = engine
        self.lib = engine.lib
        self.shape = tuple(int(v) for v in shape)   # (nz, ny, nx)
        nz, ny, nx = self.shape
        if _handle is None:
            psf = np.ascontiguousarray(psf, dtype=np.float32)
            kz, ky, kx = psf.shape
            h = C.c_void_p()
            check(self.lib.iscu_wf_plan_create(engine.h, nx, ny, nz, _ptr(psf), kx, ky, kz, C.byref(h)))
            _handle = h
        self.h = _handle
        w, hh, r = C.c_uint32(), C.c_uint32(), C.c_int32()
        check(self.lib.iscu_wf_plan_frame(self.h, C.byref(w), C.byref(hh), C.byref(r)))
        self.frame_shape = (nz, hh.value, w.value)   # the frames every render writes
        self.kernel_radius = r.value
        self._pending_io = {}   # I/O slot -> the host arrays of its enqueued render
        engine._plans.add(self)

    @classmethod
    def from_kernel(cls, engine: Engine, slot, upscale, pixel_um, kernel_cap_um, plane_nm, shape, fov):
        """The reference's widefield scene over kernel slot `slot` (iscu_wf_plan_from_kernel): a dye grid of shape
        (nz, ny, nx) cells at pixel_um / upscale, planes plane_nm thick, imaged at every plane's centre; frames are the
        camera window fov = (x0, y0, width, height) (cells x0, y0; width x height camera pixels of upscale^2 cells)."""
        nz, ny, nx = (int(v) for v in shape)
        x0, y0, w, h = (int(v) for v in fov)
        hd = C.c_void_p()
        check(engine.lib.iscu_wf_plan_from_kernel(engine.h, int(slot), int(upscale), float(pixel_um),
                                                  float(kernel_cap_um), float(plane_nm), nx, ny, nz, x0, y0, w, h,
                                                  C.byref(hd)))
        return cls(engine, (nz, ny, nx), None, _handle=hd)

    def close(self):
        if self.h:
            if self.engine.h:   # the context is still alive (Engine.close destroys its plans first)
                self.lib.iscu_wf_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grid(self):
        g = [C.c_uint32() for _ in range(3)]
        check(self.lib.iscu_wf_plan_grid(self.h, *[C.byref(x) for x in g]))
        return tuple(x.value for x in g)

    def set_timing(self, on=True):
        check(self.lib.iscu_wf_set_timing(self.h, int(on)))

    def pass_times(self):
        """The last render's pass durations (ms): x forward, y forward, z convolve, y inverse, x inverse, camera noise
        (0 without a camera)."""
        ms = (C.c_float * 6)()
        check(self.lib.iscu_wf_pass_times(self.h, ms))
        return list(ms)

    def convolve_dev(self, density_dev, image_dev=None, sync=True):
        import torch
        if image_dev is None:
            image_dev = torch.empty(self.frame_shape, dtype=torch.float32, device=density_dev.device)
        self.engine._before(sync)
        check(self.lib.iscu_wf_convolve_dev(self.h, _ptr(density_dev), _ptr(image_dev)))
        self.engine._after(sync)
        return image_dev

    def render_dev(self, density_dev, background, camera: CameraParams | None, seed, frame0=0, image_dev=None,
                   adu_dev=None, sync=True):
        cam = camera.c() if camera is not None else None
        self.engine._before(sync)
        check(self.lib.iscu_wf_render_dev(self.h, _ptr(density_dev), float(background),
                                          C.byref(cam) if cam is not None else None, seed, frame0, _ptr(image_dev),
                                          _ptr(adu_dev)))
        self.engine._after(sync)

    def render(self, density, background, camera: CameraParams | None, seed, frame0=0, want_image=False, adu=None,
               image=None):
        """Host path: density (nz, ny, nx) float32 -> (image | None, adu | None)."""
        density = np.ascontiguousarray(density, dtype=np.float32)
        if want_image and image is None:
            image = np.empty(self.frame_shape, np.float32)
        if camera is not None and adu is None:
            adu = np.empty(self.frame_shape, np.uint16)
        cam = camera.c() if camera is not None else None
        check(self.lib.iscu_wf_render(self.h, _ptr(density), float(background),
                                      C.byref(cam) if cam is not None else None, seed, frame0,
                                      _ptr(image) if want_image else None, _ptr(adu) if cam is not None else None))
        return (image if want_image else None), (adu if camera is not None else None)

    def render_async(self, io_slot, density, background, camera: CameraParams | None, seed, frame0=0, adu=None,
                     image=None):
        """Enqueues render() in I/O slot io_slot (0..3) and returns at once (iscu_wf_render_async): the volume's
        upload, the passes and the frames' download run behind the calls before it. density, adu and image are
        caller-owned contiguous arrays (page-locked for the copies to overlap) that stay untouched until
        render_wait(io_slot)."""
        if density.dtype != np.float32 or not density.flags.c_contiguous or density.shape != self.shape:
            raise ValueError("density: a C-contiguous float32 array of the plan's shape")
        for name, arr, dt in (("adu", adu, np.uint16), ("image", image, np.float32)):
            if arr is not None and (arr.dtype != dt or not arr.flags.c_contiguous or arr.shape != self.frame_shape):
                raise ValueError(f"{name}: a C-contiguous {np.dtype(dt).name} array of the plan's frame shape")
        cam = camera.c() if camera is not None else None
        check(self.lib.iscu_wf_render_async(self.h, int(io_slot), _ptr(density), float(background),
                                            C.byref(cam) if cam is not None else None, seed, frame0,
                                            _ptr(image) if image is not None else None,
                                            _ptr(adu) if adu is not None else None))
        self._pending_io[int(io_slot)] = (density, adu, image)   # held only once enqueued

    def render_wait(self, io_slot):
        """Waits for I/O slot io_slot's frames (iscu_wf_render_wait)."""
        check(self.lib.iscu_wf_render_wait(self.h, int(io_slot)))
        self._pending_io.pop(int(io_slot), None)


class WidefieldJob:
    """iscu_wf_job: the GPU side of a widefield scene's focus work (sim::WidefieldAccelerator) -- plane spectra
    resident by key, kernel spectra by plane index, within one geometry value."""

    def __init__(self, engine: Engine, budget_bytes=0):
        self.engine = engine
        self.lib = engine.lib
        h = C.c_void_p()
        check(self.lib.iscu_wf_job_create(engine.h, int(budget_bytes), C.byref(h)))
        self.h = h
        engine._plans.add(self)

    def close(self):
        if self.h:
            if self.engine.h:
                self.lib.iscu_wf_job_destroy(self.h)
            self.h = None

    def has_plane(self, geometry, key):
        return self.lib.iscu_wf_job_has_plane(self.h, int(geometry), int(key)) == 1

    def fits(self, geometry, nx_fft, ny_fft, planes):
        return self.lib.iscu_wf_job_fits(self.h, int(geometry), nx_fft, ny_fft, int(planes)) == 1

    def images(self, nx_fft, ny_fft, grid, fov, frac, geometry, kernels, planes, channels):
        """kernels: {p: complex64 (ny_fft, nx_fft/2 + 1) spectrum, RealFft2d's = numpy rfft2's layout}; planes: {key:
        (cells uint32, values float32)} (cells row-major in the nx x ny grid); channels: lists of deps (key, p0, p1,
        w0, w1) with p1 None for one kernel. Returns (n_channels, ch, cw) float32 images."""
        from ._abi import WfJobDep, WfJobDesc, WfJobKernel, WfJobPlane
        nx, ny = grid
        x0, y0, cw, ch = fov
        keep = []
        ks = (WfJobKernel * max(1, len(kernels)))()
        for i, (p, spec) in enumerate(kernels.items()):
            a = np.ascontiguousarray(spec, np.complex64)
            keep.append(a)
            ks[i].p, ks[i].spec = int(p), a.ctypes.data
        ps = (WfJobPlane * max(1, len(planes)))()
        for i, (key, (cells, values)) in enumerate(planes.items()):
            c_ = np.ascontiguousarray(cells, np.uint32)
            v_ = np.ascontiguousarray(values, np.float32)
            keep += [c_, v_]
            ps[i].key, ps[i].cells, ps[i].values, ps[i].count = int(key), c_.ctypes.data, v_.ctypes.data, len(c_)
        flat = [d for ch_ in channels for d in ch_]
        ds = (WfJobDep * max(1, len(flat)))()
        for i, (key, p0, p1, w0, w1) in enumerate(flat):
            ds[i].key, ds[i].p0, ds[i].w0 = int(key), int(p0), float(w0)
            two = p1 is not None
            ds[i].p1, ds[i].w1, ds[i].two = (int(p1) if two else int(p0)), (float(w1) if two else 0.0), int(two)
        start = np.concatenate([[0], np.cumsum([len(c_) for c_ in channels])]).astype(np.uint32)
        d = WfJobDesc(nx_fft=nx_fft, ny_fft=ny_fft, nx=nx, ny=ny, fov_x0=x0, fov_y0=y0, cw=cw, ch=ch,
                      frac_x=float(frac[0]), frac_y=float(frac[1]), geometry=int(geometry), kernels=C.cast(ks, C.c_void_p),
                      n_kernels=len(kernels), n_planes=len(planes), planes=C.cast(ps, C.c_void_p),
                      deps=C.cast(ds, C.c_void_p), channel_start=start.ctypes.data, n_channels=len(channels))
        out = np.zeros((len(channels), ch, cw), np.float32)
        ptrs = (C.c_void_p * max(1, len(channels)))(*[out[c].ctypes.data for c in range(len(channels))])
        check(self.lib.iscu_wf_job_images(self.h, C.byref(d), ptrs))
        return out


class WidefieldShift:
    """iscu_wf_shift: frames of a drifting widefield sample from its channels' spectra on an nx x ny grid
    (RenderShiftedImages)."""

    def __init__(self, engine: Engine, nx, ny):
        self.engine = engine
        self.lib = engine.lib
        self.nx, self.ny = int(nx), int(ny)
        h = C.c_void_p()
        check(self.lib.iscu_wf_shift_create(engine.h, self.nx, self.ny, C.byref(h)))
        self.h = h
        engine._plans.add(self)

    def frames_dev(self, spectra_dev, coef_dev, shift_dev, window, up, cam_dev, scale=1.0, sync=True):
        """cam_dev (n_frames, ch/up, cw/up) float32 CUDA += the frames (iscu_wf_shifted_frames_dev): spectra_dev
        complex64 (n_ch, ny, nx/2 + 1), coef_dev float32 (n_frames, n_ch), shift_dev float64 (n_frames, 2)."""
        x0, y0, cw, ch = window
        n_ch = spectra_dev.shape[0]
        n_frames = coef_dev.shape[0]
        self.engine._before(sync)
        check(self.lib.iscu_wf_shifted_frames_dev(self.h, _ptr(spectra_dev.contiguous()), n_ch,
                                                  _ptr(coef_dev.contiguous()), _ptr(shift_dev.contiguous()), n_frames,
                                                  x0, y0, cw, ch, up, float(scale), _ptr(cam_dev)))
        self.engine._after(sync)

    def close(self):
        if self.h:
            if self.engine.h:
                self.lib.iscu_wf_shift_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TiffWriter:
    """iscu_tiff: the CLI's movie file (cli/tiff_writer.h) byte for byte -- classic TIFF or BigTIFF, one uncompressed
    grey page per frame. Failures raise IscuError (code ISCU_ERR_IO) with the reference writer's message."""

    def __init__(self, path, expected_bytes=0, big=False):
        self.lib = load()
        self.h = None
        h = C.c_void_p()
        check(self.lib.iscu_tiff_open(str(path).encode(), int(expected_bytes), int(big), C.byref(h)))
        self.h = h

    @staticmethod
    def bytes(w, h, pages, bytes_per_sample, desc_bytes):
        """TiffWriter::Bytes: an upper bound of the file's size (the expected_bytes to pass)."""
        return int(load().iscu_tiff_bytes(w, h, pages, bytes_per_sample, desc_bytes))

    @staticmethod
    def _d(desc):
        return None if desc is None else desc.encode()

    def info(self):
        """(is a BigTIFF, pages, bytes)."""
        big, pages, n = C.c_int32(), C.c_uint64(), C.c_uint64()
        check(self.lib.iscu_tiff_info(self.h, C.byref(big), C.byref(pages), C.byref(n)))
        return bool(big.value), pages.value, n.value

    def page(self, px, desc=None):
        """One page of a (h, w) uint16 or float32 image."""
        px = np.ascontiguousarray(px)
        h, w = px.shape
        if px.dtype == np.float32:
            check(self.lib.iscu_tiff_page_f32(self.h, _ptr(px), w, h, self._d(desc)))
        else:
            px = np.ascontiguousarray(px, np.uint16)
            check(self.lib.iscu_tiff_page_u16(self.h, _ptr(px), w, h, self._d(desc)))

    def page_rows(self, px, w, h, desc=None):
        """A uint16 page of w x h of which px (rows, w) holds the first rows; rows() fills the rest."""
        px = np.ascontiguousarray(px, np.uint16)
        check(self.lib.iscu_tiff_page_rows(self.h, _ptr(px), px.shape[0], w, h, self._d(desc)))

    def rows(self, page, y0, px):
        px = np.ascontiguousarray(px, np.uint16)
        check(self.lib.iscu_tiff_rows(self.h, page, y0, px.shape[0], _ptr(px)))

    def pages_dev(self, engine: Engine, frames_dev, first_desc=None):
        """The (n, h, w) uint16 CUDA frames, one page each (iscu_tiff_pages_dev: copied out in chunks through two
        page-locked halves while the previous chunk is written)."""
        n, h, w = frames_dev.shape
        frames_dev = frames_dev.contiguous()
        check(self.lib.iscu_tiff_pages_dev(self.h, engine.h, _ptr(frames_dev), n, w, h, self._d(first_desc)))

    def close(self):
        if self.h:
            h, self.h = self.h, None
            check(self.lib.iscu_tiff_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            if self.h:
                self.lib.iscu_tiff_close(self.h)
                self.h = None
        except Exception:
            pass


class BinnedRenderer:
    """iscu_binned: the binned blink regime (sim::BinnedBlinkRenderer) for width x height frames, on kernel slot
    `slot` or (slot < 0) the in-focus Gaussian of sigma_px."""

    def __init__(self, engine: Engine, width, height, upscale, slot=-1, sigma_px=0.0):
        self.engine = engine
        self.lib = engine.lib
        self.width, self.height = int(width), int(height)
        h = C.c_void_p()
        check(self.lib.iscu_binned_create(engine.h, int(slot), float(sigma_px), self.width, self.height,
                                          int(upscale), C.byref(h)))
        self.h = h
        u, r, nz = C.c_int32(), C.c_int32(), C.c_int32()
        check(self.lib.iscu_binned_info(self.h, C.byref(u), C.byref(r), C.byref(nz)))
        self.upscale, self.radius, self.planes = u.value, r.value, nz.value
        engine._plans.add(self)

    def kernels(self):
        """The plane kernels at the cell pitch, (planes, 2R + 1, 2R + 1) float32."""
        D = 2 * self.radius + 1
        out = np.empty((self.planes, D, D), np.float32)
        check(self.lib.iscu_binned_kernels(self.h, _ptr(out)))
        return out

    def render_dev(self, emitters_dev, frames_dev, n_frames, img_dev, alone_dev=None, sync=True):
        """img_dev (n_frames, h, w) float32 CUDA += the frames' binned blink images (iscu_binned_render_dev);
        emitters / frames as Engine.render_frames_dev."""
        self.engine._before(sync)
        check(self.lib.iscu_binned_render_dev(self.h, _ptr(emitters_dev), _n_records(emitters_dev), _ptr(frames_dev),
                                              int(n_frames), _ptr(img_dev), _ptr(alone_dev)))
        self.engine._after(sync)

    def close(self):
        if self.h:
            if self.engine.h:
                self.lib.iscu_binned_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class DriftSettings:
    """sim::DriftSettings (Drift.h:57-79)."""
    xy_nm_per_sqrt_sec: float = 0.0
    z_nm_per_sqrt_sec: float = 0.0
    xy_speed_nm_per_sec: float = 0.0
    z_speed_nm_per_sec: float = 0.0
    xy_angle_deg: float = -1.0
    z_direction: int = 0
    angle_wander_deg: float = 180.0
    z_angle_wander_deg: float = 90.0
    speed_wander_pct: float = 0.0
    wander_time_sec: float = 60.0

    def c(self):
        from ._abi import DriftSettings as _D
        d = _D()
        for k in self.__dataclass_fields__:
            setattr(d, k, getattr(self, k))
        return d


def drift_trajectory(random_seed: int, frames: int, frame_sec: float, settings: DriftSettings) -> np.ndarray:
    """The sample drift (frames, 3) nm (DriftTrajectory, Drift.cpp:114-124): the reference's bits."""
    out = np.zeros((max(0, frames), 3), np.float64)
    s = settings.c()
    check(load().iscu_drift_trajectory(int(random_seed), int(frames), float(frame_sec), C.byref(s), _ptr(out)))
    return out


def illumination_field(width: int, height: int, profile: int, fwhm_pct: float):
    """(field (h, w) float32 with peak 1, or None for flat; mean factor) (BuildIlluminationField)."""
    out = np.empty((height, width), np.float32)
    mf = C.c_double()
    check(load().iscu_illumination_field(width, height, int(profile), float(fwhm_pct), _ptr(out), C.byref(mf)))
    return (None if profile == 0 else out), mf.value


def background_fade_scale(t: float, decay: float) -> float:
    return float(load().iscu_background_fade_scale(float(t), float(decay)))


def frames_table(counts, frame_ids=None, bg_scales=None):
    """A FRAME_DTYPE table for frames whose emitters are consecutive runs of `counts` records."""
    counts = np.asarray(counts, dtype=np.int64)
    t = np.zeros(len(counts), FRAME_DTYPE)
    t["em_count"] = counts
    t["em_start"] = np.concatenate([[0], np.cumsum(counts)[:-1]]) if len(counts) else []
    t["frame"] = np.arange(len(counts)) if frame_ids is None else frame_ids
    t["bg_scale"] = 1.0 if bg_scales is None else bg_scales
    return t


__all__ = ["Engine", "CameraParams", "PsfParams", "IscuError", "generate_camera_maps", "frames_table",
           "EMITTER_DTYPE", "FRAME_DTYPE", "GPU_SPLAT_EMITTER_DTYPE", "BLINK_EVENT_DTYPE", "CZT_FP32", "CZT_TF32X3", "CZT_F16X3",
           "INTERP_NEAREST", "INTERP_LINEAR", "INTERP_CUBIC"]
