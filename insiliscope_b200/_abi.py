"""ctypes declarations of include/iscu.h (libiscu.so).

Loading fails loudly when the library is missing: there is no CPU fallback in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libiscu.so")

ISCU_OK = 0
ISCU_ERR_ARG = 1
ISCU_ERR_CUDA = 2
ISCU_ERR_STATE = 3
ISCU_ERR_LIMIT = 4
ISCU_ERR_TIMEOUT = 5
ISCU_ERR_NODEV = 6
ISCU_ERR_IO = 7

INTERP_NEAREST, INTERP_LINEAR, INTERP_CUBIC = 0, 1, 2
CZT_FP32, CZT_TF32X3, CZT_F16X3 = 0, 1, 2
MAX_KERNELS = 4

u8p = C.POINTER(C.c_uint8)
u16p = C.POINTER(C.c_uint16)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p


class Camera(C.Structure):
    _fields_ = [
        ("quantum_efficiency", C.c_double),
        ("dark_electrons", C.c_double),
        ("gain", C.c_double),
        ("read_noise_e", C.c_double),
        ("emccd", C.c_int32),
        ("bit_depth", C.c_int32),
        ("em_gain", C.c_double),
        ("cic_electrons", C.c_double),
    ]


class WfJobKernel(C.Structure):
    _fields_ = [("p", C.c_int32), ("reserved", C.c_int32), ("spec", C.c_void_p)]


class WfJobPlane(C.Structure):
    _fields_ = [("key", C.c_uint64), ("cells", C.c_void_p), ("values", C.c_void_p), ("count", C.c_uint32),
                ("reserved", C.c_uint32)]


class WfJobDep(C.Structure):
    _fields_ = [("key", C.c_uint64), ("p0", C.c_int32), ("p1", C.c_int32), ("w0", C.c_float), ("w1", C.c_float),
                ("two", C.c_int32), ("reserved", C.c_int32)]


class WfJobDesc(C.Structure):
    _fields_ = [("nx_fft", C.c_uint32), ("ny_fft", C.c_uint32), ("nx", C.c_uint32), ("ny", C.c_uint32),
                ("fov_x0", C.c_uint32), ("fov_y0", C.c_uint32), ("cw", C.c_uint32), ("ch", C.c_uint32),
                ("frac_x", C.c_double), ("frac_y", C.c_double), ("geometry", C.c_uint64),
                ("kernels", C.c_void_p), ("n_kernels", C.c_uint32), ("n_planes", C.c_uint32),
                ("planes", C.c_void_p), ("deps", C.c_void_p), ("channel_start", C.c_void_p),
                ("n_channels", C.c_uint32), ("reserved", C.c_uint32)]


class PsfRequest(C.Structure):
    _fields_ = [
        ("wavelength_nm", C.c_double),
        ("na", C.c_double),
        ("immersion_index", C.c_double),
        ("sample_index", C.c_double),
        ("working_distance_um", C.c_double),
        ("sample_depth_nm", C.c_double),
        ("pixel_size_nm", C.c_double),
        ("zernike", C.c_double * 28),
        ("mask_double_helix", C.c_int32),
        ("mask_modes", C.c_int32),
        ("mask_waist", C.c_double),
        ("oversampling", C.c_int32),
        ("kernel_half_width_px", C.c_int32),
        ("nz", C.c_int32),
        ("pupil_samples", C.c_int32),
        ("z_step_nm", C.c_double),
        ("interp", C.c_int32),
        ("reserved", C.c_int32),
    ]


class Emitter(C.Structure):
    _fields_ = [("x_px", C.c_double), ("y_px", C.c_double), ("photons", C.c_double), ("plane", C.c_int32),
                ("reserved", C.c_int32)]


class GpuSplatEmitter(C.Structure):
    _fields_ = [("x0", C.c_int32), ("y0", C.c_int32), ("bx", C.c_int32), ("by", C.c_int32), ("plane", C.c_int32),
                ("n_taps", C.c_int32), ("photons", C.c_float), ("cut_radius2", C.c_int32),
                ("wx", C.c_float * 4), ("wy", C.c_float * 4)]


class Frame(C.Structure):
    _fields_ = [("em_start", C.c_uint32), ("em_count", C.c_uint32), ("frame", C.c_uint32), ("reserved", C.c_uint32),
                ("bg_scale", C.c_double)]


class BlinkEvent(C.Structure):
    _fields_ = [("x_um", C.c_double), ("y_um", C.c_double), ("z_nm", C.c_double), ("t_start", C.c_double),
                ("t_end", C.c_double), ("brightness", C.c_double), ("excite", C.c_double),
                ("slot", C.c_int32), ("reserved", C.c_int32)]


# name -> (restype, argtypes); every function include/iscu.h declares.
class DriftSettings(C.Structure):
    _fields_ = [("xy_nm_per_sqrt_sec", C.c_double), ("z_nm_per_sqrt_sec", C.c_double),
                ("xy_speed_nm_per_sec", C.c_double), ("z_speed_nm_per_sec", C.c_double),
                ("xy_angle_deg", C.c_double), ("z_direction", C.c_int32), ("reserved", C.c_int32),
                ("angle_wander_deg", C.c_double), ("z_angle_wander_deg", C.c_double),
                ("speed_wander_pct", C.c_double), ("wander_time_sec", C.c_double)]


class Kinetics(C.Structure):
    _fields_ = [("activation_rate_per_sec", C.c_double), ("on_sec", C.c_double), ("off_sec", C.c_double),
                ("bleach_prob", C.c_double), ("photon_cv", C.c_double), ("initial_on_sec", C.c_double)]


class Label(C.Structure):
    _fields_ = [("mode", C.c_int32), ("reserved", C.c_int32), ("kin", Kinetics)]


class NllSpec(C.Structure):
    _fields_ = [("wavelength_nm", C.c_double), ("na", C.c_double), ("n_imm", C.c_double), ("pixel_nm", C.c_double),
                ("roi", C.c_int32), ("os", C.c_int32), ("pupil", C.c_int32), ("n_zern", C.c_int32),
                ("noll", C.c_int32 * 32)]


SIGNATURES = {
    "iscu_last_error": (C.c_char_p, []),
    "iscu_abi_version": (C.c_int, []),
    "iscu_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "iscu_destroy": (None, [vp]),
    "iscu_synchronize": (C.c_int, [vp]),
    "iscu_stream": (vp, [vp]),
    "iscu_launch_count": (C.c_uint64, [vp]),
    "iscu_pcg4d_dev": (C.c_int, [vp, vp, vp, C.c_size_t]),
    "iscu_counter_uniforms_dev": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp]),
    "iscu_set_static": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp, vp, vp, C.c_double]),
    "iscu_generate_camera_maps": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                            C.c_double, C.c_double, C.c_double, C.c_uint32, C.c_uint32, vp, vp,
                                            vp]),
    "iscu_noise_frames_dev": (C.c_int, [vp, vp, C.c_uint32, vp, C.POINTER(Camera), C.c_uint32, vp]),
    "iscu_psf_geometry": (C.c_int, [C.POINTER(PsfRequest), i32p, i32p, i32p]),
    "iscu_psf_library_dev": (C.c_int, [vp, C.POINTER(PsfRequest), C.c_uint32, vp, vp, C.c_uint32, C.c_int32,
                                       C.c_int32, C.c_int32, vp]),
    "iscu_psf_library_noalloc_dev": (C.c_int, [vp, C.POINTER(PsfRequest), C.c_uint32, vp, vp, C.c_uint32,
                                               C.c_int32, C.c_int32, vp]),
    "iscu_psf_plan_create": (C.c_int, [vp, C.POINTER(PsfRequest), C.c_uint32, C.c_int32, C.c_int32,
                                       C.POINTER(vp)]),
    "iscu_psf_plan_destroy": (None, [vp]),
    "iscu_psf_plan_info": (C.c_int, [vp, i32p, i32p]),
    "iscu_psf_plan_run_dev": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_int32, vp]),
    "iscu_psf_plan_check": (C.c_int, [vp]),
    "iscu_psf_plan_run": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_int32, vp]),
    "iscu_kernel_build": (C.c_int, [vp, C.c_int32, C.POINTER(PsfRequest), C.c_int32]),
    "iscu_kernel_set_planes": (C.c_int, [vp, C.c_int32, vp, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                         C.c_int32]),
    "iscu_kernel_set_halo": (C.c_int, [vp, C.c_int32, C.c_double]),
    "iscu_kernel_get_halo": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
    "iscu_kernel_info": (C.c_int, [vp, C.c_int32, i32p, i32p, i32p, i32p]),
    "iscu_kernel_get_planes": (C.c_int, [vp, C.c_int32, vp]),
    "iscu_kernel_get_block_sums": (C.c_int, [vp, C.c_int32, vp]),
    "iscu_render_frames_dev": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(Camera), C.c_uint32, vp,
                                         vp]),
    "iscu_render_frames": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(Camera), C.c_uint32, vp, vp]),
    "iscu_collect_emitters_dev": (C.c_int, [vp, C.c_int32, vp, C.c_uint32, vp, vp, C.c_int64, C.c_uint32,
                                            C.c_double, C.c_double, vp, vp, vp, vp, vp, C.c_double, vp, vp,
                                            C.c_uint32, vp, vp, vp]),
    "iscu_render_events": (C.c_int, [vp, C.c_int32, vp, C.c_uint32, vp, vp, C.c_int64, C.c_uint32, C.c_double,
                                     C.c_double, vp, vp, vp, vp, C.c_int32, C.c_double, C.POINTER(Camera),
                                     C.c_uint32, vp, vp, vp, vp]),
    "iscu_render_events_async": (C.c_int, [vp, C.c_int32, C.c_int32, vp, C.c_uint32, vp, vp, C.c_int64, C.c_uint32,
                                           C.c_double, C.c_double, vp, vp, vp, vp, C.c_int32, C.c_double,
                                           C.POINTER(Camera), C.c_uint32, vp, vp]),
    "iscu_render_events_wait": (C.c_int, [vp, C.c_int32, u32p, C.POINTER(C.c_int64)]),
    "iscu_buffer_create": (C.c_int, [vp, C.c_size_t, vp, C.POINTER(vp)]),
    "iscu_buffer_destroy": (None, [vp]),
    "iscu_buffer_bytes": (C.c_size_t, [vp]),
    "iscu_buffer_write": (C.c_int, [vp, C.c_size_t, vp, C.c_size_t]),
    "iscu_buffer_copy": (C.c_int, [vp, vp, C.c_size_t]),
    "iscu_buffer_read": (C.c_int, [vp, C.c_size_t, vp]),
    "iscu_buffer_read_low16": (C.c_int, [vp, C.c_size_t, vp]),
    "iscu_dispatch": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, vp, C.c_size_t, C.c_uint32, C.c_uint32,
                                C.c_uint32]),
    "iscu_fft_place_dev": (C.c_int, [vp, C.c_int32, vp, C.c_uint32, vp, vp]),
    "iscu_render_fft_frames_dev": (C.c_int, [vp, C.c_int32, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(Camera), C.c_uint32,
                                             vp, vp]),
    "iscu_csv_numbers_dev": (C.c_int, [vp, vp, C.c_uint32, C.c_char_p, vp, vp]),
    "iscu_csv_table_dev": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, vp, vp, C.c_uint64, vp]),
    "iscu_tiff_bytes": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]),
    "iscu_tiff_open": (C.c_int, [C.c_char_p, C.c_uint64, C.c_int32, vp]),
    "iscu_tiff_info": (C.c_int, [vp, vp, vp, vp]),
    "iscu_tiff_page_u16": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_char_p]),
    "iscu_tiff_page_f32": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_char_p]),
    "iscu_tiff_page_rows": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_char_p]),
    "iscu_tiff_rows": (C.c_int, [vp, C.c_uint64, C.c_uint32, C.c_uint32, vp]),
    "iscu_tiff_pages_dev": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_char_p]),
    "iscu_tiff_close": (C.c_int, [vp]),
    "iscu_binned_create": (C.c_int, [vp, C.c_int32, C.c_double, C.c_uint32, C.c_uint32, C.c_int32, vp]),
    "iscu_binned_info": (C.c_int, [vp, vp, vp, vp]),
    "iscu_binned_kernels": (C.c_int, [vp, vp]),
    "iscu_binned_destroy": (None, [vp]),
    "iscu_binned_render_dev": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, vp, vp]),
    "iscu_dye_blinks_dev": (C.c_int, [vp, vp, vp, vp, C.c_uint32, vp, C.c_uint32, C.c_double, C.c_double, vp,
                                      C.c_uint32, vp, vp]),
    "iscu_drift_trajectory": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.POINTER(DriftSettings), vp]),
    "iscu_illumination_field": (C.c_int, [C.c_uint32, C.c_uint32, C.c_int32, C.c_double, vp, f64p]),
    "iscu_background_fade_scale": (C.c_double, [C.c_double, C.c_double]),
    "iscu_nll_model_create": (C.c_int, [vp, C.POINTER(NllSpec), C.POINTER(vp)]),
    "iscu_nll_model_destroy": (None, [vp]),
    "iscu_nll_model_info": (C.c_int, [vp, f64p, i32p]),
    "iscu_nll_eval_dev": (C.c_int, [vp, C.c_uint32, vp, vp, C.c_uint32, vp, f64p, vp, vp, vp, vp, vp, vp, vp]),
    "iscu_render_set_config": (C.c_int, [vp, C.c_int32]),
    "iscu_render_set_timing": (C.c_int, [vp, C.c_int32]),
    "iscu_render_pass_times": (C.c_int, [vp, f32p, u32p]),
    "iscu_render_set_contrib_limit": (C.c_int, [vp, C.c_uint64]),
    "iscu_render_get_config": (C.c_int, [vp, i32p, i32p, i32p, i32p, i32p]),
    "iscu_render_autotune": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(Camera), C.c_uint32, vp,
                                       f32p]),
    "iscu_render_graph_create": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(Camera), C.c_uint32, vp,
                                           vp, C.POINTER(vp)]),
    "iscu_render_graph_launch": (C.c_int, [vp]),
    "iscu_render_graph_destroy": (None, [vp]),
    "iscu_render_gpu_records": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.POINTER(Camera), C.c_uint32,
                                          vp]),
    "iscu_collect_frame_emitters": (C.c_int, [vp, C.c_int32, vp, C.c_uint32, C.c_int64, C.c_uint32, C.c_uint32,
                                              C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, vp,
                                              C.c_double, vp, C.c_uint32, u32p, i64p]),
    "iscu_wf_plan_create": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint32, C.c_uint32,
                                      C.c_uint32, C.POINTER(vp)]),
    "iscu_wf_plan_destroy": (None, [vp]),
    "iscu_wf_plan_from_kernel": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint32,
                                           C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                           C.POINTER(vp)]),
    "iscu_wf_job_create": (C.c_int, [vp, C.c_uint64, C.POINTER(vp)]),
    "iscu_wf_job_destroy": (None, [vp]),
    "iscu_wf_job_has_plane": (C.c_int, [vp, C.c_uint64, C.c_uint64]),
    "iscu_wf_job_fits": (C.c_int, [vp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64]),
    "iscu_wf_job_images": (C.c_int, [vp, vp, vp]),
    "iscu_wf_plan_frame": (C.c_int, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]),
    "iscu_wf_plan_grid": (C.c_int, [vp, u32p, u32p, u32p]),
    "iscu_wf_convolve_dev": (C.c_int, [vp, vp, vp]),
    "iscu_wf_set_timing": (C.c_int, [vp, C.c_int32]),
    "iscu_wf_pass_times": (C.c_int, [vp, f32p]),
    "iscu_wf_render": (C.c_int, [vp, vp, C.c_double, C.POINTER(Camera), C.c_uint32, C.c_uint32, vp, vp]),
    "iscu_wf_shift_create": (C.c_int, [vp, C.c_uint32, C.c_uint32, vp]),
    "iscu_wf_shift_destroy": (None, [vp]),
    "iscu_wf_shifted_frames_dev": (C.c_int, [vp, vp, C.c_uint32, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32,
                                             C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, vp]),
    "iscu_wf_render_async": (C.c_int, [vp, C.c_int32, vp, C.c_double, C.POINTER(Camera), C.c_uint32, C.c_uint32,
                                       vp, vp]),
    "iscu_wf_render_wait": (C.c_int, [vp, C.c_int32]),
    "iscu_wf_render_dev": (C.c_int, [vp, vp, C.c_double, C.POINTER(Camera), C.c_uint32, C.c_uint32, vp, vp]),
    "iscu_collect_emitters": (C.c_int, [vp, C.c_int32, vp, vp, vp, C.c_int64, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.c_double, C.c_double, vp, vp, vp, vp, vp, C.c_double, vp, C.c_uint32, vp,
                                        u32p, i64p]),
}

_lib = None


def load() -> C.CDLL:
    """The loaded libiscu.so, with argtypes set. Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libiscu.so is not built ({LIB_PATH}); run insiliscope_b200.build.build_library()")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class IscuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"iscu error {code}: {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != ISCU_OK:
        raise IscuError(rc, load().iscu_last_error().decode())
