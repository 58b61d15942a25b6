"""insiliscope_b200: a B200-native (sm_100a) engine for inSiliScope's fluorescence image-formation path.

The compute lives in libiscu.so (CUDA kernels + C ABI, include/iscu.h); this package is its Python host side.
"""
from .engine import (BLINK_EVENT_DTYPE, CZT_FP32, CZT_TF32X3, CZT_F16X3, DYE_DTYPE, EMITTER_DTYPE, EVENT_STRIDE, FRAME_DTYPE,
                     GPU_SPLAT_EMITTER_DTYPE, INTERP_CUBIC, INTERP_LINEAR, INTERP_NEAREST, LABEL_DNA_PAINT,
                     LABEL_DSTORM, LABEL_PALM, LABEL_WIDEFIELD, BinnedRenderer, CameraParams, Engine, IscuError,
                     PsfParams, PsfPlan, RenderGraph, TiffWriter, WidefieldJob, WidefieldPlan, WidefieldShift, frames_table,
                     generate_camera_maps)

__all__ = ["Engine", "CameraParams", "PsfParams", "PsfPlan", "RenderGraph", "IscuError", "WidefieldPlan", "BinnedRenderer",
           "TiffWriter", "WidefieldShift", "WidefieldJob",
           "generate_camera_maps",
           "frames_table",
           "EMITTER_DTYPE", "FRAME_DTYPE", "GPU_SPLAT_EMITTER_DTYPE", "BLINK_EVENT_DTYPE", "CZT_FP32", "CZT_TF32X3", "CZT_F16X3",
           "INTERP_NEAREST", "INTERP_LINEAR", "INTERP_CUBIC", "DYE_DTYPE", "EVENT_STRIDE", "LABEL_DSTORM",
           "LABEL_PALM", "LABEL_DNA_PAINT", "LABEL_WIDEFIELD"]
