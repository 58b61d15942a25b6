/*
 * iscu.h -- C ABI of the B200 image-formation engine (libiscu.so).
 *
 * The engine replaces, on an NVIDIA B200 (sm_100a), the fluorescence image-formation path of inSiliScope's render
 * engine: the Gibson-Lanni/Zernike chirp-Z PSF stack, the blink splat, the camera noise chain with its counter-based
 * pcg4d stream, and the widefield mean-field FFT convolution. Every entry point is extern "C" with plain pointers and
 * sizes, so a C++ host (the engine's GpuSimulator / SplatGpuHost / WidefieldAccelerator seams), a ctypes caller or a
 * JNI/cgo stub binds it alike.
 *
 * Conventions
 *  - Every function returns ISCU_OK (0) or an ISCU_ERR_* code; iscu_last_error() gives the calling thread's message.
 *    No C++ exception crosses this boundary (the reference seam's `bool` + `std::string& err`,
 *    adapter/inSiliScope/Simulation/GpuSimD3D11.h:61-111).
 *  - A context (iscu_ctx) owns one device, one CUDA stream and the resident buffers (kernel stacks, camera maps),
 *    the way one GpuSimulator owns its D3D11 device (GpuSimD3D11.h:28-30: one instance per thread). Calls on one
 *    context are serialized by its mutex (WidefieldGpuHost.h:74-75's GpuBackend::mu).
 *  - Functions whose pointer arguments end in `_dev` take device pointers and enqueue work on the context's stream
 *    without synchronizing; the others take host pointers and return when the results are in host memory.
 *  - Images are row-major (x fastest). Photon images are float32, camera frames uint16 ADU.
 */
#ifndef ISCU_H
#define ISCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ISCU_ABI_VERSION 1

enum iscu_status {
   ISCU_OK = 0,
   ISCU_ERR_ARG = 1,     /* an argument is out of range or inconsistent */
   ISCU_ERR_CUDA = 2,    /* a CUDA runtime or launch error (the message names the call) */
   ISCU_ERR_STATE = 3,   /* the context lacks what the call needs (no kernel in the slot, no camera maps) */
   ISCU_ERR_LIMIT = 4,   /* a size beyond a documented maximum */
   ISCU_ERR_TIMEOUT = 5, /* a bounded device-side wait ran out (the context stays usable) */
   ISCU_ERR_NODEV = 6,   /* no CUDA device, or not an sm_100 device */
   ISCU_ERR_IO = 7       /* a file could not be opened or written (the message is the reference writer's) */
};

/* Interpolation of the splat's sub-pixel read (sim::PsfInterpMode, PsfGeneratorBridge.h:68-74). Fft has no GPU path
 * in the reference and none here. */
enum iscu_interp { ISCU_INTERP_NEAREST = 0, ISCU_INTERP_LINEAR = 1, ISCU_INTERP_CUBIC = 2 };

/* Which chirp-Z product a PSF build uses. */
enum iscu_czt_method {
   ISCU_CZT_FP32 = 0,   /* the plain FP32 form: SIMT complex matmuls in shared memory */
   ISCU_CZT_TF32X3 = 1, /* split precision on the tensor cores: hi/lo TF32 operands, three tcgen05 MMAs per product,
                           FP32 accumulation in tensor memory */
   ISCU_CZT_F16X3 = 2   /* the same with hi/lo FP16 operands (exact power-of-two scales keep them in range): twice
                           the inputs per MMA, the DFT operand resident in shared memory per request set */
};

typedef struct iscu_ctx iscu_ctx;

/* ---------------------------------------------------------------- context ------------------------------------- */

/* The calling thread's last error message ("" after a success). */
const char* iscu_last_error(void);
int iscu_abi_version(void);
/* A context on CUDA device `device`; ISCU_ERR_NODEV when it is not an sm_100 device. */
int iscu_create(int device, iscu_ctx** out);
void iscu_destroy(iscu_ctx* ctx);
/* Waits for the context's stream. Returns the first asynchronous error, if any. */
int iscu_synchronize(iscu_ctx* ctx);
/* The context's cudaStream_t (as void*), for callers that order their own work with it. */
void* iscu_stream(iscu_ctx* ctx);
/* Number of kernel launches this context has issued (all entry points), for launch accounting. */
uint64_t iscu_launch_count(iscu_ctx* ctx);

/* ---------------------------------------------------------------- counter RNG --------------------------------- */
/* pcg4d (adapter/inSiliScope/Simulation/SMLMCounterRng.h:37-56, core/src/rng.h:18-33): in4_dev[4i..4i+3] = (a, b, c,
 * d) -> out4_dev[4i..4i+3], for i < n. */
int iscu_pcg4d_dev(iscu_ctx* ctx, const uint32_t* in4_dev, uint32_t* out4_dev, size_t n);
/* sim::CounterRng (SMLMCounterRng.h:60-91): the first `per_pixel` uniforms of pixel p's stream, p = pixel0 + i,
 * into out_dev[i * per_pixel + j] (float64). */
int iscu_counter_uniforms_dev(iscu_ctx* ctx, uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix,
                              uint32_t per_pixel, double* out_dev);

/* ---------------------------------------------------------------- camera --------------------------------------- */

/* sim::CameraNoiseParams (SMLMNoise.h:35-50). gain is photons (electrons) per ADU. */
typedef struct iscu_camera {
   double quantum_efficiency;
   double dark_electrons;
   double gain;              /* used where no gain map is set */
   double read_noise_e;      /* used where no read-noise map is set */
   int32_t emccd;
   int32_t bit_depth;        /* EMCCD: ADU clipped to [0, 2^bit_depth - 1] */
   double em_gain;           /* EMCCD: divides the read noise only */
   double cic_electrons;     /* EMCCD: clock-induced charge per pixel and frame */
} iscu_camera;

/* Static per-pixel inputs of a width x height frame (sim::GpuSimulator::SetStatic, GpuSimD3D11.h:88-90; the window
 * offset of SplatGpuHost::SetStatic, SplatGpu.h:51-55). offset (ADU), gain (photons/ADU), read_noise (e-) are host
 * arrays of width*height floats or NULL (offset 0, the camera's scalar gain / read noise: ApplyNoiseChain's rule,
 * SMLMNoise.cpp:148-153). background: width*height photons/pixel/frame before the per-frame scale, or NULL for the
 * flat value flat_bg. illum: the illumination field (peak 1), or NULL for flat; it multiplies the background
 * (RenderPhotonImage, SMLMSimulation.cpp:129-136) -- emitters carry their own illumination factor already.
 * pixel_base: the frame's first pixel's index on the sensor (the noise stream is the sensor's). */
int iscu_set_static(iscu_ctx* ctx, uint32_t width, uint32_t height, uint32_t pixel_base, const float* offset,
                    const float* gain, const float* read_noise, const float* background, const float* illum,
                    double flat_bg);

/* sim::PixelOffsetMap / PixelGainMap / PixelReadNoiseMap::Generate (SMLMNoise.cpp:89-140) on the host, from one
 * std::mt19937_64(seed) in the order offset, gain, read noise (SplatGpu.cpp:500-502). Any output may be NULL (its
 * draws are still taken). keep_y0/keep_rows: a window's rows (0 rows: all). */
int iscu_generate_camera_maps(uint32_t width, uint32_t height, uint64_t seed, double offset_mean_adu,
                              double offset_std_adu, double gain_nominal, double gain_std_fraction,
                              double read_noise_nominal, double read_noise_std_fraction, uint32_t keep_y0,
                              uint32_t keep_rows, float* offset, float* gain, float* read_noise);

/* ApplyNoiseChain (SMLMNoise.cpp:142-216) on n_frames photon images: photons_dev[k*w*h ..] -> adu_dev[k*w*h ..],
 * noise keyed by (seed, frames_dev[k], pixel_base + pixel). Needs iscu_set_static for the maps. */
int iscu_noise_frames_dev(iscu_ctx* ctx, const float* photons_dev, uint32_t n_frames, const uint32_t* frames_dev,
                          const iscu_camera* cam, uint32_t seed, uint16_t* adu_dev);

/* ---------------------------------------------------------------- PSF ------------------------------------------ */

/* sim::PsfGeneratorRequest for the GibsonLanniZernike model (PsfGeneratorBridge.h:91-158) with the Zernike string
 * parsed (ParseZernikeCoefficients, SMLMZernike.h:50-51): OSA/ANSI 0-27, waves, unnormalized. */
typedef struct iscu_psf_request {
   double wavelength_nm;
   double na;
   double immersion_index;
   double sample_index;
   double working_distance_um;
   double sample_depth_nm;
   double pixel_size_nm;
   double zernike[28];
   int32_t mask_double_helix;
   int32_t mask_modes;
   double mask_waist;
   int32_t oversampling;
   int32_t kernel_half_width_px;
   int32_t nz;               /* made odd and >= 3, as GeometryFor does (ZernikePsf.cpp:118-129) */
   int32_t pupil_samples;    /* 0: ZernikePupilSamples' automatic choice (ZernikePsf.cpp:139-158) */
   double z_step_nm;
   int32_t interp;           /* iscu_interp */
   int32_t reserved;
} iscu_psf_request;

/* A request's plane geometry (GeometryFor + ZernikePupilSamples): plane size, planes, pupil samples M. */
int iscu_psf_geometry(const iscu_psf_request* req, int32_t* size, int32_t* nz, int32_t* pupil_samples);

/* One PSF library: n_psf planes of size x size float32 into out_dev (device), each the squared modulus of the
 * chirp-Z image of a Gibson-Lanni + Zernike (+ double-helix) pupil (ComputeZernikePsfPlanes, ZernikePsf.cpp:160-337).
 * PSF i uses request set_of_psf[i] (host array) of the `sets` requests (host array) at defocus defocus_nm[i]
 * (host array; the reference's plane k sits at (k - (nz-1)/2) * z_step_nm). size overrides the request's
 * 2*half*os+1 (0: keep it); the pupil samples M come from the request. normalize != 0 divides each plane by its sum
 * (BuildZernikePsfKernelCache, ZernikePsf.cpp:400-410). method: iscu_czt_method. All sets must share M and size. */
int iscu_psf_library_dev(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t n_sets, const uint32_t* set_of_psf,
                         const double* defocus_nm, uint32_t n_psf, int32_t size, int32_t normalize, int32_t method,
                         float* out_dev);

/* A PSF library plan: the per-set work of ComputeZernikePsfPlanes (pupil tables, DFT matrices, and for
 * the split methods the split stacked operand) done once for `sets` at plane size `size` (0: the first request's),
 * then runs of any number of PSFs (set index + defocus each). The memo of ComputePsfKernelCache
 * (PsfGeneratorBridge.h:317-364) keeps kernel stacks the same way. ISCU_CZT_TF32X3 and ISCU_CZT_F16X3 need M <= 128
 * (a multiple of 16) and planes of at most 64 x 64. */
typedef struct iscu_psf_plan iscu_psf_plan;
int iscu_psf_plan_create(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t n_sets, int32_t size, int32_t method,
                         iscu_psf_plan** out);
void iscu_psf_plan_destroy(iscu_psf_plan* plan);
/* The plan's plane size P and pupil samples M. */
int iscu_psf_plan_info(iscu_psf_plan* plan, int32_t* size, int32_t* pupil_samples);
/* n_psf planes (P x P floats each) into out_dev from device arrays of set indices and defocus (nm); enqueued on the
 * context's stream. iscu_psf_plan_check waits and reports a bad set index or a tensor-core wait that ran out. */
int iscu_psf_plan_run_dev(iscu_psf_plan* plan, const uint32_t* set_of_psf_dev, const double* defocus_nm_dev,
                          uint32_t n_psf, int32_t normalize, float* out_dev);
int iscu_psf_plan_check(iscu_psf_plan* plan);
/* The same from host arrays into host memory (the copies are part of the call; from 2,048 PSFs on, the library runs in
 * four launches and each one's planes come back while the next computes, which pays with page-locked out). */
int iscu_psf_plan_run(iscu_psf_plan* plan, const uint32_t* set_of_psf, const double* defocus_nm, uint32_t n_psf,
                      int32_t normalize, float* out);

/* No counterpart in the reference. iscu_psf_library_dev with the plain FP32 method, for callers that must not
 * allocate GPU memory: a host whose device memory belongs to someone else (a framework's caching allocator that has
 * reserved the free memory, a fixed budget shared with other plug-ins), or a loop that cannot afford the device-wide
 * synchronization a cudaFree implies. Its temporaries (set parameters, PSF items, pupil tables, DFT matrices) live in
 * one statically sized device array of ISCU_NOALLOC_SCRATCH_BYTES that every GPU loading libiscu.so holds until exit;
 * the call itself allocates nothing on the device. Limits: at most ISCU_NOALLOC_MAX_SETS sets and
 * ISCU_NOALLOC_MAX_PSF PSFs, pupil samples M <= 128, plane size P <= 129 with (M*M + P*M)*8 bytes beside the FP32
 * chirp-Z kernel's static shared memory within one CTA's limit (227 KB on a B200: at M = 128, P <= 98), and the
 * layout within the array (sets, items, M*M*24 bytes of tables and 2*P*M*8 bytes of DFT matrices per set) must fit;
 * beyond: ISCU_ERR_LIMIT, before any copy or launch.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture. All calls share the array: calls whose work overlaps on the GPU (other threads or
 * contexts) race. Returns when the planes are in out_dev. */
#define ISCU_NOALLOC_SCRATCH_BYTES (4u << 20)
#define ISCU_NOALLOC_MAX_SETS 4
#define ISCU_NOALLOC_MAX_PSF 4096
int iscu_psf_library_noalloc_dev(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t n_sets,
                                 const uint32_t* set_of_psf, const double* defocus_nm, uint32_t n_psf, int32_t size,
                                 int32_t normalize, float* out_dev);

/* ---------------------------------------------------------------- kernel slots -------------------------------- */
/* At most this many kernel stacks per context (GpuSimulator::kMaxKernels, GpuSimD3D11.h:70). */
#define ISCU_MAX_KERNELS 4

/* Builds a kernel stack on the device from a request (BuildZernikePsfKernelCache, ZernikePsf.cpp:382-415: sum-1
 * planes, then the block sums, PsfGeneratorBridge.cpp:1021-1088) into slot 0..3. */
int iscu_kernel_build(iscu_ctx* ctx, int32_t slot, const iscu_psf_request* req, int32_t method);
/* Uploads a kernel stack made elsewhere (the engine's PsfKernelCache planes, already sum-1): nz planes of size x size
 * (host). The block sums are built on the device (GpuSimulator::SetKernels, GpuSimD3D11.h:72-77). */
int iscu_kernel_set_planes(iscu_ctx* ctx, int32_t slot, const float* planes, int32_t size, int32_t nz,
                           int32_t oversampling, double z_step_nm, int32_t interp);
/* The halo cut (WithHaloCut, PsfGeneratorBridge.cpp:1137-1243) for a slot's stack; threshold <= 0 removes it. */
int iscu_kernel_set_halo(iscu_ctx* ctx, int32_t slot, double threshold);
/* A cut slot's spans (PsfHaloSpans::lo / hi / radius2, PsfGeneratorBridge.h:228-237): lo and hi nz * (2 camRad + 1)
 * int16 each (camRad = the half width in camera pixels; a row with lo > hi is empty), radius2 nz int32 (-1: nothing
 * kept). ISCU_ERR_STATE when the slot has no cut. */
int iscu_kernel_get_halo(iscu_ctx* ctx, int32_t slot, int16_t* lo, int16_t* hi, int32_t* radius2);
/* Geometry of a slot: size, nz, oversampling, block-sum width. */
int iscu_kernel_info(iscu_ctx* ctx, int32_t slot, int32_t* size, int32_t* nz, int32_t* oversampling,
                     int32_t* block_sum_width);
/* Reads a slot's planes (nz*size*size floats) or block sums (nz*bw*bw floats, row-major) back to the host. */
int iscu_kernel_get_planes(iscu_ctx* ctx, int32_t slot, float* out);
int iscu_kernel_get_block_sums(iscu_ctx* ctx, int32_t slot, float* out);

/* ---------------------------------------------------------------- splat + noise ------------------------------- */

/* One emitter of one frame as the splat places it (sim::FrameEmitter, SMLMSimulation.h:158-173): camera-pixel
 * position (drift included), photons (overlap x brightness x excitation x illumination), and its kernel plane
 * (z index | kernel slot << 16). 32 bytes. The device derives SplatSetup (PsfGeneratorBridge.cpp:1382-1422) from
 * it in float64, so the splat is bit for bit the CPU's. */
typedef struct iscu_emitter {
   double x_px;
   double y_px;
   double photons;
   int32_t plane;
   int32_t reserved;
} iscu_emitter;

/* sim::GpuSplatEmitter (GpuSimD3D11.h:50-59): the reference's 64-byte device record (float weights). */
typedef struct iscu_gpu_splat_emitter {
   int32_t x0, y0, bx, by;
   int32_t plane;
   int32_t n_taps;
   float photons;
   int32_t cut_radius2;
   float wx[4];
   float wy[4];
} iscu_gpu_splat_emitter;

/* One frame of a batch: its emitters are [em_start, em_start + em_count) of the batch's array; frame is the noise
 * stream's frame index; bg_scale multiplies the background (BackgroundFadeScale). */
typedef struct iscu_frame {
   uint32_t em_start;
   uint32_t em_count;
   uint32_t frame;
   uint32_t reserved;
   double bg_scale;
} iscu_frame;

/* Frames k < n_frames: the background, then every emitter of the frame splatted in list order (emitters_dev holds
 * n_emitters records; a frame's run is cut at n_emitters)
 * (RenderPhotonImage, SMLMSimulation.cpp:103-160: the same float additions in the same order), then, unless
 * cam is NULL, the noise chain (ApplyNoiseChain). photons_dev (nullable) receives the noise-free images,
 * adu_dev (nullable) the frames; both n_frames*w*h. Needs iscu_set_static and the kernels the emitters name. */
int iscu_render_frames_dev(iscu_ctx* ctx, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                           const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                           float* photons_dev, uint16_t* adu_dev);
/* The same with host arrays (emitters: sum of em_count records; frames: n_frames; outputs host, nullable): the
 * copies in and out are part of the call. */
int iscu_render_frames(iscu_ctx* ctx, const iscu_emitter* emitters, uint32_t n_emitters, const iscu_frame* frames,
                       uint32_t n_frames, const iscu_camera* cam, uint32_t seed, float* photons, uint16_t* adu);

/* The render kernel's form (no reference counterpart: the reference renders a frame per CPU task, ParallelFor over
 * frames, ScopeMovie.cpp:7059-7110). config % 3: the CTA's tile, 16x16, 32x8 or 8x32 pixels; (config / 3) % 2: one
 * CTA per (frame, tile), or a persistent grid that takes (frame, tile) items heaviest frame first (for batches whose
 * frames carry very different emitter counts). Configs 0..11 render in one pass, config / 6 emitters per step of a
 * pixel's loop (*paired 0 or 1); configs 12..17 in two passes (*paired 2): every emitter's float contribution to
 * each pixel of its square first, computed by groups of emitters that read the same block sums (kernel slot, plane,
 * tap origin), then the tiles add them in emitter order. The two-pass forms keep up to a quarter of the device's
 * memory for contributions (n_emitters x square pixels floats); a batch beyond that renders in the one-pass form of
 * the same tile and scheduling. Every form gives the same bits. */
#define ISCU_RENDER_CONFIGS 18
int iscu_render_set_config(iscu_ctx* ctx, int32_t config);
/* Pass timing of the renders that follow (CUDA events on the context's stream; not inside a graph capture):
 * iscu_render_pass_times gives the mean milliseconds per render of grouping (setup, group offsets, lists),
 * contributions, and the tile pass (splat or gather + noise; a one-pass form's whole render), and how many renders were
 * timed. set_timing restarts the count. */
int iscu_render_set_timing(iscu_ctx* ctx, int32_t on);
int iscu_render_pass_times(iscu_ctx* ctx, float* ms3, uint32_t* calls);
/* The most device bytes the two-pass forms' contributions may take (0: a quarter of the device's memory). */
int iscu_render_set_contrib_limit(iscu_ctx* ctx, uint64_t bytes);
int iscu_render_get_config(iscu_ctx* ctx, int32_t* config, int32_t* tile_w, int32_t* tile_h, int32_t* persistent,
                           int32_t* paired);
/* Times the ISCU_RENDER_CONFIGS forms on the given device batch (one warm-up and two timed renders each, adu_dev
 * overwritten), keeps the fastest as the context's form; ms (nullable, ISCU_RENDER_CONFIGS floats) receives each
 * form's milliseconds per render. */
int iscu_render_autotune(iscu_ctx* ctx, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                         const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                         uint16_t* adu_dev, float* ms);
/* iscu_render_frames_dev with the context's current form captured once into a CUDA graph on the context's stream;
 * each launch replays it (the same device pointers, so refill them in place between launches). Kernel slots and
 * camera statics must not be rebuilt while the graph lives. */
typedef struct iscu_render_graph iscu_render_graph;
int iscu_render_graph_create(iscu_ctx* ctx, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                             const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                             float* photons_dev, uint16_t* adu_dev, iscu_render_graph** out);
int iscu_render_graph_launch(iscu_render_graph* graph);
void iscu_render_graph_destroy(iscu_render_graph* graph);

/* GpuSimulator::RenderFrames / SplatGpuHost::RenderFrames (GpuSimD3D11.h:98-107, SplatGpu.h:57-62) over the
 * reference's 64-byte records: the D3D11/WGSL shader's semantics (GpuSimD3D11.cpp:169-248) -- the record's float
 * weights, the halo radius test, an optional extra photon image per frame (extras: n_frames*w*h host floats, or NULL;
 * the blinks are splatted onto background + extra, as SplatGpuHost does) -- with the taps summed in float64. Host
 * arrays. */
int iscu_render_gpu_records(iscu_ctx* ctx, const iscu_gpu_splat_emitter* emitters, uint32_t n_emitters,
                            const iscu_frame* frames, uint32_t n_frames, const float* extras,
                            const iscu_camera* cam, uint32_t seed, uint16_t* adu);

/* ---------------------------------------------------------------- host-side emitter collection ---------------- */

/* sim::BlinkEvent (SMLMSimulation.h:82-102), the fields the render reads, plus the kernel slot of the event's dye
 * group (the engine renders each group with its own PSF kernel, ScopeMovie.cpp:7059-7110). */
typedef struct iscu_blink_event {
   double x_um, y_um, z_nm;
   double t_start, t_end;
   double brightness;
   double excite;
   int32_t slot;       /* used when the collecting call's slot is -1 */
   int32_t reserved;
} iscu_blink_event;

/* CollectFrameEmitters (SMLMSimulation.cpp:55-101) for one frame: the events overlapping [frame, frame+1), in order,
 * as iscu_emitter records (kernel slot `slot`, or each event's own slot when slot is -1; z plane from that slot's
 * stack by NearestZIndex, PsfGeneratorBridge.cpp:40-61), min_photons applied (RenderPhotonImage's
 * blink-min-photons). Several dye groups in one frame: put each group's events in the bucket one group after the
 * other, as the engine renders them (one RenderPhotonImage per group, accumulating). illum: the
 * illumination field (w*h host floats) or NULL. Writes at most max_out records; *n_out gets the count. Returns
 * ISCU_ERR_LIMIT when max_out is too small. *n_clamped (nullable) += emitters whose z was clamped. */
int iscu_collect_frame_emitters(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, uint32_t n_events,
                                int64_t frame, uint32_t width, uint32_t height, double pixel_size_nm,
                                double photons_per_blink, double drift_x_px, double drift_y_px,
                                double global_z_offset_um, const float* illum, double min_photons,
                                iscu_emitter* out, uint32_t max_out, uint32_t* n_out, int64_t* n_clamped);

/* The same for the frames frame0 .. frame0 + n_frames - 1 of a batch, into one emitter array and its frame table
 * (the batch a render call takes). Frame k's candidate events are bucket k: events[bucket_index[j]] for j in
 * [bucket_start[k], bucket_start[k+1]) (BucketEventsByFrame's index lists, SMLMSimulation.cpp:203-217, in event
 * order), or events[j] itself when bucket_index is NULL. drift_x_px / drift_y_px / global_z_offset_um / bg_scale:
 * per-frame arrays or NULL (0, 0, 0, 1). frames_out[k]: the frame's emitter run, frame0 + k, its bg scale. */
int iscu_collect_emitters(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, const uint32_t* bucket_index,
                          const uint32_t* bucket_start, int64_t frame0, uint32_t n_frames, uint32_t width,
                          uint32_t height, double pixel_size_nm, double photons_per_blink, const double* drift_x_px,
                          const double* drift_y_px, const double* global_z_offset_um, const double* bg_scale,
                          const float* illum, double min_photons, iscu_emitter* out, uint32_t max_out,
                          iscu_frame* frames_out, uint32_t* n_out, int64_t* n_clamped);

/* The same on the device (no reference counterpart: the reference collects on the CPU): events_dev (n_events),
 * bucket_index_dev (nullable) and bucket_start_dev (n_frames + 1) as above, the per-frame arrays and illum_dev
 * (width*height of the context's frame) device pointers or NULL. Writes out_dev (at most max_out records) and
 * event_index_dev (nullable: each record's index into the events -- the frame's ground-truth emitter list),
 * frames_out_dev (n_frames) and *n_out_dev = the records kept (more than max_out: the batch did not fit);
 * *n_clamped_dev (nullable, zero it first) += the emitters whose z was clamped. Events whose slot holds no kernel stack
 * are dropped (the host form fails on them). Needs iscu_set_static (the frame size). Asynchronous. */
int iscu_collect_emitters_dev(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events_dev, uint32_t n_events,
                              const uint32_t* bucket_index_dev, const uint32_t* bucket_start_dev, int64_t frame0,
                              uint32_t n_frames, double pixel_size_nm, double photons_per_blink,
                              const double* drift_x_px_dev, const double* drift_y_px_dev,
                              const double* global_z_offset_um_dev, const double* bg_scale_dev, const float* illum_dev,
                              double min_photons, iscu_emitter* out_dev, uint32_t* event_index_dev,
                              uint32_t max_out, iscu_frame* frames_out_dev, uint32_t* n_out_dev,
                              int64_t* n_clamped_dev);

/* Host blink events to host frames in one call (the movie engine's frame loop for one dye group batch,
 * ScopeMovie.cpp:7059-7110: CollectFrameEmitters + RenderPhotonImage + ApplyNoiseChain per frame): the events, bucket
 * arrays and per-frame arrays (as iscu_collect_emitters; use_illum: the context's illumination field weights the
 * emitters) go to the device, are collected and rendered there, and photons (nullable, n_frames*w*h floats) and adu
 * (n_frames*w*h) come back. *n_emitters (nullable) = the emitters splatted; *n_clamped (nullable) += clamped z
 * planes. Page-locked host buffers make the copies direct. */
int iscu_render_events(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, uint32_t n_events,
                       const uint32_t* bucket_index, const uint32_t* bucket_start, int64_t frame0, uint32_t n_frames,
                       double pixel_size_nm, double photons_per_blink, const double* drift_x_px,
                       const double* drift_y_px, const double* global_z_offset_um, const double* bg_scale,
                       int32_t use_illum, double min_photons, const iscu_camera* cam, uint32_t seed, float* photons,
                       uint16_t* adu, uint32_t* n_emitters, int64_t* n_clamped);

/* iscu_render_events in two halves, so that the copies of one batch overlap the render of another (the movie engine's
 * frame loop pipelined across batches). _async enqueues the batch in I/O slot io_slot (0 .. ISCU_EVENT_IO_SLOTS - 1,
 * each with its own device staging) and returns at once: the events go in on the context's upload stream, the
 * collection, render and noise run on its stream, the frames come out on its download stream. Until
 * iscu_render_events_wait(ctx, io_slot, ...) returns, the host inputs must stay unchanged and the outputs unread;
 * the wait blocks until the batch's frames are in the host buffers and reports its counts as iscu_render_events does.
 * A slot holds one batch: _async on a slot not yet waited for fails with ISCU_ERR_STATE, and so does a wait on an
 * idle slot. Page-locked host buffers let the copies run beside the kernels (pageable ones are copied synchronously).
 * A batch that fails to enqueue leaves its slot idle. */
#define ISCU_EVENT_IO_SLOTS 4
int iscu_render_events_async(iscu_ctx* ctx, int32_t io_slot, int32_t slot, const iscu_blink_event* events,
                             uint32_t n_events, const uint32_t* bucket_index, const uint32_t* bucket_start,
                             int64_t frame0, uint32_t n_frames, double pixel_size_nm, double photons_per_blink,
                             const double* drift_x_px, const double* drift_y_px, const double* global_z_offset_um,
                             const double* bg_scale, int32_t use_illum, double min_photons, const iscu_camera* cam,
                             uint32_t seed, float* photons, uint16_t* adu);
int iscu_render_events_wait(iscu_ctx* ctx, int32_t io_slot, uint32_t* n_emitters, int64_t* n_clamped);

/* ---------------------------------------------------------------- blink schedules ----------------------------- */

/* The world core's blink kinetics (core/src/dyes.h Kinetics): rates per second, times in seconds. */
typedef struct iscu_kinetics {
   double activation_rate_per_sec;
   double on_sec;
   double off_sec;
   double bleach_prob;
   double photon_cv;
   double initial_on_sec;       /* dSTORM: ON from t = 0 for Exp(initial_on_sec) before the blinks (0: none) */
} iscu_kinetics;

/* core LabelMode */
#define ISCU_LABEL_DSTORM 0
#define ISCU_LABEL_PALM 1
#define ISCU_LABEL_DNA_PAINT 2
#define ISCU_LABEL_WIDEFIELD 3
typedef struct iscu_label {
   int32_t mode;                /* ISCU_LABEL_* */
   int32_t reserved;
   iscu_kinetics kin;
} iscu_label;

/* One fluorescent dye: its address in the core's hash scheme (h1: its structure element's H1, e.g. DyeH1 of a
 * microtubule; k: the site, e.g. the protofilament; n: the index), its id (H2.a), structure and position (um). */
typedef struct iscu_dye {
   double x, y, z;
   uint32_t h1;
   int32_t k, n;
   uint32_t id;
   int32_t structure;
   int32_t reserved;
} iscu_dye;

/* The blink rows of isc_events_in_window (insiliscope.h:304-313): x, y, z, tOn, tOff, brightness, id, structure,
 * state (0: a blink), aux (0). */
#define ISCU_EVENT_STRIDE 10

/* Each dye's blinks overlapping [t0, t1) (tOn < t1, tOff > t0), as the world core schedules them (dyes.cpp: dSTORM
 * and PALM LabelSchedule, DNA-PAINT PersistentBlinks, WideField none), bit for bit: the same address-keyed draws and
 * float64 arithmetic with fdlibm's log / exp / cos. Rows per dye in the order the core appends them, dyes in input
 * order. History: n_seg = 0 the label's kinetics; n_seg >= 1 segments of constant kinetics starting at
 * hist_t_start[s] (host arrays, the first 0, increasing, at most 64), as isc_world_set_kinetics_history. dyes_dev,
 * rows_dev (max_rows x ISCU_EVENT_STRIDE doubles), dye_first_dev (nullable, n_dyes + 1: each dye's first row, then
 * the total) and *n_rows_dev (the total rows, written even past max_rows; rows at or beyond max_rows are dropped)
 * are device memory. Bounds on the per-dye work (ISCU_ERR_LIMIT beyond): a finite window of at most 36000 s ending by
 * 1e6 s, activation rates at most 1e5 per s, ON times at most 1000 s. Asynchronous. */
int iscu_dye_blinks_dev(iscu_ctx* ctx, const iscu_label* label, const double* hist_t_start,
                        const iscu_kinetics* hist_kin, uint32_t n_seg, const iscu_dye* dyes_dev, uint32_t n_dyes,
                        double t0, double t1, double* rows_dev, uint32_t max_rows, uint32_t* dye_first_dev,
                        uint32_t* n_rows_dev);

/* ---------------------------------------------------------------- per-movie host models ----------------------- */

/* sim::DriftSettings (Drift.h:57-79). */
typedef struct iscu_drift_settings {
   double xy_nm_per_sqrt_sec;   /* random walk: RMS displacement after 1 s, x and y each */
   double z_nm_per_sqrt_sec;
   double xy_speed_nm_per_sec;  /* directed part */
   double z_speed_nm_per_sec;
   double xy_angle_deg;         /* < 0: drawn per seed */
   int32_t z_direction;         /* +1 away from the coverslip, -1 towards, 0 drawn per seed */
   int32_t reserved;
   double angle_wander_deg;     /* 180 */
   double z_angle_wander_deg;   /* 90 */
   double speed_wander_pct;     /* 0 */
   double wander_time_sec;      /* 60 */
} iscu_drift_settings;

/* sim::DriftTrajectory (Drift.cpp:24-124; host): the sample's drift (nm, camera axes, +z away from the coverslip) at
 * frames 0 .. frames - 1 into xyz_nm[3 f + (0, 1, 2)], zero at frame 0, every draw from the counter stream of
 * (DriftSeed(random_seed), frame): bit for bit the reference's. */
int iscu_drift_trajectory(int64_t random_seed, int64_t frames, double frame_sec, const iscu_drift_settings* settings,
                          double* xyz_nm);
/* sim::BuildIlluminationField (SMLMBackground.cpp:8-38; host): profile 0 flat (out untouched), 1 Gaussian, 2 flat-top
 * with FWHM fwhm_pct % of the width; out: width*height floats with peak 1; *mean_factor (nullable) the field's mean. */
int iscu_illumination_field(uint32_t width, uint32_t height, int32_t profile, double fwhm_pct, float* out,
                            double* mean_factor);
/* sim::BackgroundFadeScale (SMLMBackground.cpp:52-55): 0.3 + 0.7 exp(-t / decay), 1 when decay <= 0. */
double iscu_background_fade_scale(double t, double decay);

/* ---------------------------------------------------------------- Poisson-likelihood gradient ---------------- */

/* The differentiable ROI model (no reference counterpart: the reference has no gradient): the Gibson-Lanni/Zernike
 * pupil (ZernikePsf.cpp:188-248) at matched indices and depth 0, each emitter at a continuous defocus z (nm) and
 * position (x, y) (ROI pixels), its field the separable DFT of the pupil to the ROI's os x os sub-pixel samples:
 *   U = a exp(i (z kz + 2 pi sum_j c_j Z_j - p (kx x + ky y))),  E = A U A^T,  A[s][m] = exp(i k_m p (s + 0.5) / os)
 *   mu = N kappa (sum of |E|^2 over a pixel's samples) + b_frame,   NLL = sum over ROI pixels of mu - k log mu
 * with the pupil grid k_i = (i - M/2) dk, dk = 2 kMax / (M - 4) (ZernikePsf.cpp:192-193), Z_j Noll's orthonormal
 * Zernike polynomials on rho = k / kMax (coefficients in waves rms), kappa = (p / os)^2 / (L^2 sum a), L = 2 pi / dk.
 * This build takes a 32 x 32 pupil and roi * os = 64. */
typedef struct iscu_nll_spec {
   double wavelength_nm;
   double na;
   double n_imm;          /* immersion = sample index */
   double pixel_nm;
   int32_t roi;           /* ROI side in pixels */
   int32_t os;            /* samples per pixel per axis */
   int32_t pupil;         /* M */
   int32_t n_zern;        /* <= 32 */
   int32_t noll[32];      /* the Zernike modes' Noll indices */
} iscu_nll_spec;

typedef struct iscu_nll_model iscu_nll_model;
int iscu_nll_model_create(iscu_ctx* ctx, const iscu_nll_spec* spec, iscu_nll_model** out);
void iscu_nll_model_destroy(iscu_nll_model* model);
int iscu_nll_model_info(iscu_nll_model* model, double* kappa, int32_t* n_zern);
/* NLL of n_emitters ROIs (params_dev: n x (x, y, z, N) float; frame_dev: each ROI's frame < n_frames; bg_dev:
 * n_frames float; zern: n_zern float64 host; counts_dev: n x roi x roi float) into *nll_dev (float64, device);
 * mu_dev (nullable): the expected counts. With grad_params_dev (n x 4 float: dNLL/dx, /dy, /dz, /dN) the adjoint
 * runs too (the field recomputed, no per-emitter PSF stored): grad_bg_dev (n_frames float64) and grad_zern_dev
 * (n_zern float64) receive the rest. *err_dev (int32, device) = 1 when an emitter names a frame outside the batch.
 * Asynchronous on the context's stream. */
int iscu_nll_eval_dev(iscu_nll_model* model, uint32_t n_emitters, const float* params_dev, const int32_t* frame_dev,
                      uint32_t n_frames, const float* bg_dev, const double* zern, const float* counts_dev,
                      float* mu_dev, double* nll_dev, float* grad_params_dev, double* grad_bg_dev,
                      double* grad_zern_dev, int32_t* err_dev);

/* ---------------------------------------------------------------- widefield ----------------------------------- */

/* Widefield mean-field 3D convolution: the dye density volume (nx x ny x nz float32, x fastest, photons per voxel
 * at focus) convolved with a 3D PSF (kx x ky x kz float32, centred on voxel (kx/2, ky/2, kz/2)), linear (zero-padded)
 * and cropped to the volume ("same"), so image plane f is sum_k dye plane k (x) PSF plane f - k + kz/2 -- the focus
 * series of WidefieldScene (WidefieldRender.h:588, one image per focus at every dye plane). A plan holds the PSF's
 * spectrum resident (the reference caches kernel spectra, WidefieldRender.cpp:1408). */
typedef struct iscu_wf_plan iscu_wf_plan;
int iscu_wf_plan_create(iscu_ctx* ctx, uint32_t nx, uint32_t ny, uint32_t nz, const float* psf, uint32_t kx,
                        uint32_t ky, uint32_t kz, iscu_wf_plan** out);
void iscu_wf_plan_destroy(iscu_wf_plan* plan);
/* The reference's widefield scene as a plan (WidefieldScene::UpdateFromGrid + FocusSeries + WidefieldImages::Render,
 * WidefieldRender.cpp:1180, :2845, :547; the kernel KernelWidefieldPsf, :263-330): the dye grid is nx x ny x nz cells
 * at pixel_um / upscale (dye plane i at its centre, planes plane_nm thick) and the series images it at every dye
 * plane's centre. The PSF comes from kernel slot `slot` (upscale must divide its oversampling): each cell the float64
 * sum of its (os / upscale)^2 oversampled samples, the radius capped at kernel_cap_um; dye plane k seen from focus f
 * through the slot's plane at t = (k - f) plane_nm / z_step + (nz_slot - 1) / 2 -- clamped to the stack, between two
 * planes the linear blend (PlanFocus, :1460-1522). Frames are the camera window: cells [fov_x0, fov_x0 + upscale
 * fov_w) x [fov_y0, fov_y0 + upscale fov_h) of the grid, each pixel the float64 sum of its upscale x upscale cells
 * clamped at 0, + background, then the noise chain: fov_w x fov_h x nz frames from every render call
 * (iscu_wf_render*, iscu_wf_convolve_dev). */
int iscu_wf_plan_from_kernel(iscu_ctx* ctx, int32_t slot, int32_t upscale, double pixel_um, double kernel_cap_um,
                             double plane_nm, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t fov_x0, uint32_t fov_y0,
                             uint32_t fov_w, uint32_t fov_h, iscu_wf_plan** out);
/* A plan's frame size (the grid's nx x ny, or a from-kernel plan's camera window) and its kernel radius in cells. */
int iscu_wf_plan_frame(iscu_wf_plan* plan, uint32_t* width, uint32_t* height, int32_t* kernel_radius);
/* The padded FFT grid of a plan (each axis a power of two holding the kernel and the volume's "same" window,
 * n + k/2 points, of the circular convolution). */
int iscu_wf_plan_grid(iscu_wf_plan* plan, uint32_t* gx, uint32_t* gy, uint32_t* gz);
/* density_dev (nx*ny*nz) -> image_dev (the frames: nx*ny*nz, or a from-kernel plan's window): the convolution,
 * max(0, .) per voxel (WidefieldImages::Render's clamp, WidefieldRender.cpp:547). */
int iscu_wf_convolve_dev(iscu_wf_plan* plan, const float* density_dev, float* image_dev);
/* Convolution, max(0, .) + background, then the noise chain per image plane (frame f = frame0 + plane; cam NULL: no
 * noise), host buffers: the widefield movie of one focus series. adu: nx*ny*nz uint16 (needed with cam). image
 * (nullable): the noise-free expected frames. */
int iscu_wf_render(iscu_wf_plan* plan, const float* density, double background, const iscu_camera* cam,
                   uint32_t seed, uint32_t frame0, float* image, uint16_t* adu);
/* Phase timing of a plan's renders (the reference's ISC_TIMING phases, Timing.h:123): with it on, every render
 * records CUDA events around its ISCU_WF_PASSES passes; iscu_wf_pass_times gives the last render's pass durations
 * in ms (x forward, y forward, z convolve, y inverse, x inverse, camera noise -- 0 without a camera), waiting for
 * it. */
#define ISCU_WF_PASSES 6
int iscu_wf_set_timing(iscu_wf_plan* plan, int32_t on);
int iscu_wf_pass_times(iscu_wf_plan* plan, float* ms);
/* The focus series pipelined across calls (a movie of volumes, or one volume's repeats): _async enqueues a render of
 * host buffers in I/O slot io_slot (0 .. ISCU_EVENT_IO_SLOTS - 1) -- the volume's H2D on an upload stream, the passes
 * on the context's stream after it and after everything enqueued before, the frames' D2H on a download stream after
 * them -- and returns; _wait waits for that slot's frames. One slot's copies run beside another's passes. The host
 * buffers (page-locked for the copies to overlap) are not touched by the caller until the wait; a slot takes a new
 * render only after its wait. Arguments as iscu_wf_render. */
int iscu_wf_render_async(iscu_wf_plan* plan, int32_t io_slot, const float* density, double background,
                         const iscu_camera* cam, uint32_t seed, uint32_t frame0, float* image, uint16_t* adu);
int iscu_wf_render_wait(iscu_wf_plan* plan, int32_t io_slot);
/* Frames of a drifting sample from its channels' spectra (WidefieldDriftFrames::Render / RenderShiftedImages,
 * WidefieldRender.cpp:2905-2935; ShiftedCamera and ApplyShiftRamp, DriftShift.cpp:23-71) on an nx x ny grid (powers
 * of two: the reference's GPU-mode grid, WidefieldRender.h:336). Per frame f: S = sum_c coef[f][c] spectra[c] (float
 * complex, channels in the order the reference adds them -- the near focus's persistent and bleach channels, then
 * the far focus's -- coefficients already multiplied as it does: float(a_j) x float(w_i); zero coefficients skipped),
 * times exp(2 pi i (kx sx / nx + ky' sy / ny)) with (sx, sy) = shift[f] cells (ky' the signed row frequency, the
 * Nyquist terms their cosine only), the inverse real transform (1 / (nx ny)), the window [y0, y0 + ch) x [x0, x0 +
 * cw), each cell clamped at 0, up x up cells summed in float64 x scale and added to cam[f] ((ch / up) x (cw / up)).
 * spectra_dev: n_channels x ny x (nx / 2 + 1) complex (interleaved float pairs) in RealFft2d's layout; coef_dev:
 * n_frames x n_channels floats; shift_dev: n_frames x 2 doubles. */
typedef struct iscu_wf_shift iscu_wf_shift;
int iscu_wf_shift_create(iscu_ctx* ctx, uint32_t nx, uint32_t ny, iscu_wf_shift** out);
void iscu_wf_shift_destroy(iscu_wf_shift* s);
int iscu_wf_shifted_frames_dev(iscu_wf_shift* s, const float* spectra_dev, uint32_t n_channels, const float* coef_dev,
                               const double* shift_dev, uint32_t n_frames, uint32_t x0, uint32_t y0, uint32_t cw,
                               uint32_t ch, uint32_t up, float scale, float* cam_dev);
/* Focus jobs: the GPU side of a widefield scene (sim::WidefieldAccelerator, WidefieldRender.h:342-359; the job is
 * WidefieldGpuJob, :306-337, as WidefieldScene::JobFor builds it, WidefieldRender.cpp:1953-2029). A job engine keeps
 * plane spectra resident by key and kernel spectra by plane index, both within one geometry value (a new geometry or
 * transform size drops them). iscu_wf_job_images: the job's kernel spectra not yet resident are uploaded (RealFft2d's
 * layout: ny_fft rows of nx_fft/2 + 1 complex, interleaved float pairs), its new planes (sparse cells of the nx x ny
 * dye grid, row-major, and their values) scattered and transformed, then each channel's image: sum over its deps of
 * plane spectrum x (w0 K[p0] + w1 K[p1]) (ChannelImageStep, :1790-1801), the sub-cell shift (ApplyShiftRamp,
 * DriftShift.cpp:24-48), the inverse transform (1 / (nx_fft ny_fft)) and the FOV window [fov_y0, + ch) x [fov_x0, + cw)
 * (ChannelImageFinish, WidefieldRender.cpp:1844-1878) into images[c] (host, cw x ch floats, not clamped). FFT sizes:
 * powers of two in 16..2048. budget_bytes (0: a quarter of the device) caps the plane spectra; iscu_wf_job_fits says
 * whether `planes` spectra of that size fit it (WidefieldAccelerator::Fits). */
typedef struct iscu_wf_job iscu_wf_job;
typedef struct iscu_wf_job_kernel {
   int32_t p;
   int32_t reserved;
   const float* spec;
} iscu_wf_job_kernel;
typedef struct iscu_wf_job_plane {
   uint64_t key;
   const uint32_t* cells;
   const float* values;
   uint32_t count;
   uint32_t reserved;
} iscu_wf_job_plane;
typedef struct iscu_wf_job_dep {
   uint64_t key;
   int32_t p0, p1;
   float w0, w1;
   int32_t two;
   int32_t reserved;
} iscu_wf_job_dep;
typedef struct iscu_wf_job_desc {
   uint32_t nx_fft, ny_fft, nx, ny, fov_x0, fov_y0, cw, ch;
   double frac_x, frac_y;
   uint64_t geometry;
   const iscu_wf_job_kernel* kernels;
   uint32_t n_kernels;
   uint32_t n_planes;
   const iscu_wf_job_plane* planes;
   const iscu_wf_job_dep* deps;            /* channel c: deps[channel_start[c] .. channel_start[c + 1]) */
   const uint32_t* channel_start;          /* n_channels + 1 entries */
   uint32_t n_channels;
   uint32_t reserved;
} iscu_wf_job_desc;
int iscu_wf_job_create(iscu_ctx* ctx, uint64_t budget_bytes, iscu_wf_job** out);
void iscu_wf_job_destroy(iscu_wf_job* job);
int iscu_wf_job_has_plane(iscu_wf_job* job, uint64_t geometry, uint64_t key);
int iscu_wf_job_fits(iscu_wf_job* job, uint64_t geometry, uint32_t nx_fft, uint32_t ny_fft, uint64_t planes);
int iscu_wf_job_images(iscu_wf_job* job, const iscu_wf_job_desc* desc, float* const* images);
/* The same on device buffers (the camera maps of iscu_set_static apply when their size is nx x ny). */
int iscu_wf_render_dev(iscu_wf_plan* plan, const float* density_dev, double background, const iscu_camera* cam,
                       uint32_t seed, uint32_t frame0, float* image_dev, uint16_t* adu_dev);

/* ---------------------------------------------------------------- the named-kernel backend ---------------------- */

/* sim::GpuBackend (WidefieldGpuHost.h:42-77) on the device, so that the reference's hosts over it -- SplatGpuHost
 * (SplatGpu.h:40-75) and WidefieldGpuHost (WidefieldGpuHost.h:79-114), self-checks included -- run unmodified:
 * storage buffers of 32-bit words, and the kernels those hosts dispatch by name, with their parameter blocks (up to
 * 16 words), their buffers bound in order and their dispatch sizes in workgroups:
 *   splat_frames (SplatGpu.wgsl; 16 x 16 pixels a workgroup, 7 buffers: 4 block-sum buffers, Stat, Dyn, Out),
 *   wf_clear, wf_scatter, wf_mac (256 invocations a workgroup), wf_fft (256, one transform of n <= 2048 a
 *   workgroup), wf_split, wf_expand, wf_crop, wf_frame (16 x 16) (WidefieldGpu.wgsl).
 * Each computes what its WGSL source defines, in float32 (the noise chain included: the counter stream's float
 * uniforms, Box-Muller, Knuth / normal Poisson, Marsaglia-Tsang). Every buffer access is checked against the bound
 * buffers' sizes: a read out of range gives 0 and a write out of range is dropped (WebGPU's robust buffer access),
 * and loop counts taken from buffers are bounded by the buffers' sizes, so a malformed dispatch cannot fault or
 * hang; parameters a kernel cannot run with (an FFT length that is not a power of two up to 2048, a zero grid size)
 * fail with ISCU_ERR_ARG. All work runs in order on the context's stream; buffers must be destroyed before their
 * context. */
typedef struct iscu_buffer iscu_buffer;
/* A buffer of bytes rounded up to 4, holding data (bytes of it; nullable: zeros). */
int iscu_buffer_create(iscu_ctx* ctx, size_t bytes, const void* data, iscu_buffer** out);
void iscu_buffer_destroy(iscu_buffer* buf);
size_t iscu_buffer_bytes(const iscu_buffer* buf);
/* bytes of data into buf at offset (the host buffer may be reused when the call returns). */
int iscu_buffer_write(iscu_buffer* buf, size_t offset, const void* data, size_t bytes);
/* The first bytes of src into dst. */
int iscu_buffer_copy(iscu_buffer* dst, const iscu_buffer* src, size_t bytes);
/* The first bytes of src into dst (host), after the work before it. */
int iscu_buffer_read(const iscu_buffer* src, size_t bytes, void* dst);
/* The low 16 bits of src's first `words` words (GpuBackend::ReadBackLow16: the splat's ADU), narrowed on the
 * device so that half the bytes cross to the host. */
int iscu_buffer_read_low16(const iscu_buffer* src, size_t words, uint16_t* dst);
/* GpuBackend::Dispatch: kernel by name, params (n_params <= 16 words; the rest of the block reads 0), bufs in
 * binding order (their count as the kernel's source binds them), x * y * z workgroups (y, z <= 65535). */
int iscu_dispatch(iscu_ctx* ctx, const char* kernel, const uint32_t* params, size_t n_params,
                  iscu_buffer* const* bufs, size_t n_bufs, uint32_t x, uint32_t y, uint32_t z);

/* ---------------------------------------------------------------- movie files ------------------------------------ */

/* The CLI's movie file (TiffWriter, cli/tiff_writer.h), byte for byte: a little-endian baseline TIFF, one
 * uncompressed grey page per frame -- uint16 ADU, or float32 -- with an optional description (the CLI gives one on
 * page 1); a BigTIFF (64-bit offsets) when big_tiff is set or expected_bytes + 64 MB reaches 2^32 - 1, else a
 * classic file that refuses a page that would pass 4 GB. Every page is flushed and checked; a failure leaves the
 * writer failed (ISCU_ERR_IO, the reference writer's message) and the file as written so far. Not thread-safe per
 * writer. iscu_tiff_bytes is TiffWriter::Bytes: an upper bound of a file's size, the expected_bytes to pass. */
typedef struct iscu_tiff iscu_tiff;
uint64_t iscu_tiff_bytes(uint64_t width, uint64_t height, uint64_t pages, uint64_t bytes_per_sample,
                         uint64_t desc_bytes);
int iscu_tiff_open(const char* path, uint64_t expected_bytes, int32_t big_tiff, iscu_tiff** out);
/* Whether the file is a BigTIFF, its pages so far and its bytes (any output NULL). */
int iscu_tiff_info(iscu_tiff* t, int32_t* big, uint64_t* pages, uint64_t* bytes);
/* A page of w x h samples (desc NULL or "": none). */
int iscu_tiff_page_u16(iscu_tiff* t, const uint16_t* px, uint32_t w, uint32_t h, const char* desc);
int iscu_tiff_page_f32(iscu_tiff* t, const float* px, uint32_t w, uint32_t h, const char* desc);
/* A uint16 page of which only rows 0 .. rows - 1 are given (rows x w samples), the rest left for iscu_tiff_rows
 * (TiffWriter::PageRows / Rows: a movie written in strips; the finished file equals whole-page writes). */
int iscu_tiff_page_rows(iscu_tiff* t, const uint16_t* px, uint32_t rows, uint32_t w, uint32_t h, const char* desc);
int iscu_tiff_rows(iscu_tiff* t, uint64_t page, uint32_t y0, uint32_t rows, const uint16_t* px);
/* n_frames uint16 frames of w x h from device memory (after the work enqueued on ctx's stream), one page each,
 * first_desc on the first: the frames cross to the host in chunks of about 8 MB through two page-locked halves
 * that the context keeps for all its writers, the copy of one chunk on a copy stream while the previous one is
 * written. */
int iscu_tiff_pages_dev(iscu_tiff* t, iscu_ctx* ctx, const uint16_t* frames_dev, uint32_t n_frames, uint32_t w,
                        uint32_t h, const char* first_desc);
/* Closes the file and frees the writer; ISCU_ERR_IO when a write (or this close) failed. */
int iscu_tiff_close(iscu_tiff* t);

/* The splat's Fft placement (PlanSplat with PsfInterpMode::Fft, PsfGeneratorBridge.cpp:1441-1456; the reference
 * computes it on the CPU only): for emitters k < n of emitters_dev (z index = plane & 0xFFFF of slot `slot`'s stack),
 * the kernel plane shifted by the emitter's sub-cell offset (FftShiftKernelTile, :1293-1370: g(i) = f(i + s),
 * band-limited, s = t - floor(t + 0.5) of the nearest setup's tap coordinate t per axis) and its block sums
 * (BuildBlockSums) into sums_dev[k * bw * bw ..] (bw = size + os - 1), and origins_dev[4k ..] = (x0, y0, bx, by): the
 * centre pixel and the tap the one-tap splat reads those sums at. An emitter PlanSplat refuses (photons <= 0, a plane
 * outside the stack) gets x0 = INT32_MIN and zero sums. Computed in float64 as the shift's convolution form (no
 * transform); planes up to 157 x 157 samples. */
int iscu_fft_place_dev(iscu_ctx* ctx, int32_t slot, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                       float* sums_dev, int32_t* origins_dev);
/* Frames rendered with the Fft placement (RenderPhotonImage for a kernel whose interpolation is Fft): as
 * iscu_render_frames_dev -- background, every emitter of the frame in list order, the noise chain unless cam is
 * NULL -- with every emitter on slot `slot` (z index = plane & 0xFFFF) placed by iscu_fft_place_dev and splatted at
 * its one tap from its own shifted block sums, inside its square and the slot's halo cut. The placements live in a
 * context buffer of n_emitters x (size + os - 1)^2 floats (batches up to 16 GB of it). */
int iscu_render_fft_frames_dev(iscu_ctx* ctx, int32_t slot, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                               const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                               float* photons_dev, uint16_t* adu_dev);

/* Ground-truth table text. Numbers as sim::AppendCsvNumber writes them (CsvNumber.cpp:13-32): printf's conversion of
 * "%.<p>f" or "%.<p>g" (p one digit) in the "C" locale -- the exact binary value rounded half to even -- at most 47
 * characters, nothing for NaN and infinities; "%d": the value (an integer, |v| < 2^53) as GroundTruth.cpp's Int
 * writes it (std::to_chars). iscu_csv_numbers_dev: n values into 48-byte fields (the text, NUL-padded) and their
 * lengths. */
int iscu_csv_numbers_dev(iscu_ctx* ctx, const double* values_dev, uint32_t n, const char* fmt, char* fields_dev,
                         uint8_t* lengths_dev);
/* A numeric table's rows as GroundTruth's tables lay them out (GroundTruth::FramesCsv, GroundTruth.cpp:307-339):
 * row r = its n_cols cells joined by ',' and ended by '
', cell (r, c) = columns_dev[c * n_rows + r] in format
 * fmts[c] (host array of n_cols <= 64 formats as above). The text goes to out_dev, *out_bytes its length; returns when
 * it is written (synchronizes). When it needs more than out_capacity bytes, the first out_capacity are written,
 * *out_bytes says how many it needs and the call returns ISCU_ERR_LIMIT. */
int iscu_csv_table_dev(iscu_ctx* ctx, const double* columns_dev, uint32_t n_rows, uint32_t n_cols,
                       const char* const* fmts, char* out_dev, uint64_t out_capacity, uint64_t* out_bytes);

/* ------------------------------------------------------- binned blinks (approximate SMLM) ----------------------- */

/* sim::BinnedBlinkRenderer (BinnedBlinks.h:35-60, BinnedBlinks.cpp:150-248): a frame's emitters deposited at the
 * nearest cell of a grid of u cells per camera pixel (cell floor((x + 0.5) u), per axis), one density per PSF plane,
 * each convolved with that plane's kernel at the cell pitch out to R cells, summed, max(0, .) per cell, u x u cells
 * summed into each pixel. The plane kernels are KernelWidefieldPsf::Kernel (WidefieldRender.cpp:300-322): cell
 * (dx, dy) = the sum of the oversampled plane over the r x r block from (s0 + dx r, s0 + dy r), r = os / u,
 * s0 = floor((n - 1) / 2 - r / 2 + 1); R the kernel's reach (KernelWidefieldPsf::Radius), capped by the slot's halo
 * cut at ceil((sqrt(max radius2) + 1) u). The convolution is a direct sum in float64 (the reference runs it as float
 * FFTs over a grid padded by R; the two agree to the float FFT's rounding).
 * create: kernel slot `slot` (u = the largest divisor of its oversampling up to `upscale`,
 * KernelWidefieldPsf::ValidUpscale) or, slot < 0, the in-focus Gaussian of sigma_px (u = upscale clamped to 1..8,
 * R = ceil(3 sigma u), exp(-(x^2 + y^2) / (2 (sigma u)^2)) normalized to sum 1), for width x height frames. */
typedef struct iscu_binned iscu_binned;
int iscu_binned_create(iscu_ctx* ctx, int32_t slot, double sigma_px, uint32_t width, uint32_t height,
                       int32_t upscale, iscu_binned** out);
/* The renderer's u (cells per pixel), R (kernel radius in cells) and plane count (any output NULL). */
int iscu_binned_info(iscu_binned* b, int32_t* upscale, int32_t* radius_cells, int32_t* planes);
/* The plane kernels, nz x (2R + 1)^2 floats (row-major, dy outer), into host memory. */
int iscu_binned_kernels(iscu_binned* b, float* out);
void iscu_binned_destroy(iscu_binned* b);
/* Frames k < n_frames of a batch (as iscu_render_frames_dev: frame k's emitters are emitters_dev[em_start ..
 * em_start + em_count), z index = plane & 0xFFFF, clamped to the kernel's planes; emitters with photons <= 0 and
 * those whose cell lies more than R outside the frame are skipped): img_dev[k * w * h ..] += the binned photon image
 * (BinnedBlinkRenderer::Render); alone_dev (nullable) += the same values. */
int iscu_binned_render_dev(iscu_binned* b, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                           const iscu_frame* frames_dev, uint32_t n_frames, float* img_dev, float* alone_dev);

#ifdef __cplusplus
}
#endif

#endif /* ISCU_H */
