#!/usr/bin/env python
"""Benchmark of the B200 image-formation engine; prints ONE JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload smlm]

Workload `smlm` (the plain dSTORM SMLM render): one step renders a 200-frame 128 x 128 sCMOS movie -- every frame's
background, ~160 Catmull-Rom PSF splats and the sCMOS noise chain -- from emitter records resident in HBM
(`value`: the autotuned render form, replayed from a CUDA graph of the batch), and end to end from host blink events to host ADU frames through the C ABI (`e2e`: emitter collection,
host->device copy, render, device->host copy). Frames shard across ranks (weak scaling: each rank renders its own
200 frames; no collective on the data path). L2 is flushed (a 256 MB write) before every timed step.

--impl reference: the reference's own CPU renderer (RenderPhotonImage + ApplyNoiseChain under its ParallelFor,
compiled from its sources: oracle/_ref) on all host cores, same workload and metric; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


# ----------------------------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while len(self.lines) < 2 and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
            self.skip = len(self.lines)   # samples from before the timed region
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        lines = self.lines[getattr(self, "skip", 0):] or self.lines[-1:]
        for l in lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the dominant kernels, from one ncu
# capture each; the summaries with their commands are the named files.
NCU_TRAFFIC = {
    ("smlm", "GatherTilesKernel"): (138334464, "profiles/GatherTilesKernel_smlm_dstorm.md"),
    ("smlm", "ContribKernel"): (96654336, "profiles/ContribKernel_smlm_dstorm.md"),
    ("psflib", "CztTf32x3Kernel"): (52487168, "profiles/CztTf32x3Kernel_psf_library.md"),
    ("psflib", "CztF16x3Kernel"): (28717824, "profiles/CztF16x3Kernel_psf_library.md"),
    ("two-colour", "GatherTilesKernel"): (2182043649, "profiles/GatherTilesKernel_two_colour.md"),
    ("widefield", "WfNoiseKernel"): (73900000, "profiles/widefield_cells_launches.md"),
    ("widefield", "ZKernel<convolve>"): (1046200000, "profiles/widefield_cells_launches.md"),
    ("wfshift", "ShiftColumnsKernel+ShiftRowsKernel"): (636056576, "profiles/shift_frames_launches.md"),
}


# ----------------------------------------------------------------------------------------------------- dist
def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------------------------------------------- SMLM
class SmlmWorkload:
    name = "smlm-dstorm sCMOS 128x128 px, 200 frames, 4000 sites, ~160 ON/frame, 129^2x49 cubic PSF"
    metric = "frames/s"

    FRAMES_PER_RANK = 200

    def __init__(self, rank: int):
        from insiliscope_b200.shard import frame_range
        from insiliscope_b200.workloads import smlm_dstorm
        # weak scaling: the whole job renders a 200 N-frame movie, rank r its frame_range (200 frames from 200 r)
        world = int(os.environ.get("WORLD_SIZE", "1"))
        first, end = frame_range(rank, world, self.FRAMES_PER_RANK * world)
        self.mv = smlm_dstorm(seed=42, frames=end - first, frame0=first)
        self.frame0 = first

    # -------------------------------------------------- ours
    def setup(self, device: int, form=None):
        import torch
        from insiliscope_b200 import CZT_FP32, Engine, generate_camera_maps
        mv = self.mv
        self.eng = eng = Engine(device)
        t0 = time.perf_counter()
        for slot, psf in enumerate(self.psfs()):
            eng.kernel_build(slot, psf, CZT_FP32)
        eng.synchronize()
        self.psf_build_ms = (time.perf_counter() - t0) * 1e3
        off, gain, rn = generate_camera_maps(mv.width, mv.height, mv.map_seed, mv.offset_mean, mv.offset_std,
                                             mv.gain_nominal, mv.gain_std_fraction, mv.read_noise_nominal,
                                             mv.read_noise_std_fraction)
        eng.set_static(mv.width, mv.height, offset=off, gain=gain, read_noise=rn, flat_bg=mv.background)
        self.ems, self.frames, _ = eng.collect_emitters(self.slot, mv.events, mv.bucket_start, self.frame0,
                                                        mv.width, mv.height, mv.pixel_nm, mv.photons_per_blink)
        self.ems = self.ems.copy()
        dev = f"cuda:{device}"
        self.d_em = torch.from_numpy(self.ems.view(np.uint8)).to(dev)
        self.d_fr = torch.from_numpy(self.frames.view(np.uint8)).to(dev)
        self.d_adu = torch.empty((mv.frames, mv.height, mv.width), dtype=torch.uint16, device=dev)
        t0 = time.perf_counter()
        self.autotune_ms = eng.render_autotune(self.d_em, self.d_fr, mv.frames, mv.camera, mv.noise_seed, self.d_adu)
        self.autotune_wall_ms = (time.perf_counter() - t0) * 1e3
        self.autotuned = eng.render_config()[0]
        if form is not None:
            eng.set_render_config(form)   # a fixed form (profiling runs), the autotuner's table still reported
        self.form = eng.render_config()
        # page-locked host buffers of the end-to-end call: the events and buckets in, the frames out
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).pin_memory().numpy().view(a.dtype)
        self.h_events = pin(mv.events)
        self.h_bucket = pin(np.ascontiguousarray(mv.bucket_start, np.uint32))
        # one page-locked frame buffer per I/O slot of the pipelined run (e2e_run): up to three batches in flight
        self.h_adu_ring = [torch.empty((mv.frames, mv.height, mv.width), dtype=torch.uint16).pin_memory().numpy()
                           for _ in range(3)]
        self.h_adu = self.h_adu_ring[0]
        self.stream = eng.torch_stream()
        self.frames_per_step = mv.frames
        self.n_emitters = len(self.ems)
        # one step replays the batch's render (the form above) captured in a CUDA graph
        from insiliscope_b200 import RenderGraph
        self.graph = RenderGraph(eng, self.d_em, self.d_fr, mv.frames, mv.camera, mv.noise_seed, None, self.d_adu)

    slot = 0

    def direct_step(self):
        """The render launched directly (no graph): the pass timing and the plain-form comparison use it."""
        self.eng.render_frames_dev(self.d_em, self.d_fr, self.mv.frames, self.mv.camera, self.mv.noise_seed,
                                   None, self.d_adu, sync=False)

    def device_step(self):
        self.graph.launch(sync=False)

    def e2e_step(self):
        """Host blink events (page-locked) -> host ADU frames (page-locked) in one C-ABI call: H2D of the events,
        emitter collection, render and noise on the device, D2H of the frames."""
        mv = self.mv
        _, adu, _ = self.eng.render_events(self.slot, self.h_events, self.h_bucket, self.frame0, mv.pixel_nm,
                                           mv.photons_per_blink, mv.camera, mv.noise_seed, adu_out=self.h_adu)
        return adu

    def e2e_run(self, steps):
        """steps end-to-end steps pipelined over the I/O slots (iscu_render_events_async / _wait): each step's events
        go up, are collected, rendered and noised, and its frames come down into the slot's page-locked buffer, while
        the copies of one step run beside the kernels of the next. Returns when every step's frames are on the host."""
        mv = self.mv
        depth = len(self.h_adu_ring)
        for i in range(steps):
            io = i % depth
            if i >= depth:
                self.eng.render_events_wait(io)
            self.eng.render_events_async(io, self.slot, self.h_events, self.h_bucket, self.frame0, mv.pixel_nm,
                                         mv.photons_per_blink, mv.camera, mv.noise_seed, adu_out=self.h_adu_ring[io])
        for i in range(max(0, steps - depth), steps):
            self.eng.render_events_wait(i % depth)

    def e2e_bytes(self):
        return self.h_events.nbytes + self.h_bucket.nbytes, self.h_adu.nbytes

    def timing(self, on):
        pass   # graph replays carry no timing marks: dominant() times three direct renders

    def dominant(self):
        """The render's passes, CUDA events inside the library over three direct renders: the slowest, with the
        movie's algorithmic bytes (movie_bytes) as the bytes it is judged by; each pass's own traffic as this design
        moves it (pass_bytes: the two-pass forms' contribution buffer included) in the breakdown."""
        self.eng.set_render_timing(True)
        for _ in range(3):
            self.direct_step()
        ms, calls = self.eng.render_pass_times()
        self.eng.set_render_timing(False)
        name = max(ms, key=ms.get)
        kernel = {"grouping": "ContribSetup/Scan/Scatter", "contributions": "ContribKernel",
                  "tiles": "GatherTilesKernel" if self.form[4] == 2 else "RenderTilesKernel"}[name]
        passes = ("grouping", "contributions", "tiles") if self.form[4] == 2 else ("tiles",)
        return kernel, self.movie_bytes(), ms[name], {"pass_ms": {k: round(v, 4) for k, v in ms.items()},
                                                      "design_bytes": {k: self.pass_bytes(k) for k in passes}}

    def time_render(self, form, reps=5, graph=None):
        """ms per render of the batch in render form `form` (direct launches; or a captured graph's replays)."""
        import torch
        if graph is None:
            self.eng.set_render_config(form)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        step = graph.launch if graph is not None else self.direct_step
        with torch.cuda.stream(self.stream):
            step() if graph is None else step(sync=False)
            s.record(self.stream)
            for _ in range(reps):
                step() if graph is None else step(sync=False)
            e.record(self.stream)
        e.synchronize()
        return s.elapsed_time(e) / reps

    def plain_form(self, step_ms):
        """The batching pattern against the plain form on this GPU: the autotuned form (launched directly and, where
        the step replays a captured graph, as the step), the same tile's persistent heaviest-frame-first form, and
        the plain grid form (form 0: one pass, one CTA per 16 x 16 tile, no persistence, no graph)."""
        auto = self.form[0]
        persistent = 6 * (auto // 6) + 3 + auto % 3
        grid = 6 * (auto // 6) + auto % 3
        out = {"step_ms": round(step_ms, 4), "autotuned_form": auto,
               "autotuned_direct_ms": round(self.time_render(auto), 4),
               "persistent_form": persistent, "persistent_ms": round(self.time_render(persistent), 4),
               "grid_form": grid, "grid_ms": round(self.time_render(grid), 4),
               "plain_form": 0, "plain_ms": round(self.time_render(0), 4)}
        self.eng.set_render_config(auto)
        out["graph_replay_ms"] = round(self.time_render(None, graph=self.graph), 4)
        out["speedup_vs_plain"] = round(out["plain_ms"] / step_ms, 3)
        return out

    def movie_bytes(self):
        """The step's algorithmic HBM bytes: per frame the ADU written (2 B/px) and the camera maps read as one float4
        per pixel (16 B/px), per emitter its 64-byte device record; the kernels' block sums (L2-resident) once."""
        mv = self.mv
        sums = 0
        for s in self.slots_used():
            _, nz, _, bw = self.eng.kernel_info(s)
            sums += nz * bw * bw * 4
        return mv.frames * mv.width * mv.height * 18 + self.n_emitters * 64 + sums

    def pass_bytes(self, name):
        """Algorithmic HBM bytes of a render pass. Tiles: the ADU written (2 B/px per frame), the three float camera
        maps read once (12 B/px), the frame table, each emitter's setup record (16 B), and every (emitter, square pixel)
        contribution read once (4 B; the two-pass forms) or the emitter records (32 B; one pass). Contributions: each
        emitter's staged record (88 B) read and its square's contributions written (4 B/px). Grouping: the emitter
        records read (32 B) and their setup and staged records written (96 + 16 + 88 B)."""
        mv = self.mv
        px = mv.width * mv.height
        two = self.form[4] == 2
        def side(s):
            size, _, os_, _ = self.eng.kernel_info(s)
            return 2 * (((size - 1) // 2) // os_) + 1
        sq = sum(side(s) ** 2 for s in self.slots_used()) / len(self.slots_used())
        if name == "tiles":
            per_em = 16 + 4 * sq if two else 32
            return mv.frames * (px * 2 + 24) + px * 12 + self.n_emitters * per_em
        if name == "contributions":
            return self.n_emitters * (88 + 4 * sq)
        return self.n_emitters * (32 + 96 + 16 + 88)

    def psfs(self):
        return [self.mv.psf]

    def slots_used(self):
        return list(range(len(self.psfs())))

    def config_extra(self):
        tw, th = self.form[1], self.form[2]
        return {"render_form": {"config": self.form[0], "tile": f"{tw}x{th}", "persistent": self.form[3],
                                "passes": 2 if self.form[4] == 2 else 1, "autotuned_config": self.autotuned,
                                "autotune_ms_per_form": [round(x, 4) for x in self.autotune_ms]},
                "mean_emitters_per_frame": self.n_emitters / self.mv.frames,
                "max_emitters_per_frame": int(self.frames["em_count"].max()), "cuda_graph": True}

    def alg_bytes_per_launch(self):
        return self.movie_bytes()

    # -------------------------------------------------- the reference on the host cores
    dtype = "f64"
    cpu_kind = "reference"
    cpu_sample = ("the whole 200-frame movie per step: the reference's RenderPhotonImage + ApplyNoiseChain per frame, "
                  "frames in parallel on its own thread pool (ParallelFor), PSF kernel built once before timing as the "
                  "reference memoizes it")
    frames_per_step_cpu = 200

    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        mv = self.mv
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)
        self.rk = self.ref.kernel(req=mv.psf)
        # the reference's own map generators (PixelOffsetMap / GainMap / ReadNoiseMap), nothing of this package
        self.maps = self.ref.camera_maps(mv.width, mv.height, mv.map_seed, mv.offset_mean, mv.offset_std,
                                         mv.gain_nominal, mv.gain_std_fraction, mv.read_noise_nominal,
                                         mv.read_noise_std_fraction)

    def reference_step(self):
        mv = self.mv
        t, _, adu = self.rk.render_movie(mv.events, self.frame0, mv.frames, mv.width, mv.height, mv.pixel_nm,
                                         mv.photons_per_blink, mv.background, mv.camera, *self.maps, mv.noise_seed)
        return t


class TwoColourWorkload(SmlmWorkload):
    """The uneven two-colour movie: 256 x 256 px, 1,024 frames of 10 to ~8,000 ON emitters (Poisson, lognormal
    per-frame mean), channel 0 (670 nm double helix) then channel 1 (580 nm astigmatic) splatted onto each frame,
    then the sCMOS chain. The render form (tile shape, grid or persistent heaviest-frame-first, one or two passes) is
    autotuned once on the batch, and one step replays the batch's render captured in a CUDA graph."""
    name = ("two-colour uneven SMLM 256x256 px, 1024 frames, Poisson ON counts with lognormal per-frame mean "
            "(median 300, clipped 10-8000), 670 nm double-helix + 580 nm astigmatic (Noll 5 = 0.1 lambda) 129^2x49 "
            "cubic PSFs, sCMOS")
    slot = -1

    def __init__(self, rank: int):
        from insiliscope_b200.workloads import two_colour_uneven
        self.frame0 = rank * 1024
        self.mv = two_colour_uneven(seed=42, frame0=self.frame0)

    def psfs(self):
        return self.mv.psfs

    cpu_sample = ("the movie's last 256 frames per step (25 % of its emitters, its heaviest frame among them): per "
                  "frame the reference's RenderPhotonImage for channel 0, then for channel 1 accumulating onto it "
                  "(each with its own kernel), then ApplyNoiseChain; frames in parallel on its own thread pool "
                  "(ParallelFor), kernels built once before timing")
    frames_per_step_cpu = 256

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        mv = self.mv
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)
        self.rks = [self.ref.kernel(req=p) for p in mv.psfs]
        self.maps = self.ref.camera_maps(mv.width, mv.height, mv.map_seed, mv.offset_mean, mv.offset_std,
                                         mv.gain_nominal, mv.gain_std_fraction, mv.read_noise_nominal,
                                         mv.read_noise_std_fraction)

    def reference_step(self):
        mv = self.mv
        first = self.frame0 + mv.frames - self.frames_per_step_cpu
        t, _, _ = self.ref.render_movie_groups(self.rks, mv.events, first, self.frames_per_step_cpu, mv.width,
                                               mv.height,
                                               mv.pixel_nm, mv.photons_per_blink, mv.background, mv.camera,
                                               *self.maps, mv.noise_seed)
        return t


class WidefieldWorkload:
    """The widefield mean-field focus series as the reference's widefield scene: a 512 x 512 x 64 dye grid of
    100 x 100 x 200 nm cells imaged at every plane's centre through the 3D Gibson-Lanni kernel stack (513 x 513
    samples, 65 planes 200 nm apart, built on the device; a dye plane beyond the stack's reach seen through its last
    plane, as PlanFocus clamps), the kernel radius uncapped (256 cells), linear convolution on a 1024 x 1024 x 128 FFT
    grid, max(0, .) + 5 photons/px background, EMCCD chain; one step = 64 frames."""
    name = ("widefield 3D FFT convolution 512x512x64 volume (50 cells, nuclei, 200 filaments each) x 513x513x65 "
            "Gibson-Lanni kernel stack (NA 1.4, 520 nm), EMCCD gain 300, 5 photons/px background")
    metric = "frames/s"

    # pass names and their algorithmic bytes (computed in setup)
    PASSES = ("XForwardKernel", "YForwardKernel", "ZKernel<convolve>", "YInverseKernel", "XInverseKernel",
              "WfNoiseKernel")
    e2e_stages = "the six FFT-convolution and noise passes"
    KERNEL_CAP_UM = 30.0

    def __init__(self, rank: int):
        from insiliscope_b200.workloads import widefield_cells
        self.rank = rank
        self.wv = widefield_cells(seed=42 + rank)
        self.frame0 = rank * 64
        req = self.wv.psf
        req.nz = 65
        req.kernel_half_width_px = 256
        self.req = req

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import CZT_FP32, Engine, WidefieldPlan, generate_camera_maps
        wv = self.wv
        nz, ny, nx = wv.density.shape
        self.eng = eng = Engine(device)
        t0 = time.perf_counter()
        eng.kernel_build(0, self.req, CZT_FP32)
        eng.synchronize()
        self.psf_build_ms = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        self.plan = WidefieldPlan.from_kernel(eng, 0, 1, wv.voxel_nm[0] / 1000.0, self.KERNEL_CAP_UM, wv.voxel_nm[2],
                                              (nz, ny, nx), (0, 0, nx, ny))
        self.plan_ms = (time.perf_counter() - t0) * 1e3
        off, _, _ = generate_camera_maps(nx, ny, wv.map_seed, wv.offset_mean, wv.offset_std, 1.0, 0.0, 50.0, 0.0)
        eng.set_static(nx, ny, offset=off)
        self.d_vol = torch.from_numpy(wv.density).to(f"cuda:{device}")
        self.d_adu = torch.empty((nz, ny, nx), dtype=torch.uint16, device=f"cuda:{device}")
        self.h_vol = torch.from_numpy(wv.density).pin_memory().numpy()
        self.h_adu = torch.empty((nz, ny, nx), dtype=torch.uint16).pin_memory().numpy()
        self.h_adu_ring = [self.h_adu] + [torch.empty((nz, ny, nx), dtype=torch.uint16).pin_memory().numpy()
                                          for _ in range(2)]
        self.stream = eng.torch_stream()
        self.frames_per_step = nz
        self.n_emitters = 0
        G = self.plan.grid()
        NK = G[0] // 2 + 1
        vox = nx * ny * nz
        self.pass_bytes = [vox * 4 + NK * ny * nz * 8,                    # x forward: reals in, half spectra out
                           NK * ny * nz * 8 + NK * G[1] * nz * 8,          # y forward
                           2 * NK * G[1] * nz * 8 + NK * G[1] * G[2] * 8,  # z: spectra in/out + the PSF spectrum
                           NK * G[1] * nz * 8 + NK * ny * nz * 8,          # y inverse
                           NK * ny * nz * 8 + vox * 4,                     # x inverse: photon frames out
                           vox * 4 + vox * 2 + nx * ny * 4]                # noise: photons in, ADU out + offset map

    def device_step(self):
        wv = self.wv
        self.plan.render_dev(self.d_vol, wv.background, wv.camera, wv.noise_seed, self.frame0, None, self.d_adu,
                             sync=False)

    def e2e_step(self):
        wv = self.wv
        self.plan.render(self.h_vol, wv.background, wv.camera, wv.noise_seed, self.frame0, adu=self.h_adu)
        return self.h_adu

    def e2e_run(self, steps):
        """steps end-to-end focus series pipelined over three I/O slots (iscu_wf_render_async / _wait): each step's
        volume goes up, is convolved and noised, and its frames come down into the slot's page-locked buffer, the
        copies of one step beside the passes of the next. Returns when every step's frames are on the host."""
        wv = self.wv
        depth = len(self.h_adu_ring)
        for i in range(steps):
            io = i % depth
            if i >= depth:
                self.plan.render_wait(io)
            self.plan.render_async(io, self.h_vol, wv.background, wv.camera, wv.noise_seed, self.frame0,
                                   adu=self.h_adu_ring[io])
        for i in range(max(0, steps - depth), steps):
            self.plan.render_wait(i % depth)

    def e2e_bytes(self):
        return self.h_vol.nbytes, self.h_adu.nbytes

    def dominant(self):
        """Pass times over 3 steps (CUDA events inside the plan); the slowest pass with its algorithmic bytes."""
        self.plan.set_timing(True)
        times = []
        for _ in range(3):
            self.device_step()
            times.append(self.plan.pass_times())
        self.plan.set_timing(False)
        mean = [statistics.mean(t[i] for t in times) for i in range(len(self.PASSES))]
        i = int(np.argmax(mean))
        return self.PASSES[i], self.pass_bytes[i], mean[i], dict(zip(self.PASSES, [round(m, 4) for m in mean]))

    def alg_bytes_per_launch(self):
        return sum(self.pass_bytes)

    def kernel_name(self):
        return "widefield step (6 passes)"

    def config_extra(self):
        return {"plan_ms": round(self.plan_ms, 3), "fft_grid": list(self.plan.grid()),
                "kernel_radius_cells": self.plan.kernel_radius}

    # -------------------------------------------------- CPU: the reference's widefield scene on the host cores
    dtype = "f32"
    frames_per_step_cpu = 8
    cpu_kind = "reference"
    cpu_sample = ("8 of the 64 foci per step: the reference's WidefieldScene::FocusSeries (its plane and kernel "
                  "spectra cached from the scene's set-up, as the reference keeps them; GPU mode: power-of-two FFTs) "
                  "+ WidefieldImages::Render per focus on its thread pool, then its ApplyNoiseChain (EMCCD) per frame "
                  "with the background; the scene over the reference's own 513 x 513 x 65 kernel stack "
                  "(ComputeZernikePsfPlanes), compiled from its sources")

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        wv = self.wv
        nz, ny, nx = wv.density.shape
        self.ref = Reference()
        self.ref.set_threads(threads)
        self.rk = self.ref.kernel(req=self.req)
        gx, gy, fx, fy = self.rk.wf_grid(1, 0.1, nx, ny, (0.05, 0.05), 0.0, wv.voxel_nm[2])
        counts = np.zeros((nz, gy, gx), np.float32)
        counts[:, fy:fy + ny, fx:fx + nx] = wv.density
        self.scene = self.rk.wf_scene(counts, 1, self.KERNEL_CAP_UM, 0.1, nx, ny, (0.05, 0.05), 0.0, wv.voxel_nm[2],
                                      focus0_um=0.1, gpu_mode=True)
        self.ref_off, _, _ = self.ref.camera_maps(nx, ny, wv.map_seed, wv.offset_mean, wv.offset_std, 1.0, 0.0, 50.0,
                                                  0.0)
        self.ref_off = self.ref_off.reshape(ny, nx)
        self.focus_planes = np.arange(0, nz, nz // self.frames_per_step_cpu)[:self.frames_per_step_cpu]
        self.foci = (self.focus_planes + 0.5) * (wv.voxel_nm[2] / 1000.0)

    def cpu_cores(self):
        return self.ref.threads()

    def reference_step(self):
        wv = self.wv
        t0 = time.perf_counter()
        frames, _ = self.scene.series(self.foci)
        frames += np.float32(wv.background)
        for i, f in enumerate(self.focus_planes):
            self.ref.noise_chain(frames[i], wv.camera, self.ref_off, None, None, wv.noise_seed, self.frame0 + int(f),
                                 parallel=True)
        return time.perf_counter() - t0


class PsfLibraryWorkload:
    """The batched PSF library: 4,096 PSFs (64 z x 4 wavelengths x 16 Noll 4-15 aberration sets), each a 128 x 128
    pupil (float64 OPD/chirp phases) chirp-Z'd to 64 x 64 as two complex products on the tensor cores (FP16 x 3 split
    operands, float32 accumulation in TMEM, the DFT operand resident in shared memory per request set), |E|^2, sum-1
    planes. One step = the whole library. The TF32 x 3 tensor-core form and the plain FP32 GPU form (SIMT complex
    products in shared memory) are timed beside it."""
    name = ("psf library 4096 x (128^2 pupil -> 64^2, NA 1.45, 520/580/670/750 nm, Noll 4-15 ~ N(0, 0.05 wave rms), "
            "64 z at 25 nm), chirp-Z as FP16x3 tcgen05 GEMMs")
    metric = "PSFs/s"
    dtype = "f16x3"
    roofline_kind = "tensor"
    cpu_kind = "reference"
    frames_per_step_cpu = 130
    cpu_sample = ("2 of the library's 64 requests (65 planes each at the reference-native 65 x 65, M = 128): "
                  "ComputeZernikePsfPlanes (float64 Bluestein chirp-Z, planes in parallel on its thread pool)")

    def __init__(self, rank: int):
        from insiliscope_b200.shard import library_shard
        from insiliscope_b200.workloads import psf_library
        # weak scaling: the whole job's library has 64 N z-planes per set (4,096 N PSFs), rank r its contiguous range
        world = int(os.environ.get("WORLD_SIZE", "1"))
        self.lib = library_shard(psf_library(seed=42, n_z=64 * world), rank, world)

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import CZT_F16X3, CZT_FP32, CZT_TF32X3, Engine, PsfPlan
        L = self.lib
        self.eng = eng = Engine(device)
        t0 = time.perf_counter()
        self.plan = PsfPlan(eng, L.sets, size=L.size, method=CZT_F16X3)
        self.psf_build_ms = (time.perf_counter() - t0) * 1e3
        self.plan32 = PsfPlan(eng, L.sets, size=L.size, method=CZT_FP32)
        self.plan_tf32 = PsfPlan(eng, L.sets, size=L.size, method=CZT_TF32X3)
        n = len(L.set_of_psf)
        dev = f"cuda:{device}"
        self.d_set = torch.from_numpy(L.set_of_psf.view(np.int32)).to(dev)
        self.d_dz = torch.from_numpy(L.defocus_nm).to(dev)
        self.d_out = torch.empty((n, L.size, L.size), dtype=torch.float32, device=dev)
        self.h_out = torch.empty((n, L.size, L.size), dtype=torch.float32).pin_memory().numpy()
        self.stream = eng.torch_stream()
        self.frames_per_step = n
        self.n_emitters = 0

    def device_step(self):
        self.plan.run_dev(self.d_set, self.d_dz, self.d_out, sync=False)

    def timing(self, on):
        if not on:   # after the timed steps: keep the library they made for the accuracy check
            self.h_acc = self.d_out.cpu().numpy()

    def e2e_step(self):
        L = self.lib
        self.plan.run(L.set_of_psf, L.defocus_nm, out=self.h_out)
        return self.h_out

    def e2e_bytes(self):
        return self.lib.set_of_psf.nbytes + self.lib.defocus_nm.nbytes, self.h_out.nbytes

    def flops_per_launch(self):
        P, M = self.plan.P, self.plan.M
        return 8.0 * (P * M * M + P * P * M) * self.frames_per_step   # 8 real flops per complex MAC

    def time_plan(self, plan, reps=5):
        import torch
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            plan.run_dev(self.d_set, self.d_dz, self.d_out, sync=False)   # warm
            s.record(self.stream)
            for _ in range(reps):
                plan.run_dev(self.d_set, self.d_dz, self.d_out, sync=False)
            e.record(self.stream)
        e.synchronize()
        return s.elapsed_time(e) / reps

    def dominant(self):
        self.plan.check()
        ms = self.time_plan(self.plan)
        return "CztF16x3Kernel", self.flops_per_launch(), ms, {"f16x3_ms": round(ms, 4)}

    def plain_form(self, step_ms):
        """The precision pattern against the plain FP32 form on this GPU: the same library through the SIMT float32
        chirp-Z (both products in shared memory, FP32 FMA)."""
        tc, tf32, fp32 = self.time_plan(self.plan), self.time_plan(self.plan_tf32), self.time_plan(self.plan32)
        return {"f16x3_ms": round(tc, 4), "tf32x3_ms": round(tf32, 4), "plain_fp32_ms": round(fp32, 4),
                "speedup_vs_plain": round(fp32 / tc, 3), "speedup_vs_tf32x3": round(tf32 / tc, 3)}

    def accuracy(self):
        """Every PSF of the library (the device's FP16 x 3 planes) against the float64 oracle: per PSF
        max |I - I64| / max I64 and ||I - I64|| / ||I64||, worst and median over the 4,096."""
        from concurrent.futures import ThreadPoolExecutor
        from oracle.oracle import Oracle
        L = self.lib
        got = self.h_acc
        orc = Oracle()
        n = len(L.set_of_psf)
        err, l2 = np.zeros(n), np.zeros(n)

        def one(si):
            idx = np.nonzero(L.set_of_psf == si)[0]
            if len(idx) == 0:
                return
            want = orc.psf_planes(L.sets[si], L.defocus_nm[idx] * 1e-9, size=L.size, normalize=True)
            d = got[idx].astype(np.float64) - want
            err[idx] = np.abs(d).max(axis=(1, 2)) / want.max(axis=(1, 2))
            l2[idx] = np.sqrt((d ** 2).sum(axis=(1, 2)) / (want ** 2).sum(axis=(1, 2)))

        with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
            list(ex.map(one, range(len(L.sets))))
        return {"psfs": n, "max_rel_err_worst": float(err.max()), "max_rel_err_median": float(np.median(err)),
                "rel_l2_worst": float(l2.max()), "target": 1e-5, "against": "float64 oracle (direct DFT chirp-Z)"}

    def alg_bytes_per_launch(self):
        return self.frames_per_step * self.lib.size ** 2 * 4

    def kernel_name(self):
        return "CztF16x3Kernel"

    # -------------------------------------------------- the reference's CPU PSF on the host cores
    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)
        self.reqs = []
        for s in self.lib.sets[:2]:
            r = type(s)(**{k: getattr(s, k) for k in s.__dataclass_fields__})
            r.nz = 65
            self.reqs.append(r)

    def reference_step(self):
        t0 = time.perf_counter()
        for r in self.reqs:
            self.ref.zernike_planes(r)
        return time.perf_counter() - t0


class NllGradWorkload:
    """The Poisson-likelihood gradient: 256 frames x 1,000 emitters, each in a 32 x 32 px ROI (64 x 64 sub-pixel
    samples from a 32 x 32 pupil), per emitter x, y, z, N, one background per frame, 21 Zernike coefficients. One step
    = the NLL and its adjoint gradient (the field recomputed per emitter) for all 256 frames; the data (Poisson counts
    drawn by the engine's noise chain) stay resident, the parameters come in and the gradients go out."""
    name = ("poisson NLL + adjoint gradient, 256 frames x 1000 emitters, 32x32 px ROIs (64^2 samples, 32^2 pupil), "
            "x/y/z/N, 256 backgrounds, 21 Zernike (Noll 4-24)")
    metric = "frames/s"
    dtype = "f32"
    cpu_kind = "port"
    frames_per_step_cpu = 2
    cpu_sample = ("2 of the 256 frames (2,000 ROIs): the float64 adjoint of oracle/nll_oracle.py (numpy, batched "
                  "matmuls), data drawn by numpy's Poisson at the float64 expectation")

    def __init__(self, rank: int):
        from insiliscope_b200.nll import shard_problem
        from insiliscope_b200.workloads import nll_rois
        # N ranks: one problem of 256 N frames, each rank its 256 (weak scaling); the Zernike gradient is summed
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        whole = nll_rois(seed=42, frames=256 * self.world)
        self.prob = shard_problem(whole, rank, self.world) if self.world > 1 else whole

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import Engine
        from insiliscope_b200.nll import NllModel
        from insiliscope_b200.workloads import nll_counts
        P = self.prob
        self.eng = eng = Engine(device)
        t0 = time.perf_counter()
        self.model = NllModel(eng, P.spec)
        self.psf_build_ms = (time.perf_counter() - t0) * 1e3
        dev = f"cuda:{device}"
        self.counts = nll_counts(eng, self.model, P, device=dev)
        self.d_params = torch.from_numpy(P.params).to(dev)
        self.d_frame = torch.from_numpy(P.frame).to(dev)
        self.d_bg = torch.from_numpy(P.bg).to(dev)
        self.zern = np.ascontiguousarray(P.zern, np.float64)
        n, F = len(P.frame), len(P.bg)
        # [NLL, d/dzern]: the values every rank contributes to, summed over the ranks by one all-reduce
        self.packed = torch.zeros(1 + len(self.zern), dtype=torch.float64, device=dev)
        self.d_nll, self.g_zern = self.packed[:1], self.packed[1:]
        self.d_err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.g_params = torch.empty((n, 4), dtype=torch.float32, device=dev)
        self.g_bg = torch.empty(F, dtype=torch.float64, device=dev)
        pin = lambda a: torch.from_numpy(a).pin_memory()
        self.h_params, self.h_bg = pin(P.params), pin(P.bg)
        self.h_gp = torch.empty((n, 4), dtype=torch.float32).pin_memory()
        self.h_gb = torch.empty(F, dtype=torch.float64).pin_memory()
        self.stream = eng.torch_stream()
        self.frames_per_step = F
        self.n_emitters = n

    def device_step(self):
        from insiliscope_b200.nll import reduce_shared
        self.model.run_dev(self.d_params, self.d_frame, self.d_bg, self.zern, self.counts, self.d_nll, self.d_err,
                           self.g_params, self.g_bg, self.g_zern, sync=False)
        reduce_shared(self.packed)

    def e2e_step(self):
        """Page-locked parameters in, the NLL and every gradient out, through the library's model."""
        import torch
        from insiliscope_b200.nll import reduce_shared
        # the copies on torch's own stream (ordered with the library's by the synchronizing calls)
        self.d_params.copy_(self.h_params, non_blocking=True)
        self.d_bg.copy_(self.h_bg, non_blocking=True)
        self.model.run_dev(self.d_params, self.d_frame, self.d_bg, self.zern, self.counts, self.d_nll, self.d_err,
                           self.g_params, self.g_bg, self.g_zern, sync=True)
        reduce_shared(self.packed)
        self.h_gp.copy_(self.g_params, non_blocking=True)
        self.h_gb.copy_(self.g_bg, non_blocking=True)
        torch.cuda.synchronize()
        return float(self.d_nll.item()), self.g_zern.cpu().numpy()

    def e2e_bytes(self):
        return self.h_params.numel() * 4 + self.h_bg.numel() * 4 + self.zern.nbytes, \
            self.h_gp.numel() * 4 + self.h_gb.numel() * 8 + self.zern.nbytes + 8

    def plain_form(self, step_ms):
        """The differentiation pattern against the plain FP32 form on this GPU: the same gradient by central
        differences of the FP32 forward kernel (no adjoint) -- each ROI's x, y, z and N perturbed for all emitters at
        once (an ROI depends only on its own emitter), every frame's background at once, each Zernike coefficient on
        its own: 2 x (4 + 1 + 21) = 52 forward passes writing the expected counts, and per-ROI NLLs reduced by torch."""
        import torch
        m, k = self.model, self.counts
        mu = torch.empty_like(k)
        nll = torch.zeros(1, dtype=torch.float64, device=k.device)
        fr = self.d_frame.long()
        F = self.d_bg.shape[0]

        def roi_nll(params, bg, zern):
            m.run_dev(params, self.d_frame, bg, zern, k, nll, self.d_err, mu=mu, sync=False)
            return (mu - k * torch.log(mu)).sum(dim=(1, 2))

        def fd():
            with torch.cuda.stream(self.stream):
                gp = torch.empty_like(self.d_params)
                for col, h in enumerate((1e-2, 1e-2, 0.5, None)):
                    hh = h if h is not None else 1e-3 * self.d_params[:, 3]
                    pp, pm = self.d_params.clone(), self.d_params.clone()
                    pp[:, col] += hh
                    pm[:, col] -= hh
                    gp[:, col] = (roi_nll(pp, self.d_bg, self.zern) - roi_nll(pm, self.d_bg, self.zern)) / (2 * hh)
                hb = 1e-3 * self.d_bg
                dp = roi_nll(self.d_params, self.d_bg + hb, self.zern) - roi_nll(self.d_params, self.d_bg - hb,
                                                                                self.zern)
                gb = torch.zeros(F, dtype=torch.float32, device=k.device).index_add_(0, fr, dp) / (2 * hb)
                gz = []
                for j in range(len(self.zern)):
                    zp, zm = self.zern.copy(), self.zern.copy()
                    zp[j] += 1e-4
                    zm[j] -= 1e-4
                    gz.append((roi_nll(self.d_params, self.d_bg, zp).sum() -
                               roi_nll(self.d_params, self.d_bg, zm).sum()) / 2e-4)
                return gp, gb, torch.stack(gz)

        fd()   # warm
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(self.stream)
        fd()
        e.record(self.stream)
        e.synchronize()
        fd_ms = s.elapsed_time(e)
        return {"adjoint_ms": round(step_ms, 4), "plain_central_differences_ms": round(fd_ms, 4),
                "forward_passes_plain": 52, "speedup_vs_plain": round(fd_ms / step_ms, 3)}

    def alg_bytes_per_launch(self):
        # the counts read once (4 B per ROI pixel), per emitter its parameters in and gradients out (32 B)
        R = self.prob.spec.roi
        return self.n_emitters * (R * R * 4 + 32) + self.frames_per_step * 12

    def kernel_name(self):
        return "NllKernel"

    def cpu_cores(self):
        return os.cpu_count() or 1

    def reference_setup(self, threads=0):
        from oracle.nll_oracle import NllSpec, expected, tables
        P = self.prob
        self.ospec = NllSpec()
        self.t = tables(self.ospec)
        sel = P.frame < 2
        self.s_params = P.params[sel].astype(np.float64)
        self.s_frame = P.frame[sel]
        self.s_bg = P.bg.astype(np.float64)[:2]
        mu = expected(self.ospec, P.params_true[sel].astype(np.float64), self.s_frame,
                      P.bg_true.astype(np.float64)[:2], P.zern_true, self.t)
        self.s_counts = np.random.default_rng(P.noise_seed).poisson(mu).astype(np.float64)

    def reference_step(self):
        from oracle.nll_oracle import gradient
        t0 = time.perf_counter()
        gradient(self.ospec, self.s_params, self.s_frame, self.s_bg, self.prob.zern, self.s_counts, self.t)
        return time.perf_counter() - t0


class ScheduleWorkload:
    """The step before the render: the blinks of 1,048,576 dSTORM dyes (the world core's schedules: first
    activation, ON / dark cycles with log-normal brightness, bleaching) overlapping one 1 s window late in a movie,
    [100, 101) s, so each dye's schedule is walked from its activation. The dyes stay resident; one step = the count,
    scan and row passes of iscu_dye_blinks_dev. e2e: page-locked dyes in, the window's event rows out."""
    name = ("blink schedules: 1,048,576 dSTORM dyes (activation 0.05/s, ON 40 ms, dark 2 s, bleach 0.3, photon CV "
            "0.5, initial ON 0.2 s), events of the window [100, 101) s")
    metric = "dyes/s"
    dtype = "f64"
    cpu_kind = "reference"
    KIN = [0.05, 0.04, 2.0, 0.3, 0.5, 0.2]
    T0, T1 = 100.0, 101.0

    def __init__(self, rank: int):
        from insiliscope_b200 import DYE_DTYPE
        rng = np.random.default_rng(42 + rank)
        n = 1 << 20
        d = np.zeros(n, DYE_DTYPE)
        d["h1"] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        d["k"] = rng.integers(0, 13, n)
        d["n"] = rng.integers(0, 5000, n)
        d["id"] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        d["x"], d["y"], d["z"] = rng.uniform(-50, 50, (3, n))
        self.dyes = d
        self.frames_per_step_cpu = 1 << 17
        self.cpu_sample = (f"{self.frames_per_step_cpu} of the 1,048,576 dyes per step: the core's LabelSchedule per "
                           "dye (dyes.cpp, compiled from its sources) on the reference's thread pool (ParallelFor)")

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import EVENT_STRIDE, LABEL_DSTORM, Engine
        self.eng = eng = Engine(device)
        self.mode = LABEL_DSTORM
        dev = f"cuda:{device}"
        n = len(self.dyes)
        self.d_dyes = torch.from_numpy(self.dyes.view(np.uint8)).to(dev)
        self.d_n = torch.zeros(1, dtype=torch.int32, device=dev)
        self.d_first = torch.zeros(n + 1, dtype=torch.int32, device=dev)
        eng.dye_blinks_dev(self.mode, self.KIN, self.d_dyes, n, self.T0, self.T1, None, self.d_n,
                           dye_first_dev=self.d_first)
        self.n_rows = int(self.d_n.item())
        self.d_rows = torch.empty((max(1, self.n_rows), EVENT_STRIDE), dtype=torch.float64, device=dev)
        self.h_dyes = torch.from_numpy(self.dyes.view(np.uint8)).pin_memory()
        self.h_rows = torch.empty((max(1, self.n_rows), EVENT_STRIDE), dtype=torch.float64).pin_memory()
        self.stream = eng.torch_stream()
        self.frames_per_step = n
        self.n_emitters = self.n_rows
        self.psf_build_ms = 0.0

    def device_step(self):
        self.eng.dye_blinks_dev(self.mode, self.KIN, self.d_dyes, len(self.dyes), self.T0, self.T1, self.d_rows,
                                self.d_n, dye_first_dev=self.d_first, sync=False)

    def e2e_step(self):
        """Page-locked dyes in, the window's rows out; the copies on torch's own stream, ordered with the library's by
        the synchronizing call (a pinned block used on the library's stream would outlive that stream)."""
        import torch
        self.d_dyes.copy_(self.h_dyes, non_blocking=True)
        self.eng.dye_blinks_dev(self.mode, self.KIN, self.d_dyes, len(self.dyes), self.T0, self.T1, self.d_rows,
                                self.d_n, dye_first_dev=self.d_first, sync=True)
        self.h_rows.copy_(self.d_rows, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_rows

    def e2e_bytes(self):
        return self.h_dyes.numel(), self.h_rows.numel() * 8

    def kernel_name(self):
        return "CountKernel+ScanSumsKernel+ScanOffsetsKernel+ScanWriteKernel+RowsKernel"

    def alg_bytes_per_launch(self):
        # the dyes read by the count and the row pass (48 B each), per-dye counts and first rows (8 B), the rows (80 B)
        return len(self.dyes) * (2 * 48 + 8) + self.n_rows * 80

    def config_extra(self):
        return {"rows_per_step": self.n_rows}

    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)

    def reference_step(self):
        _, sec = self.ref.dye_blinks_batch(0, self.KIN, self.dyes[:self.frames_per_step_cpu], self.T0, self.T1)
        return sec


class WfShiftWorkload:
    """Frames of a drifting widefield sample (RenderShiftedImages, a next-row widefield extra): 64 frames on a 1024 x
    1024 grid from 6 channels' spectra (two foci of a persistent and two bleaching populations), each frame its own
    bleach coefficients, focus weight and xy drift (sub-cell pose included), a 1024 x 1024 window at 2 cells per pixel
    -> 512 x 512 camera frames. The spectra stay resident; one step = iscu_wf_shifted_frames_dev. e2e: the frames'
    coefficients and shifts in, the camera frames out."""
    name = ("drifting widefield frames: 64 frames from 6 channel spectra on a 1024x1024 grid (two foci, bleach "
            "basis, drift phase ramp), 2 cells per pixel -> 512x512")
    metric = "frames/s"
    dtype = "f32"
    cpu_kind = "reference"
    NX = NY = 1024
    UP = 2

    def __init__(self, rank: int):
        rng = np.random.default_rng(42 + rank)
        nx, ny = self.NX, self.NY
        fy = np.fft.fftfreq(ny)[:, None]
        fx = np.fft.rfftfreq(nx)[None, :]
        band = np.exp(-(fx ** 2 + fy ** 2) / (2 * 0.08 ** 2))
        self.spectra = np.stack([(np.fft.rfft2(rng.random((ny, nx)).astype(np.float32) ** 4 * 50) * band)
                                 .astype(np.complex64) for _ in range(6)])
        n = 64
        self.a = rng.uniform(0.2, 1.0, (n, 2))
        self.w = rng.uniform(0.0, 1.0, n)
        self.drift = rng.uniform(-6.0, 6.0, (n, 2))
        self.frac = (0.25, -0.125)
        f32 = np.float32
        coef = np.zeros((n, 6), np.float32)
        for f in range(n):
            w0, w1 = f32(1.0 - self.w[f]), f32(self.w[f])
            coef[f] = [w0, f32(self.a[f, 0]) * w0, f32(self.a[f, 1]) * w0, w1, f32(self.a[f, 0]) * w1,
                       f32(self.a[f, 1]) * w1]
        self.coef = coef
        self.shift = np.stack([self.frac[0] - self.drift[:, 0], self.frac[1] - self.drift[:, 1]], axis=1)
        self.window = (0, 0, nx, ny)
        self.frames_per_step_cpu = 8
        self.cpu_sample = ("8 of the 64 frames per step: the reference's RenderShiftedImages (WidefieldRender.cpp, "
                           "RealFft2d's float transforms on its thread pool; compiled from its sources) per frame")

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import Engine, WidefieldShift
        self.eng = Engine(device)
        dev = f"cuda:{device}"
        self.plan = WidefieldShift(self.eng, self.NX, self.NY)
        self.d_spec = torch.from_numpy(self.spectra).to(dev)
        self.d_coef = torch.from_numpy(self.coef).to(dev)
        self.d_shift = torch.from_numpy(self.shift).to(dev)
        n = len(self.coef)
        shape = (n, self.NY // self.UP, self.NX // self.UP)
        self.d_cam = torch.zeros(shape, dtype=torch.float32, device=dev)
        self.h_coef = torch.from_numpy(self.coef).pin_memory()
        self.h_shift = torch.from_numpy(self.shift).pin_memory()
        self.h_cam = torch.empty(shape, dtype=torch.float32).pin_memory()
        self.stream = self.eng.torch_stream()
        # end-to-end pipeline: two slots of inputs and frames on the device and the host, a copy stream for the frames
        self.d_coef_io = [torch.empty_like(self.d_coef) for _ in range(2)]
        self.d_shift_io = [torch.empty_like(self.d_shift) for _ in range(2)]
        self.d_cam_io = [torch.empty_like(self.d_cam) for _ in range(2)]
        self.h_cam_io = [torch.empty(shape, dtype=torch.float32).pin_memory() for _ in range(2)]
        self.copy_stream = torch.cuda.Stream(device=dev)
        self.up_stream = torch.cuda.Stream(device=dev)   # (page-locked copies stay off the library's stream)
        self.uploaded = [torch.cuda.Event() for _ in range(2)]
        self.rendered = [torch.cuda.Event() for _ in range(2)]
        self.copied = [torch.cuda.Event() for _ in range(2)]
        self.e2e_slots = 2
        self.e2e_stages = "the frames' passes"
        self.frames_per_step = n
        self.n_emitters = 0
        self.psf_build_ms = 0.0

    def device_step(self):
        self.d_cam.zero_()
        self.plan.frames_dev(self.d_spec, self.d_coef, self.d_shift, self.window, self.UP, self.d_cam, sync=False)

    def e2e_step(self):
        import torch
        self.d_coef.copy_(self.h_coef, non_blocking=True)
        self.d_shift.copy_(self.h_shift, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        self.d_cam.zero_()
        self.plan.frames_dev(self.d_spec, self.d_coef, self.d_shift, self.window, self.UP, self.d_cam, sync=True)
        self.h_cam.copy_(self.d_cam, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_cam

    def e2e_run(self, steps):
        """steps end-to-end steps over two slots: each step's coefficients and shifts go up on an upload stream, its
        frames are rendered on the library's stream and come down on a copy stream into the slot's page-locked
        buffer, so one step's download runs beside the next step's passes. Returns when every step's frames are on
        the host."""
        import torch
        comp, copy, up = self.stream, self.copy_stream, self.up_stream
        for i in range(steps):
            io = i % 2
            up.wait_event(self.rendered[io])   # the slot's inputs of two steps back are read
            with torch.cuda.stream(up):
                self.d_coef_io[io].copy_(self.h_coef, non_blocking=True)
                self.d_shift_io[io].copy_(self.h_shift, non_blocking=True)
                self.uploaded[io].record(up)
            comp.wait_event(self.uploaded[io])
            comp.wait_event(self.copied[io])   # the slot's frames of two steps back are on the host
            with torch.cuda.stream(comp):
                self.d_cam_io[io].zero_()
                self.plan.frames_dev(self.d_spec, self.d_coef_io[io], self.d_shift_io[io], self.window, self.UP,
                                     self.d_cam_io[io], sync=False)
                self.rendered[io].record(comp)
            copy.wait_event(self.rendered[io])
            with torch.cuda.stream(copy):
                self.h_cam_io[io].copy_(self.d_cam_io[io], non_blocking=True)
                self.copied[io].record(copy)
        for io in range(2):
            self.copied[io].synchronize()

    def e2e_bytes(self):
        return self.h_coef.numel() * 4 + self.h_shift.numel() * 8, self.h_cam.numel() * 4

    def kernel_name(self):
        return "ShiftColumnsKernel+ShiftRowsKernel"

    def alg_bytes_per_launch(self):
        n = len(self.coef)
        spec = self.spectra[0].nbytes
        # per frame: the 6 channels read, the column-pass spectrum written and read back, the camera frame out
        return n * (6 * spec + 2 * spec + self.h_cam[0].numel() * 8)

    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)

    def reference_step(self):
        t0 = time.perf_counter()
        for f in range(self.frames_per_step_cpu):
            self.ref.shifted_images(self.NX, self.NY, self.spectra[:3], self.a[f], self.frac, self.drift[f],
                                    self.window, self.UP, spec1=self.spectra[3:], w=float(self.w[f]))
        return time.perf_counter() - t0


class FftPlaceWorkload:
    """The splat's Fft placement (a next-row extra the reference runs on the CPU only): for 32,000 emitters (the
    SMLM movie's 200 frames at 160 ON each: positions uniform over 128 x 128 px, planes over the 49 of its kernel,
    129 x 129 samples at oversampling 4) each emitter's kernel plane shifted by its sub-cell offset and the shifted
    plane's block sums (iscu_fft_place_dev). The records stay resident; one step = one call. e2e: records in, the
    block sums and origins out."""
    name = ("Fft placement: 32,000 emitters' shifted kernel planes (129 x 129 samples, 49 planes, oversampling 4) "
            "and their block sums")
    metric = "emitters/s"
    dtype = "f64"
    cpu_kind = "reference"

    def __init__(self, rank: int):
        from insiliscope_b200 import EMITTER_DTYPE
        rng = np.random.default_rng(42 + rank)
        n = 32000
        em = np.zeros(n, EMITTER_DTYPE)
        em["x_px"], em["y_px"] = rng.uniform(-0.5, 127.5, (2, n))
        em["photons"] = 2000.0 * np.exp(0.5 * rng.normal(size=n))
        em["plane"] = rng.integers(0, 49, n)
        self.em = em
        self.frames_per_step_cpu = 1024
        self.cpu_sample = ("1,024 of the 32,000 emitters per step: the reference's PlanSplat with the Fft placement "
                           "(FftShiftKernelTile's FFT row and column shifts, then BuildBlockSums; compiled from its "
                           "sources) on its thread pool")

    def _psf(self):
        from insiliscope_b200.workloads import smlm_dstorm
        return smlm_dstorm(frames=1).psf

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import Engine
        self.eng = eng = Engine(device)
        t0 = time.perf_counter()
        eng.kernel_build(0, self._psf())
        eng.synchronize()
        self.psf_build_ms = (time.perf_counter() - t0) * 1e3
        dev = f"cuda:{device}"
        self.d_em = torch.from_numpy(self.em.view(np.uint8)).to(dev)
        size, nz, os_, bw = eng.kernel_info(0)
        n = len(self.em)
        self.bw = bw
        self.d_sums = torch.empty((n, bw, bw), dtype=torch.float32, device=dev)
        self.d_org = torch.empty((n, 4), dtype=torch.int32, device=dev)
        self.h_em = torch.from_numpy(self.em.view(np.uint8)).pin_memory()
        self.h_sums = torch.empty((n, bw, bw), dtype=torch.float32).pin_memory()
        self.h_org = torch.empty((n, 4), dtype=torch.int32).pin_memory()
        self.stream = eng.torch_stream()
        self.frames_per_step = n
        self.n_emitters = n
        self.plane_bytes = size * size * 4

    def device_step(self):
        from insiliscope_b200.engine import _ptr
        from insiliscope_b200._abi import check
        check(self.eng.lib.iscu_fft_place_dev(self.eng.h, 0, _ptr(self.d_em), len(self.em), _ptr(self.d_sums),
                                              _ptr(self.d_org)))

    def e2e_step(self):
        import torch
        self.d_em.copy_(self.h_em, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        self.device_step()
        self.eng.synchronize()
        self.h_sums.copy_(self.d_sums, non_blocking=True)
        self.h_org.copy_(self.d_org, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_sums

    def e2e_bytes(self):
        return self.h_em.numel(), self.h_sums.numel() * 4 + self.h_org.numel() * 4

    def kernel_name(self):
        return "FftPlaceKernel"

    def alg_bytes_per_launch(self):
        # per emitter: its record, its plane read, its block sums and origin written
        return len(self.em) * (32 + self.plane_bytes + self.bw * self.bw * 4 + 16)

    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)
        self.ref_kernel = self.ref.kernel(req=self._psf())
        k = self.frames_per_step_cpu
        self.ref_xy = np.stack([self.em["x_px"][:k], self.em["y_px"][:k]], axis=1)
        self.ref_z = self.em["plane"][:k].astype(np.int32)

    def reference_step(self):
        return self.ref_kernel.plan_splat_fft_batch(self.ref_xy, self.ref_z)


class CsvWorkload:
    """Ground-truth table text: 482,304 rows (the two-colour movie's emitter rows) of 20 numeric columns in the
    tables' formats (frame %d, times and world positions %.6f, camera positions %.3f, photons %.4f, fractions %.6g,
    wavelength %.4g), formatted as AppendCsvNumber writes each number and laid out as GroundTruth's rows. The
    columns stay resident; one step = iscu_csv_table_dev (row lengths, scan, rows written; its total read back).
    e2e: the float64 columns in, the text out."""
    name = ("ground-truth table text: 482,304 rows x 20 numeric columns (%d, %.6f, %.3f, %.4f, %.6g, %.4g as the "
            "emitter table uses them), AppendCsvNumber's printf rounding")
    metric = "rows/s"
    dtype = "f64"
    cpu_kind = "reference"
    FMTS = ["%d", "%.6f", "%.3f", "%.3f", "%.3f", "%.6f", "%.6f", "%.6f", "%.6f", "%.6f", "%.6f", "%.6g", "%.4f",
            "%.4f", "%.4f", "%.4f", "%.4f", "%.4f", "%.4g", "%.6g"]

    def __init__(self, rank: int):
        rng = np.random.default_rng(42 + rank)
        n = 482304
        cols = [np.sort(rng.integers(0, 1024, n)).astype(np.float64), rng.integers(0, 1024, n) * 0.05]
        cols += [rng.uniform(0, 27648, n), rng.uniform(0, 27648, n), rng.normal(0, 300, n)]   # x, y, z [nm]
        cols += [rng.uniform(-14, 14, n) for _ in range(6)]                                     # world / site [um]
        cols += [rng.random(n)]                                                                # on fraction
        cols += [rng.lognormal(7, 1, n) for _ in range(6)]                                     # photons
        cols += [rng.choice([580.0, 670.0], n), rng.random(n)]                                 # wavelength, excite
        self.cols = np.ascontiguousarray(np.stack(cols))
        self.frames_per_step_cpu = n
        self.cpu_sample = ("all 482,304 rows per step: the reference's AppendCsvNumber per cell (CsvNumber.cpp, "
                           "compiled from its sources) in GroundTruth's Rows chunks of 16,384 rows on its thread pool")

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import Engine
        self.eng = Engine(device)
        dev = f"cuda:{device}"
        self.d_cols = torch.from_numpy(self.cols).to(dev)
        text = self.eng.csv_table_dev(self.d_cols, self.FMTS)
        self.n_text = text.numel()
        self.d_out = torch.empty(self.n_text, dtype=torch.uint8, device=dev)
        self.h_cols = torch.from_numpy(self.cols).pin_memory()
        self.h_out = torch.empty(self.n_text, dtype=torch.uint8).pin_memory()
        self.stream = self.eng.torch_stream()
        self.frames_per_step = self.cols.shape[1]
        self.n_emitters = 0
        self.psf_build_ms = 0.0

    def device_step(self):
        self.eng.csv_table_dev(self.d_cols, self.FMTS, out_dev=self.d_out)

    def e2e_step(self):
        import torch
        self.d_cols.copy_(self.h_cols, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        self.eng.csv_table_dev(self.d_cols, self.FMTS, out_dev=self.d_out)
        self.h_out.copy_(self.d_out, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_out

    def e2e_bytes(self):
        return self.cols.nbytes, self.n_text

    def kernel_name(self):
        return "CsvRowLengthsKernel+CsvScanBlocksKernel+CsvWriteRowsKernel"

    def alg_bytes_per_launch(self):
        return 2 * self.cols.nbytes + self.n_text + self.cols.shape[1] * 4 * 2   # columns twice, text, row lengths

    def config_extra(self):
        return {"text_bytes": self.n_text}

    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)

    def reference_step(self):
        _, sec = self.ref.csv_table(self.cols, self.FMTS)
        return sec


class TiffWorkload:
    """The movie file: 200 frames of 512 x 512 uint16 ADU (100 MB) from device memory into a classic TIFF in
    memory-backed storage (/dev/shm where the box has it, so that both arms time the writer, not the disk's
    writeback; the temporary directory otherwise) (iscu_tiff_pages_dev: 8 MB chunks through the context's two
    page-locked halves, each chunk's copy beside the previous chunk's file writes; the description on page 1). No
    kernel runs: the pages are the ADU frames as they are, so the device work is the copies. One step = open, 200
    pages, close."""
    name = ("movie file: 200 frames of 512x512 uint16 ADU from device memory to a classic TIFF (description on "
            "page 1) in memory-backed storage")
    metric = "frames/s"
    dtype = "u16"
    cpu_kind = "reference"
    DESC = "insiliscope movie frames=200 w=512 h=512"

    def __init__(self, rank: int):
        import tempfile
        self.rank = rank
        self.frames = np.random.default_rng(42 + rank).integers(0, 65536, (200, 512, 512)).astype(np.uint16)
        shm = "/dev/shm"
        self.dir = tempfile.mkdtemp(prefix="iscu_tiff_", dir=shm if os.path.isdir(shm) else None)
        self.frames_per_step_cpu = 200
        self.cpu_sample = ("all 200 frames per step: the reference's TiffWriter (cli/tiff_writer.h, compiled from its "
                           "sources) writing them from host vectors, as the CLI does")

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import Engine
        self.eng = Engine(device)
        self.d_frames = torch.from_numpy(self.frames).to(f"cuda:{device}")
        self.path = os.path.join(self.dir, f"movie_{self.rank}.tif")
        self.stream = self.eng.torch_stream()
        self.frames_per_step = len(self.frames)
        self.n_emitters = 0
        self.psf_build_ms = 0.0

    def device_step(self):
        from insiliscope_b200 import TiffWriter
        with TiffWriter(self.path) as t:
            t.pages_dev(self.eng, self.d_frames, self.DESC)

    def e2e_step(self):
        self.device_step()

    def e2e_bytes(self):
        return 0, self.frames.nbytes

    def kernel_name(self):
        return "pages from device memory (copies + file writes)"

    def alg_bytes_per_launch(self):
        return self.frames.nbytes   # each frame read from HBM once

    def cpu_cores(self):
        return 1

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref_path = os.path.join(self.dir, f"movie_ref_{self.rank}.tif")

    def reference_step(self):
        t0 = time.perf_counter()
        t = self.ref.tiff(self.ref_path)
        for k in range(len(self.frames)):
            t.page(self.frames[k], 512, 512, self.DESC if k == 0 else None)
        t.close()
        return time.perf_counter() - t0


class BinnedWorkload:
    """The binned blink regime (the reference's approximate SMLM render of dense frames): 200 frames of 128 x 128 px
    with about 2,400 ON emitters each (12.7 per um^2, just above the reference's switch to binned at 12.5), deposited
    on 2 x 2 cells per pixel and convolved with the SMLM kernel's 49 planes at the cell pitch (R = 33 cells); then
    20 photons/px background and the EMCCD chain. The emitter records stay resident; one step = background fill,
    iscu_binned_render_dev, iscu_noise_frames_dev. e2e: page-locked emitter records and frame table in, ADU out."""
    name = ("binned blinks: 128x128 px, 200 frames, ~2,400 ON emitters per frame (12.7 per um^2), u = 2 cells per "
            "pixel, SMLM kernel (NA 1.45, 670 nm, 49 planes), 20 photons/px background, EMCCD gain 300")
    metric = "frames/s"
    dtype = "f64"
    cpu_kind = "reference"
    BACKGROUND = 20.0

    def __init__(self, rank: int):
        from insiliscope_b200.workloads import binned_dense
        self.mv = binned_dense(seed=42 + rank)
        self.frames_per_step_cpu = 40
        self.cpu_sample = (f"{self.frames_per_step_cpu} of the 200 frames per step: the reference's "
                           "BinnedBlinkRenderer::Render per frame (BinnedBlinks.cpp, float FFTs, compiled from its "
                           "sources; frames in parallel on its thread pool) and ApplyNoiseChain per frame")

    def setup(self, device: int):
        import torch
        from insiliscope_b200 import BinnedRenderer, Engine, generate_camera_maps
        mv = self.mv
        self.eng = eng = Engine(device)
        dev = f"cuda:{device}"
        t0 = time.perf_counter()
        eng.kernel_build(0, mv.psf)
        eng.synchronize()
        self.psf_build_ms = (time.perf_counter() - t0) * 1e3
        self.binned = BinnedRenderer(eng, mv.width, mv.height, mv.upscale, slot=0)
        off, _, _ = generate_camera_maps(mv.width, mv.height, 7, 100.0, 2.0, 1.0, 0.0, 50.0, 0.0)
        self.offset = off
        eng.set_static(mv.width, mv.height, offset=off)
        n = mv.n_frames
        self.d_em = torch.from_numpy(mv.emitters.view(np.uint8)).to(dev)
        self.d_fr = torch.from_numpy(mv.frames.view(np.uint8)).to(dev)
        self.d_idx = torch.arange(n, dtype=torch.int32, device=dev)
        self.d_img = torch.empty((n, mv.height, mv.width), dtype=torch.float32, device=dev)
        self.d_adu = torch.empty((n, mv.height, mv.width), dtype=torch.uint16, device=dev)
        self.h_em = torch.from_numpy(mv.emitters.view(np.uint8)).pin_memory()
        self.h_fr = torch.from_numpy(mv.frames.view(np.uint8)).pin_memory()
        self.h_adu = torch.empty((n, mv.height, mv.width), dtype=torch.uint16).pin_memory()
        self.stream = eng.torch_stream()
        self.frames_per_step = n
        self.n_emitters = len(mv.emitters)

    def _step(self, sync):
        mv = self.mv
        self.d_img.fill_(self.BACKGROUND)
        self.binned.render_dev(self.d_em, self.d_fr, mv.n_frames, self.d_img, sync=False)
        self.eng.noise_frames_dev(self.d_img, self.d_idx, mv.camera, mv.noise_seed, out=self.d_adu, sync=sync)

    def device_step(self):
        self._step(False)

    def e2e_step(self):
        """Page-locked records in, ADU out, the copies on torch's own stream ordered with the library's by the
        synchronizing calls."""
        import torch
        self.d_em.copy_(self.h_em, non_blocking=True)
        self.d_fr.copy_(self.h_fr, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        self._step(True)
        self.h_adu.copy_(self.d_adu, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_adu

    def e2e_bytes(self):
        return self.h_em.numel() + self.h_fr.numel(), self.h_adu.numel() * 2

    def kernel_name(self):
        return "BinnedRenderKernel+noise"

    def alg_bytes_per_launch(self):
        # the emitter records (32 B) and frame table, the photon frames written by the fill, read and written by the
        # render and read by the noise chain (4 x 4 B per pixel), the ADU out and the offset map
        px = self.mv.n_frames * self.mv.width * self.mv.height
        return len(self.mv.emitters) * 32 + self.mv.n_frames * 24 + px * 16 + px * 2 + self.mv.width * self.mv.height * 4

    def config_extra(self):
        return {"upscale": self.binned.upscale, "radius_cells": self.binned.radius,
                "emitters_per_frame": round(len(self.mv.emitters) / self.mv.n_frames, 1)}

    def cpu_cores(self):
        return self.ref.threads()

    def reference_setup(self, threads=0):
        from oracle.oracle import Reference
        if not Reference.available():
            raise RuntimeError("the reference harness oracle/_ref/libiscref.so is not built (it needs the reference "
                               "tree at build time)")
        self.ref = Reference()
        self.ref.set_threads(threads)
        self.ref_kernel = self.ref.kernel(req=self.mv.psf)
        k = self.frames_per_step_cpu
        fr = self.mv.frames[:k].copy()
        last = int(fr[-1]["em_start"] + fr[-1]["em_count"])
        self.ref_em = self.mv.emitters[:last]
        self.ref_fr = fr
        self.ref_offset, _, _ = self.ref.camera_maps(self.mv.width, self.mv.height, 7, 100.0, 2.0, 1.0, 0.0, 50.0, 0.0)

    def reference_step(self):
        mv = self.mv
        t0 = time.perf_counter()
        img = np.full((len(self.ref_fr), mv.height, mv.width), self.BACKGROUND, np.float32)
        self.ref.binned_render(self.ref_kernel, 0.0, mv.width, mv.height, mv.upscale, self.ref_em, self.ref_fr, img)
        off = self.ref_offset.reshape(mv.height, mv.width)
        for k in range(len(self.ref_fr)):
            self.ref.noise_chain(img[k], mv.camera, off, None, None, mv.noise_seed, k, parallel=True)
        return time.perf_counter() - t0


WORKLOADS = {"smlm": SmlmWorkload, "widefield": WidefieldWorkload, "psflib": PsfLibraryWorkload,
             "two-colour": TwoColourWorkload, "nll-grad": NllGradWorkload, "schedules": ScheduleWorkload,
             "binned": BinnedWorkload, "tiff": TiffWorkload, "csv": CsvWorkload, "fftplace": FftPlaceWorkload,
             "wfshift": WfShiftWorkload}
for _key, _cls in WORKLOADS.items():
    _cls.key = _key


# ----------------------------------------------------------------------------------------------------- arms
L2_NOTE = "flushed before every timed step (256 MB write)"


def common_config(w, n_gpus):
    """The workload's configuration, the same dict in both arms (the GPU arm's own details go to `details`)."""
    return {"workload": w.name, "l2": L2_NOTE, "parallelism": f"frames x{n_gpus}"}


def repo_libraries():
    """This repository's shared libraries mapped into the process (which native code ran)."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            p = line.split()[-1] if line.strip() else ""
            if p.endswith(".so") and p.startswith(ROOT):
                out.add(os.path.relpath(p, ROOT))
    except OSError:
        pass
    return sorted(out)


SUBCONFIGS = (("C1", "widefield"), ("C2", "psflib"), ("C3", "two-colour"), ("C4", "nll-grad"))


def measure_reference(w, steps, warmup, n_gpus):
    """The reference's CPU path on the host cores: warm-up steps, then the mean of `steps` timed steps."""
    try:
        w.reference_setup(threads=0)
    except RuntimeError as e:
        return {"impl": "reference", "unavailable": str(e)}
    for _ in range(warmup):
        w.reference_step()
    times = [w.reference_step() for _ in range(steps)]
    ms = 1e3 * statistics.mean(times)
    value = w.frames_per_step_cpu / (ms / 1e3)
    return {"metric": w.metric, "value": value, "unit": w.metric, "n_gpus": n_gpus, "steps": steps,
            "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": w.dtype, "data": "synthetic", "impl": "reference",
            "config": common_config(w, n_gpus),
            "cpu_baseline": {"value": value, "unit": w.metric, "cores": w.cpu_cores(), "kind": w.cpu_kind,
                             "sample": w.cpu_sample, "units_per_step": w.frames_per_step_cpu},
            "e2e": {"value": value, "unit": w.metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload != "all":
        line = measure_reference(WORKLOADS[args.workload](0), args.steps, args.warmup, args.gpus)
    else:
        line = measure_reference(SmlmWorkload(0), args.steps, args.warmup, args.gpus)
        line["configs"] = {key: compact(measure_reference(WORKLOADS[name](0), min(args.steps, 5),
                                                          min(args.warmup, 2), args.gpus))
                           for key, name in SUBCONFIGS}
    line["native_libraries"] = repo_libraries()
    print(json.dumps(line))
    return 0


def cpu_leg(w, repeats=3):
    """The CPU path on this box's host cores, a bounded sample (the workload's own), best of `repeats` after one
    warm-up; and, where a workload checks its output against the float64 oracle at full size, that check."""
    try:
        w.reference_setup(threads=0)
    except RuntimeError:
        return None, None
    w.reference_step()
    best = min(w.reference_step() for _ in range(repeats))
    base = {"value": w.frames_per_step_cpu / best, "unit": w.metric, "cores": w.cpu_cores(), "kind": w.cpu_kind,
            "sample": w.cpu_sample + f"; best of {repeats}"}
    return base, (w.accuracy() if hasattr(w, "accuracy") else None)


COMPACT_KEYS = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "dtype", "config", "details", "e2e",
                "roofline", "cpu_baseline", "plain_form", "accuracy", "gpu_launches", "clocks", "unavailable", "impl")


def compact(line):
    return {k: line[k] for k in COMPACT_KEYS if k in line}


def measure_ours(w, args, world, rank, local, steps, warmup, cpu=True):
    """One workload on this rank's GPU: W untimed steps, K steps timed with CUDA events (L2 flushed before each,
    clocks sampled), the slowest pass's roofline, the end-to-end run through the C ABI with host buffers, the plain
    form beside it where the workload has one, and (rank 0, one GPU) the CPU baseline. Returns the JSON line."""
    import torch
    if args.form is not None and isinstance(w, SmlmWorkload):
        w.setup(local, form=args.form)
    else:
        w.setup(local)
    eng = w.eng
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")   # 256 MB > L2 (126 MB)
    start = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stop = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(w.stream):
        for i in range(warmup):
            flush.fill_(float(i))
            w.device_step()
    eng.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    launches0 = eng.launch_count
    if hasattr(w, "timing"):
        w.timing(True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier(world)
        with torch.cuda.stream(w.stream):
            for i in range(steps):
                flush.fill_(float(i + 1))
                start[i].record(w.stream)
                w.device_step()
                stop[i].record(w.stream)
        eng.synchronize()
        torch.cuda.synchronize()
        barrier(world)
    launches = eng.launch_count - launches0
    step_ms = [s.elapsed_time(e) for s, e in zip(start, stop)]
    ms = max_over_ranks(statistics.mean(step_ms), world)
    value = world * w.frames_per_step / (ms / 1e3)
    dom = w.dominant() if hasattr(w, "dominant") else None
    if hasattr(w, "timing"):
        w.timing(False)
    plain = w.plain_form(statistics.mean(step_ms)) if hasattr(w, "plain_form") else None
    # end to end through the C ABI with host buffers
    pipelined = hasattr(w, "e2e_run")
    run = w.e2e_run if pipelined else (lambda k: [w.e2e_step() for _ in range(k)])
    run(max(1, warmup))
    barrier(world)
    t0 = time.perf_counter()
    run(steps)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / steps, world)
    h2d, d2h = w.e2e_bytes()
    hbm, bf16, peak_kind = measured_peaks()
    if dom is not None:
        kname, kbytes, kms, breakdown = dom
    else:
        kname, kbytes, kms, breakdown = w.kernel_name(), w.alg_bytes_per_launch(), statistics.mean(step_ms), None
    tensor = getattr(w, "roofline_kind", "hbm") == "tensor"
    achieved = kbytes / (kms / 1e3) / (1e12 if tensor else 1e9)
    peak = bf16 if tensor else hbm
    line = {"metric": w.metric, "value": value, "unit": w.metric, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": w.dtype, "data": "synthetic",
            "config": common_config(w, world),
            "details": {"frames_per_step": w.frames_per_step, "emitters_per_step": w.n_emitters,
                        "psf_build_ms": round(w.psf_build_ms, 3), **(w.config_extra() if hasattr(w, "config_extra")
                                                                      else {})},
            "e2e": {"value": world * w.frames_per_step / (e2e_ms / 1e3), "unit": w.metric, "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "timing": (f"host wall clock over the steps, pipelined over {getattr(w, 'e2e_slots', 3)} I/O "
                               "slots (every step's H2D, "
                               f"{getattr(w, 'e2e_stages', 'collection, render, noise')} and D2H inside; one step's "
                               "copies beside the next one's kernels), max over ranks") if pipelined else
                              "host wall clock per step (blocking C-ABI calls), max over ranks"},
            "roofline": {"bound": "tensor" if tensor else "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s" if tensor else "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": NCU_TRAFFIC.get((w.key, kname), (None,))[0],
                         ("alg_flops_per_launch" if tensor else "alg_bytes_per_launch"): kbytes, "launch_ms": kms},
            "gpu_launches": launches, "clocks": clk.summary()}
    if breakdown and tensor:
        line["roofline"]["peak_note"] = ("measured dense bf16 cuBLAS peak; the kernel issues FP16 MMAs (the bf16 "
                                         "rate) and 3 of them per product (hi*hi, hi*lo, lo*hi)")
        line["roofline"]["issued_tflops"] = 3 * achieved
    elif breakdown:
        line["roofline"]["pass_ms"] = breakdown.get("pass_ms", breakdown)
        if "design_bytes" in breakdown:
            line["roofline"]["design_bytes_per_pass"] = breakdown["design_bytes"]
        step_bytes = kbytes if "design_bytes" in breakdown else w.alg_bytes_per_launch()
        line["roofline"]["step_alg_bytes"] = step_bytes
        line["roofline"]["step_achieved"] = step_bytes / (statistics.mean(step_ms) / 1e3) / 1e9
        line["roofline"]["step_frac"] = line["roofline"]["step_achieved"] / peak
    tr = line["roofline"]["traffic"]
    if tr and not tensor:
        line["roofline"]["traffic_over_alg"] = tr / kbytes
    if plain is not None:
        line["plain_form"] = plain
    if cpu and rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], acc = cpu_leg(w, 3 if steps >= 10 else 2)
        if acc is not None:
            line["accuracy"] = acc
    torch.cuda.synchronize()
    eng.close()
    return line


def launch_ranks(args):
    """--gpus N without a launcher: run this script under torch.distributed.run with N local ranks (one per GPU,
    rendezvous on 127.0.0.1) and pass its exit code through."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args.gpus)
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE {world}")
    torch.cuda.set_device(local)
    from insiliscope_b200.build import build_library
    build_library()
    if args.workload != "all":
        line = measure_ours(WORKLOADS[args.workload](rank), args, world, rank, local, args.steps, args.warmup)
    else:
        line = measure_ours(SmlmWorkload(rank), args, world, rank, local, args.steps, args.warmup)
        line["configs"] = {key: compact(measure_ours(WORKLOADS[name](rank), args, world, rank, local,
                                                     min(args.steps, 10), args.warmup))
                           for key, name in SUBCONFIGS}
    line["native_libraries"] = repo_libraries()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["all"] + sorted(WORKLOADS), default="all",
                    help="all (default): the SMLM movie as the headline with the widefield, PSF-library, two-colour "
                         "and gradient configurations as sub-records; or one workload alone")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", type=int, default=None,
                    help="SMLM workloads: render form 0..17 instead of the autotuner's choice (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args)
    return run_reference(args) if args.impl == "reference" else run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
