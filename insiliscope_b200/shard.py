"""Frames (and PSFs) across ranks: one process per GPU, each rendering a contiguous range of a movie's frames or of a
PSF library's PSFs.

A frame is a pure function of (spec, frame) -- the emitters are per (site, frame) hashes, the noise is keyed by
(seed, frame, pixel), the drift is a precomputed per-frame table -- so ranks need no exchange on the data path: each
renders its own range, and the movie is the ranks' ranges in rank order. torch.distributed carries the plumbing (the
gather of a movie on one rank, the max of the ranks' step times), over NCCL on GPUs or gloo on CPUs.
"""
from __future__ import annotations


def frame_range(rank: int, world: int, n_frames: int) -> tuple[int, int]:
    """The [first, end) frames of `rank` when `n_frames` split as evenly as they can (the first n % world ranks get
    one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(n_frames, world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def max_over_ranks(x: float, device=None) -> float:
    """The largest of every rank's x (a step time)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_movie(frames, n_frames: int, device=None):
    """The whole movie (n_frames, ...) from every rank's frame range (this rank's `frames`, its range's length along
    dim 0), on every rank."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return frames
    world = dist.get_world_size()
    sizes = [frame_range(r, world, n_frames) for r in range(world)]
    longest = max(e - b for b, e in sizes)
    pad = torch.zeros((longest,) + tuple(frames.shape[1:]), dtype=frames.dtype, device=device or frames.device)
    pad[: frames.shape[0]] = frames
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    return torch.cat([p[: e - b] for p, (b, e) in zip(parts, sizes)])


def library_shard(lib, rank: int, world: int):
    """The rank's share of a PSF library (workloads.PsfLibrary): its contiguous range of PSFs (frame_range over the
    library's PSFs) with every request set, so each rank builds the same DFT operands and computes its PSFs alone; the
    library is the ranks' ranges in rank order (gather_movie along the PSF axis)."""
    from dataclasses import replace
    first, end = frame_range(rank, world, len(lib.set_of_psf))
    return replace(lib, set_of_psf=lib.set_of_psf[first:end], defocus_nm=lib.defocus_nm[first:end])
