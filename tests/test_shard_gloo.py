"""Frames across ranks (world size 2, gloo, CPU): each rank makes its own frame range -- here the oracle's noise chain
on a per-frame photon image, a pure function of (seed, frame) like every frame of a movie -- and the gathered movie
equals the one a single process makes; the step time reported is the slowest rank's."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from insiliscope_b200.shard import frame_range, gather_movie, max_over_ranks

W, H, FRAMES, SEED = 24, 20, 11, 1234


def _photons(f):
    yy, xx = np.mgrid[0:H, 0:W]
    return (20.0 + 15.0 * np.sin(0.3 * xx + 0.7 * f) * np.cos(0.2 * yy - 0.1 * f) + 3.0 * f).astype(np.float32)


def _frames(first, end):
    from insiliscope_b200 import CameraParams
    from oracle.oracle import Oracle
    o = Oracle()
    off, gain, rn = o.camera_maps(W, H, 42, 100.0, 2.0, 2.2, 0.1 / 2.2, 1.5, 0.2)
    cam = CameraParams(gain=2.2, read_noise_e=1.5)
    return np.stack([o.noise_chain(_photons(f), cam, off, gain, rn, SEED, f) for f in range(first, end)]) \
        if end > first else np.zeros((0, H, W), np.uint16)


def _worker(rank, world, port, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        first, end = frame_range(rank, world, FRAMES)
        mine = torch.from_numpy(_frames(first, end).astype(np.int32))
        movie = gather_movie(mine, FRAMES)
        slowest = max_over_ranks(0.5 + rank)
        if rank == 0:
            np.save(out, movie.numpy())
            with open(out + ".t", "w") as f:
                f.write(repr(slowest))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_frame_ranges_cover_the_movie():
    for n in (0, 1, 7, 200, 1024):
        for world in (1, 2, 3, 8):
            got = [frame_range(r, world, n) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            assert max(e - b for b, e in got) - min(e - b for b, e in got) <= 1
    with pytest.raises(ValueError):
        frame_range(2, 2, 10)


def test_two_ranks_gather_the_single_process_movie(tmp_path):
    out = str(tmp_path / "movie.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    movie = np.load(out)
    assert np.array_equal(movie, _frames(0, FRAMES).astype(np.int32))
    assert float(open(out + ".t").read()) == 1.5


def _library(n_z=5):
    from insiliscope_b200.workloads import psf_library
    return psf_library(seed=9, n_z=n_z, wavelengths=(580.0, 670.0), n_aberr=2, pupil=32, size=24)


def _library_planes(lib):
    from oracle.oracle import Oracle
    o = Oracle()
    out = np.zeros((len(lib.set_of_psf), lib.size, lib.size))
    for i, (s, dz) in enumerate(zip(lib.set_of_psf, lib.defocus_nm)):
        out[i] = o.psf_planes(lib.sets[s], [dz * 1e-9], size=lib.size, normalize=True)[0]
    return out


def _library_worker(rank, world, port, out):
    from insiliscope_b200.shard import library_shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        lib = _library()
        mine = library_shard(lib, rank, world)
        planes = torch.from_numpy(_library_planes(mine))
        whole = gather_movie(planes, len(lib.set_of_psf))
        if rank == 0:
            np.save(out, whole.numpy())
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_the_psf_library(tmp_path):
    """A PSF library split into contiguous PSF ranges (library_shard): each of two gloo ranks computes its range
    (the float64 oracle here; the device plan on GPUs) and the gathered library equals the single-process one."""
    from insiliscope_b200.shard import library_shard
    lib = _library()
    n = len(lib.set_of_psf)
    parts = [library_shard(lib, r, 3) for r in range(3)]
    assert sum(len(p.set_of_psf) for p in parts) == n
    assert np.array_equal(np.concatenate([p.defocus_nm for p in parts]), lib.defocus_nm)
    out = str(tmp_path / "lib.npy")
    mp.spawn(_library_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    assert np.array_equal(np.load(out), _library_planes(lib))


SM = dict(sites=300, size=40)


def _rank_movie_adu(first, end, reference_kernel, maps):
    from insiliscope_b200.workloads import smlm_dstorm
    mv = smlm_dstorm(seed=42, frames=end - first, frame0=first, **SM)
    _, _, adu = reference_kernel.render_movie(mv.events, first, end - first, mv.width, mv.height, mv.pixel_nm,
                                              mv.photons_per_blink, mv.background, mv.camera, *maps, mv.noise_seed)
    return adu


def _smlm_setup():
    from insiliscope_b200.workloads import smlm_dstorm
    from oracle.oracle import Reference
    mv = smlm_dstorm(seed=42, frames=1, **SM)
    mv.psf.kernel_half_width_px = 6
    mv.psf.nz = 13
    ref = Reference()
    ref.set_threads(1)
    k = ref.kernel(req=mv.psf)
    maps = ref.camera_maps(mv.width, mv.height, mv.map_seed, mv.offset_mean, mv.offset_std, mv.gain_nominal,
                           mv.gain_std_fraction, mv.read_noise_nominal, mv.read_noise_std_fraction)
    return k, maps


def _smlm_worker(rank, world, port, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        k, maps = _smlm_setup()
        first, end = frame_range(rank, world, 9)
        mine = torch.from_numpy(_rank_movie_adu(first, end, k, maps).astype(np.int32))
        movie = gather_movie(mine, 9)
        if rank == 0:
            np.save(out, movie.numpy())
    finally:
        dist.destroy_process_group()


def test_two_ranks_render_the_dstorm_movie_by_frame_ranges(tmp_path):
    """The SMLM movie as the bench shards it: each rank generates the movie's frames of its frame_range
    (smlm_dstorm(frames, frame0): per (site, frame) hashes) and renders them -- the reference's own RenderPhotonImage
    + ApplyNoiseChain here, on the host -- and the gathered movie equals the whole movie rendered by one process."""
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("the reference harness (oracle/_ref) is not built")
    out = str(tmp_path / "movie.npy")
    mp.spawn(_smlm_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    k, maps = _smlm_setup()
    whole = _rank_movie_adu(0, 9, k, maps)
    assert whole.any() and np.array_equal(np.load(out), whole.astype(np.int32))
