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
