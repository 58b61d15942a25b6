"""The gradient across ranks (world size 2, gloo, CPU): each rank takes its frame range of the problem
(shard_problem), evaluates its share -- here with the float64 adjoint of the oracle, the evaluator the GPU model is
checked against -- and sums the NLL and the Zernike gradient over the ranks (reduce_shared); the result equals the
whole problem's, and each rank's per-emitter and per-frame gradients are the whole problem's rows for its frames."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

FRAMES, PER_FRAME = 5, 3


def _problem():
    from insiliscope_b200.workloads import nll_rois
    from oracle.nll_oracle import NllSpec, expected
    spec = NllSpec(roi=12, os=2, pupil=24)
    prob = nll_rois(seed=5, frames=FRAMES, per_frame=PER_FRAME, spec=spec)
    mu = expected(spec, prob.params_true.astype(np.float64), prob.frame, prob.bg_true.astype(np.float64),
                  prob.zern_true)
    counts = np.random.default_rng(9).poisson(mu).astype(np.float64)
    return spec, prob, counts


def _gradient(spec, prob, counts):
    from oracle.nll_oracle import gradient
    return gradient(spec, prob.params.astype(np.float64), prob.frame, prob.bg.astype(np.float64), prob.zern, counts)


def _worker(rank, world, port, out):
    from insiliscope_b200.nll import reduce_shared, shard_problem
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        spec, prob, counts = _problem()
        part = shard_problem(prob, rank, world)
        sel = (prob.frame >= part.frame0) & (prob.frame < part.frame0 + len(part.bg))
        value, gp, gb, gz = _gradient(spec, part, counts[sel])
        packed = torch.from_numpy(np.concatenate([[value], gz]))
        reduce_shared(packed)
        np.savez(f"{out}.{rank}.npz", packed=packed.numpy(), gp=gp, gb=gb, frame0=part.frame0, n=len(part.frame))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shards_cover_the_problem():
    from insiliscope_b200.nll import shard_problem
    _, prob, _ = _problem()
    parts = [shard_problem(prob, r, 3) for r in range(3)]
    assert [p.frame0 for p in parts] == [0, 2, 4]
    assert np.array_equal(np.concatenate([p.frame + p.frame0 for p in parts]), prob.frame)
    assert np.array_equal(np.concatenate([p.params for p in parts]), prob.params)
    assert np.array_equal(np.concatenate([p.bg for p in parts]), prob.bg)
    assert all(np.array_equal(p.zern, prob.zern) for p in parts)


def test_two_ranks_sum_to_the_whole_gradient(tmp_path):
    out = str(tmp_path / "g")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    spec, prob, counts = _problem()
    value, gp, gb, gz = _gradient(spec, prob, counts)
    got = [np.load(f"{out}.{r}.npz") for r in range(2)]
    for g in got:   # every rank holds the sums
        assert np.allclose(g["packed"][0], value, rtol=1e-12)
        assert np.allclose(g["packed"][1:], gz, rtol=1e-10, atol=1e-12 * np.abs(gz).max())
    assert np.array_equal(np.concatenate([g["gp"] for g in got]), gp)
    assert np.array_equal(np.concatenate([g["gb"] for g in got]), gb)
