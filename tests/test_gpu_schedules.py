"""Blink schedules on the device (iscu_dye_blinks_dev) against the world core's own schedules (core/src/dyes.cpp,
compiled into the reference harness): every row bit for bit -- dSTORM with and without the initial ON, PALM with the
lowest bleach probability (hundreds of blinks a dye), DNA-PAINT at a low rate (inverse-CDF counts) and a high
one (the rounded normal), kinetics histories of several segments (changes inside DNA-PAINT bins), WideField (none)."""
import numpy as np
import pytest

from insiliscope_b200 import (DYE_DTYPE, EVENT_STRIDE, LABEL_DNA_PAINT, LABEL_DSTORM, LABEL_PALM, LABEL_WIDEFIELD)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dyes(reference):
    """Dyes with the core's own addresses: DyeH1 of microtubules in a few cells, sites (protofilament k, dimer n)."""
    rng = np.random.default_rng(17)
    n = 1500
    d = np.zeros(n, DYE_DTYPE)
    cells = [(0, 0), (1, -2), (-3, 5)]
    h1s = [reference.dye_h1(42, cx, cy, mt) for cx, cy in cells for mt in range(4)]
    d["h1"] = rng.choice(np.array(h1s, np.uint64), n).astype(np.uint32)
    d["k"] = rng.integers(0, 13, n)
    d["n"] = rng.integers(0, 400, n)
    d["id"] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    d["structure"] = rng.integers(0, 4, n)
    d["x"], d["y"], d["z"] = rng.uniform(-5, 5, (3, n))
    return d


def _kin(rate, on, off, bleach, cv, init_on=0.0):
    return [rate, on, off, bleach, cv, init_on]


CASES = [
    ("dstorm-initial-on", LABEL_DSTORM, _kin(0.05, 0.04, 2.0, 0.3, 0.5, 0.2), None, 0.0, 120.0),
    ("dstorm-window", LABEL_DSTORM, _kin(0.2, 0.03, 0.5, 0.05, 0.0), None, 20.0, 23.5),
    ("palm-long", LABEL_PALM, _kin(0.5, 0.01, 0.02, 0.001, 0.7), None, 0.0, 60.0),
    ("dnapaint-low", LABEL_DNA_PAINT, _kin(0.5, 0.3, 1.0, 1.0, 0.5), None, 10.0, 21.0),
    ("dnapaint-high", LABEL_DNA_PAINT, _kin(45.0, 0.02, 1.0, 1.0, 0.3), None, 3.0, 4.2),
    ("dstorm-history", LABEL_DSTORM, _kin(0.05, 0.04, 2.0, 0.3, 0.5, 0.2),
     ([0.0, 7.5, 30.25], [_kin(0.05, 0.04, 2.0, 0.3, 0.5, 0.2), _kin(0.4, 0.02, 0.7, 0.1, 0.3, 0.0),
                          _kin(0.01, 0.08, 3.0, 0.6, 0.0, 0.0)]), 0.0, 80.0),
    ("palm-history-one", LABEL_PALM, _kin(1.0, 1.0, 1.0, 1.0, 0.0),
     ([0.0], [_kin(0.3, 0.05, 0.5, 0.2, 0.4)]), 5.0, 45.0),
    ("dnapaint-history", LABEL_DNA_PAINT, _kin(0.5, 0.3, 1.0, 1.0, 0.5),
     ([0.0, 12.4, 12.9, 15.0], [_kin(0.5, 0.3, 1.0, 1.0, 0.5), _kin(3.0, 0.1, 1.0, 1.0, 0.2),
                               _kin(40.0, 0.01, 1.0, 1.0, 0.0), _kin(0.2, 0.5, 1.0, 1.0, 0.5)]), 10.0, 17.0),
    ("widefield", LABEL_WIDEFIELD, _kin(0.5, 0.3, 1.0, 1.0, 0.5), None, 0.0, 10.0),
]


@pytest.mark.parametrize("name,mode,kin,history,t0,t1", CASES, ids=[c[0] for c in CASES])
def test_blinks_match_the_core(engine, reference, dyes, name, mode, kin, history, t0, t1):
    rows, first = engine.dye_blinks(mode, kin, dyes, t0, t1, history=history)
    assert rows.shape[1] == EVENT_STRIDE and first[-1] == len(rows)
    total = 0
    for i, d in enumerate(dyes):
        want = reference.dye_blinks(mode, kin, d["h1"], d["k"], d["n"], t0, t1, history=history)
        got = rows[first[i]:first[i + 1]]
        assert got.shape[0] == want.shape[0], (name, i)
        assert got[:, 3:6].tobytes() == want.tobytes(), (name, i)
        if len(got):
            assert np.all(got[:, 0] == d["x"]) and np.all(got[:, 6] == d["id"]) and np.all(got[:, 7] == d["structure"])
            assert not got[:, 8:].any()
        total += len(want)
    if mode == LABEL_WIDEFIELD:
        assert total == 0
    else:
        assert total > 0
    if name == "palm-long":   # long schedules (bleach probability clamped at 0.01: ~100 cycles, some many more)
        assert max(first[1:] - first[:-1]) >= 500


def test_row_cap_and_empty(engine, dyes):
    """Past max_rows the rows are dropped but the total is still reported; no dyes gives no rows."""
    import torch
    kin = _kin(0.5, 0.3, 1.0, 1.0, 0.5)
    rows, first = engine.dye_blinks(LABEL_DNA_PAINT, kin, dyes[:200], 10.0, 21.0)
    d_dyes = torch.from_numpy(np.ascontiguousarray(dyes[:200]).view(np.uint8)).cuda()
    small = torch.zeros((10, EVENT_STRIDE), dtype=torch.float64, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    engine.dye_blinks_dev(LABEL_DNA_PAINT, kin, d_dyes, 200, 10.0, 21.0, small, d_n)
    assert int(d_n.item()) == len(rows) > 10
    assert np.array_equal(small.cpu().numpy(), rows[:10])
    r0, f0 = engine.dye_blinks(LABEL_DSTORM, kin, dyes[:0], 0.0, 10.0)
    assert len(r0) == 0 and list(f0) == [0]


@pytest.mark.parametrize("reps", [3, 9, 60])
def test_first_rows_over_many_scan_blocks(engine, dyes, reps):
    """The dyes' first rows (an exclusive scan of their counts, 4,096 counts per scan block) over one block and a
    part (4,500 dyes), several (13,500) and many (90,000): each dye's count and rows as in the short list."""
    kin = _kin(0.5, 0.01, 0.02, 0.001, 0.7)   # long schedules: counts up to hundreds
    rows1, first1 = engine.dye_blinks(LABEL_PALM, kin, dyes, 0.0, 20.0)
    big = np.tile(dyes, reps)
    rows, first = engine.dye_blinks(LABEL_PALM, kin, big, 0.0, 20.0)
    assert first[0] == 0 and first[-1] == len(rows) == reps * len(rows1)
    assert np.array_equal(np.diff(first), np.tile(np.diff(first1), reps))
    assert np.array_equal(rows, np.tile(rows1, (reps, 1)))
    import torch   # the same through the scratch first-row array (no caller array)
    d_dyes = torch.from_numpy(np.ascontiguousarray(big).view(np.uint8)).cuda()
    out = torch.zeros((len(rows), EVENT_STRIDE), dtype=torch.float64, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    engine.dye_blinks_dev(LABEL_PALM, kin, d_dyes, len(big), 0.0, 20.0, out, d_n)
    assert int(d_n.item()) == len(rows) and np.array_equal(out.cpu().numpy(), rows)
