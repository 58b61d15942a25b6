"""The ground-truth tables' text on the B200 (iscu_csv_numbers_dev, iscu_csv_table_dev) against the checker (printf
of the exact binary value, cut to 47 characters) and the reference's AppendCsvNumber / table rows: equal character
for character, every precision of both styles, and whole tables byte for byte, including a short output buffer."""
import numpy as np
import pytest

from insiliscope_b200 import IscuError
from test_csv_oracle import TABLE_FMTS, csv_values, printf

pytestmark = pytest.mark.gpu


def _texts(fields, lens):
    f, l = fields.cpu().numpy(), lens.cpu().numpy()
    return [bytes(f[i, :l[i]]).decode() for i in range(len(l))]


@pytest.mark.parametrize("fmt", TABLE_FMTS)
def test_numbers_table_formats(engine, reference, fmt):
    import torch
    v = csv_values(n=20000)
    got = _texts(*engine.csv_numbers_dev(torch.from_numpy(v).cuda(), fmt))
    assert got == [printf(x, fmt) for x in v]
    assert got[:3000] == reference.csv_numbers(v[:3000], fmt)


def test_numbers_every_precision(engine):
    import torch
    v = csv_values(seed=11, n=2000)
    d = torch.from_numpy(v).cuda()
    for kind in "fg":
        for p in range(10):
            fmt = f"%.{p}{kind}"
            assert _texts(*engine.csv_numbers_dev(d, fmt)) == [printf(x, fmt) for x in v], fmt


def test_table_equals_reference(engine, reference):
    import torch
    rng = np.random.default_rng(5)
    n = 70000
    fmts = ["%d", "%.6f", "%.6g", "%.6f", "%.6f", "%.6f", "%.6f", "%.4f", "%.4f", "%.4f"]   # the frames table's
    cols = np.stack([np.arange(n, dtype=np.float64), np.arange(n) * 0.05, np.full(n, 0.05),
                     rng.normal(0, 10, n), rng.normal(0, 10, n), rng.normal(0, 1, n), rng.normal(0, 1, n),
                     rng.normal(0, 30, n), rng.normal(0, 30, n), rng.normal(0, 50, n)])
    want, _ = reference.csv_table(cols, fmts)
    d = torch.from_numpy(cols).cuda()
    got = engine.csv_table_dev(d, fmts)
    assert bytes(got.cpu().numpy()) == want
    # an output too short: its first bytes written, the size needed reported
    short = torch.zeros(1000, dtype=torch.uint8, device="cuda")
    with pytest.raises(IscuError) as e:
        engine.csv_table_dev(d, fmts, out_dev=short)
    assert e.value.code == 4 and str(len(want)) in str(e.value)
    assert bytes(short.cpu().numpy()) == want[:1000]


def _checker_table(cols, fmts):
    return "".join(",".join(printf(cols[c, r], fmts[c]) for c in range(len(fmts))) + "\n"
                   for r in range(cols.shape[1])).encode()


def test_table_spans_staged_and_direct(engine):
    """Rows written through the shared-memory spans (16-byte stores) and straight from the threads (a span longer than
    the staging buffer, or an output that does not start on 16 bytes), byte for byte against the checker, with the
    bytes around the text untouched and an output that ends inside the last 16-byte chunk."""
    import torch
    rng = np.random.default_rng(9)
    n = 5000   # 20 spans of 256 rows of 64 columns, each span longer than the staging buffer
    fmts = ["%d"] + ["%.9f"] * 63
    cols = rng.normal(0, 1e3, (64, n))
    cols[0] = np.arange(n)
    cols[1:, n // 2:] *= 1e12
    cols[5, 7] = np.nan
    want = _checker_table(cols, fmts)
    d = torch.from_numpy(cols).cuda()
    for start in (0, 3, 16):
        buf = torch.full((len(want) + 64,), 0xAB, dtype=torch.uint8, device="cuda")
        got = engine.csv_table_dev(d, fmts, out_dev=buf[start:start + len(want) + 40])
        assert bytes(got.cpu().numpy()) == want, start
        b = buf.cpu().numpy()
        assert not (b[:start] != 0xAB).any() and not (b[start + len(want):] != 0xAB).any(), start
    # short rows only (every span staged when the output starts on 16 bytes), and the output ending 7 bytes before the
    # text does
    small = d[:8, :3000].contiguous()
    want8 = _checker_table(cols[:8, :3000], fmts[:8])
    for start in (0, 5, 16):
        buf = torch.full((len(want8) + 64,), 0xAB, dtype=torch.uint8, device="cuda")
        got = engine.csv_table_dev(small, fmts[:8], out_dev=buf[start:start + len(want8) + 40])
        assert bytes(got.cpu().numpy()) == want8, start
        b = buf.cpu().numpy()
        assert not (b[:start] != 0xAB).any() and not (b[start + len(want8):] != 0xAB).any(), start
    buf = torch.full((len(want8) + 32,), 0xAB, dtype=torch.uint8, device="cuda")
    with pytest.raises(IscuError):
        engine.csv_table_dev(small, fmts[:8], out_dev=buf[:len(want8) - 7])
    b = buf.cpu().numpy()
    assert bytes(b[:len(want8) - 7]) == want8[:-7] and not (b[len(want8) - 7:] != 0xAB).any()
