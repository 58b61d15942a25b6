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
