"""The ground-truth tables' number text: the checker (Python's printf-style formatting of the exact binary value, cut to
47 characters, nothing for NaN and infinities) pinned against the reference's own AppendCsvNumber (CsvNumber.cpp,
compiled into oracle/_ref), and the reference's table rows (GroundTruth's Rows: cells joined by ',', rows ended by
'\\n') against the same checker. CPU only; the device formatter is in tests/test_gpu_csv.py."""
import numpy as np
import pytest

TABLE_FMTS = ["%.6f", "%.4f", "%.3f", "%.6g", "%.4g", "%.9g"]   # the formats the tables use


def csv_values(seed=7, n=20000):
    """Values of every kind the tables' numbers meet: random magnitudes 1e-12 .. 1e12, exact binary fractions (decimal
    ties at some precisions), a few ulps either side of each precision's rounding boundaries, +-0, the extremes,
    NaN and infinities."""
    rng = np.random.default_rng(seed)
    v = [0.0, -0.0, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, -1e300, 1e-300, float("nan"),
         float("inf"), -float("inf"), 0.5, 1.5, 2.5, -2.5, 0.125, 1e15, 1e16, 1e22, 123456.5, 999999.5, 9.9999995]
    v += list(rng.choice([-1, 1], n) * rng.random(n) * 10.0 ** rng.integers(-12, 13, n))
    v += list(rng.integers(-1000000, 1000001, n) / 2.0 ** rng.integers(0, 31, n))
    for p in range(10):
        mid = (rng.integers(0, 2000000, n // 20) + 0.5) * 10.0 ** (-p)
        for k in range(-3, 4):
            v += list(np.nextafter(mid, np.inf if k > 0 else 0.0) if k else mid)
    return np.array(v, np.float64)


def printf(v, fmt):
    return (fmt % v)[:47] if np.isfinite(v) else ""


@pytest.mark.parametrize("fmt", TABLE_FMTS + ["%.0f", "%.9f", "%.0g", "%.1g"])
def test_checker_equals_reference(reference, fmt):
    v = csv_values(n=4000)
    assert reference.csv_numbers(v, fmt) == [printf(x, fmt) for x in v]


def test_reference_table_rows(reference):
    rng = np.random.default_rng(3)
    n = 40000   # several of the reference's 16,384-row chunks
    fmts = ["%d", "%.6f", "%.6g", "%.4f", "%.9g"]
    cols = np.stack([np.arange(n, dtype=np.float64), rng.random(n) * 100, rng.random(n) * 1e-3,
                     rng.normal(0, 50, n), rng.lognormal(7, 1, n)])
    text, _ = reference.csv_table(cols, fmts)
    want = "".join(",".join(str(int(cols[0, r])) if f == "%d" else printf(cols[c, r], f)
                            for c, f in enumerate(fmts)) + "\n" for r in range(n))
    assert text.decode() == want
