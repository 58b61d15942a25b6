"""The movie writer (iscu_tiff_*) against the reference's own TiffWriter (cli/tiff_writer.h, compiled into oracle/_ref):
the same page sequences give the same files byte for byte -- classic and BigTIFF, uint16 and float32 pages,
descriptions in place and at an offset, odd lengths padded, strips written row by row -- and the same refusals with
the same messages. CPU only (the device-page form is in tests/test_gpu_tiff.py)."""
import numpy as np
import pytest

from insiliscope_b200 import IscuError, TiffWriter

DESC = "spec seed=42 frames=3 w=37 h=23 camera=sCMOS version=test"


def _frames(n, h, w, dtype=np.uint16, seed=0):
    rng = np.random.default_rng(seed)
    if dtype == np.uint16:
        return rng.integers(0, 65536, (n, h, w)).astype(np.uint16)
    return rng.normal(100.0, 30.0, (n, h, w)).astype(np.float32)


def _both(reference, tmp_path, name, ops, expected=0, big=False):
    """Runs ops (a list of (method, args)) on both writers; returns the two files' bytes."""
    ours_p, ref_p = tmp_path / f"{name}_ours.tif", tmp_path / f"{name}_ref.tif"
    ours, ref = TiffWriter(ours_p, expected, big), reference.tiff(ref_p, expected, big)
    for op, args in ops:
        if op == "page":
            px, desc = args
            ours.page(px, desc)
            assert ref.page(px, px.shape[1], px.shape[0], desc)
        elif op == "page_rows":
            px, w, h, desc = args
            ours.page_rows(px, w, h, desc)
            assert ref.page_rows(px, px.shape[0], w, h, desc)
        elif op == "rows":
            page, y0, px = args
            ours.rows(page, y0, px)
            assert ref.rows(page, y0, px.shape[0], px)
    assert ours.info()[0] == ref.big()
    ours.close()
    assert ref.close()
    return ours_p.read_bytes(), ref_p.read_bytes()


@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("dtype", [np.uint16, np.float32])
@pytest.mark.parametrize("desc", [DESC, None, "abc", "abcd", "1234567", "12345678"])
def test_pages_byte_for_byte(reference, tmp_path, big, dtype, desc):
    f = _frames(3, 23, 37, dtype)
    ops = [("page", (f[0], desc)), ("page", (f[1], None)), ("page", (f[2], desc))]
    a, b = _both(reference, tmp_path, "p", ops, big=big)
    assert a == b


def test_expected_size_picks_bigtiff(reference, tmp_path):
    # TiffWriter::Bytes and the switch at expected + 64 MB >= 2^32 - 1: one byte either side
    assert TiffWriter.bytes(2048, 2048, 500, 2, 1 << 16) == reference.L.ref_tiff_bytes(2048, 2048, 500, 2, 1 << 16)
    edge = 0xFFFFFFFF - (64 << 20)
    for expected, big in ((edge - 1, False), (edge, True)):
        w = TiffWriter(tmp_path / "e.tif", expected)
        r = reference.tiff(tmp_path / "e_ref.tif", expected)
        assert w.info()[0] == big == r.big()
        w.close()
        r.close()


def test_strips_equal_whole_pages(reference, tmp_path):
    f = _frames(4, 30, 21)
    ops = [("page_rows", (f[k, :8], 21, 30, DESC if k == 0 else None)) for k in range(4)]
    for y0 in (8, 20):
        for k in range(4):
            ops.append(("rows", (k, y0, f[k, y0: min(30, y0 + 12)])))
    a, b = _both(reference, tmp_path, "s", ops)
    whole, _ = _both(reference, tmp_path, "w", [("page", (f[k], DESC if k == 0 else None)) for k in range(4)])
    assert a == b == whole


def test_refusals_match(reference, tmp_path):
    """Rows outside their page, and a classic file's page that would pass 4 GB (refused before a byte of it is
    written): the same refusal and message as the reference's writer; the writer stays failed."""
    f = _frames(1, 10, 10)
    w, r = TiffWriter(tmp_path / "x.tif"), reference.tiff(tmp_path / "x.tif.ref")
    w.page(f[0])
    assert r.page(f[0], 10, 10)
    with pytest.raises(IscuError) as e:
        w.rows(0, 5, f[0][:6])
    assert not r.rows(0, 5, 6, f[0][:6])
    assert e.value.code == 7
    assert str(e.value).split(": ", 1)[1] == r.error().replace("x.tif.ref", "x.tif")
    with pytest.raises(IscuError):
        w.close()
    r.close()

    w, r = TiffWriter(tmp_path / "g.tif"), reference.tiff(tmp_path / "g.tif.ref")
    small = np.zeros(4, np.uint16)   # never read: the size check comes first
    assert w.lib.iscu_tiff_page_u16(w.h, small.ctypes.data, 65536, 32769, None) == 7
    msg = w.lib.iscu_last_error().decode()
    assert not r.page(small, 65536, 32769)
    assert msg == r.error().replace("g.tif.ref", "g.tif")
    assert w.info()[1:] == (0, 8)
    with pytest.raises(IscuError):
        w.page(f[0])
    with pytest.raises(IscuError):
        w.close()
    r.close()


def test_open_failure_message(reference, tmp_path):
    path = tmp_path / "missing" / "m.tif"
    with pytest.raises(IscuError) as e:
        TiffWriter(path)
    r = reference.tiff(path)
    assert e.value.code == 7
    assert str(e.value).split(": ", 1)[1] == r.error()
