"""Pages straight from device memory (iscu_tiff_pages_dev): frames copied out in chunks through two page-locked halves
while the previous chunk is written give the file the reference's TiffWriter writes from host pages, byte for byte --
one chunk and several (both halves reused), classic and BigTIFF, and a second writer on the same context reusing the
context's halves."""
import numpy as np
import pytest

from insiliscope_b200 import TiffWriter

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,h,w,big", [(7, 23, 37, False), (40, 512, 512, False), (18, 512, 512, True)])
def test_device_pages_equal_host_pages(engine, reference, tmp_path, n, h, w, big):
    import torch
    frames = np.random.default_rng(n).integers(0, 65536, (n, h, w)).astype(np.uint16)
    desc = f"device movie n={n}"
    d_frames = torch.from_numpy(frames).cuda()
    for attempt in range(2):
        path = tmp_path / f"dev{attempt}.tif"
        with TiffWriter(path, big=big) as t:
            t.pages_dev(engine, d_frames, desc)
            assert t.info()[1] == n
    ref = reference.tiff(tmp_path / "ref.tif", 0, big)
    for k in range(n):
        assert ref.page(frames[k], w, h, desc if k == 0 else None)
    assert ref.close()
    want = (tmp_path / "ref.tif").read_bytes()
    assert (tmp_path / "dev0.tif").read_bytes() == want
    assert (tmp_path / "dev1.tif").read_bytes() == want
