"""The Python host refuses caller buffers the library would write past (wrong dtype, device, layout or too few
elements) before any device call: the checks themselves, on CPU tensors and arrays."""
import numpy as np
import pytest
import torch

from insiliscope_b200.engine import _require_array, _require_tensor


def test_tensor_check_accepts_and_refuses():
    t = torch.zeros(12, dtype=torch.float32)
    _require_tensor(t, "out", (torch.float32,), None, 12)           # host tensor, enough elements
    with pytest.raises(ValueError, match="at least 13"):
        _require_tensor(t, "out", (torch.float32,), None, 13)       # too small
    with pytest.raises(ValueError, match="float64"):
        _require_tensor(t, "out", (torch.float64,), None, 12)       # wrong dtype
    with pytest.raises(ValueError, match="cuda:0"):
        _require_tensor(t, "out", (torch.float32,), 0, 12)          # host tensor where a device one is needed
    with pytest.raises(ValueError):
        _require_tensor(torch.zeros(4, 6).t(), "out", (torch.float32,), None, 12)   # not contiguous
    with pytest.raises(ValueError):
        _require_tensor(np.zeros(12, np.float32), "out", (torch.float32,), None, 12)  # not a tensor
    _require_tensor(torch.zeros(3, dtype=torch.int32), "set_of", (torch.int32, torch.uint32), None, 3)


def test_array_check_accepts_and_refuses():
    a = np.zeros((2, 3, 3), np.float32)
    _require_array(a, "out", np.float32, 18)
    with pytest.raises(ValueError):
        _require_array(a, "out", np.float32, 19)
    with pytest.raises(ValueError):
        _require_array(a.astype(np.float64), "out", np.float32, 18)
    with pytest.raises(ValueError):
        _require_array(np.zeros((3, 6), np.float32).T, "out", np.float32, 18)
