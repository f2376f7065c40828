"""Host-side checks of the S= paths and the device dB wrappers (no GPU
needed): shape validation happens before any library call."""

import numpy as np
import pytest

import metalmom_b200 as M


def test_mel_project_rejects_mismatched_rows():
    # numpy's matmul in the reference raises ValueError for this shape
    with pytest.raises(ValueError):
        M.melspectrogram(S=np.ones((513, 10), np.float32), n_fft=2048)
    with pytest.raises(ValueError):  # a scalar becomes shape (1,): one row
        M.melspectrogram(S=np.float32(1.0))


def test_device_db_rejects_host_arrays():
    import torch
    with pytest.raises(ValueError):
        M.power_to_db_device(torch.ones(8))  # a CPU tensor
