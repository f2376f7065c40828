"""Full-size clips of every group of the uneven mixed batch against the oracle.

One 120 s clip (the longest length of the uneven batch) for each of its 12
parameter groups -- sr 22050 / 44100, n_fft 1024 / 2048 / 4096 with hop
n_fft / 4, 64 / 128 mels, 20 MFCC -- run as one grouped plan (one branch per
group), so the kernels, layouts and table sets of the bench's uneven leg see
clips of the full length.  Each clip's MFCC is checked within 1e-4 of max |c|
and its log-mel rows (the plan's intermediate, floored at the clip maximum -
80 dB) within 1e-3 dB for values within 60 dB of the clip maximum, and below
that within the float32 rounding bound that the reference's own float32 path
shows on the same clip (``dbcheck.check_db``).
"""

import numpy as np
import pytest

from dbcheck import check_db

pytestmark = pytest.mark.gpu

MFCC_TOL = 1e-4
GROUPS = [dict(sr=sr, n_fft=nf, hop_length=nf // 4, n_mels=nm, n_mfcc=20)
          for sr in (22050, 44100) for nf in (1024, 2048, 4096) for nm in (64, 128)]


def _device_floats(ptr, n):
    import torch

    class View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 2}

    return torch.as_tensor(View(), device="cuda").cpu().numpy().copy()


def test_120s_clips_of_every_uneven_group_vs_oracle():
    import torch
    import metalmom_b200 as M
    from metalmom_b200 import synth
    from oracle import oracle as O, refcpu
    clips = [synth.music_clip(120 * g["sr"], g["sr"], seed=500 + i) for i, g in enumerate(GROUPS)]
    with M.Plan([len(c) for c in clips], clip_params=GROUPS) as plan:
        outs = plan.execute_host(clips)
        torch.cuda.synchronize()
        for i, (y, g) in enumerate(zip(clips, GROUPS)):
            sr, n_fft, hop, n_mels = g["sr"], g["n_fft"], g["hop_length"], g["n_mels"]
            exp_db = O.mel_db(y, sr, n_fft, hop, n_fft, True, n_mels)
            exp_c = O.dct_basis(20, n_mels) @ exp_db
            assert outs[i].shape == exp_c.shape, g
            assert O.mfcc_rel_error(outs[i], exp_c) < MFCC_TOL, (g, O.mfcc_rel_error(outs[i], exp_c))
            T = plan.frames[i]
            rows = _device_floats(plan.clip_mel_db_ptr(i), T * n_mels).reshape(T, n_mels).T
            got_db = np.maximum(rows.astype(np.float64), plan.clip_max_db(i) - 80.0)
            _, ref_db = refcpu.mfcc(y, sr, 20, n_fft, hop, n_fft, n_mels, 0.0, 0.0, True, want_mel_db=True)
            check_db(got_db, exp_db, ref_db, g)
