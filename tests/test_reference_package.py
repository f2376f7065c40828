"""MetalMom's own, unchanged Python package and tests against libmetalmom.so.

The drop-in claim at the boundary: MetalMom's cffi layer
(``python/metalmom/_native.py:505-515`` loads ``_lib/libmetalmom.dylib``
from the package directory) binds this library unchanged, and MetalMom's own
parity and bridge tests pass through it.

Set ``MM_REFERENCE_DIR`` to a MetalMom checkout (its ``python/metalmom``
package and ``Tests/`` directory).  The test copies the package into a
temporary directory, installs ``libmetalmom.so`` there under the file name
the package opens, copies the selected test files and ``Tests/golden`` next
to it (MetalMom's tests skip, rather than fail, when a golden is missing),
runs them with pytest in a subprocess, and fails on any failure, error or
skip.  Without ``MM_REFERENCE_DIR`` it is skipped (the checkout is not part of
this repository).

Deselected, each for a reason outside this library:
- ``test_bridge_errors.py::test_griffinlim_error`` and
  ``::test_neural_beat_decode_error`` call ``mm_griffinlim`` (phase
  reconstruction) and ``mm_neural_beat_decode`` (beat tracking), entry points
  of other MetalMom subsystems that this library does not export;
- ``test_parity_mel_filterbank.py::TestHzMelConversions::test_hz_to_mel_known_values``
  and ``::test_mel_to_hz_known_values`` import librosa (not installed) to
  check the test file's own helper functions, not the library.
"""

import os
import re
import shutil
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "metalmom_b200", "_lib", "libmetalmom.so")

TEST_FILES = [
    "test_parity_stft.py", "test_parity_melspec.py", "test_parity_mfcc.py", "test_parity_mel_filterbank.py",
    "test_parity_scaling.py", "test_parity_delta.py", "test_onset_strength.py", "test_bridge_errors.py",
]
DESELECT = [
    "Tests/test_bridge_errors.py::test_griffinlim_error",
    "Tests/test_bridge_errors.py::test_neural_beat_decode_error",
    "Tests/test_parity_mel_filterbank.py::TestHzMelConversions::test_hz_to_mel_known_values",
    "Tests/test_parity_mel_filterbank.py::TestHzMelConversions::test_mel_to_hz_known_values",
]


def _summary_counts(text):
    counts = {}
    for n, what in re.findall(r"(\d+) (passed|failed|skipped|errors?|deselected|xfailed|xpassed)", text):
        counts[what.rstrip("s") if what.startswith("error") else what] = int(n)
    return counts


def test_reference_package_and_tests_run_unchanged(tmp_path):
    ref = os.environ.get("MM_REFERENCE_DIR")
    if not ref:
        pytest.skip("MM_REFERENCE_DIR is not set (path of a MetalMom checkout)")
    pkg_src = os.path.join(ref, "python", "metalmom")
    tests_src = os.path.join(ref, "Tests")
    assert os.path.isdir(pkg_src) and os.path.isdir(tests_src), ref
    assert os.path.exists(LIB), "build libmetalmom.so first"

    pkg_dir = tmp_path / "site"
    shutil.copytree(pkg_src, pkg_dir / "metalmom")
    (pkg_dir / "metalmom" / "_lib").mkdir(exist_ok=True)
    shutil.copy(LIB, pkg_dir / "metalmom" / "_lib" / "libmetalmom.dylib")
    work = tmp_path / "run"
    (work / "Tests").mkdir(parents=True)
    shutil.copytree(os.path.join(tests_src, "golden"), work / "Tests" / "golden")
    for f in TEST_FILES:
        shutil.copy(os.path.join(tests_src, f), work / "Tests" / f)

    env = dict(os.environ, PYTHONPATH=str(pkg_dir))
    cmd = [sys.executable, "-m", "pytest", "-q", "-rs", "-p", "no:cacheprovider", "--rootdir", str(work)]
    cmd += [f"Tests/{f}" for f in TEST_FILES]
    for d in DESELECT:
        cmd += ["--deselect", d]
    r = subprocess.run(cmd, cwd=work, env=env, capture_output=True, text=True, timeout=900)
    out = r.stdout + r.stderr
    print(out[-6000:])
    counts = _summary_counts(out.strip().splitlines()[-1] if out.strip() else "")
    assert r.returncode == 0, out[-4000:]
    assert counts.get("passed", 0) > 0, out[-2000:]
    assert counts.get("skipped", 0) == 0, out[-4000:]
    assert counts.get("failed", 0) == 0 and counts.get("error", 0) == 0, out[-4000:]
    assert counts.get("deselected", 0) == len(DESELECT), counts
