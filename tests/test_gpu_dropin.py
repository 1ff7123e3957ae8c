"""The drop-in, shown with the reference's own callers and its own GPU core (on a GPU).

1. The reference's unmodified test files for its CUDA core and its Fusion adapter
   (tests/test_core_cuda.py, tests/test_adapter_conformance.py of the reference, staged in
   baseline/_ref with its package and golden files by oracle/stage_reference.sh) run with
   `bwpm._core` bound to the shim of tests/reference_shim.py: `bwpm.fast.run_2d/run_3d(...,
   backend="cuda")` and `bwpm.adapter.apply(..., backend="cuda")` then run on this library, and
   the reference's own assertions (rel 1e-10 against its golden files and against its CPU core,
   src/bwpm/fast.py:86-200, src/bwpm/adapter.py:210-241) must hold. BWPM_REQUIRE_CUDA=1 makes a
   missing CUDA path fail instead of skip (tests/test_core_cuda.py:24-27 of the reference).
2. This library's FP64 CudaSolver against the reference's own CudaSolver (cpp/src/solver_cuda.cu,
   built for sm_100a with cuFFT) on the same device, at the reference's CUDA tolerance.
"""

from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

import reference_shim
from conftest import ROOT, load_npz
from golden_cases import volume_case

pytestmark = pytest.mark.gpu

needs_staged = pytest.mark.skipif(not reference_shim.staged(),
                                  reason="reference not staged (oracle/stage_reference.sh)")


@needs_staged
def test_reference_callers_pass_through_the_shim():
    tests = reference_shim.STAGED / "tests"
    env = dict(os.environ, BWPM_REQUIRE_CUDA="1", PYTHONDONTWRITEBYTECODE="1")
    r = subprocess.run(
        [sys.executable, str(ROOT / "tests" / "reference_shim.py"), "-q", "-m", "not slow",
         "-p", "no:cacheprovider", "-rs", str(tests / "test_core_cuda.py"),
         str(tests / "test_adapter_conformance.py")],
        capture_output=True, text=True, timeout=1800, env=env, cwd=str(reference_shim.STAGED))
    tail = r.stdout[-4000:] + r.stderr[-2000:]
    assert r.returncode == 0, tail
    assert " passed" in r.stdout and "skipped" not in r.stdout.splitlines()[-1], tail


@needs_staged
@pytest.mark.parametrize("prefix,iters", [("volume1.", 2), ("volume2.", 2), ("volume3.", 2),
                                          ("fluct1.", 1), ("backscatter.", 3)])
def test_fp64_matches_the_reference_gpu_core(prefix, iters):
    """Same inputs on the same device through both GPU cores; rel 1e-10 (the reference's
    CUDA-against-CPU tolerance, tests/test_core_cuda.py:108-110 of the reference)."""
    from bwpm_b200 import _core

    ref_core = reference_shim.reference_core()
    assert ref_core.HAS_CUDA and ref_core.cuda_device_count() > 0
    args, field, fl = volume_case(load_npz("random_volumes.npz"), prefix)
    ours = _core.CudaSolver(*args, 0, fluctuation=fl).run(field, iters, [])
    theirs = ref_core.CudaSolver(*args, 0, fluctuation=fl).run(field, iters, [])
    scale = 1e-10 * float(np.max(np.abs(field)))
    for key in ("transmitted", "reflected"):
        assert np.max(np.abs(ours[key] - theirs[key])) < scale, key
