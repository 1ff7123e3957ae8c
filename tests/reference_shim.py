"""Runs the reference's own Python callers against this library (test infrastructure).

The reference's package, tests and golden files are staged, unchanged, in baseline/_ref by
oracle/stage_reference.sh. `install()` puts the drop-in shim in front of the reference's facade:
the module `bwpm._core` (cpp/python/bindings.cpp:122-180) becomes one whose GPU names
(`CudaSolver`, `HAS_CUDA`, `cuda_device_count`, `transmission_matrix`, `reflection_matrix`,
`longitudinal_wavenumber`) are bwpm_b200._core's and whose CPU class `Solver` is the reference's
own compiled core, so that `bwpm.fast` (src/bwpm/fast.py:86-98) and `bwpm.adapter`
(src/bwpm/adapter.py:210-241) with backend="cuda" run here while backend="cpu" stays the
reference's.

Usage: python tests/reference_shim.py [pytest arguments]   (pytest with the shim installed)
"""

from __future__ import annotations

import importlib.util
import sys
import types
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
STAGED = ROOT / "baseline" / "_ref"
GPU_NAMES = ("HAS_CUDA", "CudaSolver", "cuda_device_count", "transmission_matrix",
             "reflection_matrix", "longitudinal_wavenumber")


def staged() -> bool:
    """True when the reference package, its tests and golden files are staged."""
    return ((STAGED / "bwpm" / "fast.py").exists() and (STAGED / "tests").is_dir()
            and bool(sorted((STAGED / "bwpm").glob("_core*.so"))))


def reference_core():
    """The reference's compiled bwpm._core, loaded under its init name from baseline/_ref."""
    so = sorted((STAGED / "bwpm").glob("_core*.so"))[0]
    spec = importlib.util.spec_from_file_location("_core", so)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def install() -> types.ModuleType:
    """Binds `bwpm._core` to the shim; returns the reference's own compiled core."""
    ref = reference_core()
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    from bwpm_b200 import _core as ours

    shim = types.ModuleType("bwpm._core")
    shim.Solver = ref.Solver
    for name in GPU_NAMES:
        setattr(shim, name, getattr(ours, name))
    sys.path.insert(0, str(STAGED))
    sys.modules["bwpm._core"] = shim
    import bwpm

    bwpm._core = shim
    return ref


if __name__ == "__main__":
    import pytest

    install()
    sys.exit(pytest.main(sys.argv[1:]))
