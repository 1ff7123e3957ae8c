"""The C ABI library loads and exports every entry point that include/*.h declares (no GPU)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(bwpm_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from bwpm_b200 import _lib

    names = declared_symbols()
    assert "bwpm_solver_run" in names
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) <= names


def test_device_count_without_gpu_is_an_int():
    from bwpm_b200 import _core

    assert isinstance(_core.cuda_device_count(), int)


def test_errors_map_to_value_error():
    import numpy as np
    import pytest

    from bwpm_b200 import _core

    with pytest.raises(ValueError, match="labels must have shape"):
        _core.CudaSolver(4, 1, 1.0, 1.0, 1.0, 1.0, np.array([1.0]), np.zeros((2, 4)), 1.0, None)


def test_every_batched_length_has_a_kernel_variant():
    """The lengths of the batched workload all have compiled register-resident kernels."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import variant_count

    for n in workloads.BATCH_SIZES:
        assert variant_count(n) >= 1, n
    assert variant_count(1000) == 0  # served by the generic kernels
