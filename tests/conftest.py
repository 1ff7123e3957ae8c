"""Shared test setup: the `gpu` marker, repository paths and golden-fixture loaders."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


def load_golden(case: str) -> tuple[dict, dict]:
    """(arrays, meta) of a converted golden file of the reference."""
    with np.load(GOLDEN / f"{case}.npz") as z:
        arrays = {k: z[k] for k in z.files if k != "meta"}
        meta = json.loads(str(z["meta"]))
    return arrays, meta


def load_npz(name: str) -> dict:
    with np.load(GOLDEN / name) as z:
        return {k: z[k] for k in z.files}


def close(a: np.ndarray, b: np.ndarray, rel: float, abs_: float) -> None:
    """numpy.allclose with the reference's {rel, abs} tolerance (tests/test_core_solver.py:228)."""
    assert a.shape == b.shape, (a.shape, b.shape)
    err = np.max(np.abs(a - b) - (abs_ + rel * np.abs(b)))
    assert np.allclose(a, b, rtol=rel, atol=abs_), f"excess error {err:.3e}"


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 error ‖a − b‖₂/‖b‖₂."""
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)
