"""GPU facade with the reference's `bwpm.fast` API (src/bwpm/fast.py:81-200).

`run_2d(propagator, field, iterations, keep, threads, backend, device)` and
`run_3d(solver, field, iterations, keep, threads, backend, device)` build the same
`_core.CudaSolver` call as the reference (2D as nx = 1, lateral axis y, fast.py:120-142) and
return the same result types. `backend` accepts "auto" and "cuda"; "cpu" raises ValueError
because this package has no CPU path. `threads` is accepted and ignored (GPU only).
Extension: `precision=64` (reference arithmetic) or `32` (complex64 fields).
"""

from __future__ import annotations

from typing import Any

import numpy as np

from bwpm_b200 import _core
from bwpm_b200._core import reflection_matrix, transmission_matrix
from bwpm_b200.model import (
    BidirectionalResult,
    Bidirectional3D,
    Propagator2D,
    Result3D,
    power_flux,
)

CORE_AVAILABLE = True


def cuda_available() -> bool:
    """True if a CUDA device is present."""
    return _core.cuda_device_count() > 0


def _solver(backend: str, device: int, fluctuation, precision: int, *args) -> Any:
    if backend not in ("auto", "cpu", "cuda"):
        raise ValueError("backend must be 'auto', 'cpu' or 'cuda'")
    if backend == "cpu":
        raise ValueError("bwpm_b200 has no CPU backend; use backend='cuda'")
    if not cuda_available():
        raise RuntimeError("CUDA backend requested but no device present")
    return _core.CudaSolver(*args, device, fluctuation=fluctuation, precision=precision)


def run_2d(propagator: Propagator2D, field, iterations: int = 3, keep: bool = False,
           threads: int | None = None, backend: str = "auto", device: int = 0,
           precision: int = 64) -> BidirectionalResult:
    """2D FPWPM (iterations = 0) or BWPM through the CUDA core (src/bwpm/fast.py:101-162)."""
    g = propagator.grid
    labels = np.asarray(propagator.labels, dtype=np.int32)[:, :, None]
    nz = labels.shape[0]
    mask = None if propagator.mask is None else np.asarray(propagator.mask)[:, None]
    fluctuation = None
    if propagator.fluctuation is not None:
        fluctuation = np.asarray(propagator.fluctuation, dtype=np.complex128)[:, :, None]
    solver = _solver(backend, device, fluctuation, precision, g.ny, 1, g.dy, 1.0, g.dz, g.k0,
                     np.asarray(propagator.indices, dtype=np.complex128), labels,
                     complex(propagator.index_before), mask)
    out = solver.run(np.asarray(field)[:, None, :], iterations,
                     list(range(nz + 1)) if keep else [])
    forward = backward = None
    if keep:
        forward = np.stack([out["forward"][p][:, 0] for p in range(nz + 1)])
        if iterations > 0:
            backward = np.stack([out["backward"][p][:, 0] for p in range(nz + 1)])
    residual = []
    if iterations > 0:
        p_in = power_flux(np.asarray(field), g, propagator.index_before)
        last = complex(propagator.indices[int(np.asarray(propagator.labels)[-1][g.ny // 2])])
        for t, r in zip(out["transmitted_iter"], out["reflected_iter"], strict=True):
            p_r = power_flux(r[:, 0], g, propagator.index_before, direction=-1)
            p_t = power_flux(t[:, 0], g, last)
            residual.append(1.0 - (p_r + p_t) / p_in if p_in > 0 else float("nan"))
    return BidirectionalResult(out["transmitted"][:, 0], out["reflected"][:, 0], forward,
                               backward, residual)


def run_3d(solver: Bidirectional3D, field, iterations: int = 1, keep: tuple = (),
           threads: int | None = None, backend: str = "auto", device: int = 0,
           precision: int = 64) -> Result3D:
    """3D run through the CUDA core (src/bwpm/fast.py:165-200)."""
    g = solver.grid
    fluctuation = None
    if solver.fluctuation is not None:
        fluctuation = np.asarray(solver.fluctuation, dtype=np.complex128)
    core = _solver(backend, device, fluctuation, precision, g.ny, g.nx, g.dy, g.dx, g.dz, g.k0,
                   np.asarray(solver.indices, dtype=np.complex128),
                   np.asarray(solver.labels, dtype=np.int32), complex(solver.index_before),
                   solver.mask)
    out = core.run(np.asarray(field), iterations, list(keep))
    zero = np.zeros_like(out["transmitted"])
    planes = {p: (out["forward"].get(p, zero), out["backward"].get(p, zero)) for p in keep}
    return Result3D(out["transmitted"], out["reflected"], planes, int(out["stored_values"]))


__all__ = ["CORE_AVAILABLE", "cuda_available", "reflection_matrix", "run_2d", "run_3d",
           "transmission_matrix"]
