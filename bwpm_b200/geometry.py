"""Label volumes generated on the GPU from a geometry (the C ABI's bwpm_geometry_labels).

A geometry is a dict as taken by bwpm_b200.workloads.geometry_labels (the host generator with
the same FP64 operations): kind ∈ {tilted_facet, lens_array, microlens, tilted_slab}, grid
(nz, ny, nx, dz, dy, dx) and the body's parameters. Labels follow the reference's
labels_at_centres rule (src/bwpm/geometry.py:24-37).
"""

from __future__ import annotations

import numpy as np

from bwpm_b200._lib import check, lib, ptr

KINDS = {"tilted_facet": 0, "lens_array": 1, "microlens": 2, "tilted_slab": 3}
PARAMS = ("base", "tan_tilt", "pitch", "sag", "radius", "vertex", "back")


def kind_of(g: dict) -> int:
    try:
        return KINDS[g["kind"]]
    except KeyError as e:
        raise ValueError(f"unknown geometry kind {g.get('kind')!r}") from e


def params_of(g: dict) -> np.ndarray:
    """The BWPM_GEOMETRY_PARAMS parameters in C-ABI order (absent ones 0)."""
    return np.array([float(g.get(k, 0.0)) for k in PARAMS], dtype=np.float64)


def device_labels(g: dict, device: int = 0) -> np.ndarray:
    """uint8 labels (nz, ny, nx) generated on the device, copied back (for checks)."""
    nz, ny, nx = int(g["nz"]), int(g["ny"]), int(g["nx"])
    out = np.empty((nz, ny, nx), dtype=np.uint8)
    prm = params_of(g)
    check(lib.bwpm_geometry_labels(int(device), kind_of(g), ptr(prm), prm.size, nz, ny, nx,
                                   float(g["dz"]), float(g["dy"]), float(g["dx"]), ptr(out)))
    return out
