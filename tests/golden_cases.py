"""Builds solver inputs from the converted golden files of the reference (tests/golden/*.npz).

The 2D cases use the reference facade's mapping onto the 3D core (src/bwpm/fast.py:120-142):
labels (nz, ny) -> (nz, ny, 1), field (ny, 2) -> (ny, 1, 2), mask (ny,) -> (ny, 1), nx = 1,
dx = 1.0; k0 = 2π/(λ·1e-3) (src/bwpm/fpwpm.py:50-53).
"""

from __future__ import annotations

import numpy as np

from conftest import load_golden


def k0_of(wavelength_um: float) -> float:
    return float(2.0 * np.pi / (wavelength_um * 1e-3))


def case_2d(name: str):
    """(core_args, field (ny,1,2), fluctuation or None, arrays, meta) of a 2D golden case."""
    a, meta = load_golden(name)
    ny = int(meta["parameters.ny"])
    labels = np.asarray(a["inputs.labels"], dtype=np.int32)[:, :, None]
    mask = a.get("inputs.mask")
    mask = None if mask is None else np.asarray(mask, dtype=np.float64)[:, None]
    fl = a.get("inputs.fluctuation")
    fl = None if fl is None else np.asarray(fl, dtype=np.complex128)[:, :, None]
    args = (ny, 1, float(meta["parameters.dy_mm"]), 1.0, float(meta["parameters.dz_mm"]),
            k0_of(float(meta["parameters.wavelength_um"])),
            np.asarray(a["inputs.indices"], dtype=np.complex128), labels,
            complex(a["inputs.index_before"]), mask)
    field = np.asarray(a["inputs.field"], dtype=np.complex128)[:, None, :]
    return args, field, fl, a, meta


def case_3d(name: str):
    a, meta = load_golden(name)
    mask = a.get("inputs.mask")
    fl = a.get("inputs.fluctuation")
    args = (int(meta["parameters.ny"]), int(meta["parameters.nx"]), float(meta["parameters.dy_mm"]),
            float(meta["parameters.dx_mm"]), float(meta["parameters.dz_mm"]),
            k0_of(float(meta["parameters.wavelength_um"])),
            np.asarray(a["inputs.indices"], dtype=np.complex128),
            np.asarray(a["inputs.labels"], dtype=np.int32), complex(a["inputs.index_before"]),
            None if mask is None else np.asarray(mask, dtype=np.float64))
    field = np.asarray(a["inputs.field"], dtype=np.complex128)
    return args, field, (None if fl is None else np.asarray(fl, dtype=np.complex128)), a, meta


def volume_case(d: dict, prefix: str):
    """Random-volume fixture (tests/golden/random_volumes.npz) -> (core_args, field, fl)."""
    g = d[prefix + "grid"]
    nx, ny = int(g[0]), int(g[1])
    dx, dy, dz, wl = float(g[2]), float(g[3]), float(g[4]), float(g[5])
    mask = d.get(prefix + "mask")
    fl = d.get(prefix + "fluctuation")
    args = (ny, nx, dy, dx, dz, k0_of(wl), d[prefix + "indices"],
            np.asarray(d[prefix + "labels"], dtype=np.int32), complex(d[prefix + "index_before"]),
            mask)
    return args, d[prefix + "field"], fl
