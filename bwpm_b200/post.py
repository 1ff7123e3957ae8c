"""Post-processing of fields on the GPU (FP64, compensated sums), through the C ABI.

Same quantities and conventions as the reference's host functions:
- `port_power` — bwpm.adapter.port_power (src/bwpm/adapter.py:267-284), for a PortField-like
  object (`.port` with nx, ny, dx, dy, wavelength_um, index, direction; `.field` (ny, nx, 2)) or
  for plain arrays through `port_power_array`;
- `power_flux` — bwpm.fpwpm.power_flux (src/bwpm/fpwpm.py:205-216), the 2D flux (nx = 1);
- `plane_power`, `axial_focus` — bwpm.pilot_imc3d (src/bwpm/pilot_imc3d.py:55-131), for a
  Grid3D-like grid (nx, ny, dx, dy, k0).
"""

from __future__ import annotations

import ctypes

import numpy as np

from bwpm_b200._lib import check, lib, ptr


def _k0(wavelength_um: float) -> float:
    return float(2.0 * np.pi / (wavelength_um * 1e-3))


def _field(field, ny: int, nx: int) -> np.ndarray:
    f = np.ascontiguousarray(field, dtype=np.complex128)
    if f.size != 2 * ny * nx:
        raise ValueError("field must have shape (ny, nx, 2)")
    return f


def port_power_array(field, dy: float, dx: float, k0: float, index: complex, direction: int,
                     device: int = 0) -> float:
    """Poynting flux of a (ny, nx, 2) field through a plane of a homogeneous medium."""
    f = np.asarray(field)
    ny, nx = int(f.shape[0]), int(f.shape[1]) if f.ndim == 3 else 1
    f = _field(f, ny, nx)
    index = complex(index)
    out = ctypes.c_double()
    check(lib.bwpm_port_power(int(device), ny, nx, float(dy), float(dx), float(k0), index.real,
                              index.imag, int(direction), ptr(f), ctypes.byref(out)))
    return float(out.value)


def port_power(port_field, device: int = 0) -> float:
    """bwpm.adapter.port_power on the device."""
    p = port_field.port
    return port_power_array(port_field.field, p.dy, p.dx, _k0(p.wavelength_um), p.index,
                            p.direction, device)


def power_flux(field_xy, dy: float, k0: float, index: complex, direction: int = 1,
               device: int = 0) -> float:
    """2D flux of a (ny, 2) field (bwpm.fpwpm.power_flux): the port power with nx = 1, dx = 1."""
    f = np.asarray(field_xy)
    return port_power_array(f.reshape(f.shape[0], 1, 2), dy, 1.0, k0, index, direction, device)


def plane_power(field, grid, index: float, device: int = 0) -> float:
    """bwpm.pilot_imc3d.plane_power on the device (grid: nx, ny, dx, dy, k0)."""
    f = _field(field, int(grid.ny), int(grid.nx))
    out = ctypes.c_double()
    check(lib.bwpm_plane_power(int(device), int(grid.ny), int(grid.nx), float(grid.dy),
                               float(grid.dx), float(grid.k0), float(index), ptr(f),
                               ctypes.byref(out)))
    return float(out.value)


def axial_focus(field, grid, index: float, offsets, na: float | None = None,
                device: int = 0, return_intensity: bool = False):
    """bwpm.pilot_imc3d.axial_focus on the device: (offset of the maximum, maximum), plus the
    intensity at every offset when return_intensity."""
    f = _field(field, int(grid.ny), int(grid.nx))
    off = np.ascontiguousarray(offsets, dtype=np.float64).ravel()
    inten = np.empty(off.size)
    best, peak = ctypes.c_double(), ctypes.c_double()
    check(lib.bwpm_axial_focus(int(device), int(grid.ny), int(grid.nx), float(grid.dy),
                               float(grid.dx), float(grid.k0), float(index), ptr(off), off.size,
                               0.0 if na is None else float(na), ptr(f), ctypes.byref(best),
                               ctypes.byref(peak), ptr(inten)))
    if return_intensity:
        return float(best.value), float(peak.value), inten
    return float(best.value), float(peak.value)
