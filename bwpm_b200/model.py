"""Problem descriptions of the reference's Python API, as plain data for the GPU facade.

Mirrors the attributes the reference facade reads (src/bwpm/fast.py:101-200) from
`Grid2D`/`Propagator2D` (src/bwpm/fpwpm.py:30-120), `Grid3D`/`Bidirectional3D`
(src/bwpm/volume3d.py:34-140) and the result types `BidirectionalResult`
(src/bwpm/bidirectional.py:47-65) and `Result3D` (src/bwpm/volume3d.py:85-99). Only the data and
the validation live here; stepping is done by the CUDA core (bwpm_b200._core).
`power_flux` is the reference facade's host-side energy bookkeeping (src/bwpm/fpwpm.py:205-216).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GRAZING_TOLERANCE = 1e-12


@dataclass(frozen=True)
class Grid2D:
    """Transverse grid (ny samples of dy mm), slab thickness dz (mm), wavelength (µm)."""

    ny: int
    dy: float
    dz: float
    wavelength_um: float

    def __post_init__(self) -> None:
        if self.ny < 2 or self.dy <= 0 or self.dz <= 0 or self.wavelength_um <= 0:
            raise ValueError("ny >= 2 and positive dy, dz, wavelength_um are required")

    @property
    def k0(self) -> float:
        return float(2.0 * np.pi / (self.wavelength_um * 1e-3))

    @property
    def y(self) -> np.ndarray:
        return np.asarray((np.arange(self.ny) - self.ny // 2) * self.dy, dtype=np.float64)

    @property
    def ky(self) -> np.ndarray:
        return np.asarray(2.0 * np.pi * np.fft.fftfreq(self.ny, d=self.dy), dtype=np.float64)


@dataclass(frozen=True)
class Grid3D:
    """Transverse grid (ny × nx) and step size; lengths in mm, wavelength in µm."""

    nx: int
    ny: int
    dx: float
    dy: float
    dz: float
    wavelength_um: float

    def __post_init__(self) -> None:
        if min(self.nx, self.ny) < 2 or min(self.dx, self.dy, self.dz, self.wavelength_um) <= 0:
            raise ValueError("nx, ny >= 2 and positive steps and wavelength are required")

    @property
    def k0(self) -> float:
        return float(2.0 * np.pi / (self.wavelength_um * 1e-3))

    @property
    def x(self) -> np.ndarray:
        return np.asarray((np.arange(self.nx) - self.nx // 2) * self.dx, dtype=np.float64)

    @property
    def y(self) -> np.ndarray:
        return np.asarray((np.arange(self.ny) - self.ny // 2) * self.dy, dtype=np.float64)

    def k_grid(self) -> tuple[np.ndarray, np.ndarray]:
        kx = 2.0 * np.pi * np.fft.fftfreq(self.nx, d=self.dx)
        ky = 2.0 * np.pi * np.fft.fftfreq(self.ny, d=self.dy)
        kxx, kyy = np.meshgrid(kx, ky)
        return np.asarray(kxx), np.asarray(kyy)


def _rolloff(coords: np.ndarray, width: float, order: int, edge: float) -> np.ndarray:
    a = np.abs(coords)
    if width == 0:
        return np.ones_like(a)
    u = np.clip((a - (float(np.max(a)) - width)) / width, 0.0, 1.0)
    return np.asarray(edge ** (u**order), dtype=np.float64)


def absorbing_mask(grid: Grid2D, width: float, order: int = 4, edge: float = 1e-6) -> np.ndarray:
    """Super-Gaussian absorbing mask m(y) (src/bwpm/fpwpm.py:66-85)."""
    if width < 0 or order < 1 or not 0 < edge < 1:
        raise ValueError("width >= 0, order >= 1 and 0 < edge < 1 are required")
    return _rolloff(grid.y, width, order, edge)


def absorbing_mask_2d(grid: Grid3D, width: float, order: int = 8, edge: float = 1e-6) -> np.ndarray:
    """Product of 1D masks in x and y, shape (ny, nx) (src/bwpm/volume3d.py:70-82)."""
    if width < 0 or order < 1 or not 0 < edge < 1:
        raise ValueError("width >= 0, order >= 1 and 0 < edge < 1 are required")
    return np.asarray(_rolloff(grid.y, width, order, edge)[:, None]
                      * _rolloff(grid.x, width, order, edge)[None, :])


def _check_labels(labels: np.ndarray, n_indices: int) -> None:
    if labels.size and (labels.min() < 0 or labels.max() >= n_indices):
        raise ValueError("labels must index into `indices`")


@dataclass
class Propagator2D:
    """2D volume: grid, indices per label, labels (nz, ny), medium before, mask (ny,), δn."""

    grid: Grid2D
    indices: list
    labels: np.ndarray
    index_before: complex
    mask: np.ndarray | None = None
    fluctuation: np.ndarray | None = None

    def __post_init__(self) -> None:
        labels = np.asarray(self.labels)
        if labels.ndim != 2 or labels.shape[1] != self.grid.ny:
            raise ValueError("labels must have shape (nz, ny)")
        _check_labels(labels, len(self.indices))


@dataclass
class Bidirectional3D:
    """3D volume: grid, indices, labels (nz, ny, nx), medium before, mask (ny, nx), δn."""

    grid: Grid3D
    indices: list
    labels: np.ndarray
    index_before: complex
    mask: np.ndarray | None = None
    sparse: bool = True
    workers: int | None = None
    fluctuation: np.ndarray | None = None

    def __post_init__(self) -> None:
        lab = np.asarray(self.labels)
        g = self.grid
        if lab.ndim != 3 or lab.shape[1:] != (g.ny, g.nx):
            raise ValueError("labels must have shape (nz, ny, nx)")
        _check_labels(lab, len(self.indices))


@dataclass(frozen=True)
class BidirectionalResult:
    transmitted: np.ndarray
    reflected: np.ndarray
    forward: np.ndarray | None
    backward: np.ndarray | None
    energy_residual: list


@dataclass(frozen=True)
class Result3D:
    transmitted: np.ndarray
    reflected: np.ndarray
    planes: dict
    stored_values: int


def longitudinal_wavenumber_host(index: complex, k0: float, kp2: np.ndarray) -> np.ndarray:
    """k_z for the host-side flux bookkeeping (src/bwpm/interface.py:26-48)."""
    n2k2 = complex(index) ** 2 * k0 * k0
    q = np.asarray(n2k2 - kp2, dtype=np.complex128)
    q = np.where(np.abs(q) <= GRAZING_TOLERANCE * abs(n2k2), 0.0, q)
    kz = np.sqrt(q)
    flip = (kz.imag < 0) | ((kz.imag == 0) & (kz.real < 0))
    kz = np.where(flip, -kz, kz)
    tiny = 1e-12 * k0
    return np.asarray(np.where(np.abs(kz) < tiny, 1j * tiny, kz))


def power_flux(field_xy: np.ndarray, grid: Grid2D, index: complex, direction: int = 1) -> float:
    """Power through the plane (Parseval sum of Re k_z·(|Ê|² + |Ê_z|²)), src/bwpm/fpwpm.py:205-216."""
    spectrum = np.fft.fft(field_xy, axis=0) / grid.ny
    kz = longitudinal_wavenumber_host(index, grid.k0, grid.ky**2)
    with np.errstate(divide="ignore", invalid="ignore"):
        ez = np.where(kz != 0, -direction * grid.ky * spectrum[:, 1] / kz, 0.0)
    magnitude = np.sum(np.abs(spectrum) ** 2, axis=1) + np.abs(ez) ** 2
    return float(np.sum(np.real(kz) * magnitude) * grid.ny * grid.dy)
