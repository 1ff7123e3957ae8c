"""CPU oracle for the post-processing of fields (test infrastructure only; never on the product
path): a numpy restatement of the reference's port power, plane power, axial focus and 2D
power flux, each function citing the reference lines it follows. Pinned against outputs of the
reference's own functions on seeded inputs (tests/golden/postproc.npz, generated by
tests/golden/make_fixtures.py `post`).
"""

from __future__ import annotations

import numpy as np

GRAZING_TOLERANCE = 1e-12  # src/bwpm/interface.py:34-41
GRAZING_COS = 1e-9  # src/bwpm/pilot_imc3d.py:18


def fftfreq_2pi(n: int, d: float) -> np.ndarray:
    return 2.0 * np.pi * np.fft.fftfreq(n, d=d)


def kz_of(index: complex, k0: float, kp2: np.ndarray) -> np.ndarray:
    """k_z with Im ≥ 0 and the grazing rule (src/bwpm/interface.py:26-48)."""
    n2k2 = complex(index) ** 2 * k0 * k0
    q = np.asarray(n2k2 - kp2, dtype=np.complex128)
    q = np.where(np.abs(q) <= GRAZING_TOLERANCE * abs(n2k2), 0.0, q)
    kz = np.sqrt(q)
    kz = np.where((kz.imag < 0) | ((kz.imag == 0) & (kz.real < 0)), -kz, kz)
    tiny = 1e-12 * k0
    return np.where(np.abs(kz) < tiny, 1j * tiny, kz)


def k_grid(ny: int, nx: int, dy: float, dx: float) -> tuple[np.ndarray, np.ndarray]:
    """(k_x, k_y), shape (ny, nx) (src/bwpm/volume3d.py:62-67)."""
    kxx, kyy = np.meshgrid(fftfreq_2pi(nx, dx), fftfreq_2pi(ny, dy))
    return kxx, kyy


def port_power(field: np.ndarray, dy: float, dx: float, k0: float, index: complex,
               direction: int) -> float:
    """src/bwpm/adapter.py:267-284."""
    ny, nx = field.shape[:2]
    kx, ky = k_grid(ny, nx, dy, dx)
    spectrum = np.fft.fft2(field, axes=(0, 1))
    kz = kz_of(index, k0, kx * kx + ky * ky)
    ez = -direction * (kx * spectrum[..., 0] + ky * spectrum[..., 1]) / kz
    magnitude = np.sum(np.abs(spectrum) ** 2, axis=-1) + np.abs(ez) ** 2
    return float(np.sum(np.real(kz) * magnitude) * dx * dy / (nx * ny))


def power_flux(field_xy: np.ndarray, dy: float, k0: float, index: complex,
               direction: int = 1) -> float:
    """2D flux of src/bwpm/fpwpm.py:205-216 (field (ny, 2))."""
    ny = field_xy.shape[0]
    spectrum = np.fft.fft(field_xy, axis=0) / ny
    ky = fftfreq_2pi(ny, dy)
    kz = kz_of(index, k0, ky**2)
    ez = -direction * ky * spectrum[:, 1] / kz
    magnitude = np.sum(np.abs(spectrum) ** 2, axis=1) + np.abs(ez) ** 2
    return float(np.sum(np.real(kz) * magnitude) * ny * dy)


def _cos_theta(kx, ky, index: float, k0: float) -> np.ndarray:
    """src/bwpm/pilot_imc3d.py:46-52."""
    k = index * k0
    cos_t = np.sqrt(np.maximum(1.0 - (kx**2 + ky**2) / k**2, 0.0))
    return np.where(cos_t > GRAZING_COS, cos_t, 0.0)


def plane_power(field: np.ndarray, dy: float, dx: float, k0: float, index: float) -> float:
    """src/bwpm/pilot_imc3d.py:24-67."""
    ny, nx = field.shape[:2]
    kx, ky = k_grid(ny, nx, dy, dx)
    a = np.fft.fft2(field, axes=(0, 1))
    cos_t = _cos_theta(kx, ky, index, k0)
    kp = np.hypot(kx, ky)
    safe = np.where(kp > 0, kp, 1.0)
    sx, sy = np.where(kp > 0, -ky / safe, 0.0), np.where(kp > 0, kx / safe, 1.0)
    px, py = np.where(kp > 0, kx / safe, 1.0), np.where(kp > 0, ky / safe, 0.0)
    e_s = a[..., 0] * sx + a[..., 1] * sy
    e_p = (a[..., 0] * px + a[..., 1] * py) / np.where(cos_t > GRAZING_COS, cos_t, 1.0)
    return float(index * np.sum(cos_t * (np.abs(e_s) ** 2 + np.abs(e_p) ** 2)))


def axial_focus_intensity(field: np.ndarray, dy: float, dx: float, k0: float, index: float,
                          offsets: np.ndarray, na: float | None = None) -> np.ndarray:
    """On-axis intensity per offset (src/bwpm/pilot_imc3d.py:96-131)."""
    ny, nx = field.shape[:2]
    kx, ky = k_grid(ny, nx, dy, dx)
    a = np.fft.fft2(field, axes=(0, 1))
    a = a * np.exp(1j * (kx * (nx // 2) * dx + ky * (ny // 2) * dy))[..., None]
    cos_t = _cos_theta(kx, ky, index, k0)
    prop = cos_t > 0
    if na is not None:
        prop &= np.hypot(kx, ky) <= na * k0
    kz = (index * k0 * cos_t)[prop]
    ax, ay = a[..., 0][prop], a[..., 1][prop]
    az = -(kx[prop] * ax + ky[prop] * ay) / kz
    out = []
    for d in np.asarray(offsets, dtype=np.float64):
        ph = np.exp(1j * kz * d)
        out.append(sum(abs(np.sum(c * ph)) ** 2 for c in (ax, ay, az)) / (nx * ny) ** 2)
    return np.array(out)


def axial_focus(field, dy, dx, k0, index, offsets, na=None) -> tuple[float, float]:
    """(offset of the first maximum, maximum) (src/bwpm/pilot_imc3d.py:125-131)."""
    inten = axial_focus_intensity(field, dy, dx, k0, index, offsets, na)
    best, peak = 0.0, -1.0
    for d, v in zip(np.asarray(offsets, dtype=np.float64), inten):
        if v > peak:
            best, peak = float(d), float(v)
    return best, peak
