"""Drop-in for the reference's compiled module `bwpm._core` (cpp/python/bindings.cpp:122-180).

Same names, argument meaning, result dict and exception types:
- `CudaSolver(ny, nx, dy, dx, dz, k0, indices, labels, index_before, mask, device=0,
  fluctuation=None)` with `.run(field, iterations, keep=[]) -> dict` (bindings.cpp:158-173),
- `HAS_CUDA`, `cuda_device_count()` (bindings.cpp:156-157),
- `transmission_matrix`, `reflection_matrix` (bindings.cpp:124-137),
- `longitudinal_wavenumber` (bindings.cpp:178-179).
All computation runs on the GPU through libbwpm_b200.so. The reference's CPU class `Solver` is
not provided: this package has no CPU path.

Extensions beyond the reference: keyword `precision` (64: complex128 fields, the reference's
arithmetic; 32: complex64 fields with FP64-built operator tables) and `gmres_tol`;
`CudaSolver.from_geometry` (labels generated on the device from a geometry, see
bwpm_b200.geometry).
"""

from __future__ import annotations

import ctypes

import numpy as np

from bwpm_b200._lib import check, lib, ptr

HAS_CUDA = True


def cuda_device_count() -> int:
    """Number of usable CUDA devices (0 without a driver)."""
    return int(lib.bwpm_cuda_device_count())


def _matrices(reflection: int, k_x, k_y, index_in, index_out, k0) -> np.ndarray:
    kx = np.ascontiguousarray(k_x, dtype=np.float64)
    ky = np.ascontiguousarray(k_y, dtype=np.float64)
    if kx.shape != ky.shape:
        raise ValueError("k_x and k_y must have the same shape")
    out = np.empty(kx.shape + (2, 2), dtype=np.complex128)
    a, b = complex(index_in), complex(index_out)
    check(lib.bwpm_interface_matrices(reflection, ptr(kx), ptr(ky), kx.size, a.real, a.imag,
                                      b.real, b.imag, float(k0), ptr(out)))
    return out


def transmission_matrix(k_x, k_y, index_in, index_out, k0) -> np.ndarray:
    """T of wende2023 eqs. (2), (3) without propagation factor, shape (..., 2, 2)."""
    return _matrices(0, k_x, k_y, index_in, index_out, k0)


def reflection_matrix(k_x, k_y, index_in, index_out, k0) -> np.ndarray:
    """R of wende2023 eqs. (8), (9) without propagation factor, shape (..., 2, 2)."""
    return _matrices(1, k_x, k_y, index_in, index_out, k0)


def longitudinal_wavenumber(index, k0, k_perp_sq):
    """k_z = sqrt(ñ²k₀² − k⊥²), Im k_z ≥ 0, grazing rule; scalar in, complex out (arrays too)."""
    kp2 = np.ascontiguousarray(k_perp_sq, dtype=np.float64)
    out = np.empty(kp2.shape, dtype=np.complex128)
    i = complex(index)
    check(lib.bwpm_longitudinal_wavenumber(i.real, i.imag, float(k0), ptr(kp2), kp2.size,
                                           ptr(out)))
    return complex(out) if out.ndim == 0 else out


class CudaSolver:
    """FPWPM/BWPM on the GPU (B200), the reference's `bwpm._core.CudaSolver`."""

    def __init__(self, ny, nx, dy, dx, dz, k0, indices, labels, index_before, mask,
                 device: int = 0, fluctuation=None, *, precision: int = 64,
                 gmres_tol: float | None = None):
        self._h = None
        labels = np.ascontiguousarray(labels, dtype=np.int32)
        if labels.ndim != 3:
            raise ValueError("labels must have shape (nz, ny, nx)")
        indices = np.ascontiguousarray(indices, dtype=np.complex128).ravel()
        mask_a = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        fl = None
        if fluctuation is not None:
            fl = np.ascontiguousarray(fluctuation, dtype=np.complex128)
            if fl.shape != labels.shape:
                raise ValueError("fluctuation must have the shape of labels")
        if gmres_tol is None:
            gmres_tol = 1e-12 if precision == 64 else 1e-6
        ib = complex(index_before)
        self.ny, self.nx, self.nz = int(ny), int(nx), int(labels.shape[0])
        self.precision = int(precision)
        h = ctypes.c_void_p()
        check(lib.bwpm_solver_create(self.ny, self.nx, float(dy), float(dx), float(dz), float(k0),
                                     ptr(indices), indices.size, ptr(labels), self.nz, ib.real,
                                     ib.imag, ptr(mask_a), int(device), ptr(fl), self.precision,
                                     float(gmres_tol), ctypes.byref(h)))
        self._h = h

    @classmethod
    def from_geometry(cls, ny, nx, dy, dx, dz, k0, indices, geometry: dict, index_before, mask,
                      device: int = 0, *, precision: int = 64) -> CudaSolver:
        """A solver whose labels are generated on the device from `geometry` (a dict as in
        bwpm_b200.workloads.geometry_labels); no label volume exists on the host."""
        from bwpm_b200.geometry import kind_of, params_of

        self = cls.__new__(cls)
        self._h = None
        indices = np.ascontiguousarray(indices, dtype=np.complex128).ravel()
        mask_a = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        prm = params_of(geometry)
        ib = complex(index_before)
        self.ny, self.nx, self.nz = int(ny), int(nx), int(geometry["nz"])
        self.precision = int(precision)
        h = ctypes.c_void_p()
        check(lib.bwpm_solver_create_geometry(
            self.ny, self.nx, float(dy), float(dx), float(dz), float(k0), ptr(indices),
            indices.size, kind_of(geometry), ptr(prm), prm.size, self.nz, ib.real, ib.imag,
            ptr(mask_a), int(device), self.precision, ctypes.byref(h)))
        self._h = h
        return self

    def __del__(self):
        if getattr(self, "_h", None):
            lib.bwpm_solver_destroy(self._h)
            self._h = None

    def run(self, field, iterations: int, keep=()) -> dict:
        """Returns {transmitted, reflected, transmitted_iter, reflected_iter, forward, backward,
        stored_values} like the reference (cpp/python/bindings.cpp:61-86)."""
        f = np.ascontiguousarray(field, dtype=np.complex128)
        if f.ndim != 3 or f.shape[2] != 2:
            raise ValueError("field must have shape (ny, nx, 2)")
        if f.size != 2 * self.ny * self.nx:
            raise ValueError("field must have shape (ny, nx, 2)")
        iterations = int(iterations)
        if iterations < 0:
            raise ValueError("iterations must be >= 0")
        kk = sorted({int(k) for k in keep})
        if any(k < 0 for k in kk):
            raise ValueError("keep planes must be non-negative")
        kk = [k for k in kk if k <= self.nz]
        keep_a = np.asarray(kk, dtype=np.int64)
        shape = (f.shape[0], f.shape[1], 2)
        t = np.empty(shape, dtype=np.complex128)
        r = np.empty(shape, dtype=np.complex128)
        ti = np.empty((iterations,) + shape, dtype=np.complex128) if iterations else None
        ri = np.empty((iterations,) + shape, dtype=np.complex128) if iterations else None
        fw = np.empty((len(kk),) + shape, dtype=np.complex128) if kk else None
        bw = np.empty((len(kk),) + shape, dtype=np.complex128) if kk and iterations else None
        stored = ctypes.c_int64(0)
        check(lib.bwpm_solver_run(self._h, ptr(f), iterations, ptr(keep_a) if kk else None,
                                  len(kk), ptr(t), ptr(r), ptr(ti), ptr(ri), ptr(fw), ptr(bw),
                                  ctypes.byref(stored)))
        return {
            "transmitted": t,
            "reflected": r,
            "transmitted_iter": [ti[i] for i in range(iterations)] if iterations else [],
            "reflected_iter": [ri[i] for i in range(iterations)] if iterations else [],
            "forward": {k: fw[i] for i, k in enumerate(kk)} if kk else {},
            "backward": {k: bw[i] for i, k in enumerate(kk)} if (kk and iterations) else {},
            "stored_values": int(stored.value),
        }

    def stats(self) -> dict:
        """Device bytes held, kernels launched so far, GMRES operator applications."""
        b, k, g = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib.bwpm_solver_stats(self._h, ctypes.byref(b), ctypes.byref(k), ctypes.byref(g)))
        return {"device_bytes": b.value, "kernel_launches": k.value, "gmres_applies": g.value}
