"""Batched 2D solves on one GPU: many uneven problems in one launch of persistent kernels.

Each problem uses the reference's 2D convention (src/bwpm/fast.py:120-142: the 3D core with
nx = 1, lateral axis y, labels (nz, ny), field (ny, 2)). Fields are complex64 on the device;
operator tables are built in FP64 and the power flux per iteration is accumulated in FP64, so
the energy residual ε = 1 − (P_R + P_T)/P_in of the reference facade (src/bwpm/fast.py:148-155)
comes back with every result.
"""

from __future__ import annotations

import ctypes

import numpy as np

from bwpm_b200._lib import check, lib, ptr


class Batch2D:
    """Collects 2D problems, prepares them once, then solves all of them per `run()`."""

    def __init__(self, device: int = 0):
        self._h = None
        h = ctypes.c_void_p()
        check(lib.bwpm_batch_create(int(device), ctypes.byref(h)))
        self._h = h
        self._shapes: list[tuple[int, int]] = []  # (ny, iterations) per problem
        self._prepared = False

    def __del__(self):
        if getattr(self, "_h", None):
            lib.bwpm_batch_destroy(self._h)
            self._h = None

    def add(self, ny, dy, dz, k0, indices, labels, index_before, mask, field,
            iterations: int) -> int:
        """Adds one problem; labels (nz, ny) or (nz, ny, 1), field (ny, 2) or (ny, 1, 2)."""
        labels = np.ascontiguousarray(labels, dtype=np.int32)
        if labels.ndim == 3:
            labels = np.ascontiguousarray(labels[:, :, 0])
        if labels.ndim != 2 or labels.shape[1] != int(ny):
            raise ValueError("labels must have shape (nz, ny)")
        indices = np.ascontiguousarray(indices, dtype=np.complex128).ravel()
        f = np.ascontiguousarray(field, dtype=np.complex128).reshape(-1)
        if f.size != 2 * int(ny):
            raise ValueError("field must have shape (ny, 2)")
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64).ravel()
        ib = complex(index_before)
        out = ctypes.c_int64()
        check(lib.bwpm_batch_add(self._h, int(ny), float(dy), float(dz), float(k0), ptr(indices),
                                 indices.size, ptr(labels), labels.shape[0], ib.real, ib.imag,
                                 ptr(m), ptr(f), int(iterations), ctypes.byref(out)))
        self._shapes.append((int(ny), int(iterations)))
        return int(out.value)

    def add_problem(self, prob) -> int:
        """Adds a `bwpm_b200.workloads.Problem` with nx = 1."""
        if prob.nx != 1:
            raise ValueError("Batch2D takes 2D problems (nx = 1)")
        return self.add(prob.ny, prob.dy, prob.dz, prob.k0, prob.indices, prob.labels,
                        prob.index_before, prob.mask, prob.field, prob.iterations)

    def set_autotune(self, on: bool = True) -> None:
        """Times the kernel variants of each fixed length at prepare and keeps the fastest."""
        check(lib.bwpm_batch_set_autotune(self._h, int(bool(on))))

    def set_variant(self, ny: int, variant: int) -> None:
        """Forces kernel variant `variant` for length ny (see variant_count)."""
        check(lib.bwpm_batch_set_variant(self._h, int(ny), int(variant)))

    def classes(self) -> list[dict]:
        """Kernel classes of the prepared batch: length, threads, CTAs per line, variant."""
        out = []
        for k in range(self.stats()["classes"]):
            v = [ctypes.c_int64() for _ in range(5)]
            ms = ctypes.c_float()
            check(lib.bwpm_batch_class_info(self._h, k, *[ctypes.byref(x) for x in v],
                                            ctypes.byref(ms)))
            out.append({"ny": v[0].value, "threads": v[1].value, "cluster": v[2].value,
                        "variant": v[3].value, "items": v[4].value, "tuned_ms": ms.value})
        return out

    def prepare(self) -> None:
        check(lib.bwpm_batch_prepare(self._h))
        self._prepared = True

    def run(self) -> float:
        """Solves every problem once (inputs resident); returns the device time in ms."""
        ms = ctypes.c_float()
        check(lib.bwpm_batch_run(self._h, ctypes.byref(ms)))
        return float(ms.value)

    @property
    def packed_size(self) -> int:
        return sum(2 * ny for ny, _ in self._shapes)

    def solve_packed(self, fields: np.ndarray, out: np.ndarray) -> float:
        """End to end: new incident fields (packed complex128, Σ ny·2) in, packed
        (transmitted, reflected) per problem out; returns the device time in ms."""
        assert fields.dtype == np.complex128 and out.dtype == np.complex128
        assert fields.size == self.packed_size and out.size == 2 * self.packed_size
        ms = ctypes.c_float()
        check(lib.bwpm_batch_solve_packed(self._h, ptr(fields), ptr(out), ctypes.byref(ms)))
        return float(ms.value)

    def result(self, i: int) -> dict:
        ny, iters = self._shapes[i]
        t = np.empty((ny, 2), dtype=np.complex128)
        r = np.empty((ny, 2), dtype=np.complex128)
        ft = np.empty(max(iters, 1))
        fr = np.empty(max(iters, 1))
        fin = ctypes.c_double()
        lat = ctypes.c_double()
        check(lib.bwpm_batch_result(self._h, int(i), ptr(t), ptr(r), ptr(ft), ptr(fr),
                                    ctypes.byref(fin), ctypes.byref(lat)))
        ft, fr = ft[:iters], fr[:iters]
        p_in = fin.value
        eps = [1.0 - (a + b) / p_in if p_in > 0 else float("nan") for a, b in zip(ft, fr)]
        return {"transmitted": t, "reflected": r, "flux_t": ft, "flux_r": fr, "flux_in": p_in,
                "energy_residual": eps, "latency_ms": lat.value}

    def work(self) -> dict:
        """Algorithmic transforms, FLOPs and minimal DRAM bytes of one run."""
        t, f, y = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib.bwpm_batch_work(self._h, ctypes.byref(t), ctypes.byref(f), ctypes.byref(y)))
        return {"transforms": t.value, "flops": f.value, "bytes": y.value}

    def stats(self) -> dict:
        v = [ctypes.c_int64() for _ in range(5)]
        check(lib.bwpm_batch_stats(self._h, *[ctypes.byref(x) for x in v]))
        keys = ("device_bytes", "kernel_launches", "work_items", "classes", "packed_inputs")
        return {k: x.value for k, x in zip(keys, v)}


def variant_count(ny: int) -> int:
    """Number of compiled kernel variants for length ny (0: the generic kernels serve it)."""
    return int(lib.bwpm_variant_count(int(ny)))


def flush_l2(device: int = 0, nbytes: int = 512 << 20) -> None:
    """Overwrites `nbytes` of device scratch so the next run starts with a cold L2 (126 MB)."""
    check(lib.bwpm_flush_l2(int(device), int(nbytes)))


def host_register(a: np.ndarray) -> None:
    """Page-locks an array's memory (fast, asynchronous host copies)."""
    check(lib.bwpm_host_register(ptr(a), a.nbytes))


def host_unregister(a: np.ndarray) -> None:
    check(lib.bwpm_host_unregister(ptr(a)))
