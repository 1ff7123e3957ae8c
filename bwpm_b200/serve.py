"""Served request loop: continuous batching of 2D and 3D solves on one GPU.

A `Server` takes requests at any time (`submit`) and returns a ticket at once. 2D requests (the
reference's 2D convention, src/bwpm/fast.py:120-142) are prepared on host worker threads,
admitted longest estimated chain first (then in arrival order) while the device-memory budget
holds, and launched in groups on the
batched resident engine (complex64 fields, FP64 tables and power flux); groups launched while
others are still running share the GPU. 3D requests run through the complex64 plane engine on
their own streams. Every result carries its latency (submit → result on the host), its queueing
time (submit → launch) and, for 2D, the power flux per iteration (energy residual
ε = 1 − (P_R + P_T)/P_in as src/bwpm/fast.py:148-155).

The reference has no server; it solves one problem per `CudaSolver.run` call.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from bwpm_b200._lib import check, lib, ptr


class Server:
    """Continuous-batching request loop on one GPU (see the module docstring)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, max_groups: int = 0,
                 max_group_solves: int = 0, max_3d: int = 0):
        self._h = None
        h = ctypes.c_void_p()
        check(lib.bwpm_server_create(int(device), int(budget_bytes), int(max_groups),
                                     int(max_group_solves), int(max_3d), ctypes.byref(h)))
        self._h = h
        self._shape: dict[int, tuple[int, int, int, bool]] = {}  # ticket -> (ny, nx, iters, 3d)
        self._borrowed: dict[int, np.ndarray] = {}  # ticket -> labels the server reads later

    def close(self) -> None:
        """Waits for every submitted request, then releases the server."""
        if getattr(self, "_h", None):
            lib.bwpm_server_destroy(self._h)
            self._h = None
            self._borrowed.clear()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, prob, borrow: bool = True) -> int:
        """Submits a `bwpm_b200.workloads.Problem` (nx = 1: 2D, else 3D); returns its ticket.
        A 3D problem with `labels` None and a `geometry` has its labels generated on the device.

        borrow: the server takes the labels after the call returns (2D: copied by a preparation
        worker, 3D: read in place by the set-up; the Server holds the array until the request's
        result is taken), so a large 3D submission does not stall the caller; False copies
        everything inside the call."""
        indices = np.ascontiguousarray(prob.indices, dtype=np.complex128).ravel()
        field = np.ascontiguousarray(prob.field, dtype=np.complex128)
        mask = None if prob.mask is None else np.ascontiguousarray(prob.mask, dtype=np.float64)
        ib = complex(prob.index_before)
        t = ctypes.c_int64()
        if prob.fluctuation is not None:
            raise ValueError("the server takes problems without a fluctuation term")
        if prob.nx != 1 and prob.labels is None and prob.geometry is not None:
            # 3D without a label volume: labels generated on the device from the geometry
            from bwpm_b200.geometry import kind_of, params_of

            prm = params_of(prob.geometry)
            check(lib.bwpm_server_submit_3d_geometry(
                self._h, prob.ny, prob.nx, prob.dy, prob.dx, prob.dz, prob.k0, ptr(indices),
                indices.size, kind_of(prob.geometry), ptr(prm), prm.size, prob.nz, ib.real,
                ib.imag, ptr(mask), ptr(field), int(prob.iterations), ctypes.byref(t)))
            self._shape[t.value] = (prob.ny, prob.nx, int(prob.iterations), True)
            return int(t.value)
        labels = np.ascontiguousarray(prob.ensure_labels(), dtype=np.int32)
        nz = labels.shape[0]
        if prob.nx == 1:
            fn = lib.bwpm_server_submit_2d_borrowed if borrow else lib.bwpm_server_submit_2d
            check(fn(self._h, prob.ny, prob.dy, prob.dz, prob.k0, ptr(indices), indices.size,
                     ptr(labels), nz, ib.real, ib.imag, ptr(mask), ptr(field),
                     int(prob.iterations), ctypes.byref(t)))
        else:
            fn = lib.bwpm_server_submit_3d_borrowed if borrow else lib.bwpm_server_submit_3d
            check(fn(self._h, prob.ny, prob.nx, prob.dy, prob.dx, prob.dz, prob.k0, ptr(indices),
                     indices.size, ptr(labels), nz, ib.real, ib.imag, ptr(mask), ptr(field),
                     int(prob.iterations), ctypes.byref(t)))
        if borrow:
            self._borrowed[t.value] = labels
        self._shape[t.value] = (prob.ny, prob.nx, int(prob.iterations), prob.nx != 1)
        return int(t.value)

    def wait(self, ticket: int, timeout_s: float = -1.0) -> bool:
        done = ctypes.c_int()
        check(lib.bwpm_server_wait(self._h, int(ticket), float(timeout_s), ctypes.byref(done)))
        return bool(done.value)

    def result(self, ticket: int) -> dict:
        """Waits for the request and returns its results (the ticket is released)."""
        self.wait(ticket)
        self._borrowed.pop(ticket, None)  # finished: the server no longer reads the labels
        ny, nx, iters, is3d = self._shape.pop(ticket)
        t = np.empty((ny, nx, 2), dtype=np.complex128)
        r = np.empty((ny, nx, 2), dtype=np.complex128)
        ft = np.full(max(iters, 1), np.nan)
        fr = np.full(max(iters, 1), np.nan)
        fin, lat, que, dev = (ctypes.c_double() for _ in range(4))
        check(lib.bwpm_server_result(self._h, int(ticket), ptr(t), ptr(r), ptr(ft), ptr(fr),
                                     ctypes.byref(fin), ctypes.byref(lat), ctypes.byref(que),
                                     ctypes.byref(dev)))
        out = {"transmitted": t, "reflected": r, "latency_ms": lat.value, "queue_ms": que.value,
               "device_ms": dev.value}
        if not is3d:
            out["transmitted"] = t[:, 0]
            out["reflected"] = r[:, 0]
            ft, fr = ft[:iters], fr[:iters]
            p_in = fin.value
            out.update(flux_t=ft, flux_r=fr, flux_in=p_in,
                       energy_residual=[1.0 - (a + b) / p_in if p_in > 0 else float("nan")
                                        for a, b in zip(ft, fr)])
        return out

    def stats(self) -> dict:
        v = [ctypes.c_int64() for _ in range(8)]
        check(lib.bwpm_server_stats(self._h, *[ctypes.byref(x) for x in v]))
        keys = ("submitted", "completed", "failed", "groups", "bytes_in_flight", "peak_bytes",
                "kernel_launches", "max_concurrent")
        return {k: x.value for k, x in zip(keys, v)}


def serve_stream(server: Server, stream, time_scale: float = 1.0) -> tuple[list[dict], float]:
    """Submits (arrival_s, problem) pairs at their arrival times (scaled), collects every result;
    returns the results in submission order and the wall time from first arrival to last result."""
    t0 = time.perf_counter()
    tickets = []
    for arrival, prob in stream:
        delay = t0 + arrival * time_scale - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets.append(server.submit(prob))
    results = [server.result(t) for t in tickets]
    first = t0 + (stream[0][0] * time_scale if stream else 0.0)
    return results, time.perf_counter() - first
