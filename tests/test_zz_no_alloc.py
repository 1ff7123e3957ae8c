"""The allocation-free slab step (bwpm_step2d_noalloc) against the allocating solver, on a GPU.

bwpm_step2d_noalloc serves callers that cannot allocate device memory when they need a step
(a host framework owning all device memory in its own arena, a real-time loop, a plugin with a
fixed budget): it keeps its scratch in a fixed device array inside the library. This test hands
it device buffers (made here with torch) through the C ABI and checks two calls in a row against
bwpm_solver_run (through bwpm_b200._core.CudaSolver, iterations = 0) at the tolerance of the other
FP64 GPU tests: rel 1e-10, abs 1e-11·max. The file name makes pytest collect it last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL, ATOL_REL = 1e-10, 1e-11


def _close(a, b):
    assert a.shape == b.shape
    assert np.allclose(a, b, rtol=RTOL, atol=ATOL_REL * float(np.max(np.abs(b)) or 1.0))


def _geometry(ny: int, nz: int):
    """Tilted glass/silver interfaces (several label pairs per step), mask, TE + TM field."""
    lam = 0.6e-3
    dy, dz = lam / 8, lam / 10
    y = (np.arange(ny) - ny // 2) * dy
    z = (np.arange(nz) + 0.5) * dz
    labels = np.where(z[:, None] > 0.4 * nz * dz + 0.05 * y[None, :], 1, 0).astype(np.int32)
    labels[z > 0.8 * nz * dz] = 2
    indices = np.array([1.0, 1.52, 0.135 + 3.98j])
    mask = np.exp(-((np.abs(y) / (0.45 * ny * dy)) ** 16))
    field = np.zeros((ny, 1, 2), dtype=np.complex128)
    field[:, 0, 0] = np.exp(-((y / (ny * dy / 8)) ** 2)) * np.exp(1j * 0.3 * 2 * np.pi / lam * y)
    field[:, 0, 1] = 0.4j * field[:, 0, 0]
    return dy, dz, 2 * np.pi / lam, indices, labels, mask, field


def _noalloc(torch, lib, ny, dy, dz, k0, indices, lb, la, ib, mask, field):
    dev = torch.device("cuda", 0)
    fin = torch.from_numpy(np.ascontiguousarray(field.reshape(ny, 2))).to(dev)
    fout = torch.zeros_like(fin)
    d_la = torch.from_numpy(np.ascontiguousarray(la, dtype=np.int32)).to(dev)
    d_lb = None if lb is None else torch.from_numpy(np.ascontiguousarray(lb, dtype=np.int32)).to(dev)
    d_mask = torch.from_numpy(np.ascontiguousarray(mask, dtype=np.float64)).to(dev)
    idx = np.ascontiguousarray(indices, dtype=np.complex128)
    ib = complex(ib)
    torch.cuda.synchronize()
    status = lib.bwpm_step2d_noalloc(
        0, ny, dy, dz, k0, idx.ctypes.data, idx.size, None if d_lb is None else d_lb.data_ptr(),
        d_la.data_ptr(), ib.real, ib.imag, d_mask.data_ptr(), fin.data_ptr(), fout.data_ptr(), None)
    return status, fout.cpu().numpy().reshape(ny, 1, 2)


@pytest.mark.parametrize("ny", [384, 1024])
def test_noalloc_step_matches_solver_on_two_calls(ny):
    torch = pytest.importorskip("torch")
    from bwpm_b200 import _core
    from bwpm_b200._lib import check, lib

    assert torch.cuda.is_available()
    dy, dz, k0, indices, labels, mask, field = _geometry(ny, 24)
    p = 10  # step from plane p to plane p + 1 crosses the tilted glass face (several pairs)
    solver = _core.CudaSolver(ny, 1, dy, 1.0, dz, k0, indices, labels[:, :, None], 1.0 + 0j,
                              mask[:, None], 0)
    ref = solver.run(field, 0, [p, p + 1])
    # call 1: a step inside the volume, input = the solver's plane p
    st, out1 = _noalloc(torch, lib, ny, dy, dz, k0, indices, labels[p - 1], labels[p], 1.0,
                        mask, ref["forward"][p])
    check(st)
    _close(out1, ref["forward"][p + 1])
    # call 2, right after: the first step from the medium before the volume (labels_before NULL)
    first = _core.CudaSolver(ny, 1, dy, 1.0, dz, k0, indices, labels[:1, :, None], 1.0 + 0j,
                             mask[:, None], 0).run(field, 0, [])
    st, out2 = _noalloc(torch, lib, ny, dy, dz, k0, indices, None, labels[0], 1.0, mask, field)
    check(st)
    _close(out2, first["transmitted"])


def test_noalloc_wide_staging_length_matches_oracle():
    """7776 = 2^5·3^5 needs the kernel's wider FFT staging (more than 512 threads at 16 values
    per thread); checked against the CPU oracle's first step (oracle/port.py) at the same
    tolerance, on two calls in a row."""
    torch = pytest.importorskip("torch")
    from bwpm_b200._lib import check, lib
    from oracle import port

    ny = 7776
    dy, dz, k0, indices, labels, mask, field = _geometry(ny, 4)
    lab = labels[1:3].copy()
    lab[1][: ny // 4] = 2  # air/glass, air/silver and glass/silver pairs in one step
    ref = port.Solver(ny, 1, dy, 1.0, dz, k0, indices, lab[:, :, None], 1.0 + 0j,
                      mask[:, None]).run(field, 0, [1, 2])
    for _ in range(2):
        st, out = _noalloc(torch, lib, ny, dy, dz, k0, indices, lab[0], lab[1], 1.0, mask,
                           ref["forward"][1])
        check(st)
        _close(out, ref["forward"][2])


def test_noalloc_bad_label_then_valid_call_and_no_allocation():
    """A label outside `indices` is found on the device and returns BWPM_EINVAL with the
    reference's message; the next valid call starts from a cleared status word and is correct;
    neither call changes the device's free memory."""
    torch = pytest.importorskip("torch")
    from bwpm_b200 import _core
    from bwpm_b200._lib import BWPM_EINVAL, check, last_error, lib

    ny = 512
    dy, dz, k0, indices, labels, mask, field = _geometry(ny, 8)
    dev = torch.device("cuda", 0)
    bad = labels[0].copy()
    bad[ny // 3] = indices.size  # one label equal to m
    d_bad = torch.from_numpy(bad).to(dev)
    d_good = torch.from_numpy(np.ascontiguousarray(labels[0])).to(dev)
    d_mask = torch.from_numpy(np.ascontiguousarray(mask)).to(dev)
    fin = torch.from_numpy(np.ascontiguousarray(field.reshape(ny, 2))).to(dev)
    fout = torch.zeros_like(fin)
    idx = np.ascontiguousarray(indices, dtype=np.complex128)

    def call(d_lab):
        return lib.bwpm_step2d_noalloc(0, ny, dy, dz, k0, idx.ctypes.data, idx.size, None,
                                       d_lab.data_ptr(), 1.0, 0.0, d_mask.data_ptr(),
                                       fin.data_ptr(), fout.data_ptr(), None)

    check(call(d_good))  # the module and the scratch address are set up before measuring
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    st = call(d_bad)
    assert st == BWPM_EINVAL
    assert "labels must index into" in last_error()
    fout.zero_()
    torch.cuda.synchronize()
    check(call(d_good))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    first = _core.CudaSolver(ny, 1, dy, 1.0, dz, k0, indices, labels[:1, :, None], 1.0 + 0j,
                             mask[:, None], 0).run(field, 0, [])
    _close(fout.cpu().numpy().reshape(ny, 1, 2), first["transmitted"])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from bwpm_b200._lib import BWPM_EINVAL, last_error, lib

    ny = 16384
    dy, dz, k0, indices, labels, mask, field = _geometry(ny, 2)
    st, _ = _noalloc(torch, lib, ny, dy, dz, k0, indices, None, labels[0], 1.0, mask, field)
    assert st == BWPM_EINVAL
    assert "8192" in last_error()
    assert ctypes.c_int(st).value == BWPM_EINVAL
