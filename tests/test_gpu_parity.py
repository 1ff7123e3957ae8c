"""Parity of the CUDA core (through the C ABI) with the reference, on a GPU.

Mirrors the reference's tests/test_core_cuda.py: golden files at rel 1e-10, abs 1e-11·max
(test_core_cuda.py:34-36) and the random volumes at 1e-10·max|field| (:108-110) for the FP64
drop-in path; the complex64 path (precision=32) at relative L2 ≤ 1e-4 against the same values.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, load_npz, rel_l2
from golden_cases import case_2d, case_3d, volume_case

pytestmark = pytest.mark.gpu

RTOL, ATOL_REL = 1e-10, 1e-11  # the reference's CUDA tolerance (tests/test_core_cuda.py:34-36)
L2_C64 = 1e-4                  # complex64 fields against the FP64 reference


def _close(a, b):
    assert a.shape == b.shape
    atol = ATOL_REL * float(np.max(np.abs(b)) or 1.0)
    err = float(np.max(np.abs(a - b) - RTOL * np.abs(b)))
    assert np.allclose(a, b, rtol=RTOL, atol=atol), f"max excess {err:.3e} (atol {atol:.3e})"


@pytest.fixture(scope="module")
def core():
    from bwpm_b200 import _core

    if _core.cuda_device_count() < 1:
        pytest.fail("no CUDA device")
    return _core


def _run(core, args, field, fl, iters, keep, precision=64):
    s = core.CudaSolver(*args, 0, fluctuation=fl, precision=precision)
    return s.run(field, iters, list(keep))


def test_interface_matrices(core):
    a, meta = load_golden("interface_matrices")
    kx, ky = a["inputs.k_x_per_mm"], a["inputs.k_y_per_mm"]
    k0 = meta["parameters.k0_per_mm"]
    for j, (n1, n2) in enumerate(a["inputs.index_pairs"]):
        _close(core.transmission_matrix(kx * n1.real, ky * n1.real, n1, n2, k0), a["expected.T"][j])
        _close(core.reflection_matrix(kx * n1.real, ky * n1.real, n1, n2, k0), a["expected.R"][j])


def test_longitudinal_wavenumber(core):
    from oracle import port

    kp2 = np.linspace(0, 3, 101) * (2 * np.pi / 0.5e-3) ** 2
    for idx in (1.0, 1.5, 0.213 + 6.697j):
        got = core.longitudinal_wavenumber(idx, 2 * np.pi / 0.5e-3, kp2)
        ref = port.longitudinal_wavenumber(idx, 2 * np.pi / 0.5e-3, kp2)
        assert np.allclose(got, ref, rtol=1e-14, atol=1e-9)


@pytest.mark.parametrize("precision", [64, 32])
def test_fpwpm2d_interface(core, precision):
    args, f, fl, a, meta = case_2d("fpwpm2d_interface")
    nz = args[7].shape[0]
    r = _run(core, args, f, fl, 0, range(nz + 1), precision)
    planes = np.stack([r["forward"][p][:, 0] for p in range(nz + 1)])
    if precision == 64:
        _close(planes, a["expected.planes"])
    else:
        assert rel_l2(planes, a["expected.planes"]) < L2_C64


@pytest.mark.parametrize("precision", [64, 32])
def test_bwpm2d_tilted_silver(core, precision):
    args, f, fl, a, meta = case_2d("bwpm2d_tilted_silver")
    nz = args[7].shape[0]
    r = _run(core, args, f, fl, 2, range(nz + 1), precision)
    fw = np.stack([r["forward"][p][:, 0] for p in range(nz + 1)])
    bw = np.stack([r["backward"][p][:, 0] for p in range(nz + 1)])
    if precision == 64:
        _close(fw, a["expected.forward"])
        _close(bw, a["expected.backward"])
    else:
        assert rel_l2(fw, a["expected.forward"]) < L2_C64
        assert rel_l2(bw, a["expected.backward"]) < L2_C64


@pytest.mark.parametrize("precision", [64, 32])
def test_bwpm2d_slab_exact(core, precision):
    args, f, fl, a, meta = case_2d("bwpm2d_slab_exact")
    r = _run(core, args, f, fl, 40, (), precision)
    if precision == 64:
        _close(r["transmitted"][:, 0], a["expected.transmitted"])
        _close(r["reflected"][:, 0], a["expected.reflected"])
        rte = complex(np.mean(r["reflected"][:, 0, 0] / f[:, 0, 0]))
        assert abs(rte - complex(a["reference.r_te_airy"])) < 1e-12
    else:
        assert rel_l2(r["transmitted"][:, 0], a["expected.transmitted"]) < L2_C64
        assert rel_l2(r["reflected"][:, 0], a["expected.reflected"]) < L2_C64


@pytest.mark.parametrize("precision", [64, 32])
def test_bwpm3d_tilted(core, precision):
    args, f, fl, a, meta = case_3d("bwpm3d_tilted")
    keep = (0, 10, 20)
    r = _run(core, args, f, fl, 2, keep, precision)
    if precision == 64:
        _close(r["transmitted"], a["expected.transmitted"])
        _close(r["reflected"], a["expected.reflected"])
        _close(np.stack([r["forward"][p] for p in keep]), a["expected.forward_planes"])
        _close(np.stack([r["backward"][p] for p in keep]), a["expected.backward_planes"])
    else:
        assert rel_l2(r["transmitted"], a["expected.transmitted"]) < L2_C64
        assert rel_l2(r["reflected"], a["expected.reflected"]) < L2_C64


def test_fpwpm2d_fluctuation(core):
    args, f, fl, a, meta = case_2d("fpwpm2d_fluctuation")
    nz = args[7].shape[0]
    r = _run(core, args, f, fl, 0, range(nz + 1))
    _close(np.stack([r["forward"][p][:, 0] for p in range(nz + 1)]), a["expected.planes"])


def test_bwpm3d_fluctuation(core):
    args, f, fl, a, meta = case_3d("bwpm3d_fluctuation")
    keep = (0, 8, 16)
    r = _run(core, args, f, fl, 1, keep)
    _close(r["transmitted"], a["expected.transmitted"])
    _close(r["reflected"], a["expected.reflected"])
    _close(np.stack([r["forward"][p] for p in keep]), a["expected.forward_planes"])
    _close(np.stack([r["backward"][p] for p in keep]), a["expected.backward_planes"])


@pytest.mark.parametrize("prefix,iters", [("volume1.", 2), ("volume2.", 2), ("volume3.", 2),
                                          ("fluct1.", 1), ("fluct2.", 1), ("backscatter.", 3)])
def test_random_volumes(core, prefix, iters):
    """tests/test_core_cuda.py:91-179: odd sizes (15, 12, 9), silver, masks, δn, R1-R3."""
    d = load_npz("random_volumes.npz")
    args, field, fl = volume_case(d, prefix)
    r = _run(core, args, field, fl, iters, ())
    scale = 1e-10 * float(np.max(np.abs(field)))
    assert np.max(np.abs(r["transmitted"] - d[prefix + "transmitted"])) < scale
    assert np.max(np.abs(r["reflected"] - d[prefix + "reflected"])) < scale
    if prefix + "stored_values" in d:
        assert r["stored_values"] == int(d[prefix + "stored_values"])


@pytest.mark.parametrize("name", ["slab2d_te", "slab2d_tm", "born2d_small_te", "born2d_small_tm",
                                  "lens3d_small"])
def test_workload_cases_fp64(core, name):
    """Workload-shaped inputs against the reference CPU core: FP64 at relative L2 ≤ 1e-10."""
    from bwpm_b200 import workloads

    d = load_npz("workload_cases.npz")
    prob = workloads.Problem.from_arrays(d, name + ".")
    s = core.CudaSolver(*prob.core_args(), 0, fluctuation=prob.fluctuation)
    r = s.run(prob.field, prob.iterations, [])
    assert rel_l2(r["transmitted"], d[name + ".transmitted"]) < 1e-10
    assert rel_l2(r["reflected"], d[name + ".reflected"]) < 1e-10
    assert r["stored_values"] == int(d[name + ".stored_values"])


@pytest.mark.parametrize("name", ["slab2d_te", "slab2d_tm", "lens3d_small", "born2d_small_te"])
def test_workload_cases_c64(core, name):
    from bwpm_b200 import workloads

    d = load_npz("workload_cases.npz")
    prob = workloads.Problem.from_arrays(d, name + ".")
    s = core.CudaSolver(*prob.core_args(), 0, fluctuation=prob.fluctuation, precision=32)
    r = s.run(prob.field, prob.iterations, [])
    assert rel_l2(r["transmitted"], d[name + ".transmitted"]) < L2_C64
    assert rel_l2(r["reflected"], d[name + ".reflected"]) < L2_C64


def test_fast_facade_matches_golden(core):
    """The facade (bwpm_b200.fast.run_2d) with the reference's semantics incl. ε per iteration."""
    from bwpm_b200 import fast
    from bwpm_b200.model import Grid2D, Propagator2D

    a, meta = load_golden("bwpm2d_tilted_silver")
    g = Grid2D(int(meta["parameters.ny"]), meta["parameters.dy_mm"], meta["parameters.dz_mm"],
               meta["parameters.wavelength_um"])
    prop = Propagator2D(g, list(a["inputs.indices"]), a["inputs.labels"],
                        complex(a["inputs.index_before"]), a["inputs.mask"])
    res = fast.run_2d(prop, a["inputs.field"], 2, keep=True, backend="cuda")
    _close(res.forward, a["expected.forward"])
    _close(res.backward, a["expected.backward"])
    assert np.allclose(res.energy_residual, a["expected.energy_residual"], rtol=1e-8, atol=1e-10)


def test_run_twice_is_deterministic(core):
    args, f, fl, a, meta = case_2d("bwpm2d_tilted_silver")
    s = core.CudaSolver(*args, 0)
    r1 = s.run(f, 2, [])
    r2 = s.run(f, 2, [])
    assert np.array_equal(r1["transmitted"], r2["transmitted"])
    assert np.array_equal(r1["reflected"], r2["reflected"])


@pytest.mark.parametrize("prefix,iters", [("volume1.", 2), ("volume2.", 2), ("volume3.", 2),
                                          ("fluct1.", 1), ("backscatter.", 3)])
@pytest.mark.parametrize("precision", [64, 32])
def test_device_setup_equals_host_setup(core, monkeypatch, prefix, iters, precision):
    """The per-step tables built on the device (plane_setup.cuh) give bit-identical results to
    the host set-up, FP64 and complex64, with keep planes, stored sources and Born slabs."""
    d = load_npz("random_volumes.npz")
    args, field, fl = volume_case(d, prefix)
    out = {}
    for where in ("host", "device"):
        monkeypatch.setenv("BWPM_SETUP", where)
        out[where] = core.CudaSolver(*args, 0, fluctuation=fl, precision=precision).run(
            field, iters, [0, 5])
    a, b = out["host"], out["device"]
    for key in ("transmitted", "reflected"):
        assert np.array_equal(a[key], b[key]), key
    for q in (0, 5):
        assert np.array_equal(a["forward"][q], b["forward"][q])
        assert np.array_equal(a["backward"][q], b["backward"][q])
    assert a["stored_values"] == b["stored_values"]


@pytest.mark.parametrize("prefix,iters", [("volume2.", 2), ("volume3.", 2), ("backscatter.", 3)])
@pytest.mark.parametrize("precision", [64, 32])
def test_bulk_column_kernel_equals_plain_loads(core, monkeypatch, prefix, iters, precision):
    """The 3D column kernel that stages columns and tables with bulk copies and groups passes
    (k_cols_step_bulk) gives the same bits as the plain-load kernel (BWPM_COLS=plain)."""
    d = load_npz("random_volumes.npz")
    args, field, fl = volume_case(d, prefix)
    assert int(args[0]) % 2 == 0  # even ny: the bulk path applies
    out = {}
    for mode in ("plain", "bulk"):
        monkeypatch.setenv("BWPM_COLS", mode)
        monkeypatch.setenv("BWPM_3D_KERNELS", "general")
        out[mode] = core.CudaSolver(*args, 0, fluctuation=fl, precision=precision).run(
            field, iters, [0, 5])
    a, b = out["plain"], out["bulk"]
    for key in ("transmitted", "reflected"):
        assert np.array_equal(a[key], b[key]), key
    for q in (0, 5):
        assert np.array_equal(a["forward"][q], b["forward"][q])


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("prefix,iters", [("fluct1.", 1), ("fluct2.", 1), ("backscatter.", 3)])
def test_born_step_graph_equals_host_loop(core, monkeypatch, prefix, iters, precision):
    """The Born step run as one CUDA graph whose conditional nodes make the GMRES decisions on
    the device (the default) gives the same bits as the host-driven GMRES loop
    (BWPM_GMRES=host): same kernels, same order, only who decides to stop differs."""
    d = load_npz("random_volumes.npz")
    args, field, fl = volume_case(d, prefix)
    out = {}
    for mode in ("host", "graph"):
        monkeypatch.setenv("BWPM_GMRES", mode)
        out[mode] = core.CudaSolver(*args, 0, fluctuation=fl, precision=precision).run(
            field, iters, [])
    for key in ("transmitted", "reflected"):
        assert np.array_equal(out["host"][key], out["graph"][key]), key


@pytest.mark.parametrize("precision", [64, 32])
def test_born_step_graph_born2d(core, monkeypatch, precision):
    """As above on a 2D Born chain (4096 points, 60 slabs with δn on every slab, 2 iterations)."""
    from bwpm_b200 import workloads

    p = workloads.born2d(nz=60, iterations=2)
    out = {}
    for mode in ("host", "graph"):
        monkeypatch.setenv("BWPM_GMRES", mode)
        out[mode] = core.CudaSolver(*p.core_args(), 0, fluctuation=p.fluctuation,
                                    precision=precision).run(p.field, p.iterations, [])
    for key in ("transmitted", "reflected"):
        assert np.array_equal(out["host"][key], out["graph"][key]), key


@pytest.mark.parametrize("mode", ["graph", "host"])
def test_born_gmres_restart_limit_raises(core, monkeypatch, mode):
    """A GMRES(30) that cannot converge (tolerance 0) stops after 100 restarts with RuntimeError,
    as the reference does (cpp/src/solver.cpp:341-342). In the Born-step graph the limit sets an
    error flag that the run reads at its end; the next solver on the device runs normally."""
    monkeypatch.setenv("BWPM_GMRES", mode)
    # ≈ 400 propagating modes per component: no Krylov breakdown (an exact solve) within a cycle
    ny, lam = 1024, 0.633e-3
    dy = lam / 8
    dz = lam / 10
    y = (np.arange(ny) - ny // 2) * dy
    field = np.zeros((ny, 1, 2), complex)
    field[:, 0, 0] = np.exp(-((y / (64 * dy)) ** 2))
    labels = np.zeros((1, ny, 1), np.int32)
    fl = 0.01 * np.random.default_rng(3).standard_normal((1, ny, 1)) + 0j
    args = (ny, 1, dy, 1.0, dz, 2 * np.pi / lam, np.array([1.5 + 0j]), labels, 1.0 + 0j, None)
    s = core.CudaSolver(*args, 0, fluctuation=fl, gmres_tol=0.0)
    with pytest.raises(RuntimeError, match="GMRES did not converge"):
        s.run(field, 0, [])
    r = core.CudaSolver(*args, 0, fluctuation=fl).run(field, 0, [])
    assert np.all(np.isfinite(r["transmitted"])) and np.linalg.norm(r["transmitted"]) > 0
