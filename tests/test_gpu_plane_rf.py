"""The fixed-length complex64 3D step kernels (bwpm_b200/csrc/plane_rf.cuh) on a GPU.

Every lateral size they cover (256, 384, 512, 768, 1024) and non-square planes run a seeded
tilted-facet or lens-array volume (labels generated on the device, multi-pass steps at the
interface, reflections, sparse sources, absorbing mask, two iterations) three ways: through the
fixed-length kernels (the default for these sizes), through the general kernels
(BWPM_3D_KERNELS=general) and in FP64. Both complex64 forms hold the complex64 contract
against FP64 (relative L2 ≤ 1e-4) and agree with each other to 2e-5 (they differ only in
the radix order of their transforms, i.e. in rounding).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

C64_TOL, FORMS_TOL = 1e-4, 2e-5


def _volume(ny: int, nx: int, nz: int, kind: str):
    from bwpm_b200 import workloads

    lam = 0.633e-3
    dy = dx = lam / 6
    dz = lam / 8
    y, x = workloads.centred(ny, dy), workloads.centred(nx, dx)
    g = {"nz": nz, "ny": ny, "nx": nx, "dz": dz, "dy": dy, "dx": dx, "base": nz // 3 * dz}
    if kind == "facet":  # the tilted face crosses every slab: 2-3 passes per step
        g.update(kind="tilted_facet", tan_tilt=float(np.tan(np.deg2rad(6.0))))
        n = 1.46
    else:
        pitch, sag = 0.03, 0.006
        g.update(kind="lens_array", pitch=pitch, sag=sag,
                 radius=((pitch / 2) ** 2 + sag**2) / (2 * sag))
        n = 1.55
    w0 = min(ny * dy, nx * dx) / 8
    r2 = y[:, None] ** 2 + x[None, :] ** 2
    field = np.zeros((ny, nx, 2), complex)
    field[..., 0] = np.exp(-r2 / w0**2)
    field[..., 1] = 0.3j * np.exp(-r2 / w0**2)
    mask = (workloads.absorbing_mask_1d(y, ny * dy / 10)[:, None]
            * workloads.absorbing_mask_1d(x, nx * dx / 10)[None, :])
    return g, np.array([1.0 + 0j, n + 0j]), mask, field, workloads.k0_of(0.633)


def _run(monkeypatch, ny, nx, nz, kind, precision, kernels, iterations=2):
    from bwpm_b200 import _core

    g, idx, mask, field, k0 = _volume(ny, nx, nz, kind)
    if kernels == "general":
        monkeypatch.setenv("BWPM_3D_KERNELS", "general")
    else:
        monkeypatch.delenv("BWPM_3D_KERNELS", raising=False)
    s = _core.CudaSolver.from_geometry(ny, nx, g["dy"], g["dx"], g["dz"], k0, idx, g, 1.0, mask, 0,
                                       precision=precision)
    return s.run(field, iterations, [1, nz // 2])


@pytest.mark.parametrize("ny,nx,nz,kind", [(256, 256, 60, "facet"), (384, 384, 40, "lens"),
                                           (512, 512, 40, "facet"), (768, 768, 24, "lens"),
                                           (1024, 1024, 20, "facet"), (512, 256, 40, "facet"),
                                           (256, 1024, 24, "lens")])
def test_fixed_length_kernels_match_general_and_fp64(monkeypatch, ny, nx, nz, kind):
    rf = _run(monkeypatch, ny, nx, nz, kind, 32, "fixed")
    gen = _run(monkeypatch, ny, nx, nz, kind, 32, "general")
    f64 = _run(monkeypatch, ny, nx, nz, kind, 64, "general")
    for key in ("transmitted", "reflected"):
        assert np.linalg.norm(f64[key]) > 1e-3 * np.linalg.norm(f64["transmitted"]), key
        assert rel_l2(rf[key], f64[key]) < C64_TOL, (key, rel_l2(rf[key], f64[key]))
        assert rel_l2(gen[key], f64[key]) < C64_TOL, (key, rel_l2(gen[key], f64[key]))
        assert rel_l2(rf[key], gen[key]) < FORMS_TOL, (key, rel_l2(rf[key], gen[key]))
    for q in (1, nz // 2):  # kept planes (forward sweep of the last iteration)
        assert rel_l2(rf["forward"][q], f64["forward"][q]) < C64_TOL, q


def test_fixed_length_kernels_are_deterministic(monkeypatch):
    a = _run(monkeypatch, 512, 512, 30, "facet", 32, "fixed")
    b = _run(monkeypatch, 512, 512, 30, "facet", 32, "fixed")
    for key in ("transmitted", "reflected"):
        assert np.array_equal(a[key], b[key]), key


def test_fixed_length_kernels_born_3d(monkeypatch):
    """A 3D Born chain (δn on every slab of a 256² plane): the fixed-length column kernel also
    writes the step's spectrum that the Born step starts from. Complex64 through the fixed-length
    kernels against the general ones and against FP64."""
    from bwpm_b200 import _core, workloads

    n, nz, lam = 256, 6, 0.633e-3
    d, dz = lam / 6, lam / 8
    c = workloads.centred(n, d)
    field = np.zeros((n, n, 2), complex)
    field[..., 0] = np.exp(-(c[:, None] ** 2 + c[None, :] ** 2) / (n * d / 8) ** 2)
    labels = np.zeros((nz, n, n), np.int32)
    rng = np.random.default_rng(11)
    fl = 0.01 * rng.standard_normal((nz, n, n)) + 0j
    args = (n, n, d, d, dz, workloads.k0_of(0.633), np.array([1.5 + 0j]), labels, 1.0 + 0j, None)
    out = {}
    for name, prec, kernels in (("rf", 32, None), ("gen", 32, "general"), ("f64", 64, "general")):
        if kernels:
            monkeypatch.setenv("BWPM_3D_KERNELS", kernels)
        else:
            monkeypatch.delenv("BWPM_3D_KERNELS", raising=False)
        out[name] = _core.CudaSolver(*args, 0, fluctuation=fl, precision=prec).run(field, 1, [])
    for key in ("transmitted", "reflected"):
        assert np.linalg.norm(out["f64"][key]) > 0, key
        assert rel_l2(out["rf"][key], out["f64"][key]) < C64_TOL, (key, rel_l2(out["rf"][key], out["f64"][key]))
        assert rel_l2(out["rf"][key], out["gen"][key]) < FORMS_TOL, (key, rel_l2(out["rf"][key], out["gen"][key]))
