"""Generates the golden fixtures under tests/golden/ from the reference (run once, here).

Two sources, both read from the reference tree (BWPM_REFERENCE, default: a `reference`
directory beside this repository); nothing under tests/ reads the reference at run time, only
these fixtures:

1. The reference's own golden files `reference/<case>.result.json` (format "raytatouille-result",
   written by the reference's tools/export_reference.py from tools/reference_cases.py). Each is
   decoded and stored as `<case>.npz` with its inputs, expected outputs and tolerance.
2. Extra cases computed by the reference itself:
   - the random volumes of the reference's CUDA parity tests (tests/test_core_cuda.py:91-196),
     run through the reference's Python `Bidirectional3D` (src/bwpm/volume3d.py:246-319);
   - workload-shaped cases (the 2D slab at full size, reduced Born and 3D microlens cases), run
     through the reference's compiled CPU core `bwpm._core.Solver` (cpp/src/solver.cpp:444-528)
     built by oracle/build_ref.sh.

Usage: python tests/golden/make_fixtures.py          (golden files, random volumes, workloads)
       python tests/golden/make_fixtures.py full     (the Born chain and the microlens at full size)
       python tests/golden/make_fixtures.py post     (post-processing of fields)
"""

from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF = Path(os.environ.get("BWPM_REFERENCE", str(REPO.parent / "reference")))

GOLDEN_CASES = (
    "interface_matrices",
    "fpwpm2d_interface",
    "bwpm2d_tilted_silver",
    "bwpm2d_slab_exact",
    "bwpm3d_tilted",
    "fpwpm2d_fluctuation",
    "bwpm3d_fluctuation",
)

_SPECIAL = {"NaN": math.nan, "Infinity": math.inf, "-Infinity": -math.inf}


def _num(x: object) -> float:
    return _SPECIAL[x] if isinstance(x, str) else float(x)  # type: ignore[arg-type]


def decode(value: object) -> object:
    """Decodes the value encoding of the raytatouille-result envelope (arrays, complex, NaN)."""
    if isinstance(value, list):
        return [decode(v) for v in value]
    if not isinstance(value, dict):
        return value
    if set(value) == {"dtype", "shape", "values"}:
        dtype = np.dtype(value["dtype"])
        if dtype.kind == "f":
            flat = [_num(x) for x in value["values"]]
        elif dtype.kind == "c":
            flat = [complex(_num(a), _num(b)) for a, b in value["values"]]
        else:
            flat = value["values"]
        return np.array(flat, dtype=dtype).reshape(value["shape"])
    if set(value) == {"float"}:
        return _num(value["float"])
    if set(value) == {"complex"}:
        a, b = value["complex"]
        return complex(_num(a), _num(b))
    return {k: decode(v) for k, v in value.items()}


def _flatten(prefix: str, d: dict, out: dict, meta: dict) -> None:  # type: ignore[type-arg]
    for k, v in d.items():
        key = f"{prefix}{k}"
        if isinstance(v, np.ndarray):
            out[key] = v
        elif isinstance(v, complex):
            out[key] = np.array(v, dtype=np.complex128)
        elif isinstance(v, (int, float)):
            meta[key] = v
        elif isinstance(v, dict):
            _flatten(key + ".", v, out, meta)
        else:
            meta[key] = v


def convert_golden() -> None:
    for case in GOLDEN_CASES:
        src = REF / "reference" / f"{case}.result.json"
        envelope = json.loads(src.read_text("utf-8"))
        assert envelope["format"] == "raytatouille-result"
        data = decode(envelope["data"])
        arrays: dict[str, np.ndarray] = {}
        meta: dict[str, object] = {"case": case, "source": str(data["source"])}
        for part in ("parameters", "inputs", "expected", "tolerance", "reference",
                     "reference_tolerance"):
            _flatten(part + ".", data[part], arrays, meta)
        arrays["meta"] = np.array(json.dumps(meta))
        np.savez_compressed(HERE / f"{case}.npz", **arrays)
        print("golden", case, sorted(arrays))


def _reference_python():
    sys.path.insert(0, str(REF / "src"))
    from bwpm.volume3d import Bidirectional3D, Grid3D, absorbing_mask_2d  # noqa: PLC0415

    return Bidirectional3D, Grid3D, absorbing_mask_2d


def random_volume_cases() -> None:
    """The random volumes of tests/test_core_cuda.py:91-111 (seeds 1-3) and :139-196."""
    Bidirectional3D, Grid3D, absorbing_mask_2d = _reference_python()
    out: dict[str, np.ndarray] = {}
    meta: dict[str, object] = {"source": "tests/test_core_cuda.py:91-196 via Bidirectional3D"}
    for seed in (1, 2, 3):
        rng = np.random.default_rng(seed)
        nx, ny, nz = (15, 12, 9) if seed % 2 else (8, 16, 11)
        grid = Grid3D(nx, ny, 0.04e-3, 0.05e-3, 0.03e-3, 0.6)
        labels = rng.integers(0, 4, size=(nz, 1, 1)) * np.ones((1, ny, nx), dtype=np.int64)
        labels[nz // 2] = rng.integers(0, 4, size=(ny, nx))
        indices = np.array([1.0 + 0j, 1.5 + 0j, 2.1 + 0.01j, 0.213 + 6.697j])
        field = rng.normal(size=(ny, nx, 2)) + 1j * rng.normal(size=(ny, nx, 2))
        kx, ky = grid.k_grid()
        spectrum = np.fft.fft2(field, axes=(0, 1))
        spectrum[np.sqrt(kx**2 + ky**2) >= 1.2 * grid.k0] = 0.0
        field = np.fft.ifft2(spectrum, axes=(0, 1))
        mask = absorbing_mask_2d(grid, 2 * grid.dx) if seed == 2 else None
        res = Bidirectional3D(grid, list(indices), labels, 1.2 + 0j, mask).run(field, 2, (0, 5, nz))
        p = f"volume{seed}."
        out[p + "grid"] = np.array([nx, ny, 0.04e-3, 0.05e-3, 0.03e-3, 0.6])
        out[p + "indices"] = indices
        out[p + "labels"] = labels.astype(np.int32)
        out[p + "index_before"] = np.array(1.2 + 0j)
        out[p + "field"] = field
        if mask is not None:
            out[p + "mask"] = mask
        out[p + "transmitted"] = res.transmitted
        out[p + "reflected"] = res.reflected
        out[p + "stored_values"] = np.array(res.stored_values)
        for q in (0, 5, nz):
            out[p + f"forward{q}"] = res.planes[q][0]
            out[p + f"backward{q}"] = res.planes[q][1]
    for seed in (1, 2):  # tests/test_core_cuda.py:139-158
        rng = np.random.default_rng(seed)
        nx, ny, nz = (15, 12, 9) if seed % 2 else (8, 16, 11)
        grid = Grid3D(nx, ny, 0.04e-3, 0.05e-3, 0.03e-3, 0.6)
        labels = rng.integers(0, 2, size=(nz, 1, 1)) * np.ones((1, ny, nx), dtype=np.int64)
        labels[nz // 2] = rng.integers(0, 3, size=(ny, nx))
        indices = np.array([1.33 + 0j, 1.5 + 0j, 2.1 + 0.01j])
        fl = 0.03 * rng.normal(size=(nz, ny, nx)) + 0.002j * rng.normal(size=(nz, ny, nx))
        fl[nz // 2] = 0.0
        field = rng.normal(size=(ny, nx, 2)) + 1j * rng.normal(size=(ny, nx, 2))
        mask = absorbing_mask_2d(grid, 2 * grid.dx) if seed == 2 else None
        res = Bidirectional3D(grid, list(indices), labels, 1.33 + 0j, mask, fluctuation=fl).run(
            field, 1, (0, 5, nz))
        p = f"fluct{seed}."
        out[p + "grid"] = np.array([nx, ny, 0.04e-3, 0.05e-3, 0.03e-3, 0.6])
        out[p + "indices"] = indices
        out[p + "labels"] = labels.astype(np.int32)
        out[p + "index_before"] = np.array(1.33 + 0j)
        out[p + "field"] = field
        out[p + "fluctuation"] = fl
        if mask is not None:
            out[p + "mask"] = mask
        out[p + "transmitted"] = res.transmitted
        out[p + "reflected"] = res.reflected
    # back scattering over three iterations, tests/test_core_cuda.py:161-179
    rng = np.random.default_rng(5)
    nx, ny, nz = 12, 10, 14
    grid = Grid3D(nx, ny, 0.05e-3, 0.05e-3, 0.04e-3, 0.8)
    labels = np.zeros((nz, ny, nx), dtype=np.int64)
    labels[nz - 3:] = 1
    fl = np.zeros((nz, ny, nx), dtype=np.complex128)
    fl[1: nz - 4] = 0.02 * rng.normal(size=(nz - 5, ny, nx)) + 1e-3j
    field = rng.normal(size=(ny, nx, 2)) + 1j * rng.normal(size=(ny, nx, 2))
    mask = absorbing_mask_2d(grid, 2 * grid.dx)
    indices = np.array([1.38 + 0j, 1.5 + 0.002j])
    res = Bidirectional3D(grid, list(indices), labels, 1.38 + 0j, mask, fluctuation=fl).run(
        field, 3, (0, 5, nz))
    p = "backscatter."
    out[p + "grid"] = np.array([nx, ny, 0.05e-3, 0.05e-3, 0.04e-3, 0.8])
    out[p + "indices"] = indices
    out[p + "labels"] = labels.astype(np.int32)
    out[p + "index_before"] = np.array(1.38 + 0j)
    out[p + "field"] = field
    out[p + "fluctuation"] = fl
    out[p + "mask"] = mask
    out[p + "transmitted"] = res.transmitted
    out[p + "reflected"] = res.reflected
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / "random_volumes.npz", **out)
    print("random_volumes", len(out))


def _ref_core():
    import importlib.util  # noqa: PLC0415

    so = sorted((REPO / "oracle" / "_ref").glob("_core*.so"))
    if not so:
        raise SystemExit("run oracle/build_ref.sh first")
    spec = importlib.util.spec_from_file_location("_core", so[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def baseline_shaped_cases() -> None:
    """Seeded inputs shaped like the workloads (bwpm_b200.workloads), outputs of the reference
    CPU core at FP64: the 2D slab at full size (1024 points, 250 slabs, 8 iterations, TE and
    TM), the Born case and the 3D microlens at reduced sizes."""
    sys.path.insert(0, str(REPO))
    from bwpm_b200 import workloads  # noqa: PLC0415

    core = _ref_core()
    out: dict[str, np.ndarray] = {}
    cases = {
        "slab2d_te": workloads.slab2d(polarization="te"),
        "slab2d_tm": workloads.slab2d(polarization="tm"),
        "born2d_small_te": workloads.born2d(ny=256, nz=24, iterations=2, polarization="te"),
        "born2d_small_tm": workloads.born2d(ny=256, nz=24, iterations=2, polarization="tm"),
        "lens3d_small": workloads.microlens3d(n=48, nz=40, iterations=2),
    }
    for name, prob in cases.items():
        s = core.Solver(*prob.core_args(), 1, fluctuation=prob.fluctuation)
        res = s.run(prob.field, prob.iterations, [])
        for k, v in prob.arrays().items():
            out[f"{name}.{k}"] = v
        out[f"{name}.transmitted"] = res["transmitted"]
        out[f"{name}.reflected"] = res["reflected"]
        out[f"{name}.stored_values"] = np.array(res["stored_values"])
        print("baseline-shaped", name, prob.ny, prob.nx, prob.nz)
    np.savez_compressed(HERE / "workload_cases.npz", **out)


FULL_PIXELS = 16384  # pixels of the 3D microlens fields stored in full (a seeded subset)
FULL_PROJECTIONS = 8  # seeded complex Gaussian projections of each whole 3D field


def microlens_probe(n_pixels: int, n_planes: int = 2, seed: int = 31):
    """Seeded pixel subset (sorted flat indices into (ny·nx)) and projection rows of the 3D
    microlens check; the GPU test regenerates the same arrays from the same seeds."""
    rng = np.random.default_rng(seed)
    pix = np.sort(rng.choice(n_pixels, FULL_PIXELS, replace=False))
    w = rng.standard_normal((FULL_PROJECTIONS, n_pixels * n_planes)) + 1j * rng.standard_normal(
        (FULL_PROJECTIONS, n_pixels * n_planes))
    return pix, w


def _full_case(name: str):
    """One full-size workload through the reference CPU core (run in its own process)."""
    sys.path.insert(0, str(REPO))
    from bwpm_b200 import workloads  # noqa: PLC0415

    core = _ref_core()
    if name.startswith("born2d_"):
        prob = workloads.born2d(polarization=name.split("_")[1])
        threads = 1
    else:
        prob = workloads.microlens3d()
        threads = int(os.environ.get("BWPM_FIXTURE_THREADS", "6"))
    s = core.Solver(*prob.core_args(), threads, fluctuation=prob.fluctuation)
    res = s.run(prob.field, prob.iterations, [])
    return name, res["transmitted"], res["reflected"], res["transmitted_iter"], res["reflected_iter"]


def full_size_cases() -> None:
    """The Born chain and the 3D microlens at full size through the reference CPU core, FP64:
    - born2d_te / born2d_tm: 4096 points, 2000 slabs with δn on every slab, 6 iterations
      (inputs from bwpm_b200.workloads.born2d, seed 2): full transmitted and reflected fields
      and the norms of the per-iteration fields;
    - microlens3d: 512² points, 400 slabs, 6 iterations (bwpm_b200.workloads.microlens3d, no
      random input): the fields at a seeded subset of FULL_PIXELS pixels plus FULL_PROJECTIONS
      seeded complex projections of each whole field (a 512² × 2 complex128 field is 8 MB).
    The three solves run in parallel processes (a few minutes on 8 cores)."""
    import multiprocessing as mp  # noqa: PLC0415

    ctx = mp.get_context("spawn")
    with ctx.Pool(3) as pool:
        results = pool.map(_full_case, ["born2d_te", "born2d_tm", "microlens3d"])
    out: dict[str, np.ndarray] = {}
    for name, t, r, t_it, r_it in results:
        if name.startswith("born2d_"):
            out[f"{name}.transmitted"] = t
            out[f"{name}.reflected"] = r
            out[f"{name}.transmitted_iter_norms"] = np.array(
                [np.linalg.norm(x) for x in t_it])
            out[f"{name}.reflected_iter_norms"] = np.array(
                [np.linalg.norm(x) for x in r_it])
        else:
            n_pix = t.shape[0] * t.shape[1]
            pix, w = microlens_probe(n_pix)
            for key, f in (("transmitted", t), ("reflected", r)):
                flat = f.reshape(n_pix, 2)
                out[f"{name}.{key}.pixels"] = flat[pix]
                out[f"{name}.{key}.projections"] = w @ flat.reshape(-1)
                out[f"{name}.{key}.norm"] = np.array(np.linalg.norm(f))
                out[f"{name}.{key}.max_abs"] = np.array(np.max(np.abs(f)))
        print("full-size", name, flush=True)
    out["meta"] = np.array(json.dumps({
        "source": "reference CPU core bwpm._core.Solver (cpp/src/solver.cpp:444-528) built by "
                  "oracle/build_ref.sh; inputs from bwpm_b200.workloads (born2d TE/TM, microlens3d)",
        "pixels": FULL_PIXELS, "projections": FULL_PROJECTIONS, "probe_seed": 31}))
    np.savez_compressed(HERE / "full_configs.npz", **out)


def post_cases() -> None:
    """Post-processing of fields by the reference's own functions on seeded inputs:
    bwpm.adapter.port_power (src/bwpm/adapter.py:267-284), bwpm.pilot_imc3d.plane_power and
    axial_focus (src/bwpm/pilot_imc3d.py:55-131), bwpm.fpwpm.power_flux
    (src/bwpm/fpwpm.py:205-216)."""
    sys.path.insert(0, str(REF / "src"))
    from bwpm.adapter import Port, PortField, port_power  # noqa: PLC0415
    from bwpm.fpwpm import Grid2D, power_flux  # noqa: PLC0415
    from bwpm.pilot_imc3d import axial_focus, plane_power  # noqa: PLC0415
    from bwpm.volume3d import Grid3D  # noqa: PLC0415

    rng = np.random.default_rng(41)
    out: dict[str, np.ndarray] = {}
    wl = 0.633
    lam = wl * 1e-3
    # a tilted Gaussian beam in both components plus seeded noise, 48 x 64
    ny, nx, d = 48, 64, lam / 6
    y = (np.arange(ny) - ny // 2) * d
    x = (np.arange(nx) - nx // 2) * d
    r2 = y[:, None] ** 2 + x[None, :] ** 2
    k0 = 2 * np.pi / lam
    beam = np.exp(-r2 / (8 * d) ** 2) * np.exp(1j * 0.3 * k0 * x[None, :])
    field = np.stack([beam, 0.4j * beam], axis=-1)
    field = field + 0.05 * (rng.standard_normal(field.shape) + 1j * rng.standard_normal(field.shape))
    out["beam3d.field"] = field
    out["beam3d.grid"] = np.array([ny, nx, d, d, wl])
    for tag, index, direction in (("n15_fwd", 1.5 + 0j, 1), ("absorbing_bwd", 1.0 + 0.02j, -1),
                                  ("silver_fwd", 0.135 + 3.98j, 1)):
        port = Port(0.0, direction, index, wl, nx, ny, d, d)
        out[f"beam3d.port_power.{tag}"] = np.array(port_power(PortField(port, field)))
        out[f"beam3d.port_power.{tag}.index"] = np.array(index)
        out[f"beam3d.port_power.{tag}.direction"] = np.array(direction)
    grid = Grid3D(nx, ny, d, d, d, wl)
    out["beam3d.plane_power.n15"] = np.array(plane_power(field, grid, 1.5))
    out["beam3d.plane_power.n10"] = np.array(plane_power(field, grid, 1.0))
    # a converging Gaussian beam (focus 30 µm behind the plane), 64 x 64, in air
    n, d = 64, lam / 4
    c = (np.arange(n) - n // 2) * d
    r2 = c[:, None] ** 2 + c[None, :] ** 2
    f = 30e-3
    beam = np.exp(-r2 / (14 * d) ** 2) * np.exp(-1j * k0 * r2 / (2 * f))
    lens = np.stack([beam, 0.2 * beam], axis=-1)
    offsets = np.linspace(0.0, 60e-3, 61)
    out["focus.field"] = lens
    out["focus.grid"] = np.array([n, n, d, d, wl])
    out["focus.offsets"] = offsets
    g = Grid3D(n, n, d, d, d, wl)
    for tag, na in (("all", None), ("na04", 0.4)):
        best, peak = axial_focus(lens, g, 1.0, offsets, na=na)
        out[f"focus.{tag}.best"] = np.array(best)
        out[f"focus.{tag}.peak"] = np.array(peak)
    # 2D power flux (nx = 1), 256 points
    ny, d = 256, lam / 8
    y = (np.arange(ny) - ny // 2) * d
    prof = np.exp(-(y / (20 * d)) ** 2) * np.exp(1j * 0.2 * k0 * y)
    f2 = np.stack([prof, 0.5 * prof], axis=-1) + 0.02 * rng.standard_normal((ny, 2))
    g2 = Grid2D(ny, d, d, wl)
    out["flux2d.field"] = f2
    out["flux2d.grid"] = np.array([ny, 1, d, 1.0, wl])
    out["flux2d.power_flux.n15_fwd"] = np.array(power_flux(f2, g2, 1.5 + 0j, direction=1))
    out["flux2d.power_flux.n10_bwd"] = np.array(power_flux(f2, g2, 1.0 + 0j, direction=-1))
    out["meta"] = np.array(json.dumps({"source": "reference functions (adapter.port_power, "
                                                 "pilot_imc3d.plane_power/axial_focus, "
                                                 "fpwpm.power_flux) on seeded inputs, seed 41"}))
    np.savez_compressed(HERE / "postproc.npz", **out)
    print("postproc", sorted(out))


if __name__ == "__main__":
    if sys.argv[1:] == ["full"]:
        full_size_cases()
    elif sys.argv[1:] == ["post"]:
        post_cases()
    else:
        convert_golden()
        random_volume_cases()
        baseline_shaped_cases()
