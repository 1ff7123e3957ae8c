"""Seeded synthetic workloads for the slab-stepping path (no dataset is involved).

Every generator returns a `Problem`: the constructor arguments of the solver in the reference's
`bwpm._core` call convention (cpp/python/bindings.cpp:159-173: ny, nx, dy, dx, dz, k0, indices,
labels, index_before, mask, fluctuation) plus the incident field and the iteration count. Lengths
are in mm, k0 = 2π/λ in 1/mm (src/bwpm/fpwpm.py:50-53). The 2D solver is the 3D solver with
nx = 1 and the lateral axis y (src/bwpm/fast.py:120-142), TE = E_x, TM = E_y.

Workloads (sizes as named):
- `slab2d`: 1024 points, dy = λ/8, 250 slabs of λ/10, a 5 µm slab n = 1.5 in air, 5 µm Gaussian
  beam at normal incidence, 8 iterations, λ = 0.633 µm.
- `born2d`: 4096 points, 2000 slabs, host n = 1.5 with a seeded Gaussian random δn (std 0.01,
  correlation length 0.5 µm), 10° plane wave, 6 iterations.
- `microlens3d`: 512² points, dx = λ/6, 400 slabs of λ/8, spherical-cap lens (R = 50 µm,
  n = 1.52) with a 5°-tilted flat back face coated with silver (0.135 + 3.98i), 8 µm Gaussian
  beam, absorbing mask 16·dx, 6 iterations.
- `batch2d`: 256 seeded 2D instances of uneven size (256 … 8192 points incl. 3·2^k), 100-2000
  slabs, λ in 0.4-1.0 µm, 0-30° incidence, one slab n in 1.4-1.8 with a 0-8° tilted front face.
- `request_stream`: Poisson arrivals of 70 % 2D and 30 % 3D solves (microlens arrays and tilted
  fibre facets).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SILVER_CFG3 = 0.135 + 3.98j
BATCH_SIZES = (256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096, 6144, 8192)


def k0_of(wavelength_um: float) -> float:
    """Vacuum wavenumber 2π/λ in 1/mm (src/bwpm/fpwpm.py:50-53)."""
    return float(2.0 * np.pi / (wavelength_um * 1e-3))


def centred(n: int, d: float) -> np.ndarray:
    """Centred sample positions (i − n//2)·d (src/bwpm/fpwpm.py:55-58)."""
    return (np.arange(n) - n // 2) * d


def absorbing_mask_1d(coords: np.ndarray, width: float, order: int = 8,
                      edge: float = 1e-6) -> np.ndarray:
    """Super-Gaussian absorbing roll-off of src/bwpm/fpwpm.py:66-85 (one axis)."""
    a = np.abs(coords)
    if width == 0:
        return np.ones_like(a)
    u = np.clip((a - (float(np.max(a)) - width)) / width, 0.0, 1.0)
    return np.asarray(edge ** (u**order), dtype=np.float64)


GEOMETRY_KINDS = ("tilted_facet", "lens_array", "microlens", "tilted_slab")


def geometry_labels(g: dict) -> np.ndarray:
    """uint8 labels (nz, ny, nx) of a geometry at the pixel centres (the rule of
    src/bwpm/geometry.py:24-37: slab j at z = (j + 0.5)·dz, centred lateral grid). The same FP64
    operations in the same order as the device generator (csrc/geometry.cuh), so both give
    identical labels. Keys: kind, nz, ny, nx, dz, dy, dx and per kind
    - tilted_facet: base, tan_tilt (label 1 where z ≥ base + tan_tilt·y);
    - lens_array: base, pitch, sag, radius (label 1 where z ≥ base − h(x, y), spherical caps);
    - microlens: vertex, radius, back, tan_tilt (1 inside the cap, 2 behind the tilted face);
    - tilted_slab: base, tan_tilt, back (1 where base + tan_tilt·y ≤ z < back)."""
    nz, ny, nx = int(g["nz"]), int(g["ny"]), int(g["nx"])
    z = (np.arange(nz) + 0.5) * g["dz"]
    y = centred(ny, g["dy"])
    x = centred(nx, g["dx"])
    zz = z[:, None, None]
    kind = g["kind"]
    if kind == "tilted_facet":
        surface = g["base"] + g["tan_tilt"] * y[:, None] * np.ones((1, nx))
        return (zz >= surface[None]).astype(np.uint8)
    if kind == "lens_array":
        half = g["pitch"] / 2
        coords = [y[:, None] * np.ones((1, nx))]
        if nx > 1:
            coords.append(x[None, :] * np.ones((ny, 1)))
        r2 = 0.0
        for c in coords:
            local = (c + half) % g["pitch"] - half
            r2 = r2 + local**2
        height = np.sqrt(np.maximum(g["radius"] ** 2 - r2, 0.0)) - (g["radius"] - g["sag"])
        height = np.maximum(height, 0.0)
        return (zz >= (g["base"] - height)[None]).astype(np.uint8)
    if kind == "microlens":
        r2 = x[None, :] ** 2 + y[:, None] ** 2
        radius = g["radius"]
        sag = g["vertex"] + radius - np.sqrt(np.maximum(radius**2 - r2, 0.0))
        sag = np.where(r2 < radius**2, sag, np.inf)
        back_face = g["back"] + g["tan_tilt"] * y[:, None] * np.ones((1, nx))
        labels = np.zeros((nz, ny, nx), dtype=np.uint8)
        labels[zz >= sag[None]] = 1
        labels[zz >= back_face[None]] = 2
        return labels
    if kind == "tilted_slab":
        front = g["base"] + g["tan_tilt"] * y
        glass = (z[:, None] >= front[None, :]) & (z[:, None] < g["back"])
        return np.repeat(glass.astype(np.uint8)[:, :, None], nx, axis=2)
    raise ValueError(f"unknown geometry kind {kind!r}")


@dataclass
class Problem:
    """One solve: geometry, materials, incident field and iteration count."""

    ny: int
    nx: int
    dy: float
    dx: float
    dz: float
    k0: float
    indices: np.ndarray          # complex128 (M,)
    labels: np.ndarray | None    # int32 (nz, ny, nx), or None when `geometry` describes them
    index_before: complex
    mask: np.ndarray | None      # float64 (ny, nx) or None
    field: np.ndarray            # complex128 (ny, nx, 2)
    iterations: int
    fluctuation: np.ndarray | None = None  # complex128 (nz, ny, nx) or None
    name: str = ""
    extra: dict = field(default_factory=dict)
    geometry: dict | None = None  # the body the labels come from (see geometry_labels)

    @property
    def nz(self) -> int:
        return int(self.labels.shape[0]) if self.labels is not None else int(self.geometry["nz"])

    def ensure_labels(self) -> np.ndarray:
        """The int32 labels, generated on the host from `geometry` when not stored."""
        if self.labels is None:
            self.labels = geometry_labels(self.geometry).astype(np.int32)
        return self.labels

    def core_args(self) -> tuple:
        """Positional constructor arguments of bwpm._core.Solver / CudaSolver."""
        return (self.ny, self.nx, self.dy, self.dx, self.dz, self.k0, self.indices,
                self.ensure_labels(),
                complex(self.index_before), self.mask)

    def arrays(self) -> dict[str, np.ndarray]:
        out = {
            "grid": np.array([self.ny, self.nx, self.dy, self.dx, self.dz, self.k0]),
            "indices": self.indices,
            "labels": self.ensure_labels(),
            "index_before": np.array(complex(self.index_before)),
            "field": self.field,
            "iterations": np.array(self.iterations),
        }
        if self.mask is not None:
            out["mask"] = self.mask
        if self.fluctuation is not None:
            out["fluctuation"] = self.fluctuation
        return out

    @staticmethod
    def from_arrays(d: dict[str, np.ndarray], prefix: str = "") -> Problem:
        g = d[prefix + "grid"]
        mask = d.get(prefix + "mask")
        fl = d.get(prefix + "fluctuation")
        return Problem(int(g[0]), int(g[1]), float(g[2]), float(g[3]), float(g[4]), float(g[5]),
                       np.asarray(d[prefix + "indices"], dtype=np.complex128),
                       np.asarray(d[prefix + "labels"], dtype=np.int32),
                       complex(d[prefix + "index_before"]),
                       None if mask is None else np.asarray(mask, dtype=np.float64),
                       np.asarray(d[prefix + "field"], dtype=np.complex128),
                       int(d[prefix + "iterations"]),
                       None if fl is None else np.asarray(fl, dtype=np.complex128))

    def polarization_field(self, pol: str) -> None:
        """Moves the scalar profile into E_x (TE) or E_y (TM)."""
        prof = self.field[..., 0] + self.field[..., 1]
        self.field = np.zeros_like(self.field)
        self.field[..., 0 if pol == "te" else 1] = prof


def _vec(profile: np.ndarray, pol: str) -> np.ndarray:
    f = np.zeros(profile.shape + (2,), dtype=np.complex128)
    f[..., 0 if pol == "te" else 1] = profile
    return f


def slab2d(polarization: str = "te", ny: int = 1024, nz: int = 250, iterations: int = 8,
           wavelength_um: float = 0.633) -> Problem:
    """Planar 5 µm slab n = 1.5 in air, normal-incidence 5 µm Gaussian beam, no mask."""
    lam = wavelength_um * 1e-3
    dy, dz = lam / 8, lam / 10
    labels = np.zeros((nz, ny, 1), dtype=np.int32)
    first = int(round(85 * nz / 250))
    count = int(round(5e-3 / dz))  # 79 slabs of λ/10 at 0.633 µm ≈ 5 µm
    labels[first:first + count] = 1
    y = centred(ny, dy)
    prof = np.exp(-((y / 5e-3) ** 2)).astype(np.complex128)[:, None]
    return Problem(ny, 1, dy, 1.0, dz, k0_of(wavelength_um), np.array([1.0 + 0j, 1.5 + 0j]),
                   labels, 1.0 + 0j, None, _vec(prof, polarization), iterations,
                   name=f"slab2d_{polarization}")


def gaussian_random_field(rng: np.random.Generator, nz: int, ny: int, dz: float, dy: float,
                          corr: float, std: float) -> np.ndarray:
    """White N(0,1) on (nz, ny) filtered by exp(−|q|²l_c²/8) in Fourier space, rescaled to the
    sample standard deviation `std` (real)."""
    white = rng.standard_normal((nz, ny))
    qz = 2 * np.pi * np.fft.fftfreq(nz, d=dz)
    qy = 2 * np.pi * np.fft.fftfreq(ny, d=dy)
    filt = np.exp(-(qz[:, None] ** 2 + qy[None, :] ** 2) * corr**2 / 8)
    f = np.real(np.fft.ifft2(np.fft.fft2(white) * filt))
    f -= f.mean()
    return f * (std / f.std())


def born2d(polarization: str = "te", ny: int = 4096, nz: int = 2000, iterations: int = 6,
           wavelength_um: float = 0.633, seed: int = 2) -> Problem:
    """Host n = 1.5 everywhere with Gaussian random δn (std 0.01, l_c = 0.5 µm), 10° plane
    wave with k_y snapped to the nearest grid frequency."""
    lam = wavelength_um * 1e-3
    dy, dz = lam / 8, lam / 10
    k0 = k0_of(wavelength_um)
    rng = np.random.default_rng(seed)
    dn = gaussian_random_field(rng, nz, ny, dz, dy, 0.5e-3, 0.01)
    labels = np.zeros((nz, ny, 1), dtype=np.int32)
    ky_grid = 2 * np.pi * np.fft.fftfreq(ny, d=dy)
    ky = ky_grid[np.argmin(np.abs(ky_grid - 1.5 * k0 * np.sin(np.deg2rad(10.0))))]
    y = centred(ny, dy)
    prof = np.exp(1j * ky * y)[:, None]
    return Problem(ny, 1, dy, 1.0, dz, k0, np.array([1.5 + 0j]), labels, 1.5 + 0j, None,
                   _vec(prof, polarization), iterations,
                   fluctuation=dn.astype(np.complex128)[:, :, None],
                   name=f"born2d_{polarization}")


def microlens3d(n: int = 512, nz: int = 400, iterations: int = 6,
                wavelength_um: float = 0.633) -> Problem:
    """Spherical-cap microlens (R = 50 µm, n = 1.52, vertex at z = 2 µm, convex toward −z) whose
    flat back face at z = 24 µm + tan 5°·y is coated with silver; sizes scale with n/512 and
    nz/400 so reduced cases keep all three materials."""
    lam = wavelength_um * 1e-3
    dx = dy = lam / 6
    dz = lam / 8
    sz = nz / 400.0
    sr = n / 512.0
    radius = 50e-3 * sr
    vertex = 2e-3 * sz
    back = 24e-3 * sz
    x = centred(n, dx)
    y = centred(n, dy)
    r2 = x[None, :] ** 2 + y[:, None] ** 2
    geometry = {"kind": "microlens", "nz": nz, "ny": n, "nx": n, "dz": dz, "dy": dy, "dx": dx,
                "vertex": vertex, "radius": radius, "back": back,
                "tan_tilt": float(np.tan(np.deg2rad(5.0)))}
    labels = geometry_labels(geometry).astype(np.int32)
    mask = absorbing_mask_1d(y, 16 * dy)[:, None] * absorbing_mask_1d(x, 16 * dx)[None, :]
    prof = np.exp(-r2 / (8e-3 * max(sr, 0.1)) ** 2).astype(np.complex128)
    return Problem(n, n, dy, dx, dz, k0_of(wavelength_um),
                   np.array([1.0 + 0j, 1.52 + 0j, SILVER_CFG3]), labels, 1.0 + 0j, mask,
                   _vec(prof, "te"), iterations, name=f"microlens3d_{n}", geometry=geometry)


def tilted_slab2d_params(rng: np.random.Generator, i: int, sizes=BATCH_SIZES,
                         nz_range=(100, 2000), iterations: int = 6) -> dict:
    """Parameters of one instance of the batched 2D workload (seeded by `rng`)."""
    return {"i": i, "ny": int(rng.choice(sizes)),
            "nz": int(rng.integers(nz_range[0], nz_range[1] + 1)),
            "wl": float(rng.uniform(0.4, 1.0)), "theta": float(rng.uniform(0.0, np.deg2rad(30.0))),
            "n": float(rng.uniform(1.4, 1.8)), "tilt": float(rng.uniform(0.0, np.deg2rad(8.0))),
            "iterations": iterations}


def tilted_slab2d(rng: np.random.Generator, i: int, sizes=BATCH_SIZES,
                  nz_range=(100, 2000), iterations: int = 6) -> Problem:
    """One instance of the batched 2D workload (seeded by `rng`)."""
    return tilted_slab2d_from(tilted_slab2d_params(rng, i, sizes, nz_range, iterations))


def tilted_slab2d_from(prm: dict) -> Problem:
    """Builds the instance: one slab n in air, front face tilted, back face flat (middle half
    of nz), tilted Gaussian beam w₀ = ny·dy/8, mask width ny·dy/10 (order 8), TE for even i."""
    i, ny, nz, wl = prm["i"], prm["ny"], prm["nz"], prm["wl"]
    theta, n, tilt, iterations = prm["theta"], prm["n"], prm["tilt"], prm["iterations"]
    lam = wl * 1e-3
    dy, dz = lam / 8, lam / 10
    k0 = k0_of(wl)
    y = centred(ny, dy)
    geometry = {"kind": "tilted_slab", "nz": nz, "ny": ny, "nx": 1, "dz": dz, "dy": dy, "dx": 1.0,
                "base": nz // 4 * dz, "tan_tilt": float(np.tan(tilt)), "back": (3 * nz) // 4 * dz}
    labels = geometry_labels(geometry).astype(np.int32)
    w0 = ny * dy / 8
    prof = (np.exp(-((y / w0) ** 2)) * np.exp(1j * k0 * np.sin(theta) * y))[:, None]
    mask = absorbing_mask_1d(y, ny * dy / 10)[:, None]
    pol = "te" if i % 2 == 0 else "tm"
    return Problem(ny, 1, dy, 1.0, dz, k0, np.array([1.0 + 0j, n + 0j]), labels, 1.0 + 0j, mask,
                   _vec(prof, pol), iterations, name=f"batch2d_{i}_{pol}",
                   extra={"wavelength_um": wl, "theta": theta, "tilt": tilt}, geometry=geometry)


def batch2d_params(count: int = 256, seed: int = 4, sizes=BATCH_SIZES, nz_range=(100, 2000),
                   iterations: int = 6) -> list[dict]:
    """Parameters of the batched 2D workload (cheap; build each with tilted_slab2d_from)."""
    rng = np.random.default_rng(seed)
    return [tilted_slab2d_params(rng, i, sizes, nz_range, iterations) for i in range(count)]


def batch2d(count: int = 256, seed: int = 4, sizes=BATCH_SIZES, nz_range=(100, 2000),
            iterations: int = 6) -> list[Problem]:
    """The batched 2D workload: `count` seeded instances of uneven size."""
    return [tilted_slab2d_from(p) for p in batch2d_params(count, seed, sizes, nz_range, iterations)]


def smooth_sizes(lo: int, hi: int) -> list[int]:
    """Lateral sizes in [lo, hi] whose prime factors are 2, 3 and 5."""
    out = []
    for v in range(lo, hi + 1):
        m = v
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            out.append(v)
    return out


SERVED_3D_LATERAL = (256, 384, 512, 768, 1024)


def request(rng: np.random.Generator, i: int, iterations: int = 2,
            max_lateral_3d: int = 1024, host_labels: bool = True) -> Problem:
    """One request of the served stream: 70 % 2D, 30 % 3D; microlens array or tilted facet.
    3D lateral sizes are drawn from SERVED_3D_LATERAL up to `max_lateral_3d`. The body is kept
    as `geometry`; with host_labels=False a 3D request carries no label volume (labels = None:
    they are generated where they are used, e.g. on the device)."""
    is2d = rng.uniform() < 0.7
    wl = 0.633
    lam = wl * 1e-3
    k0 = k0_of(wl)
    if is2d:
        ny, nx = int(rng.choice(smooth_sizes(1024, 4096))), 1
        nz = int(rng.integers(500, 2001))
        dy, dx, dz = lam / 8, 1.0, lam / 10
    else:
        ny = nx = int(rng.choice([v for v in SERVED_3D_LATERAL if v <= max_lateral_3d]))
        nz = int(rng.integers(200, 601))
        dy = dx = lam / 6
        dz = lam / 8
    y = centred(ny, dy)
    x = centred(nx, dx)
    geometry = {"nz": nz, "ny": ny, "nx": nx, "dz": dz, "dy": dy, "dx": dx,
                "base": nz // 3 * dz}
    if rng.uniform() < 0.5:
        # a square array of spherical caps of height `sag` over half the pitch, bulging toward
        # −z from the substrate at `base`
        pitch = float(rng.uniform(20e-3, 60e-3))
        sag = float(rng.uniform(2e-3, 10e-3))
        n = float(rng.uniform(1.46, 1.6))
        half = pitch / 2
        geometry.update(kind="lens_array", pitch=pitch, sag=sag,
                        radius=(half**2 + sag**2) / (2 * sag))
        kind = "lens_array"
    else:
        n = float(rng.uniform(1.44, 1.47))
        tilt = float(rng.uniform(0.0, np.deg2rad(8.0)))
        geometry.update(kind="tilted_facet", tan_tilt=float(np.tan(tilt)))
        kind = "fiber_facet"
    labels = geometry_labels(geometry).astype(np.int32) if (host_labels or is2d) else None
    if is2d:
        w0 = ny * dy / 8
        prof = np.exp(-((y / w0) ** 2))[:, None]
        mask = absorbing_mask_1d(y, ny * dy / 10)[:, None]
    else:
        w0 = ny * dy / 8
        r2 = (y[:, None] * np.ones((1, nx))) ** 2 + (x[None, :] * np.ones((ny, 1))) ** 2
        prof = np.exp(-r2 / w0**2)
        mask = absorbing_mask_1d(y, ny * dy / 10)[:, None] * absorbing_mask_1d(x, nx * dx / 10)[None, :]
    pol = "te" if rng.uniform() < 0.5 else "tm"
    return Problem(ny, nx, dy, dx, dz, k0, np.array([1.0 + 0j, n + 0j]), labels, 1.0 + 0j, mask,
                   _vec(prof.astype(np.complex128), pol), iterations,
                   name=f"request_{i}_{kind}_{'2d' if is2d else '3d'}", geometry=geometry)


def request_stream(count: int, rate_hz: float, seed: int = 5, iterations: int = 2,
                   max_lateral_3d: int = 1024,
                   host_labels: bool = True) -> list[tuple[float, Problem]]:
    """Seeded Poisson arrivals: (arrival time in s, problem)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate_hz))
        out.append((t, request(rng, i, iterations, max_lateral_3d, host_labels)))
    return out


def poisson_arrivals(count: int, rate_hz: float, seed: int = 5) -> np.ndarray:
    """Seeded Poisson arrival times (s) of `count` requests at `rate_hz`."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=count))
