"""CPU oracle: a numpy restatement of the reference's FP64 slab-stepping algorithm.

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA path (tests/, the smoke check
and the CPU-baseline leg of bench.py); the product never imports it.

It follows the reference's C++ CPU core `bwpm::Solver` (cpp/src/solver.cpp) step for step,
vectorised over grid points with numpy's FFT (pocketfft, as the reference core):
- k grid:        cpp/src/solver.cpp:17-24, :40-46  (2π·(m·(1/(n·d))) rounding of fftfreq)
- k_z, Fresnel:  cpp/src/interface.cpp:8-28
- T and R:       cpp/src/interface.cpp:30-52
- operator:      cpp/src/solver.cpp:73-106  (table 1 propagation factors)
- apply:         cpp/src/solver.cpp:384-417 (Σ I_r,s F⁻¹{M F{E}}, mask on transmissions)
- sources:       cpp/src/solver.cpp:419-441 (store/add at interface pixels)
- Born:          cpp/src/solver.cpp:215-382 (sources, G operator, Cayley step, emission)
- GMRES:         cpp/src/solver.cpp:127-207 (restarted, MGS, Givens; tol 1e-12, m = 30)
- run:           cpp/src/solver.cpp:444-528 (forward/backward sweeps, iterations)

Pinned against the reference's golden files (reference/*.result.json, converted to
tests/golden/*.npz) and against the reference core built from source (oracle/_ref).
"""

from __future__ import annotations

import numpy as np

GRAZING = 1e-12  # cpp/include/bwpm/interface.hpp:17
GAUSS = ((1.0 - 1.0 / np.sqrt(3.0)) / 2.0, (1.0 + 1.0 / np.sqrt(3.0)) / 2.0)  # solver.cpp:212
FWD_T, FWD_R, BWD_T, BWD_R = 0, 1, 2, 3


def fftfreq(n: int, d: float) -> np.ndarray:
    """2π·numpy.fft.fftfreq(n, d) with the rounding 2π·(m·(1/(n·d))) (solver.cpp:17-24)."""
    i = np.arange(n)
    m = np.where(i < (n + 1) // 2, i, i - n).astype(np.float64)
    val = 1.0 / (float(n) * d)
    return 2.0 * np.pi * (m * val)


def longitudinal_wavenumber(index: complex, k0: float, kp2: np.ndarray) -> np.ndarray:
    """k_z with Im ≥ 0 and the grazing rule (interface.cpp:8-18)."""
    index = complex(index)
    n2k2 = index * index * (k0 * k0)
    q = np.asarray(n2k2 - np.asarray(kp2, dtype=np.float64), dtype=np.complex128)
    q = np.where(np.abs(q) <= GRAZING * abs(n2k2), 0.0 + 0.0j, q)
    kz = np.sqrt(q)
    flip = (kz.imag < 0.0) | ((kz.imag == 0.0) & (kz.real < 0.0))
    kz = np.where(flip, -kz, kz)
    tiny = 1e-12 * k0
    return np.where(np.abs(kz) < tiny, 1j * tiny, kz)


def fresnel(kx, ky, n1: complex, n2: complex, k0: float):
    """Convention A coefficients (interface.cpp:20-28)."""
    kp2 = kx * kx + ky * ky
    kz1 = longitudinal_wavenumber(n1, k0, kp2)
    kz2 = longitudinal_wavenumber(n2, k0, kp2)
    q1, q2 = kz1 / k0, kz2 / k0
    den_p = n2 * n2 * q1 + n1 * n1 * q2
    return ((q1 - q2) / (q1 + q2), (n2 * n2 * q1 - n1 * n1 * q2) / den_p,
            2.0 * q1 / (q1 + q2), 2.0 * n1 * n2 * q1 / den_p, kz1, kz2)


def transmission_matrix(kx, ky, n1, n2, k0) -> np.ndarray:
    """T of interface.cpp:30-40, shape (..., 2, 2)."""
    kx = np.asarray(kx, dtype=np.float64)
    ky = np.asarray(ky, dtype=np.float64)
    n1, n2 = complex(n1), complex(n2)
    r_s, r_p, t_s, t_p, kz1, kz2 = fresnel(kx, ky, n1, n2, k0)
    kp2 = kx * kx + ky * ky
    kr, ks = n1 * k0, n2 * k0
    with np.errstate(divide="ignore", invalid="ignore"):
        gamma = kz1 * kz2 + kz2 * kp2 / kz1
        scale = 1.0 / (kp2 * kr * ks)
        off = (t_p * gamma - t_s * kr * ks) * kx * ky * scale
        m00 = (t_p * kx * kx * gamma + t_s * ky * ky * kr * ks) * scale
        m11 = (t_p * ky * ky * gamma + t_s * kx * kx * kr * ks) * scale
    zero = kp2 == 0.0
    m00 = np.where(zero, t_s, m00)
    m11 = np.where(zero, t_s, m11)
    off = np.where(zero, 0.0, off)
    return np.stack([np.stack([m00, off], -1), np.stack([off, m11], -1)], -2)


def reflection_matrix(kx, ky, n1, n2, k0) -> np.ndarray:
    """R of interface.cpp:42-52, shape (..., 2, 2)."""
    kx = np.asarray(kx, dtype=np.float64)
    ky = np.asarray(ky, dtype=np.float64)
    n1, n2 = complex(n1), complex(n2)
    r_s, r_p, t_s, t_p, kz1, kz2 = fresnel(kx, ky, n1, n2, k0)
    kp2 = kx * kx + ky * ky
    kr = n1 * k0
    with np.errstate(divide="ignore", invalid="ignore"):
        gamma = kz1 * kz1 + kp2
        scale = 1.0 / (kp2 * kr * kr)
        off = -(r_p * gamma + r_s * kr * kr) * kx * ky * scale
        m00 = (-r_p * kx * kx * gamma + r_s * ky * ky * kr * kr) * scale
        m11 = (-r_p * ky * ky * gamma + r_s * kx * kx * kr * kr) * scale
    zero = kp2 == 0.0
    m00 = np.where(zero, r_s, m00)
    m11 = np.where(zero, r_s, m11)
    off = np.where(zero, 0.0, off)
    return np.stack([np.stack([m00, off], -1), np.stack([off, m11], -1)], -2)


class GmresNotConverged(RuntimeError):
    pass


def gmres(apply, b: np.ndarray, x: np.ndarray, tol: float = 1e-12, restart: int = 30,
          max_restarts: int = 100) -> tuple[np.ndarray, int]:
    """Restarted GMRES of solver.cpp:130-207; returns (x, number of operator applications)."""
    n_apply = 0
    bnorm = np.linalg.norm(b)
    if bnorm == 0.0:
        return np.zeros_like(x), 0
    m = restart
    for _ in range(max_restarts):
        w = apply(x)
        n_apply += 1
        v0 = b - w
        beta = np.linalg.norm(v0)
        if beta <= tol * bnorm:
            return x, n_apply
        basis = [v0 / beta]
        h = np.zeros((m + 1, m), dtype=np.complex128)
        g = np.zeros(m + 1, dtype=np.complex128)
        cs = np.zeros(m, dtype=np.complex128)
        sn = np.zeros(m, dtype=np.complex128)
        g[0] = beta
        used, done = 0, False
        for j in range(m):
            w = apply(basis[j])
            n_apply += 1
            for i in range(j + 1):
                hij = np.vdot(basis[i], w)
                h[i, j] = hij
                w = w - hij * basis[i]
            hnext = np.linalg.norm(w)
            basis.append(w / hnext if hnext > 0.0 else np.zeros_like(w))
            for i in range(j):
                a, c = h[i, j], h[i + 1, j]
                h[i, j] = cs[i] * a + sn[i] * c
                h[i + 1, j] = -np.conj(sn[i]) * a + cs[i] * c
            a = h[j, j]
            r = np.sqrt(abs(a) ** 2 + hnext * hnext)
            if abs(a) == 0.0:
                cs[j], sn[j] = 0.0, 1.0
            else:
                cs[j] = abs(a) / r
                sn[j] = (a / abs(a)) * hnext / r
            h[j, j] = cs[j] * a + sn[j] * hnext
            g[j + 1] = -np.conj(sn[j]) * g[j]
            g[j] = cs[j] * g[j]
            used = j + 1
            if abs(g[j + 1]) <= tol * bnorm or hnext == 0.0:
                done = True
                break
        y = np.zeros(used, dtype=np.complex128)
        for i in range(used - 1, -1, -1):
            s = g[i] - np.dot(h[i, i + 1:used], y[i + 1:used])
            y[i] = s / h[i, i]
        for i in range(used):
            x = x + y[i] * basis[i]
        if done:
            w = apply(x)
            n_apply += 1
            if np.linalg.norm(b - w) <= tol * bnorm * 10.0:
                return x, n_apply
    raise GmresNotConverged("GMRES did not converge in the Born step")


class Solver:
    """FP64 BWPM on the CPU with the reference core's semantics (cpp/src/solver.cpp:27-528)."""

    def __init__(self, ny, nx, dy, dx, dz, k0, indices, labels, index_before, mask,
                 fluctuation=None, gmres_tol: float = 1e-12):
        self.ny, self.nx = int(ny), int(nx)
        self.dy, self.dx, self.dz, self.k0 = float(dy), float(dx), float(dz), float(k0)
        self.indices = np.asarray(indices, dtype=np.complex128)
        self.labels = np.asarray(labels, dtype=np.int32)
        self.nz = self.labels.shape[0]
        n = self.ny * self.nx
        if self.labels.size != self.nz * n:
            raise ValueError("labels must have shape (nz, ny, nx)")
        self.labels = self.labels.reshape(self.nz, self.ny, self.nx)
        self.index_before = complex(index_before)
        self.mask = None if mask is None else np.asarray(mask, dtype=np.float64).reshape(
            self.ny, self.nx)
        if self.labels.min(initial=0) < 0 or self.labels.max(initial=0) >= len(self.indices):
            raise ValueError("labels must index into `indices`")
        kx1 = fftfreq(self.nx, self.dx)
        ky1 = fftfreq(self.ny, self.dy)
        self.kx = np.broadcast_to(kx1[None, :], (self.ny, self.nx)).copy()
        self.ky = np.broadcast_to(ky1[:, None], (self.ny, self.nx)).copy()
        self.gmres_tol = gmres_tol
        self.gmres_applies: list[int] = []
        self.fluct = None
        self.host = [None] * self.nz
        if fluctuation is not None:  # solver.cpp:49-62
            fl = np.asarray(fluctuation, dtype=np.complex128).reshape(self.nz, self.ny, self.nx)
            self.fluct = fl
            for j in range(self.nz):
                nzmask = fl[j] != 0
                if not nzmask.any():
                    continue
                found = set(complex(v) for v in self.indices[self.labels[j][nzmask]])
                if len(found) > 1:
                    raise ValueError(f"slab {j}: fluctuation must lie in one host index")
                self.host[j] = found.pop()
        self._cache: dict = {}

    # -- helpers ----------------------------------------------------------------------------
    def plane_labels(self, p: int) -> np.ndarray:
        if p == 0:
            return np.full((self.ny, self.nx), -1, dtype=np.int32)
        return self.labels[p - 1]

    def index_of(self, label: int) -> complex:
        return self.index_before if label < 0 else complex(self.indices[label])

    def op(self, kind: int, r: int, s: int) -> np.ndarray:
        """Operator M (ny, nx, 2, 2) of (kind, r, s) with the table-1 phase (solver.cpp:73-106)."""
        key = (kind, r, s)
        if key in self._cache:
            return self._cache[key]
        nr, ns = self.index_of(r), self.index_of(s)
        kx, ky, k0, dz = self.kx, self.ky, self.k0, self.dz
        kp2 = kx * kx + ky * ky
        if kind == FWD_T:
            a = transmission_matrix(kx, ky, nr, ns, k0)
            phase = np.exp(1j * longitudinal_wavenumber(ns, k0, kp2) * dz)
        elif kind == FWD_R:
            a = reflection_matrix(kx, ky, nr, ns, k0)
            phase = np.ones(kp2.shape, dtype=np.complex128)
        elif kind == BWD_T:
            a = transmission_matrix(kx, ky, nr, ns, k0)
            phase = np.exp(1j * longitudinal_wavenumber(nr, k0, kp2) * dz)
        else:
            a = reflection_matrix(kx, ky, nr, ns, k0)
            phase = np.exp(2.0 * 1j * longitudinal_wavenumber(nr, k0, kp2) * dz)
        m = a * phase[..., None, None]
        self._cache[key] = m
        return m

    @staticmethod
    def fft(v: np.ndarray, forward: bool) -> np.ndarray:
        """2D FFT over (ny, nx) per component; inverse scaled 1/N (solver.cpp:108-125)."""
        if forward:
            return np.fft.fft2(v, axes=(0, 1))
        return np.fft.ifft2(v, axes=(0, 1))

    def apply(self, kind: int, e: np.ndarray, p_r: int, p_s: int) -> np.ndarray:
        """Σ_(r,s) I_r,s F⁻¹{M_rs F{e}}; reflections skip equal indices; mask on transmissions
        (solver.cpp:384-417)."""
        lr, ls = self.plane_labels(p_r), self.plane_labels(p_s)
        pairs = sorted(set(zip(lr.ravel().tolist(), ls.ravel().tolist())))
        spec = self.fft(e, True)
        out = np.zeros_like(e)
        refl = kind in (FWD_R, BWD_R)
        for r, s in pairs:
            if refl and self.index_of(r) == self.index_of(s):
                continue
            m = self.op(kind, r, s)
            w = np.empty_like(spec)
            w[..., 0] = m[..., 0, 0] * spec[..., 0] + m[..., 0, 1] * spec[..., 1]
            w[..., 1] = m[..., 1, 0] * spec[..., 0] + m[..., 1, 1] * spec[..., 1]
            w = self.fft(w, False)
            sel = (lr == r) & (ls == s)
            out[sel] = w[sel]
        if not refl and self.mask is not None:
            out = out * self.mask[..., None]
        return out

    # -- Born (solver.cpp:215-382) -----------------------------------------------------------
    def _born_common(self, slab: int):
        host = complex(self.host[slab])
        kx, ky = self.kx, self.ky
        kp2 = kx * kx + ky * ky
        host2k2 = host * host * self.k0 * self.k0
        kabs2 = abs(host2k2)
        kz = longitudinal_wavenumber(host, self.k0, kp2)
        prop = (kp2 < kabs2) & (np.abs(host2k2 - kp2) > GRAZING * kabs2)
        return host, kp2, kz, prop

    def born_sources(self, e: np.ndarray, direction: int, slab: int) -> np.ndarray:
        host, kp2, kz, prop = self._born_common(slab)
        kx, ky = self.kx, self.ky
        spec = self.fft(e, True)
        ex, ey = spec[..., 0], spec[..., 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            ez = np.where(prop, -float(direction) * (kx * ex + ky * ey) / kz, 0.0)
        full = np.stack([ex, ey, ez], -1)
        scale = 2.0 * host * self.k0 * self.k0
        v = scale * self.fluct[slab]
        out = []
        for m in range(2):
            dist = (GAUSS[m] if direction > 0 else 1.0 - GAUSS[m]) * self.dz
            phase = np.where(prop, np.exp(1j * kz * dist), 0.0)
            w = self.fft(full * phase[..., None], False)
            w = v[..., None] * w
            out.append(self.fft(w, True))
        return np.stack(out)

    def born_operator(self, spec: np.ndarray, direction: int, slab: int) -> np.ndarray:
        host, kp2, kz, prop = self._born_common(slab)
        kx, ky = self.kx, self.ky
        k2 = (host * self.k0) ** 2
        d = float(direction)
        ex = np.where(prop, spec[..., 0], 0.0)
        ey = np.where(prop, spec[..., 1], 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            ez = np.where(prop, -d * (kx * ex + ky * ey) / kz, 0.0)
        w = self.fft(np.stack([ex, ey, ez], -1), False)
        w = (2.0 * host * self.k0 * self.k0 * self.fluct[slab])[..., None] * w
        w = self.fft(w, True)
        with np.errstate(divide="ignore", invalid="ignore"):
            green = 1j * self.dz / (2.0 * kz)
            lon = (kx * w[..., 0] + ky * w[..., 1] + d * kz * w[..., 2]) / k2
            o0 = np.where(prop, green * (w[..., 0] - kx * lon), 0.0)
            o1 = np.where(prop, green * (w[..., 1] - ky * lon), 0.0)
        return np.stack([o0, o1], -1)

    def born_step(self, e: np.ndarray, direction: int, slab: int) -> np.ndarray:
        host, kp2, kz, prop = self._born_common(slab)
        x = self.fft(e, True)
        half = np.where(prop, np.exp(1j * kz * (self.dz / 2.0)), 0.0)
        x = x * half[..., None]
        rhs = self.born_operator(x, direction, slab)

        def apply(v):
            return v - 0.5 * self.born_operator(v.reshape(rhs.shape), direction,
                                                slab).ravel()

        y, napp = gmres(apply, rhs.ravel(), rhs.ravel().copy(), self.gmres_tol)
        self.gmres_applies.append(napp)
        y = y.reshape(rhs.shape)
        if direction > 0:
            f = half
        else:
            with np.errstate(divide="ignore", invalid="ignore"):
                f = np.where(half == 0, half, 1.0 / half)
        return self.fft(y * f[..., None], False)

    def born_emission(self, sources: np.ndarray, direction: int, slab: int) -> np.ndarray:
        host, kp2, kz, prop = self._born_common(slab)
        kx, ky = self.kx, self.ky
        k2 = (host * self.k0) ** 2
        d = float(direction)
        skz = d * kz
        total = np.zeros((self.ny, self.nx, 2), dtype=np.complex128)
        with np.errstate(divide="ignore", invalid="ignore"):
            for m in range(2):
                green = 0.5 * np.exp(1j * skz * ((1.0 - GAUSS[m]) * self.dz)) * (
                    1j * self.dz / (2.0 * kz))
                s = sources[m]
                lon = (kx * s[..., 0] + ky * s[..., 1] + skz * s[..., 2]) / k2
                total[..., 0] += np.where(prop, green * (s[..., 0] - kx * lon), 0.0)
                total[..., 1] += np.where(prop, green * (s[..., 1] - ky * lon), 0.0)
        return self.fft(total, False)

    # -- the sweep (solver.cpp:444-528) ------------------------------------------------------
    def run(self, field_in: np.ndarray, iterations: int, keep=()) -> dict:
        n_ = (self.ny, self.nx, 2)
        field_in = np.asarray(field_in, dtype=np.complex128)
        if field_in.size != self.ny * self.nx * 2:
            raise ValueError("field must have shape (ny, nx, 2)")
        field_in = field_in.reshape(n_)
        keep = set(int(k) for k in keep)
        iface = []
        idx_before = np.vectorize(self.index_of, otypes=[np.complex128])
        planes_idx = [idx_before(self.plane_labels(p)) for p in range(self.nz + 1)]
        for p in range(self.nz):
            iface.append(planes_idx[p] != planes_idx[p + 1])
        anyi = [bool(m.any()) for m in iface]
        res = {"transmitted": None, "reflected": None, "transmitted_iter": [],
               "reflected_iter": [], "forward": {}, "backward": {}, "stored_values": 0}
        src_fwd: dict[int, tuple] = {}
        src_bwd: dict[int, tuple] = {}
        born_fwd: dict[int, np.ndarray] = {}
        born_bwd: dict[int, np.ndarray] = {}
        mask = self.mask

        def store(v, where):
            return (where, v[where].copy())

        def add(v, s):
            where, vals = s
            v = v.copy()
            v[where] += vals
            return v

        for _ in range(max(iterations, 1)):
            src_bwd, born_bwd = {}, {}
            e = field_in.copy()
            if 0 in src_fwd:
                e = add(e, src_fwd[0])
            if 0 in keep:
                res["forward"][0] = e.copy()
            for p in range(self.nz):
                if iterations > 0 and anyi[p]:
                    src_bwd[p] = store(self.apply(FWD_R, e, p, p + 1), iface[p])
                nxt = self.apply(FWD_T, e, p, p + 1)
                if self.host[p] is not None:
                    inc = self.born_step(e, +1, p)
                    m = 1.0 if mask is None else mask[..., None]
                    nxt = nxt + inc * m
                    if iterations > 0:
                        born_bwd[p + 1] = self.born_emission(self.born_sources(e, +1, p), -1, p)
                e = nxt
                if p + 1 in src_fwd:
                    e = add(e, src_fwd[p + 1])
                if p + 1 in born_fwd:
                    e = e + born_fwd[p + 1]
                if p + 1 in keep:
                    res["forward"][p + 1] = e.copy()
            res["transmitted"] = e
            if iterations == 0:
                break
            src_fwd, born_fwd = {}, {}
            e = np.zeros(n_, dtype=np.complex128)
            if self.nz in src_bwd:
                e = add(e, src_bwd[self.nz])
            if self.nz in born_bwd:
                e = e + born_bwd[self.nz]
            if self.nz in keep:
                res["backward"][self.nz] = e.copy()
            for p in range(self.nz, 0, -1):
                if self.host[p - 1] is not None:
                    born_fwd[p] = self.born_emission(self.born_sources(e, -1, p - 1), +1, p - 1)
                    e = e + self.born_step(e, -1, p - 1)
                if anyi[p - 1]:
                    src_fwd[p] = store(self.apply(BWD_R, e, p, p - 1), iface[p - 1])
                e = self.apply(BWD_T, e, p, p - 1)
                if p - 1 in src_bwd:
                    e = add(e, src_bwd[p - 1])
                if p - 1 in born_bwd:
                    e = e + born_bwd[p - 1]
                if p - 1 in keep:
                    res["backward"][p - 1] = e.copy()
            res["reflected"] = e
            res["transmitted_iter"].append(res["transmitted"])
            res["reflected_iter"].append(res["reflected"])
            stored = sum(int(s[0].sum()) for s in src_bwd.values()) + sum(
                int(s[0].sum()) for s in src_fwd.values())
            res["stored_values"] = max(res["stored_values"], stored)
        if res["reflected"] is None:
            res["reflected"] = np.zeros(n_, dtype=np.complex128)
        return res


def power_flux(field_y: np.ndarray, ny: int, dy: float, k0: float, index: complex,
               direction: int = 1) -> float:
    """2D power flux Σ Re k_z (|Ê|² + |Ê_z|²) (src/bwpm/fpwpm.py:205-216), field (ny, 2)."""
    spectrum = np.fft.fft(field_y, axis=0) / ny
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=dy)
    kz = longitudinal_wavenumber(index, k0, ky**2)
    with np.errstate(divide="ignore", invalid="ignore"):
        ez = np.where(kz != 0, -direction * ky * spectrum[:, 1] / kz, 0.0)
    magnitude = np.sum(np.abs(spectrum) ** 2, axis=1) + np.abs(ez) ** 2
    return float(np.sum(np.real(kz) * magnitude) * ny * dy)
