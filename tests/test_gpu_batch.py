"""Batched resident 2D engine (complex64) against the FP64 references, on a GPU.

Tolerances: relative L2 ≤ 1e-4 on transmitted/reflected fields against FP64 (the reference's
golden files, the reference CPU core outputs, or the FP64 GPU path that matches them at 1e-10),
and |ε_c64 − ε_FP64| ≤ 1e-6·max(1, (P_R + P_T)/P_in) on the energy residual
ε = 1 − (P_R + P_T)/P_in (the balance relative to the largest of the fluxes involved).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_npz, rel_l2
from golden_cases import case_2d

pytestmark = pytest.mark.gpu

L2_C64 = 1e-4
EPS_TOL = 1e-6


def _add_case(b, name, iters):
    args, f, fl, a, meta = case_2d(name)
    ny, _, dy, _, dz, k0, indices, labels, ib, mask = args
    i = b.add(ny, dy, dz, k0, indices, labels, ib, None if mask is None else mask[:, 0],
              f[:, 0, :], iters)
    return i, a


def test_batch_golden_2d_cases():
    from bwpm_b200.batch import Batch2D

    b = Batch2D()
    i1, a1 = _add_case(b, "fpwpm2d_interface", 0)
    i2, a2 = _add_case(b, "bwpm2d_tilted_silver", 2)
    i3, a3 = _add_case(b, "bwpm2d_slab_exact", 40)
    b.prepare()
    b.run()
    r1, r2, r3 = b.result(i1), b.result(i2), b.result(i3)
    assert rel_l2(r1["transmitted"], a1["expected.planes"][-1]) < L2_C64
    assert rel_l2(r2["transmitted"], a2["expected.forward"][-1]) < L2_C64
    assert rel_l2(r2["reflected"], a2["expected.backward"][0]) < L2_C64
    assert np.max(np.abs(np.array(r2["energy_residual"]) - a2["expected.energy_residual"])) < EPS_TOL
    assert rel_l2(r3["transmitted"], a3["expected.transmitted"]) < L2_C64
    assert rel_l2(r3["reflected"], a3["expected.reflected"]) < L2_C64
    assert np.all(r1["reflected"] == 0)


@pytest.mark.parametrize("name", ["slab2d_te", "slab2d_tm"])
def test_batch_slab_full_size(name):
    """1024 points, 250 slabs, 8 iterations against the reference CPU core (FP64)."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D

    d = load_npz("workload_cases.npz")
    prob = workloads.Problem.from_arrays(d, name + ".")
    b = Batch2D()
    i = b.add_problem(prob)
    b.run()
    r = b.result(i)
    assert rel_l2(r["transmitted"], d[name + ".transmitted"][:, 0]) < L2_C64
    assert rel_l2(r["reflected"], d[name + ".reflected"][:, 0]) < L2_C64


def _fp64(prob):
    from bwpm_b200 import _core

    s = _core.CudaSolver(*prob.core_args(), 0)
    return s.run(prob.field, prob.iterations, [])


def test_batch_uneven_instances_against_fp64_and_energy():
    """Uneven sizes incl. 3·2^k, tilted faces, masks, TE and TM, 0-30° incidence."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D
    from bwpm_b200.model import Grid2D, power_flux

    probs = workloads.batch2d(count=12, seed=11, sizes=(256, 384, 768, 1536, 3072, 6144),
                              nz_range=(40, 120), iterations=3)
    b = Batch2D()
    ids = [b.add_problem(p) for p in probs]
    b.run()
    for p, i in zip(probs, ids):
        r = b.result(i)
        ref = _fp64(p)
        assert rel_l2(r["transmitted"], ref["transmitted"][:, 0]) < L2_C64, p.name
        assert rel_l2(r["reflected"], ref["reflected"][:, 0]) < L2_C64, p.name
        g = Grid2D(p.ny, p.dy, p.dz, p.extra["wavelength_um"])
        p_in = power_flux(p.field[:, 0], g, p.index_before)
        last = complex(p.indices[int(p.labels[-1, p.ny // 2, 0])])
        for k in range(p.iterations):
            pt = power_flux(ref["transmitted_iter"][k][:, 0], g, last)
            pr = power_flux(ref["reflected_iter"][k][:, 0], g, p.index_before, direction=-1)
            eps64 = 1.0 - (pt + pr) / p_in
            scale = max(1.0, (pt + pr) / p_in)
            assert abs(r["energy_residual"][k] - eps64) < EPS_TOL * scale, (p.name, k)


# Energy balance of full-length chains: the FP32 rounding of ~24,000 dependent slab steps
# (2000 slabs, 6 iterations) moves the transmitted power by a random 1-4e-6 of P_in per
# iteration (measured on these items: at most 4.1e-6), so full-length chains are held to 1e-5
# and chains up to 120 slabs (test above) to 1e-6.
EPS_TOL_FULL = 1e-5


@pytest.mark.parametrize("ny", [8192, 6144, 3072])
def test_full_length_chains_against_fp64_and_energy(ny):
    """2000 slabs × 6 iterations (the longest chains of the batched workload), TE and TM, on the
    4-CTA cluster (8192, 6144) and single-CTA (3072) kernels: relative L2 ≤ 1e-4 against the FP64
    drop-in path and the energy balance on every iteration. The FP64 iteration converges on
    these items (it diverges on some instances of the workload whose light is trapped in the
    tilted slab, in the reference's algorithm as here)."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D
    from bwpm_b200.model import Grid2D, power_flux

    base = dict(wl=0.633, theta=0.2, n=1.5, tilt=0.05, iterations=6, ny=ny, nz=2000)
    probs = [workloads.tilted_slab2d_from(dict(base, i=i)) for i in (0, 1)]
    b = Batch2D()
    ids = [b.add_problem(p) for p in probs]
    b.run()
    for p, i in zip(probs, ids):
        r = b.result(i)
        ref = _fp64(p)
        assert rel_l2(r["transmitted"], ref["transmitted"][:, 0]) < L2_C64, p.name
        assert rel_l2(r["reflected"], ref["reflected"][:, 0]) < L2_C64, p.name
        g = Grid2D(p.ny, p.dy, p.dz, p.extra["wavelength_um"])
        p_in = power_flux(p.field[:, 0], g, p.index_before)
        last = complex(p.indices[int(p.labels[-1, p.ny // 2, 0])])
        for k in range(p.iterations):
            pt = power_flux(ref["transmitted_iter"][k][:, 0], g, last)
            pr = power_flux(ref["reflected_iter"][k][:, 0], g, p.index_before, direction=-1)
            eps64 = 1.0 - (pt + pr) / p_in
            scale = max(1.0, (pt + pr) / p_in)
            assert abs(r["energy_residual"][k] - eps64) < EPS_TOL_FULL * scale, (p.name, k)


def test_two_classes_in_one_batch():
    """A 6144-point and a 256-point solve (two CTA-width classes run concurrently)."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D

    probs = workloads.batch2d(count=12, seed=11, sizes=(256, 384, 768, 1536, 3072, 6144),
                              nz_range=(40, 120), iterations=3)
    b = Batch2D()
    ids = [b.add_problem(probs[2]), b.add_problem(probs[0])]
    b.run()
    for p, i in zip((probs[2], probs[0]), ids):
        ref = _fp64(p)
        assert rel_l2(b.result(i)["transmitted"], ref["transmitted"][:, 0]) < L2_C64


def test_result_alone_equals_result_in_mix():
    """A solve run alone and inside a batch of other solves gives the same result."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D

    probs = workloads.batch2d(count=9, seed=12, sizes=(256, 512, 1024, 3072),
                              nz_range=(30, 80), iterations=2)
    alone = Batch2D()
    ia = alone.add_problem(probs[0])
    alone.run()
    ra = alone.result(ia)
    mix = Batch2D()
    ids = [mix.add_problem(p) for p in probs[1:5]] + [mix.add_problem(probs[0])] + [
        mix.add_problem(p) for p in probs[5:]]
    mix.run()
    rm = mix.result(ids[4])
    assert np.array_equal(ra["transmitted"], rm["transmitted"])
    assert np.array_equal(ra["reflected"], rm["reflected"])


def test_solve_packed_round_trip():
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D

    probs = workloads.batch2d(count=5, seed=13, sizes=(256, 1024), nz_range=(20, 40), iterations=2)
    b = Batch2D()
    ids = [b.add_problem(p) for p in probs]
    b.run()
    fields = np.concatenate([p.field[:, 0, :].ravel() for p in probs])
    out = np.empty(2 * fields.size, dtype=np.complex128)
    b.solve_packed(fields, out)
    off = 0
    for p, i in zip(probs, ids):
        r = b.result(i)
        n2 = 2 * p.ny
        assert np.array_equal(out[off:off + n2].reshape(p.ny, 2), r["transmitted"])
        assert np.array_equal(out[off + n2:off + 2 * n2].reshape(p.ny, 2), r["reflected"])
        off += 2 * n2


FIXED_LENGTHS = (256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096, 6144, 8192)


def _variant_problem(n):
    from bwpm_b200 import workloads

    prm = dict(i=n, ny=n, nz=40, wl=0.55, theta=0.2, n=1.6, tilt=0.1, iterations=2)
    return workloads.tilted_slab2d_from(prm)


@pytest.mark.parametrize("n", FIXED_LENGTHS)
def test_every_kernel_variant_matches_fp64(n):
    """Each compiled kernel variant of a length (threads, radices, CTAs per line) against FP64."""
    from bwpm_b200.batch import Batch2D, variant_count

    p = _variant_problem(n)
    ref = _fp64(p)
    count = variant_count(n)
    assert count >= 1
    for k in range(count):
        b = Batch2D()
        b.set_variant(n, k)
        i = b.add_problem(p)
        b.run()
        cls = b.classes()
        assert cls[0]["variant"] == k and cls[0]["ny"] == n
        r = b.result(i)
        assert rel_l2(r["transmitted"], ref["transmitted"][:, 0]) < L2_C64, (n, k, cls[0])
        assert rel_l2(r["reflected"], ref["reflected"][:, 0]) < L2_C64, (n, k, cls[0])


def _seven_pass_problem(n, pol):
    """Three dielectrics behind two parallel tilted faces that cross the line on every slab: each
    step has 5 transmission passes (air, glass, n = 2 and the two interfaces) and 2 reflection
    passes, more than one group of passes per exchange in every cluster kernel."""
    from bwpm_b200.workloads import Problem, _vec, absorbing_mask_1d, centred, k0_of

    wl, nz, tilt, theta = 0.55, 40, 0.1, 0.15
    lam = wl * 1e-3
    dy, dz, k0 = lam / 8, lam / 10, k0_of(wl)
    y = centred(n, dy)
    z = (np.arange(nz) + 0.5) * dz
    front = 10 * dz + np.tan(tilt) * y
    back = front + 10 * dz
    labels = ((z[:, None] >= front[None, :]).astype(np.int32) +
              (z[:, None] >= back[None, :]).astype(np.int32))[:, :, None]
    w0 = n * dy / 8
    prof = (np.exp(-((y / w0) ** 2)) * np.exp(1j * k0 * np.sin(theta) * y))[:, None]
    mask = absorbing_mask_1d(y, n * dy / 10)[:, None]
    return Problem(n, 1, dy, 1.0, dz, k0, np.array([1.0 + 0j, 1.5 + 0j, 2.0 + 0j]), labels,
                   1.0 + 0j, mask, _vec(prof, pol), 2, name=f"seven_pass_{n}_{pol}")


@pytest.mark.parametrize("n", (4096, 6144, 8192))
def test_cluster_variants_on_steps_with_more_passes_than_a_group(n):
    """Steps with 7 passes: the inverse transforms go out in several groups (4 + 3 or 2 + 2 + 2 + 1
    per exchange); every variant of the length against FP64, TE and TM."""
    from bwpm_b200.batch import Batch2D, variant_count

    for pol in ("te", "tm"):
        p = _seven_pass_problem(n, pol)
        ref = _fp64(p)
        for k in range(variant_count(n)):
            b = Batch2D()
            b.set_variant(n, k)
            i = b.add_problem(p)
            b.run()
            r = b.result(i)
            assert rel_l2(r["transmitted"], ref["transmitted"][:, 0]) < L2_C64, (n, pol, k)
            assert rel_l2(r["reflected"], ref["reflected"][:, 0]) < L2_C64, (n, pol, k)


def test_autotuned_batch_equals_forced_variant():
    """Autotuning picks a variant per length; the results equal a run forced to that variant."""
    from bwpm_b200 import workloads
    from bwpm_b200.batch import Batch2D, variant_count

    probs = workloads.batch2d(count=8, seed=31, sizes=(1024, 4096, 6144, 8192), nz_range=(30, 60),
                              iterations=2)
    b = Batch2D()
    b.set_autotune(True)
    ids = [b.add_problem(p) for p in probs]
    b.run()
    cls = {c["ny"]: c for c in b.classes()}
    assert all((c["tuned_ms"] > 0) == (variant_count(n) > 1) for n, c in cls.items())
    forced = Batch2D()
    for n, c in cls.items():
        forced.set_variant(n, c["variant"])
    fids = [forced.add_problem(p) for p in probs]
    forced.run()
    for i, j in zip(ids, fids):
        assert np.array_equal(b.result(i)["transmitted"], forced.result(j)["transmitted"])


@pytest.mark.parametrize("n", [1000, 1125, 1200, 1944, 2160, 2187, 2700, 3645, 4000, 4050, 3125])
def test_runtime_length_kernels_match_fp64(n):
    """Lengths without a compiled kernel: the run-time-length register kernels (E values per
    thread, radices 2/3/4/5/8 dividing E), or the generic kernel (3125 = 5^5), against FP64."""
    from bwpm_b200.batch import Batch2D

    p = _variant_problem(n)
    ref = _fp64(p)
    b = Batch2D()
    i = b.add_problem(p)
    b.run()
    cls = b.classes()[0]
    assert cls["variant"] <= -1 and cls["ny"] == n
    assert (cls["variant"] == -1) == (n == 3125), cls  # −1: generic kernel, ≤ −2: run-time length
    r = b.result(i)
    assert rel_l2(r["transmitted"], ref["transmitted"][:, 0]) < L2_C64, cls
    assert rel_l2(r["reflected"], ref["reflected"][:, 0]) < L2_C64, cls


def test_wide_runtime_length_kernel_runs_4050_points():
    """4050 = 2·3⁴·5²: the default kernels with E ≥ 9 take at most 256 threads, where only E = 30
    (135 threads) fits; the wide form (512 threads) runs it with E = 9 on 450 threads."""
    from bwpm_b200.batch import Batch2D

    p = _variant_problem(4050)
    b = Batch2D()
    b.add_problem(p)
    b.prepare()
    cls = b.classes()[0]
    assert cls["variant"] <= -2 and 256 < cls["threads"] <= 512, cls


@pytest.mark.parametrize("n", [1024, 2048])
def test_runtime_length_kernel_forced_at_a_fixed_length(n):
    """set_variant(n, −1): the run-time-length kernel serves a length that has compiled ones."""
    from bwpm_b200.batch import Batch2D

    p = _variant_problem(n)
    ref = _fp64(p)
    b = Batch2D()
    b.set_variant(n, -1)
    i = b.add_problem(p)
    b.run()
    assert b.classes()[0]["variant"] <= -2
    r = b.result(i)
    assert rel_l2(r["transmitted"], ref["transmitted"][:, 0]) < L2_C64
    assert rel_l2(r["reflected"], ref["reflected"][:, 0]) < L2_C64
