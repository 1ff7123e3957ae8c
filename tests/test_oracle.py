"""The CPU oracle (oracle/port.py) pinned against the reference's golden vectors.

Golden files: the reference's reference/*.result.json (converted by tests/golden/make_fixtures.py)
with the tolerances they carry (rel 1e-12, abs 1e-13·max; tools/reference_cases.py:26-27), and
the reference's own outputs for the random volumes of tests/test_core_cuda.py:91-196 and for
workload-shaped cases (reference CPU core, cpp/src/solver.cpp).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import close, load_golden, load_npz
from golden_cases import case_2d, case_3d, volume_case
from oracle import port


def test_interface_matrices_golden():
    a, meta = load_golden("interface_matrices")
    kx, ky = a["inputs.k_x_per_mm"], a["inputs.k_y_per_mm"]
    k0 = meta["parameters.k0_per_mm"]
    for j, (n1, n2) in enumerate(a["inputs.index_pairs"]):
        t = port.transmission_matrix(kx * n1.real, ky * n1.real, n1, n2, k0)
        r = port.reflection_matrix(kx * n1.real, ky * n1.real, n1, n2, k0)
        close(t, a["expected.T"][j], meta["tolerance.rel"], meta["tolerance.abs"])
        close(r, a["expected.R"][j], meta["tolerance.rel"], meta["tolerance.abs"])


def test_fpwpm2d_interface_golden():
    args, f, fl, a, meta = case_2d("fpwpm2d_interface")
    nz = args[7].shape[0]
    r = port.Solver(*args, fluctuation=fl).run(f, 0, range(nz + 1))
    planes = np.stack([r["forward"][p][:, 0] for p in range(nz + 1)])
    close(planes, a["expected.planes"], meta["tolerance.rel"], meta["tolerance.abs"])


def test_bwpm2d_tilted_silver_golden():
    args, f, fl, a, meta = case_2d("bwpm2d_tilted_silver")
    nz = args[7].shape[0]
    r = port.Solver(*args, fluctuation=fl).run(f, 2, range(nz + 1))
    close(np.stack([r["forward"][p][:, 0] for p in range(nz + 1)]), a["expected.forward"],
          meta["tolerance.rel"], meta["tolerance.abs"])
    close(np.stack([r["backward"][p][:, 0] for p in range(nz + 1)]), a["expected.backward"],
          meta["tolerance.rel"], meta["tolerance.abs"])


def test_bwpm2d_slab_exact_golden_and_airy():
    args, f, fl, a, meta = case_2d("bwpm2d_slab_exact")
    r = port.Solver(*args, fluctuation=fl).run(f, 40)
    close(r["transmitted"][:, 0], a["expected.transmitted"], meta["tolerance.rel"], meta["tolerance.abs"])
    close(r["reflected"][:, 0], a["expected.reflected"], meta["tolerance.rel"], meta["tolerance.abs"])
    rte = complex(np.mean(r["reflected"][:, 0, 0] / f[:, 0, 0]))
    assert abs(rte - complex(a["reference.r_te_airy"])) < meta["reference_tolerance.abs"]


@pytest.mark.parametrize("name,iters,keep", [("bwpm3d_tilted", 2, (0, 10, 20)),
                                             ("bwpm3d_fluctuation", 1, (0, 8, 16))])
def test_3d_golden(name, iters, keep):
    args, f, fl, a, meta = case_3d(name)
    r = port.Solver(*args, fluctuation=fl).run(f, iters, keep)
    tol = (meta["tolerance.rel"], meta["tolerance.abs"])
    close(r["transmitted"], a["expected.transmitted"], *tol)
    close(r["reflected"], a["expected.reflected"], *tol)
    close(np.stack([r["forward"][p] for p in keep]), a["expected.forward_planes"], *tol)
    close(np.stack([r["backward"][p] for p in keep]), a["expected.backward_planes"], *tol)


def test_fpwpm2d_fluctuation_golden():
    args, f, fl, a, meta = case_2d("fpwpm2d_fluctuation")
    nz = args[7].shape[0]
    r = port.Solver(*args, fluctuation=fl).run(f, 0, range(nz + 1))
    close(np.stack([r["forward"][p][:, 0] for p in range(nz + 1)]), a["expected.planes"],
          meta["tolerance.rel"], meta["tolerance.abs"])


@pytest.mark.parametrize("prefix,iters", [("volume1.", 2), ("volume2.", 2), ("volume3.", 2),
                                          ("fluct1.", 1), ("fluct2.", 1), ("backscatter.", 3)])
def test_random_volumes_against_reference_python(prefix, iters):
    d = load_npz("random_volumes.npz")
    args, field, fl = volume_case(d, prefix)
    r = port.Solver(*args, fluctuation=fl).run(field, iters)
    scale = 1e-12 * float(np.max(np.abs(field)))
    assert np.max(np.abs(r["transmitted"] - d[prefix + "transmitted"])) < scale
    assert np.max(np.abs(r["reflected"] - d[prefix + "reflected"])) < scale
    if prefix + "stored_values" in d:
        assert r["stored_values"] == int(d[prefix + "stored_values"])


def test_errors_match_reference_messages():
    args, f, fl, a, meta = case_2d("fpwpm2d_interface")
    bad = np.array(args[7])
    bad[0, 0, 0] = 7
    with pytest.raises(ValueError, match="labels must index"):
        port.Solver(*args[:7], bad, *args[8:])
