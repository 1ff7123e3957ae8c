"""The oracle restatement against the reference CPU core built from source (oracle/_ref).

Skipped where oracle/build_ref.sh has not been run (e.g. a machine without the reference tree).
"""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import pytest

from bwpm_b200 import workloads
from conftest import load_npz, rel_l2
from oracle import port

REF = sorted((Path(__file__).resolve().parents[1] / "oracle" / "_ref").glob("_core*.so"))


def _ref():
    spec = importlib.util.spec_from_file_location("_core", REF[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


pytestmark = pytest.mark.skipif(not REF, reason="oracle/_ref not built (oracle/build_ref.sh)")


@pytest.mark.parametrize("name", ["slab2d_te", "born2d_small_tm", "lens3d_small"])
def test_workload_fixtures_are_reference_outputs(name):
    """The committed workload fixtures equal a fresh reference-core run (fixture freshness)."""
    d = load_npz("workload_cases.npz")
    prob = workloads.Problem.from_arrays(d, name + ".")
    s = _ref().Solver(*prob.core_args(), 1, fluctuation=prob.fluctuation)
    r = s.run(prob.field, prob.iterations, [])
    assert rel_l2(r["transmitted"], d[name + ".transmitted"]) < 1e-13
    assert rel_l2(r["reflected"], d[name + ".reflected"]) < 1e-13


def test_port_equals_reference_core_small_lens():
    d = load_npz("workload_cases.npz")
    prob = workloads.Problem.from_arrays(d, "lens3d_small.")
    r = port.Solver(*prob.core_args(), fluctuation=prob.fluctuation).run(prob.field, prob.iterations)
    assert rel_l2(r["transmitted"], d["lens3d_small.transmitted"]) < 1e-11
    assert rel_l2(r["reflected"], d["lens3d_small.reflected"]) < 1e-11
    assert r["stored_values"] == int(d["lens3d_small.stored_values"])


def test_port_equals_reference_core_born():
    d = load_npz("workload_cases.npz")
    prob = workloads.Problem.from_arrays(d, "born2d_small_te.")
    r = port.Solver(*prob.core_args(), fluctuation=prob.fluctuation).run(prob.field, prob.iterations)
    assert rel_l2(r["transmitted"], d["born2d_small_te.transmitted"]) < 1e-11
    assert rel_l2(r["reflected"], d["born2d_small_te.reflected"]) < 1e-10


def test_reference_core_interface_matrices_equal_port():
    core = _ref()
    rng = np.random.default_rng(3)
    k0 = 2 * np.pi / 0.6e-3
    kx = rng.uniform(-2, 2, 200) * k0
    ky = rng.uniform(-2, 2, 200) * k0
    for n1, n2 in [(1.0, 1.5), (1.5, 1.0), (1.0, 0.213 + 6.697j), (1.33, 2.1 + 0.01j)]:
        a = core.transmission_matrix(kx, ky, n1, n2, k0)
        b = port.transmission_matrix(kx, ky, n1, n2, k0)
        assert np.allclose(a, b, rtol=1e-12, atol=1e-13 * np.max(np.abs(a)))
