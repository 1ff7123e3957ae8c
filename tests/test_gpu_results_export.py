"""A GPU result exported in the reference's golden-file envelope and read back (on a GPU).

The 5 µm slab at full size (1024 points, 250 slabs, 8 iterations, TE and TM) runs through the
FP64 drop-in path and the batched complex64 engine; each result becomes a `FieldReference`
record (bwpm_b200.results.solve_record) in a "raytatouille-result" file, which is read back by
this package and, where the reference package is staged (oracle/stage_reference.sh), by the
reference's own reader (src/bwpm/results.py:125-135). The read-back fields equal the written
ones exactly and match the reference CPU core's result for the same inputs (fixture
workload_cases.npz) at the tolerance the record states (FP64: 1e-10; complex64: 1e-4).
"""

from __future__ import annotations

import importlib
import sys

import numpy as np
import pytest

import reference_shim
from conftest import load_npz, rel_l2

pytestmark = pytest.mark.gpu


def _reference_reader():
    if not reference_shim.staged():
        return None
    sys.path.insert(0, str(reference_shim.STAGED))
    try:
        return importlib.import_module("bwpm.results")
    finally:
        sys.path.remove(str(reference_shim.STAGED))


@pytest.mark.parametrize("pol", ["te", "tm"])
def test_config1_results_exported_and_read_back(tmp_path, pol):
    from bwpm_b200 import _core, results, workloads
    from bwpm_b200.batch import Batch2D

    fixture = load_npz("workload_cases.npz")
    name = f"slab2d_{pol}"
    p = workloads.Problem.from_arrays(fixture, name + ".")
    r64 = _core.CudaSolver(*p.core_args(), 0).run(p.field, p.iterations, [])
    b = Batch2D(0)
    i = b.add_problem(p)
    b.prepare()
    b.run()
    r32 = b.result(i)
    records = {
        "fp64": results.solve_record(f"{name}_fp64", p, r64, "bwpm_b200 CudaSolver, FP64",
                                     {"rel": 1e-10, "abs": 0.0}),
        "c64": results.solve_record(f"{name}_c64", p,
                                    {"transmitted": r32["transmitted"][:, None, :],
                                     "reflected": r32["reflected"][:, None, :],
                                     "energy_residual": r32["energy_residual"]},
                                    "bwpm_b200 batched engine, complex64", {"rel": 1e-4, "abs": 0.0}),
    }
    ref_reader = _reference_reader()
    for kind, rec in records.items():
        path = tmp_path / f"{name}_{kind}.result.json"
        path.write_text(results.to_json(results.FIELD_REFERENCE, rec), encoding="utf-8")
        text = path.read_text(encoding="utf-8")
        readers = [results.load_json] + ([ref_reader.load_json] if ref_reader else [])
        for load in readers:
            kind_name, data = load(text)
            assert kind_name == results.FIELD_REFERENCE
            tol = data["tolerance"]["rel"]
            for key in ("transmitted", "reflected"):
                back = np.asarray(data["expected"][key])
                assert np.array_equal(back, rec["expected"][key])
                assert rel_l2(back, fixture[f"{name}.{key}"]) < tol, (kind, key)
            assert np.array_equal(np.asarray(data["inputs"]["labels"]), p.labels)
