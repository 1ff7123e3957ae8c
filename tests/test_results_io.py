"""The golden-file envelope ("raytatouille-result") written and read by bwpm_b200.results.

The reference's golden files use this envelope (src/bwpm/results.py); tests/golden holds them
converted to npz. Here: round trips of every value kind, the decoder of the fixture generator
(tests/golden/make_fixtures.py) reading what this module writes, and a solve record of the
oracle's result for a golden case.
"""

from __future__ import annotations

import json
import math

import numpy as np
import pytest

from conftest import load_golden


def test_round_trip_of_every_value_kind():
    from bwpm_b200 import results

    data = {
        "f64": np.array([[1.5, math.nan], [math.inf, -math.inf]]),
        "c128": np.array([1 + 2j, complex(math.nan, 1.0), complex(0.0, -math.inf)]),
        "i32": np.arange(6, dtype=np.int32).reshape(2, 3),
        "u8": np.array([0, 255], dtype=np.uint8),
        "b": np.array([True, False]),
        "scalar": 0.1,
        "nan": math.nan,
        "z": 0.25 - 3j,
        "nested": {"list": [1, 2.5, "text"], "k": np.float64(2.0)},
    }
    kind, back = results.load_json(results.to_json(results.FIELD_REFERENCE, data))
    assert kind == results.FIELD_REFERENCE
    for key in ("f64", "c128", "i32", "u8", "b"):
        assert back[key].dtype == data[key].dtype and back[key].shape == data[key].shape
        assert np.array_equal(back[key], data[key], equal_nan=True)
    assert back["scalar"] == 0.1 and math.isnan(back["nan"]) and back["z"] == 0.25 - 3j
    assert back["nested"] == {"list": [1, 2.5, "text"], "k": 2.0}


def test_text_is_strict_json_with_markers():
    from bwpm_b200 import results

    text = results.to_json("T", {"a": np.array([math.nan]), "s": math.inf})
    env = json.loads(text)  # no NaN literals
    assert env["format"] == "raytatouille-result" and env["schema_version"].startswith("0.1.")
    assert env["data"]["a"]["values"] == ["NaN"] and env["data"]["s"] == {"float": "Infinity"}


def test_rejects_other_formats_and_versions():
    from bwpm_b200 import results

    with pytest.raises(ValueError):
        results.load_json(json.dumps({"format": "other", "schema_version": "0.1.0", "data": {}}))
    with pytest.raises(ValueError):
        results.load_json(json.dumps({"format": results.FORMAT, "schema_version": "1.0", "data": {}}))
    with pytest.raises(ValueError):
        results.encode(np.array(["x"]))


def test_fixture_decoder_reads_what_this_module_writes():
    from golden import make_fixtures
    from bwpm_b200 import results

    data = {"x": np.array([1 + 1j, complex(math.inf, 0.0)]), "y": np.array([2.0, math.nan])}
    env = json.loads(results.to_json("T", data))
    dec = make_fixtures.decode(env["data"])
    assert np.array_equal(dec["x"], data["x"]) and np.array_equal(dec["y"], data["y"], equal_nan=True)


def test_solve_record_of_a_golden_case():
    """A record of the oracle's run of bwpm2d_tilted_silver round-trips and matches the file."""
    from bwpm_b200 import results, workloads
    from oracle import port

    a, meta = load_golden("bwpm2d_tilted_silver")
    ny = int(meta["parameters.ny"])
    lam = meta["parameters.wavelength_um"]
    prob = workloads.Problem(ny, 1, meta["parameters.dy_mm"], 1.0, meta["parameters.dz_mm"],
                             workloads.k0_of(lam), np.asarray(a["inputs.indices"]),
                             np.asarray(a["inputs.labels"], dtype=np.int32)[:, :, None],
                             complex(a["inputs.index_before"]), a["inputs.mask"][:, None],
                             np.asarray(a["inputs.field"])[:, None, :], 2)
    r = port.Solver(*prob.core_args()).run(prob.field, prob.iterations)
    rec = results.solve_record("bwpm2d_tilted_silver_oracle", prob,
                               {"transmitted": r["transmitted"], "reflected": r["reflected"]},
                               source="oracle/port.py")
    kind, back = results.load_json(results.to_json(results.FIELD_REFERENCE, rec))
    assert kind == "FieldReference"
    assert np.array_equal(back["expected"]["transmitted"], r["transmitted"])
    assert np.allclose(back["expected"]["transmitted"][:, 0], a["expected.forward"][-1],
                       rtol=1e-12, atol=1e-13 * np.max(np.abs(a["expected.forward"][-1])))
