"""Results in the reference's golden-file envelope ("raytatouille-result").

The reference keeps its golden files (`reference/<case>.result.json`, written by
`src/bwpm/results.py:110-167`) in a JSON envelope {"format", "schema_version", "type", "data"}
whose values follow one encoding:

- arrays: {"dtype", "shape", "values"} in C order, complex entries as [re, im];
- non-finite floats inside arrays as "NaN" / "Infinity" / "-Infinity", as scalars
  {"float": ...}; complex scalars {"complex": [re, im]};
- `allow_nan=False` JSON.

This module writes and reads that envelope so that results of this implementation (drop-in,
batched or served) can be exchanged with tools that read the reference's files, and so that a
`FieldReference` record (parameters, inputs, expected outputs, tolerance) can be produced from a
run here. The encoding must be the reference's for the files to be interchangeable; the code is
this package's own.
"""

from __future__ import annotations

import json
import math
from typing import Any

import numpy as np

FORMAT = "raytatouille-result"
SCHEMA_VERSION = "0.1.13"  # the version of the reference's files (reference/*.result.json)
FIELD_REFERENCE = "FieldReference"

_ARRAY_DTYPES = ("bool", "int8", "int16", "int32", "int64", "uint8", "uint16", "uint32",
                 "uint64", "float32", "float64", "complex64", "complex128")
_NONFINITE = {"NaN": math.nan, "Infinity": math.inf, "-Infinity": -math.inf}


def _fin(x: float) -> float | str:
    """A float, or its marker string when it is not finite."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    return x


def _num(x: Any) -> float:
    return _NONFINITE[x] if isinstance(x, str) else float(x)


def encode(value: Any) -> Any:
    """JSON-compatible data of a value (nested dicts, lists, NumPy arrays and scalars)."""
    if isinstance(value, np.ndarray):
        name = value.dtype.name
        if name not in _ARRAY_DTYPES:
            raise ValueError(f"results: arrays of dtype {name} cannot be written")
        flat = value.reshape(-1).tolist()
        if value.dtype.kind == "f":
            flat = [_fin(x) for x in flat]
        elif value.dtype.kind == "c":
            flat = [[_fin(z.real), _fin(z.imag)] for z in flat]
        return {"dtype": name, "shape": list(value.shape), "values": flat}
    if isinstance(value, dict):
        return {str(k): encode(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [encode(v) for v in value]
    if isinstance(value, np.generic):
        return encode(value.item())
    if isinstance(value, complex):
        return {"complex": [_fin(value.real), _fin(value.imag)]}
    if isinstance(value, float) and not math.isfinite(value):
        return {"float": _fin(value)}
    return value


def decode(value: Any) -> Any:
    """Inverse of `encode`: arrays come back as NumPy arrays of their dtype and shape."""
    if isinstance(value, list):
        return [decode(v) for v in value]
    if not isinstance(value, dict):
        return value
    keys = set(value)
    if keys == {"dtype", "shape", "values"}:
        dt = np.dtype(value["dtype"])
        vals = value["values"]
        if dt.kind == "f":
            vals = [_num(x) for x in vals]
        elif dt.kind == "c":
            vals = [complex(_num(a), _num(b)) for a, b in vals]
        return np.asarray(vals, dtype=dt).reshape(value["shape"])
    if keys == {"float"}:
        return _num(value["float"])
    if keys == {"complex"}:
        a, b = value["complex"]
        return complex(_num(a), _num(b))
    return {k: decode(v) for k, v in value.items()}


def to_json(type_name: str, data: dict[str, Any], indent: int | None = None) -> str:
    """The envelope text of `data` under the result type `type_name`."""
    return json.dumps({"format": FORMAT, "schema_version": SCHEMA_VERSION, "type": type_name,
                       "data": encode(data)}, allow_nan=False, indent=indent, ensure_ascii=False)


def load_json(text: str) -> tuple[str, dict[str, Any]]:
    """(type, decoded data) of an envelope text; only schema versions 0.1.x are read."""
    env = json.loads(text)
    if env.get("format") != FORMAT:
        raise ValueError(f"results: format must be '{FORMAT}'")
    if not str(env.get("schema_version", "")).startswith("0.1."):
        raise ValueError("results: only schema versions 0.1.x are read")
    data = decode(env["data"])
    if not isinstance(data, dict):
        raise ValueError("results: data must be an object")
    return str(env["type"]), data


def field_reference(case: str, description: str, source: str, parameters: dict[str, Any],
                    inputs: dict[str, Any], expected: dict[str, Any], tolerance: dict[str, float],
                    reference: dict[str, Any] | None = None,
                    reference_tolerance: dict[str, float] | None = None) -> dict[str, Any]:
    """A `FieldReference` record: one case with its parameters, inputs, expected outputs and
    tolerance (and, where there is one, an independent value with its tolerance)."""
    return {"case": case, "description": description, "source": source,
            "parameters": parameters, "inputs": inputs, "expected": expected,
            "tolerance": tolerance, "reference": reference or {},
            "reference_tolerance": reference_tolerance or {}}


def solve_record(case: str, prob, result: dict[str, Any], source: str,
                 tolerance: dict[str, float] | None = None) -> dict[str, Any]:
    """A `FieldReference` record of one solve of this implementation: the problem
    (`bwpm_b200.workloads.Problem`) as parameters and inputs, its transmitted and reflected
    fields (and energy residual, when the result has one) as expected values."""
    params = {"ny": int(prob.ny), "nx": int(prob.nx), "dy_mm": float(prob.dy),
              "dx_mm": float(prob.dx), "dz_mm": float(prob.dz), "k0_per_mm": float(prob.k0),
              "iterations": int(prob.iterations)}
    inputs = {"indices": np.asarray(prob.indices, dtype=np.complex128),
              "labels": np.asarray(prob.labels, dtype=np.int32),
              "index_before": complex(prob.index_before),
              "field": np.asarray(prob.field, dtype=np.complex128)}
    if prob.mask is not None:
        inputs["mask"] = np.asarray(prob.mask, dtype=np.float64)
    expected = {"transmitted": np.asarray(result["transmitted"], dtype=np.complex128),
                "reflected": np.asarray(result["reflected"], dtype=np.complex128)}
    if "energy_residual" in result:
        expected["energy_residual"] = np.asarray(result["energy_residual"], dtype=np.float64)
    return field_reference(case, f"{case}: one solve of bwpm_b200", source, params, inputs,
                           expected, tolerance or {"rel": 1e-4, "abs": 0.0})
