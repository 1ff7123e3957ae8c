"""Label volumes generated on the device from a geometry (bwpm_geometry_labels) against the host
generator with the same operations (bwpm_b200.workloads.geometry_labels): integer output, so
identical or it fails. Then solves whose labels come from the device generator against the same
solves with host labels (bit for bit), alone and through the server."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    from bwpm_b200 import workloads

    out = [workloads.microlens3d(n=128, nz=100).geometry, workloads.microlens3d().geometry]
    prm = workloads.batch2d_params(24, 4)
    out += [workloads.tilted_slab2d_from(p).geometry for p in prm[:12]]
    stream = workloads.request_stream(40, 1.0, seed=5, iterations=2, max_lateral_3d=512,
                                      host_labels=False)
    out += [p.geometry for _, p in stream]
    rng = np.random.default_rng(3)
    big = workloads.request(rng, 0, max_lateral_3d=1024, host_labels=False).geometry
    out.append(dict(big, nz=40, ny=1024, nx=1024))
    return out


def test_device_labels_equal_host_labels():
    from bwpm_b200 import geometry, workloads

    kinds = set()
    for g in _cases():
        host = workloads.geometry_labels(g)
        dev = geometry.device_labels(g)
        assert dev.shape == host.shape
        assert np.array_equal(dev, host), (g["kind"], g["ny"], g["nx"], g["nz"])
        kinds.add(g["kind"])
    assert kinds == set(geometry.KINDS)


def test_rejects_bad_geometry():
    from bwpm_b200 import geometry

    g = {"kind": "lens_array", "nz": 4, "ny": 8, "nx": 8, "dz": 1e-4, "dy": 1e-4, "dx": 1e-4,
         "pitch": 0.0}
    with pytest.raises(ValueError):
        geometry.device_labels(g)
    with pytest.raises(ValueError):
        geometry.device_labels(dict(g, kind="cube"))


@pytest.mark.parametrize("precision", [64, 32])
def test_solver_from_geometry_equals_host_labels(precision):
    from bwpm_b200 import _core, workloads

    p = workloads.microlens3d(n=96, nz=60, iterations=2)
    a = _core.CudaSolver(*p.core_args(), 0, precision=precision).run(p.field, 2, [0, 30])
    b = _core.CudaSolver.from_geometry(p.ny, p.nx, p.dy, p.dx, p.dz, p.k0, p.indices, p.geometry,
                                       p.index_before, p.mask, 0, precision=precision).run(
        p.field, 2, [0, 30])
    for key in ("transmitted", "reflected"):
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(a["forward"][30], b["forward"][30])
    assert a["stored_values"] == b["stored_values"]


def test_served_geometry_requests_equal_solves_alone():
    from bwpm_b200 import _core, workloads
    from bwpm_b200.serve import Server, serve_stream

    stream = workloads.request_stream(30, 1.0, seed=5, iterations=2, max_lateral_3d=384,
                                      host_labels=False)
    probs3d = [p for _, p in stream if p.nx != 1][:4]
    assert probs3d and all(p.labels is None for p in probs3d)
    with Server(0) as srv:
        res, _ = serve_stream(srv, [(0.0, p) for p in probs3d])
    for p, r in zip(probs3d, res):
        alone = _core.CudaSolver.from_geometry(p.ny, p.nx, p.dy, p.dx, p.dz, p.k0, p.indices,
                                               p.geometry, p.index_before, p.mask, 0,
                                               precision=32).run(p.field, p.iterations, [])
        for key in ("transmitted", "reflected"):
            assert np.array_equal(r[key], alone[key]), key
