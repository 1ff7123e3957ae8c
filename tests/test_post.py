"""Post-processing of fields: the CPU oracle (oracle/post.py) and the device functions
(bwpm_b200.post, -m gpu) against the reference's own functions on seeded inputs
(tests/golden/postproc.npz): bwpm.adapter.port_power (src/bwpm/adapter.py:267-284),
bwpm.fpwpm.power_flux (src/bwpm/fpwpm.py:205-216), bwpm.pilot_imc3d.plane_power and
axial_focus (src/bwpm/pilot_imc3d.py:55-131). Tolerance rel 1e-12 (FP64 with a different FFT
and compensated sums); the focus offset is exact.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from conftest import load_npz
from oracle import post as oracle

TOL = 1e-12
PORTS = ("n15_fwd", "absorbing_bwd", "silver_fwd")


@pytest.fixture(scope="module")
def z():
    return load_npz("postproc.npz")


def _grid(g):
    ny, nx, dy, dx, wl = g
    return SimpleNamespace(ny=int(ny), nx=int(nx), dy=float(dy), dx=float(dx),
                           k0=float(2 * np.pi / (wl * 1e-3)))


def _rel(a, b):
    return abs(a - b) / abs(b)


def test_oracle_port_and_plane_power(z):
    g = _grid(z["beam3d.grid"])
    for tag in PORTS:
        got = oracle.port_power(z["beam3d.field"], g.dy, g.dx, g.k0,
                                complex(z[f"beam3d.port_power.{tag}.index"]),
                                int(z[f"beam3d.port_power.{tag}.direction"]))
        assert _rel(got, float(z[f"beam3d.port_power.{tag}"])) < TOL, tag
    for tag, n in (("n15", 1.5), ("n10", 1.0)):
        got = oracle.plane_power(z["beam3d.field"], g.dy, g.dx, g.k0, n)
        assert _rel(got, float(z[f"beam3d.plane_power.{tag}"])) < TOL, tag


def test_oracle_power_flux_and_focus(z):
    g = _grid(z["flux2d.grid"])
    f = z["flux2d.field"]
    assert _rel(oracle.power_flux(f, g.dy, g.k0, 1.5, 1), float(z["flux2d.power_flux.n15_fwd"])) < TOL
    assert _rel(oracle.power_flux(f, g.dy, g.k0, 1.0, -1), float(z["flux2d.power_flux.n10_bwd"])) < TOL
    g = _grid(z["focus.grid"])
    for tag, na in (("all", None), ("na04", 0.4)):
        best, peak = oracle.axial_focus(z["focus.field"], g.dy, g.dx, g.k0, 1.0, z["focus.offsets"], na)
        assert best == float(z[f"focus.{tag}.best"])
        assert _rel(peak, float(z[f"focus.{tag}.peak"])) < TOL


@pytest.mark.gpu
def test_device_port_and_plane_power(z):
    from bwpm_b200 import post

    g = _grid(z["beam3d.grid"])
    for tag in PORTS:
        got = post.port_power_array(z["beam3d.field"], g.dy, g.dx, g.k0,
                                    complex(z[f"beam3d.port_power.{tag}.index"]),
                                    int(z[f"beam3d.port_power.{tag}.direction"]))
        assert _rel(got, float(z[f"beam3d.port_power.{tag}"])) < TOL, tag
    for tag, n in (("n15", 1.5), ("n10", 1.0)):
        got = post.plane_power(z["beam3d.field"], g, n)
        assert _rel(got, float(z[f"beam3d.plane_power.{tag}"])) < TOL, tag


@pytest.mark.gpu
def test_device_power_flux_and_focus(z):
    from bwpm_b200 import post

    g = _grid(z["flux2d.grid"])
    f = z["flux2d.field"]
    assert _rel(post.power_flux(f, g.dy, g.k0, 1.5, 1), float(z["flux2d.power_flux.n15_fwd"])) < TOL
    assert _rel(post.power_flux(f, g.dy, g.k0, 1.0, -1), float(z["flux2d.power_flux.n10_bwd"])) < TOL
    g = _grid(z["focus.grid"])
    for tag, na in (("all", None), ("na04", 0.4)):
        best, peak, inten = post.axial_focus(z["focus.field"], g, 1.0, z["focus.offsets"], na,
                                             return_intensity=True)
        assert best == float(z[f"focus.{tag}.best"])
        assert _rel(peak, float(z[f"focus.{tag}.peak"])) < TOL
        ref = oracle.axial_focus_intensity(z["focus.field"], g.dy, g.dx, g.k0, 1.0,
                                           z["focus.offsets"], na)
        assert np.allclose(inten, ref, rtol=TOL, atol=0)


@pytest.mark.gpu
def test_device_post_rejects_bad_input():
    from bwpm_b200 import post

    g = SimpleNamespace(ny=8, nx=8, dy=1e-4, dx=1e-4, k0=1e4)
    with pytest.raises(ValueError):
        post.plane_power(np.zeros((8, 8, 2)), g, -1.0)
    with pytest.raises(ValueError):
        post.port_power_array(np.zeros((8, 8, 2)), 1e-4, 1e-4, 1e4, 1.0, 2)
    with pytest.raises(ValueError):
        post.axial_focus(np.zeros((8, 8, 2)), g, 1.0, [])
