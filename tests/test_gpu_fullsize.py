"""Whole 1-degree sweeps of the two large workloads through TomoSh_CUDA,
bit for bit against the reference INT3 engine's own outputs for every
orientation (tests/golden/make_fullsize.py wrote them, running the engine
compiled from the reference sources).

* the 81,920-triangle solid at 0.5 mm, 21,960 orientations: its exact Vo
  passes 2^24, so the float32 accumulators VoF exercise the fold replay;
* the manikin-like thin open shell in shell mode at 1 mm, 21,960
  orientations, ~1.3 M slot entries per orientation.

The meshes are regenerated from their seeds; a SHA-256 of the arrays pins
that the bytes are the ones the reference engine saw.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.golden.make_fullsize import cases, mesh_sha256
from tests.test_golden import GOLDEN_DIR
from tomo_shell2026_b200 import meshgen

CASES = {name: (factory, opts) for name, factory, opts, _ in cases()}


def _load(name):
    path = GOLDEN_DIR / f"{name}.npz"
    assert path.exists(), f"missing fixture {path.name}: run tests/golden/make_fullsize.py"
    return np.load(path)


def _bits(a):
    return np.asarray(a, np.float32).view(np.int32)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fixture_mesh_regenerates(name):
    """The seeded generator reproduces the exact mesh bytes of the fixture."""
    d = _load(name)
    factory, _ = CASES[name]
    assert mesh_sha256(factory()) == str(d["mesh_sha256"])
    assert d["Vss64"].shape[0] == d["yaw_deg"].shape[0] * d["pitch_deg"].shape[0]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_full_sweep_matches_reference_engine(name):
    from tomo_shell2026_b200 import native
    d = _load(name)
    factory, opts = CASES[name]
    mesh = factory()
    assert mesh_sha256(mesh) == str(d["mesh_sha256"])
    ypr = meshgen.ypr_grid(d["yaw_deg"], d["pitch_deg"])
    res = native.sweep(mesh, ypr, opts)
    for k in ("Vo64", "Vss64", "Vtc64"):
        got, want = getattr(res, k), d[k]
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"{name}: {k} differs at {bad.size} orientations, first {bad[:8]}"
    for k in ("VoF", "VssF", "Mo", "Mss", "Vtc"):
        bad = np.nonzero(_bits(getattr(res, k)) != _bits(d[k]))[0]
        assert bad.size == 0, f"{name}: {k} bits differ at {bad.size} orientations, first {bad[:8]}"
    assert res.optID == int(d["optID"]), f"{name}: optID {res.optID} != {int(d['optID'])}"
    # the argmin of the exact int64 Vss (lowest index on ties) names the same orientation
    assert int(np.argmin(res.Vss64)) == res.optID
