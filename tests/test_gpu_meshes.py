"""The reference's own mesh files on the CUDA path: TomoSh_CUDA against the
reference INT3 engine's outputs stored in tests/golden/mesh_*.npz
(tests/golden/make_meshes.py), per orientation and bit for bit, for every
printer setup the fixture holds.  The mesh arrays travel in the fixtures,
so no mesh file is read here."""
from __future__ import annotations

import json

import numpy as np
import pytest

from tests.test_golden import GOLDEN_DIR
from tomo_shell2026_b200 import meshgen
from tomo_shell2026_b200.options import PrintOptions

MESH_FIXTURES = sorted(GOLDEN_DIR.glob("mesh_*.npz"))


def _mesh(d):
    return meshgen.MeshArrays(d["vertices"], d["faces"], d["vertex_normals"], d["face_normals"], float(d["area"]))


def _bits(a):
    return np.asarray(a, np.float32).view(np.int32)


def test_mesh_fixtures_present():
    names = {p.stem for p in MESH_FIXTURES}
    assert {"mesh_manikin_ply", "mesh_bunny_stl", "mesh_body_gltf", "mesh_sphere_ply"} <= names
    for p in MESH_FIXTURES:
        d = np.load(p)
        m = _mesh(d)
        assert m.faces.min() >= 0 and m.faces.max() < m.n_vtx
        assert d["explicit_Vss64"].shape[0] == d["yaw_deg"].shape[0] * d["pitch_deg"].shape[0]


@pytest.mark.gpu
@pytest.mark.parametrize("path", MESH_FIXTURES, ids=[p.stem for p in MESH_FIXTURES])
def test_reference_mesh_on_cuda_path(path):
    from tomo_shell2026_b200 import native
    d = np.load(path)
    m = _mesh(d)
    ypr = meshgen.ypr_grid(d["yaw_deg"], d["pitch_deg"])
    for tag in d["variants"]:
        opts = PrintOptions(**json.loads(str(d[f"{tag}_options"])))
        res = native.sweep(m, ypr, opts)
        for k in ("Vo64", "Vss64", "Vtc64"):
            bad = np.nonzero(getattr(res, k) != d[f"{tag}_{k}"])[0]
            assert bad.size == 0, f"{path.stem}/{tag}: {k} differs at {bad[:8]}"
        for k in ("VoF", "VssF", "Mo", "Mss", "Vtc"):
            bad = np.nonzero(_bits(getattr(res, k)) != _bits(d[f"{tag}_{k}"]))[0]
            assert bad.size == 0, f"{path.stem}/{tag}: {k} bits differ at {bad[:8]}"
        assert res.optID == int(d[f"{tag}_optID"]), f"{path.stem}/{tag}: optID"
