"""The reference-compatible Python surface on the CPU: mesh files, the
ctypes helpers and optimum ranking against the reference's own modules, and
the argument arrays TomoDLLInterface packs against the fixture made from the
reference engine (tests/golden/make_golden.py)."""
from __future__ import annotations

import importlib.util
import json
import struct
import sys
from pathlib import Path

import numpy as np
import pytest

from tomo_shell2026_b200 import meshgen
from tomo_shell2026_b200.cfms_tomo import SlicingOptions, TomoDLLInterface, TriMesh, enumBedType, enumPixelType, load
from tomo_shell2026_b200.cfms_tomo import tomo_io
from tomo_shell2026_b200.cfms_tomo.meshio import OrientedBox

from oracle.build import REF_ROOT  # noqa: E402  (the reference checkout, where present)

REF = REF_ROOT / "cfms_tomo"
GOLD = Path(__file__).parent / "golden" / "manager_two_parts.npz"


def _ref_module(name):
    if not (REF / f"{name}.py").exists():
        pytest.skip("reference checkout not present")
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))
    spec = importlib.util.spec_from_file_location(f"_ref_{name}", REF / f"{name}.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _tri_set(v, f):
    t = np.round(np.asarray(v, np.float64)[np.asarray(f)], 5)
    # rotate each triangle so its smallest corner comes first (winding kept)
    keys = [tuple(map(tuple, np.roll(x, -int(np.lexsort(x.T[::-1])[0]), axis=0))) for x in t]
    return sorted(keys)


@pytest.fixture(scope="module")
def small():
    m = meshgen.small_solid(0, with_hull=False)
    return m.vertices.astype(np.float64), m.faces.astype(np.int64)


def _write_ply(path, v, f, binary):
    head = (f"ply\nformat {'binary_little_endian' if binary else 'ascii'} 1.0\nelement vertex {len(v)}\n"
            "property float x\nproperty float y\nproperty float z\n"
            f"element face {len(f)}\nproperty list uchar int vertex_indices\nend_header\n").encode()
    with open(path, "wb") as fh:
        fh.write(head)
        if binary:
            fh.write(np.asarray(v, "<f4").tobytes())
            rec = np.zeros(len(f), dtype=[("n", "u1"), ("i", "<i4", 3)])
            rec["n"], rec["i"] = 3, f
            fh.write(rec.tobytes())
        else:
            for p in v:
                fh.write(("%r %r %r\n" % tuple(float(np.float32(x)) for x in p)).encode())
            for t in f:
                fh.write(("3 %d %d %d\n" % tuple(t)).encode())


def _write_stl(path, v, f, binary):
    t = np.asarray(v, np.float32)[f]
    if binary:
        rec = np.zeros(len(f), dtype=[("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")])
        rec["v"] = t
        with open(path, "wb") as fh:
            fh.write(b"\0" * 80 + struct.pack("<I", len(f)) + rec.tobytes())
    else:
        with open(path, "w") as fh:
            fh.write("solid s\n")
            for x in t:
                fh.write("facet normal 0 0 0\nouter loop\n")
                for p in x:
                    fh.write("vertex %r %r %r\n" % tuple(float(c) for c in p))
                fh.write("endloop\nendfacet\n")
            fh.write("endsolid s\n")


def _write_gltf(path, v, f, glb, offset):
    pos = np.asarray(v, "<f4").tobytes()
    idx = np.asarray(f, "<u4").tobytes()
    blob = pos + idx
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0]}],
           "nodes": [{"children": [1], "translation": list(offset)}, {"mesh": 0}],
           "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]}],
           "accessors": [{"bufferView": 0, "componentType": 5126, "count": len(v), "type": "VEC3"},
                         {"bufferView": 1, "componentType": 5125, "count": f.size, "type": "SCALAR"}],
           "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": len(pos)},
                           {"buffer": 0, "byteOffset": len(pos), "byteLength": len(idx)}],
           "buffers": [{"byteLength": len(blob)}]}
    if glb:
        js = json.dumps(doc).encode()
        js += b" " * (-len(js) % 4)
        blob += b"\0" * (-len(blob) % 4)
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(blob), 0x004E4942) + blob
        Path(path).write_bytes(b"glTF" + struct.pack("<II", 2, 12 + len(body)) + body)
    else:
        Path(path).with_suffix(".bin").write_bytes(blob)
        doc["buffers"][0]["uri"] = Path(path).with_suffix(".bin").name
        Path(path).write_text(json.dumps(doc))


@pytest.mark.parametrize("kind", ["ply_ascii", "ply_binary", "stl_ascii", "stl_binary", "obj", "gltf", "glb"])
def test_mesh_files_round_trip(tmp_path, small, kind):
    v, f = small
    v32 = v.astype(np.float32).astype(np.float64)
    offset = (0.0, 0.0, 0.0)
    if kind.startswith("ply"):
        p = tmp_path / "m.ply"; _write_ply(p, v, f, kind.endswith("binary"))
    elif kind.startswith("stl"):
        p = tmp_path / "m.stl"; _write_stl(p, v, f, kind.endswith("binary"))
    elif kind == "obj":
        p = tmp_path / "m.obj"
        p.write_text("".join("v %r %r %r\n" % tuple(float(c) for c in x) for x in v.astype(np.float32)) +
                     "".join("f %d %d %d\n" % tuple(t + 1) for t in f))
    else:
        offset = (1.5, -2.0, 4.0)
        p = tmp_path / ("m.glb" if kind == "glb" else "m.gltf"); _write_gltf(p, v, f, kind == "glb", offset)
    m = load(p)
    assert m.faces.shape == f.shape
    assert m.vertices.shape == v.shape, "duplicate corners must merge back to the shared vertices"
    assert m.is_watertight
    assert _tri_set(m.vertices, m.faces) == _tri_set(v32 + np.asarray(offset), f)


def test_trimesh_properties(small):
    v, f = small
    m = TriMesh(v, f, process=False)
    ref = meshgen.mesh_from_arrays(v, f, with_hull=False)
    assert abs(m.area - ref.area) < 1e-6 * ref.area
    assert np.allclose(m.face_normals, ref.face_normals, atol=1e-6)
    # angle-weighted normals of a smooth closed surface stay close to area-weighted ones
    assert np.min(np.einsum("ij,ij->i", m.vertex_normals, ref.vertex_normals)) > 0.99
    h = m.convex_hull
    assert h.is_watertight
    c = h.vertices.mean(0)
    assert np.all(np.einsum("ij,ij->i", h.face_normals, h.triangles.mean(1) - c) > 0), "hull normals point outward"
    box = m.bounding_box_oriented
    assert isinstance(box, OrientedBox) and box.extents.shape == (3,)
    assert np.all(box.extents <= np.linalg.norm(m.extents) + 1e-9)
    # an open mesh is not watertight
    assert not TriMesh(v, f[:-10], process=False).is_watertight


@pytest.mark.parametrize("name,faces,watertight", [("(1)sphere.ply", 39200, True), ("(3)manikin.ply", 13672, False),
                                                   ("Bunny_69k.stl", 69662, False)])
def test_reference_mesh_files(name, faces, watertight):
    path = REF_ROOT / "MeshData" / name
    if not path.exists():
        pytest.skip("reference mesh data not present")
    m = load(path)
    assert m.faces.shape[0] == faces
    assert m.is_watertight == watertight


def test_ranking_matches_reference_tomo_io():
    ref = _ref_module("tomo_io")
    rng = np.random.default_rng(5)
    for n in (1, 7, 169, 1000):
        data = (rng.random(n) * 50).astype(np.float32)
        data[rng.integers(0, n, n // 5)] = data[0]   # ties
        for N in (1, 3, 2000):
            a, b = tomo_io.smallestN_indices(data, N)
            ra, rb = ref.smallestN_indices(data, N)
            assert np.array_equal(a, ra) and np.array_equal(b, rb)
    assert tomo_io.FStr(1.234, precision=2) == ref.FStr(1.234, precision=2)
    assert np.array_equal(tomo_io.toRadian([0, 90, 360]), ref.toRadian([0, 90, 360]))


def test_options_match_reference():
    ref = _ref_module("tomo_slicingOptions")
    for k in ("wall_thickness", "PLA_density", "Fclad", "Fcore", "Fss", "Css", "dVoxel", "nVoxel", "theta_c",
              "bUseExplicitSS", "BedType", "Yaw", "Pitch", "Roll", "theta_YP", "bVerbose", "bUseCUDA", "bShellMesh",
              "ShellThickness"):
        assert getattr(SlicingOptions, k) == getattr(ref.SlicingOptions, k), k
    for e in enumPixelType:
        assert getattr(ref.enumPixelType, e.name).value == e.value
    for e in enumBedType:
        assert getattr(ref.enumBedType, e.name).value == e.value


def test_interface_packs_the_reference_arrays():
    """YPR grid and info arrays of TomoDLLInterface equal those the fixture
    was made with (no GPU call: the library is only loaded)."""
    d = np.load(GOLD)
    s_o = SlicingOptions()
    s_o.theta_YP = 30
    s_o.bVerbose = False
    itf = TomoDLLInterface("Tomo_Shell2026.dll", s_o, True, True)
    assert np.array_equal(itf.YPR, d["YPR"])
    # reference layout: np.meshgrid(yaw, pitch, [0]) raveled, yaw fastest
    assert np.array_equal(itf.YPR[:13, 0], itf.yaw_range) and np.all(itf.YPR[:13, 1] == 0)
    for k in range(2):
        tm = TriMesh(d[f"p{k}_vertices"].astype(np.float64), d[f"p{k}_faces"], d[f"p{k}_vertex_normals"], process=False)
        itf.bShellMesh = s_o.bShellMesh and not tm.is_watertight
        itf.pack(tm, itf.YPR.shape[0], False)
        assert np.array_equal(itf.Float32Info.view(np.int32), d[f"p{k}_f32info"].view(np.int32))
        assert np.array_equal(itf.Int32Info, d[f"p{k}_i32info"])
