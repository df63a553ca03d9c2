"""Mesh files and the mesh properties the orientation search reads, without trimesh.

The reference front-end loads meshes with trimesh 4.4.0
(cfms_tomo/shell_test/tomoSh_io_trimesh.py:540, ``trimesh.load(filename,
force='mesh')``) and reads from the result: ``vertices``, ``faces``,
``vertex_normals``, ``face_normals``, ``area``, ``is_watertight``,
``convex_hull`` (``vertices``, ``faces``/``triangles``, ``face_normals``) and
``bounding_box_oriented.extents`` (cfms_tomo/tomo_dll_interface.py:56-70,
tomo_result.py:31).  trimesh is not a dependency here; :class:`TriMesh`
restates those properties from their published definitions:

* loading merges vertices whose positions agree to 8 decimals (and whose
  file normals agree, when the file has normals), as trimesh's default
  ``process=True`` does; polygons are split into triangle fans;
* face normals are the normalised ``(b - a) x (c - a)``; vertex normals are
  the file's when it has them, else the sum of adjacent face normals
  weighted by the face's interior angle at the vertex, normalised;
* ``is_watertight``: every undirected edge is shared by exactly two faces;
* the convex hull is scipy's Qhull hull of the vertices, outward normals;
* the oriented box is aligned to the principal axes of the hull vertices
  (trimesh fits a minimum-volume box; the extents only feed a reported
  beam length, never the search).

These are inputs to the search, so the GPU library and the oracles always
receive identical bytes; their agreement with trimesh itself is not pinned
(trimesh is absent).

Formats: PLY (ascii, binary little/big endian), STL (ascii, binary), OBJ,
glTF 2.0 (.gltf with external or data-URI buffers, and .glb); glTF scenes
are flattened with every mesh node's world transform (skins ignored).
"""
from __future__ import annotations

import base64
import json
import os
import struct
from dataclasses import dataclass

import numpy as np

__all__ = ["TriMesh", "load", "OrientedBox"]


@dataclass
class OrientedBox:
    extents: np.ndarray
    transform: np.ndarray


class TriMesh:
    """Triangle mesh with the trimesh-style properties the search reads."""

    def __init__(self, vertices, faces, vertex_normals=None, process: bool = True, name: str = "mesh"):
        v = np.asarray(vertices, dtype=np.float64).reshape(-1, 3)
        f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
        vn = None if vertex_normals is None else np.asarray(vertex_normals, dtype=np.float64).reshape(-1, 3)
        if f.size and (f.min() < 0 or f.max() >= len(v)):
            raise ValueError("face index out of range")
        if process and len(v):
            v, f, vn = _merge_vertices(v, f, vn)
        self.vertices = v
        self.faces = f
        self._vn = vn
        self.name = name
        self._cache: dict = {}

    # -- geometry ---------------------------------------------------------
    @property
    def triangles(self) -> np.ndarray:
        return self.vertices[self.faces]

    def _cross(self):
        if "cross" not in self._cache:
            t = self.triangles
            self._cache["cross"] = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
        return self._cache["cross"]

    @property
    def face_normals(self) -> np.ndarray:
        c = self._cross()
        n = np.linalg.norm(c, axis=1)
        out = np.zeros_like(c)
        ok = n > 0
        out[ok] = c[ok] / n[ok, None]
        return out

    @property
    def area_faces(self) -> np.ndarray:
        return 0.5 * np.linalg.norm(self._cross(), axis=1)

    @property
    def area(self) -> float:
        return float(self.area_faces.sum())

    @property
    def vertex_normals(self) -> np.ndarray:
        if self._vn is not None:
            return self._vn
        if "vn" not in self._cache:
            t = self.triangles
            fn = self.face_normals
            acc = np.zeros_like(self.vertices)
            for k in range(3):
                e1 = t[:, (k + 1) % 3] - t[:, k]
                e2 = t[:, (k + 2) % 3] - t[:, k]
                cosang = np.einsum("ij,ij->i", e1, e2) / np.maximum(
                    np.linalg.norm(e1, axis=1) * np.linalg.norm(e2, axis=1), 1e-300)
                ang = np.arccos(np.clip(cosang, -1.0, 1.0))
                np.add.at(acc, self.faces[:, k], fn * ang[:, None])
            n = np.linalg.norm(acc, axis=1)
            ok = n > 0
            acc[ok] /= n[ok, None]
            self._cache["vn"] = acc
        return self._cache["vn"]

    @property
    def edges_sorted(self) -> np.ndarray:
        f = self.faces
        return np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)

    @property
    def is_watertight(self) -> bool:
        if len(self.faces) == 0:
            return False
        _, counts = np.unique(self.edges_sorted, axis=0, return_counts=True)
        return bool(np.all(counts == 2))

    @property
    def bounds(self) -> np.ndarray:
        return np.stack([self.vertices.min(0), self.vertices.max(0)])

    @property
    def extents(self) -> np.ndarray:
        b = self.bounds
        return b[1] - b[0]

    @property
    def convex_hull(self) -> "TriMesh":
        if "hull" not in self._cache:
            from scipy.spatial import ConvexHull
            h = ConvexHull(self.vertices)
            used = np.unique(h.simplices)
            remap = -np.ones(len(self.vertices), np.int64)
            remap[used] = np.arange(used.size)
            f = remap[h.simplices]
            hv = self.vertices[used]
            # orient every hull face outward (Qhull's simplices are unordered)
            t = hv[f]
            c = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
            flip = np.einsum("ij,ij->i", c, h.equations[:, :3]) < 0
            f[flip] = f[flip][:, ::-1]
            self._cache["hull"] = TriMesh(hv, f, process=False, name=self.name + "_hull")
        return self._cache["hull"]

    @property
    def bounding_box_oriented(self) -> OrientedBox:
        p = self.convex_hull.vertices if len(self.vertices) >= 4 else self.vertices
        c = p.mean(0)
        _, _, vt = np.linalg.svd(p - c, full_matrices=False)
        local = (p - c) @ vt.T
        lo, hi = local.min(0), local.max(0)
        m = np.eye(4)
        m[:3, :3] = vt.T
        m[:3, 3] = c + vt.T @ ((lo + hi) * 0.5)
        return OrientedBox(hi - lo, m)

    # -- editing ----------------------------------------------------------
    def copy(self) -> "TriMesh":
        return TriMesh(self.vertices.copy(), self.faces.copy(),
                       None if self._vn is None else self._vn.copy(), process=False, name=self.name)

    def apply_transform(self, m4) -> "TriMesh":
        m = np.asarray(m4, dtype=np.float64).reshape(4, 4)
        self.vertices = self.vertices @ m[:3, :3].T + m[:3, 3]
        if self._vn is not None:
            n = self._vn @ np.linalg.inv(m[:3, :3])
            self._vn = n / np.maximum(np.linalg.norm(n, axis=1), 1e-300)[:, None]
        self._cache.clear()
        return self

    def to_arrays(self, with_hull: bool = True):
        """The reference C-ABI arrays (float32 / int32) as a MeshArrays."""
        from ..meshgen import MeshArrays
        e3 = lambda dt: np.zeros((0, 3), dt)  # noqa: E731
        if with_hull and len(self.vertices) >= 4:
            h = self.convex_hull
            hv, hf, hn = h.vertices.astype(np.float32), h.faces.astype(np.int32), h.face_normals.astype(np.float32)
        else:
            hv, hf, hn = e3(np.float32), e3(np.int32), e3(np.float32)
        return MeshArrays(np.ascontiguousarray(self.vertices, np.float32), np.ascontiguousarray(self.faces, np.int32),
                          np.ascontiguousarray(self.vertex_normals, np.float32),
                          np.ascontiguousarray(self.face_normals, np.float32), self.area, hv, hf, hn,
                          self.is_watertight, self.name)


def _merge_vertices(v, f, vn):
    key = np.round(v, 8)
    if vn is not None:
        key = np.concatenate([key, np.round(vn, 8)], axis=1)
    _, first, inverse = np.unique(key, axis=0, return_index=True, return_inverse=True)
    inverse = inverse.reshape(-1)
    # keep the first occurrence order (trimesh keeps file order of first use)
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    new_index = rank[inverse]
    keep = first[order]
    return v[keep], new_index[f], (None if vn is None else vn[keep])


# ------------------------------------------------------------------ loaders

def load(filename, force: str = "mesh", process: bool = True) -> TriMesh:
    """Load a PLY / STL / OBJ / glTF / GLB file as one :class:`TriMesh`."""
    if force != "mesh":
        raise ValueError("only force='mesh' is supported")
    path = os.fspath(filename)
    ext = os.path.splitext(path)[1].lower()
    name = os.path.splitext(os.path.basename(path))[0]
    if ext == ".ply":
        v, f, vn = _load_ply(path)
    elif ext == ".stl":
        v, f, vn = _load_stl(path)
    elif ext == ".obj":
        v, f, vn = _load_obj(path)
    elif ext in (".gltf", ".glb"):
        v, f, vn = _load_gltf(path)
    else:
        raise ValueError(f"unsupported mesh format: {ext}")
    return TriMesh(v, f, vn, process=process, name=name)


def _fan(polys):
    tris = []
    for p in polys:
        for k in range(1, len(p) - 1):
            tris.append((p[0], p[k], p[k + 1]))
    return np.asarray(tris, dtype=np.int64).reshape(-1, 3)


_PLY_TYPES = {"char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2",
              "ushort": "u2", "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
              "float": "f4", "float32": "f4", "double": "f8", "float64": "f8"}


def _load_ply(path):
    with open(path, "rb") as fh:
        data = fh.read()
    end = data.find(b"end_header")
    if not data.startswith(b"ply") or end < 0:
        raise ValueError("not a PLY file")
    body = data[data.index(b"\n", end) + 1:]
    fmt = None
    elements = []   # (name, count, [(prop, type) | (prop, ('list', count_type, item_type))])
    for line in data[:end].decode("ascii", "replace").splitlines():
        w = line.split()
        if not w:
            continue
        if w[0] == "format":
            fmt = w[1]
        elif w[0] == "element":
            elements.append((w[1], int(w[2]), []))
        elif w[0] == "property" and elements:
            if w[1] == "list":
                elements[-1][2].append((w[4], ("list", _PLY_TYPES[w[2]], _PLY_TYPES[w[3]])))
            else:
                elements[-1][2].append((w[2], _PLY_TYPES[w[1]]))
    verts = faces = None
    if fmt == "ascii":
        tokens = body.split()
        pos = 0
        for name, count, props in elements:
            rows = []
            for _ in range(count):
                row = {}
                for pname, ptype in props:
                    if isinstance(ptype, tuple):
                        n = int(tokens[pos]); pos += 1
                        row[pname] = [int(t) for t in tokens[pos:pos + n]]; pos += n
                    else:
                        row[pname] = float(tokens[pos]); pos += 1
                rows.append(row)
            if name == "vertex":
                verts = rows
            elif name == "face":
                faces = rows
    elif fmt in ("binary_little_endian", "binary_big_endian"):
        bo = "<" if fmt == "binary_little_endian" else ">"
        pos = 0
        for name, count, props in elements:
            if all(not isinstance(t, tuple) for _, t in props):
                dt = np.dtype([(p, bo + t) for p, t in props])
                arr = np.frombuffer(body, dtype=dt, count=count, offset=pos)
                pos += dt.itemsize * count
                if name == "vertex":
                    verts = arr
            else:
                rows = []
                for _ in range(count):
                    row = {}
                    for pname, ptype in props:
                        if isinstance(ptype, tuple):
                            ct_, it_ = np.dtype(bo + ptype[1]), np.dtype(bo + ptype[2])
                            n = int(np.frombuffer(body, ct_, 1, pos)[0]); pos += ct_.itemsize
                            row[pname] = np.frombuffer(body, it_, n, pos).astype(np.int64); pos += it_.itemsize * n
                        else:
                            t = np.dtype(bo + ptype)
                            row[pname] = np.frombuffer(body, t, 1, pos)[0]; pos += t.itemsize
                    rows.append(row)
                if name == "face":
                    faces = rows
    else:
        raise ValueError(f"unsupported PLY format {fmt}")
    if verts is None:
        raise ValueError("PLY has no vertex element")
    get = (lambda k: np.asarray([r[k] for r in verts], np.float64)) if isinstance(verts, list) else \
        (lambda k: np.asarray(verts[k], np.float64))
    v = np.stack([get("x"), get("y"), get("z")], 1)
    names = [p for p, _ in next(e for e in elements if e[0] == "vertex")[2]]
    vn = np.stack([get("nx"), get("ny"), get("nz")], 1) if {"nx", "ny", "nz"} <= set(names) else None
    key = None
    if faces:
        key = "vertex_indices" if "vertex_indices" in faces[0] else ("vertex_index" if "vertex_index" in faces[0] else None)
    f = _fan([list(r[key]) for r in faces]) if key else np.zeros((0, 3), np.int64)
    return v, f, vn


def _load_stl(path):
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) >= 84:
        n = struct.unpack("<I", data[80:84])[0]
        if 84 + 50 * n == len(data):
            dt = np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("attr", "<u2")])
            rec = np.frombuffer(data, dtype=dt, count=n, offset=84)
            v = rec["v"].reshape(-1, 3).astype(np.float64)
            return v, np.arange(3 * n, dtype=np.int64).reshape(-1, 3), None
    pts = [list(map(float, line.split()[1:4])) for line in data.decode("ascii", "replace").splitlines()
           if line.strip().startswith("vertex")]
    v = np.asarray(pts, np.float64).reshape(-1, 3)
    return v, np.arange(len(v), dtype=np.int64).reshape(-1, 3), None


def _load_obj(path):
    v, polys = [], []
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            w = line.split()
            if not w:
                continue
            if w[0] == "v":
                v.append([float(x) for x in w[1:4]])
            elif w[0] == "f":
                idx = []
                for t in w[1:]:
                    i = int(t.split("/")[0])
                    idx.append(i - 1 if i > 0 else len(v) + i)
                polys.append(idx)
    return np.asarray(v, np.float64).reshape(-1, 3), _fan(polys), None


_GL_TYPES = {5120: "i1", 5121: "u1", 5122: "i2", 5123: "u2", 5125: "u4", 5126: "f4"}
_GL_COUNT = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


def _quat_matrix(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _node_matrix(node):
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).T   # column-major in the file
    m = np.eye(4)
    s = np.asarray(node.get("scale", [1, 1, 1]), np.float64)
    r = _quat_matrix(node.get("rotation", [0, 0, 0, 1]))
    m[:3, :3] = r * s[None, :]
    m[:3, 3] = node.get("translation", [0, 0, 0])
    return m


def _load_gltf(path):
    with open(path, "rb") as fh:
        raw = fh.read()
    bin_chunk = None
    if raw[:4] == b"glTF":
        pos, doc = 12, None
        while pos + 8 <= len(raw):
            length, kind = struct.unpack("<II", raw[pos:pos + 8])
            chunk = raw[pos + 8:pos + 8 + length]
            if kind == 0x4E4F534A:
                doc = json.loads(chunk.decode("utf-8"))
            elif kind == 0x004E4942:
                bin_chunk = chunk
            pos += 8 + length
    else:
        doc = json.loads(raw.decode("utf-8"))
    base = os.path.dirname(os.path.abspath(path))
    buffers = []
    for b in doc.get("buffers", []):
        uri = b.get("uri")
        if uri is None:
            buffers.append(bin_chunk)
        elif uri.startswith("data:"):
            buffers.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            with open(os.path.join(base, uri), "rb") as fh:
                buffers.append(fh.read())

    def accessor(i):
        a = doc["accessors"][i]
        bv = doc["bufferViews"][a["bufferView"]]
        comp = np.dtype("<" + _GL_TYPES[a["componentType"]])
        n = _GL_COUNT[a["type"]]
        off = bv.get("byteOffset", 0) + a.get("byteOffset", 0)
        stride = bv.get("byteStride", comp.itemsize * n)
        buf = buffers[bv["buffer"]]
        if stride == comp.itemsize * n:
            out = np.frombuffer(buf, comp, a["count"] * n, off).reshape(a["count"], n)
        else:
            rows = [np.frombuffer(buf, comp, n, off + k * stride) for k in range(a["count"])]
            out = np.stack(rows) if rows else np.zeros((0, n), comp)
        return out

    vs, fs, base_n = [], [], 0
    scene = doc.get("scenes", [{}])[doc.get("scene", 0)] if doc.get("scenes") else {"nodes": list(range(len(doc.get("nodes", []))))}

    def visit(i, parent):
        node = doc["nodes"][i]
        m = parent @ _node_matrix(node)
        nonlocal base_n
        if "mesh" in node:
            for prim in doc["meshes"][node["mesh"]]["primitives"]:
                if prim.get("mode", 4) != 4:
                    continue
                p = accessor(prim["attributes"]["POSITION"]).astype(np.float64)
                idx = accessor(prim["indices"]).reshape(-1).astype(np.int64) if "indices" in prim \
                    else np.arange(len(p), dtype=np.int64)
                vs.append(p @ m[:3, :3].T + m[:3, 3])
                fs.append(idx.reshape(-1, 3) + base_n)
                base_n += len(p)
        for c in node.get("children", []):
            visit(c, m)

    for r in scene.get("nodes", []):
        visit(r, np.eye(4))
    if not vs:
        raise ValueError("glTF file has no triangle primitives")
    return np.concatenate(vs), np.concatenate(fs), None
