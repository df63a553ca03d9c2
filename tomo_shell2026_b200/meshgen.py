"""Seeded synthetic meshes and orientation grids for the orientation search.

The workloads the orientation search is measured on are described by shape
only (no mesh files ship with them), so they are generated here with numpy:

* ``perturbed_icosphere`` -- a closed icosphere whose vertices are displaced
  radially by a sum of seeded real spherical harmonics, optionally plus
  Gaussian bumps and dents (the small "plain method" mesh: subdivision 4,
  5,120 triangles, r = 50 mm, 6 harmonics of degree <= 3, amplitude 0.15;
  the 82k-triangle solid: subdivision 6, 81,920 triangles, r = 80 mm,
  harmonics of degree <= 8 at amplitude 0.25 and 4 bumps/dents with
  sigma 10 mm and height +-20 mm).
* ``ypr_grid`` -- the (yaw, pitch, roll) array in the layout the reference
  Python surface builds with ``np.meshgrid(yaw, pitch, [0])`` + ravel
  (cfms_tomo/tomo_dll_interface.py:38-43): pitch-major, yaw fastest,
  float32 radians.

A mesh is returned as :class:`MeshArrays`, the same float32/int32 arrays the
reference hands to its C-ABI (tomo_dll_interface.py:59-70): vertices, vertex
normals, faces, face normals, surface area and convex hull.  Vertex normals
are area-weighted face-normal sums; they are inputs to the search, so the
GPU path and the oracle always receive identical bytes.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = ["MeshArrays", "icosphere", "geodesic_sphere", "perturbed_icosphere", "uv_sphere", "perturbed_sphere",
           "ypr_grid",
           "small_solid", "solid_82k", "random_mesh", "mesh_from_arrays"]


@dataclass
class MeshArrays:
    """Mesh arrays in the dtypes of the reference C-ABI."""

    vertices: np.ndarray          # [V, 3] float32
    faces: np.ndarray             # [T, 3] int32
    vertex_normals: np.ndarray    # [V, 3] float32
    face_normals: np.ndarray      # [T, 3] float32
    area: float                   # total surface area (float64, cast to float32 at the ABI)
    hull_vertices: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    hull_faces: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    hull_face_normals: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    is_watertight: bool = True
    name: str = "mesh"

    @property
    def n_tri(self) -> int:
        return int(self.faces.shape[0])

    @property
    def n_vtx(self) -> int:
        return int(self.vertices.shape[0])


def _normals(v: np.ndarray, f: np.ndarray) -> tuple[np.ndarray, np.ndarray, float]:
    v64 = v.astype(np.float64)
    a, b, c = v64[f[:, 0]], v64[f[:, 1]], v64[f[:, 2]]
    cr = np.cross(b - a, c - a)
    dbl_area = np.linalg.norm(cr, axis=1)
    fn = cr / np.maximum(dbl_area, 1e-300)[:, None]
    vn = np.zeros_like(v64)
    for k in range(3):
        np.add.at(vn, f[:, k], cr)          # area-weighted
    vn /= np.maximum(np.linalg.norm(vn, axis=1), 1e-300)[:, None]
    return vn.astype(np.float32), fn.astype(np.float32), float(dbl_area.sum() * 0.5)


def _hull(v: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    try:
        from scipy.spatial import ConvexHull
    except Exception:  # pragma: no cover - scipy is in the image
        return (np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32), np.zeros((0, 3), np.float32))
    h = ConvexHull(v.astype(np.float64))
    used = np.unique(h.simplices)
    remap = -np.ones(v.shape[0], np.int64)
    remap[used] = np.arange(used.size)
    hv = v[used].astype(np.float32)
    hf = remap[h.simplices].astype(np.int32)
    hn = h.equations[:, :3].astype(np.float32)
    return hv, hf, hn


def mesh_from_arrays(vertices, faces, name: str = "mesh", with_hull: bool = True,
                     vertex_normals=None, watertight: bool | None = None) -> MeshArrays:
    """Build :class:`MeshArrays` from raw vertices/faces."""
    v = np.ascontiguousarray(vertices, dtype=np.float32)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    vn, fn, area = _normals(v, f)
    if vertex_normals is not None:
        vn = np.ascontiguousarray(vertex_normals, dtype=np.float32)
    hv, hf, hn = _hull(v) if (with_hull and v.shape[0] >= 4) else (
        np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32), np.zeros((0, 3), np.float32))
    if watertight is None:
        watertight = _is_watertight(f)
    return MeshArrays(v, f, vn, fn, area, hv, hf, hn, watertight, name)


def _is_watertight(f: np.ndarray) -> bool:
    e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return bool(np.all(counts == 2))


def icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**subdivisions faces (float64 vertices)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
         (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, np.float64)
    verts /= np.linalg.norm(verts, axis=1)[:, None]
    faces = np.array(f, np.int64)
    for _ in range(subdivisions):
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        es = np.sort(e, axis=1)
        uniq, inv = np.unique(es, axis=0, return_inverse=True)
        mids = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1)[:, None]
        base = verts.shape[0]
        verts = np.vstack([verts, mids])
        inv = inv.reshape(3, -1).T + base          # [T, 3]: mid of (0,1), (1,2), (2,0)
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        ab, bc, ca = inv[:, 0], inv[:, 1], inv[:, 2]
        faces = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                                np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return verts, faces


def _real_sh(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    from scipy.special import sph_harm_y
    if m == 0:
        return np.real(sph_harm_y(l, 0, theta, phi))
    y = sph_harm_y(l, abs(m), theta, phi)
    s = np.sqrt(2.0) * (-1.0) ** m
    return s * (np.real(y) if m > 0 else np.imag(y))


def perturbed_icosphere(subdivisions: int, radius: float, seed: int, n_harmonics: int = 6,
                        max_degree: int = 3, amplitude: float = 0.15, n_bumps: int = 0,
                        bump_sigma: float = 10.0, bump_height: float = 20.0, scale: float = 1.0,
                        name: str | None = None, with_hull: bool = True) -> MeshArrays:
    """Closed icosphere, radially displaced by seeded real spherical harmonics
    (and optionally Gaussian bumps/dents), coordinates multiplied by ``scale``
    (2.0 expresses 0.5 mm voxels on the reference's 1-unit grid)."""
    u, f = icosphere(subdivisions)
    return _perturbed(u, f, radius, seed, n_harmonics, max_degree, amplitude, n_bumps, bump_sigma, bump_height,
                      scale, name or f"ico{subdivisions}_s{seed}", with_hull)


def geodesic_sphere(frequency: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit geodesic sphere: every icosahedron face cut into frequency^2
    triangles (20 * frequency^2 faces, outward winding, vertex valence 5 or 6),
    points placed on each flat face and projected onto the sphere."""
    nu = max(1, int(frequency))
    base_v, base_f = icosphere(0)
    ii, jj = np.meshgrid(np.arange(nu + 1), np.arange(nu + 1), indexing="ij")
    keep = (ii + jj) <= nu
    ii, jj = ii[keep], jj[keep]
    local = -np.ones((nu + 1, nu + 1), np.int64)
    local[ii, jj] = np.arange(ii.size)
    pts = []
    for a, b, c in base_f:
        A, B, C = base_v[a], base_v[b], base_v[c]
        P = A[None, :] + np.outer(ii / nu, B - A) + np.outer(jj / nu, C - A)
        pts.append(P / np.linalg.norm(P, axis=1)[:, None])
    pts = np.concatenate(pts)
    _, first, inv = np.unique(np.round(pts, 9), axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    gid = rank[inv]
    verts = pts[first[order]]
    tris = []
    ti, tj = np.meshgrid(np.arange(nu), np.arange(nu), indexing="ij")
    up = (ti + tj) <= nu - 1
    dn = (ti + tj) <= nu - 2
    for k in range(len(base_f)):
        off = k * ii.size
        g = lambda i, j: gid[off + local[i, j]]  # noqa: E731
        i1, j1 = ti[up], tj[up]
        tris.append(np.stack([g(i1, j1), g(i1 + 1, j1), g(i1, j1 + 1)], 1))
        i2, j2 = ti[dn], tj[dn]
        tris.append(np.stack([g(i2 + 1, j2), g(i2 + 1, j2 + 1), g(i2, j2 + 1)], 1))
    return verts, np.concatenate(tris).astype(np.int64)


def uv_sphere(n_tri: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit latitude/longitude sphere with about n_tri triangles (outward winding):
    n_lon segments and n_lat rings give 2 * n_lon * (n_lat - 1) triangles."""
    n_lon = max(8, int(round(np.sqrt(max(n_tri, 32)))))
    n_lat = max(3, int(round(n_tri / (2.0 * n_lon))) + 1)
    th = np.pi * np.arange(1, n_lat) / n_lat
    ph = 2.0 * np.pi * np.arange(n_lon) / n_lon
    ring = np.stack([np.outer(np.sin(th), np.cos(ph)), np.outer(np.sin(th), np.sin(ph)),
                     np.outer(np.cos(th), np.ones(n_lon))], -1).reshape(-1, 3)
    verts = np.vstack([[0.0, 0.0, 1.0], [0.0, 0.0, -1.0], ring])
    vid = lambda k, j: 2 + (k - 1) * n_lon + (j % n_lon)  # noqa: E731
    faces = []
    for j in range(n_lon):
        faces.append((0, vid(1, j), vid(1, j + 1)))
        faces.append((1, vid(n_lat - 1, j + 1), vid(n_lat - 1, j)))
        for k in range(1, n_lat - 1):
            a, b, c, d = vid(k, j), vid(k, j + 1), vid(k + 1, j), vid(k + 1, j + 1)
            faces.append((a, c, d))
            faces.append((a, d, b))
    return verts, np.asarray(faces, np.int64)


def perturbed_sphere(n_tri: int, radius: float, seed: int, **kw) -> MeshArrays:
    """A geodesic sphere of about n_tri triangles (20 * round(sqrt(n_tri / 20))^2)
    with the same seeded radial displacement as :func:`perturbed_icosphere`
    (keyword arguments as there)."""
    u, f = geodesic_sphere(max(1, int(round(np.sqrt(n_tri / 20.0)))))
    name = kw.pop("name", None) or f"geo{f.shape[0]}_s{seed}"
    with_hull = kw.pop("with_hull", True)
    args = dict(n_harmonics=6, max_degree=3, amplitude=0.15, n_bumps=0, bump_sigma=10.0, bump_height=20.0, scale=1.0)
    args.update(kw)
    return _perturbed(u, f, radius, seed, args["n_harmonics"], args["max_degree"], args["amplitude"], args["n_bumps"],
                      args["bump_sigma"], args["bump_height"], args["scale"], name, with_hull)


def _perturbed(u, f, radius, seed, n_harmonics, max_degree, amplitude, n_bumps, bump_sigma, bump_height, scale,
               name, with_hull) -> MeshArrays:
    rng = np.random.default_rng(seed)
    theta = np.arccos(np.clip(u[:, 2], -1.0, 1.0))
    phi = np.arctan2(u[:, 1], u[:, 0])
    s = np.zeros(u.shape[0])
    for _ in range(n_harmonics):
        l = int(rng.integers(1, max_degree + 1))
        m = int(rng.integers(-l, l + 1))
        s += rng.uniform(-1.0, 1.0) * _real_sh(l, m, theta, phi)
    r = radius * (1.0 + amplitude * s)
    for _ in range(n_bumps):
        c = rng.normal(size=3)
        c /= np.linalg.norm(c)
        h = bump_height * (1.0 if rng.random() < 0.5 else -1.0)
        d2 = np.sum((u * radius - c * radius) ** 2, axis=1)
        r = r + h * np.exp(-d2 / (2.0 * bump_sigma ** 2))
    r = np.maximum(r, 0.05 * radius)
    v = (u * r[:, None]) * scale
    return mesh_from_arrays(v, f, name, with_hull=with_hull, watertight=True)


def small_solid(seed: int = 0, with_hull: bool = True) -> MeshArrays:
    """Plain-method mesh: subdivision 4 (5,120 triangles), r = 50 mm, 1 mm voxels."""
    return perturbed_icosphere(4, 50.0, seed, n_harmonics=6, max_degree=3, amplitude=0.15,
                               name=f"solid5k_s{seed}", with_hull=with_hull)


def solid_82k(seed: int = 0, with_hull: bool = True) -> MeshArrays:
    """82k-triangle solid: subdivision 6 (81,920 triangles), r = 80 mm, SH degree <= 8 at
    amplitude 0.25 plus 4 Gaussian bumps/dents (sigma 10 mm, +-20 mm), 0.5 mm voxels
    (coordinates x2)."""
    return perturbed_icosphere(6, 80.0, seed, n_harmonics=12, max_degree=8, amplitude=0.25,
                               n_bumps=4, bump_sigma=10.0, bump_height=20.0, scale=2.0,
                               name=f"solid82k_s{seed}", with_hull=with_hull)


def random_mesh(n_tri: int, seed: int, extent: float = 60.0, open_fraction: float = 0.0) -> MeshArrays:
    """Triangle soup for edge-case tests: random small and sliver triangles
    (not watertight)."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0.2 * extent, 0.8 * extent, size=(n_tri, 3))
    sizes = rng.lognormal(mean=0.0, sigma=1.0, size=(n_tri, 1))
    offs = rng.normal(size=(n_tri, 3, 3)) * sizes[:, :, None]
    sliver = rng.random(n_tri) < 0.15
    offs[sliver, 2, :] = offs[sliver, 1, :] * rng.uniform(-1.2, 1.2, size=(int(sliver.sum()), 1))
    v = (centers[:, None, :] + offs).reshape(-1, 3)
    f = np.arange(3 * n_tri, dtype=np.int32).reshape(-1, 3)
    return mesh_from_arrays(v, f, f"soup{n_tri}_s{seed}", with_hull=True, watertight=False)


def ypr_grid(yaw_deg, pitch_deg, roll_deg=(0.0,)) -> np.ndarray:
    """[n, 3] float32 radians, pitch-major / yaw-fastest like the reference's
    np.meshgrid(yaw, pitch, roll) + ravel (tomo_dll_interface.py:38-43)."""
    yaw = np.asarray(yaw_deg, np.float64) * np.pi / 180.0
    pitch = np.asarray(pitch_deg, np.float64) * np.pi / 180.0
    roll = np.asarray(roll_deg, np.float64) * np.pi / 180.0
    xx, yy, zz = np.meshgrid(yaw.astype(np.float32), pitch.astype(np.float32), roll.astype(np.float32))
    return np.ascontiguousarray(np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()]).astype(np.float32))


# ------------------------------------------------------------------ thin open shell

def _surface_nets(f: np.ndarray, origin: np.ndarray, h: float) -> tuple[np.ndarray, np.ndarray]:
    """Triangulate the zero level set of a sampled signed distance f[nx, ny, nz]
    (negative inside) by surface nets: one vertex per sign-changing cube at
    the mean of its edge crossings, one quad (two triangles) per
    sign-changing grid edge, wound so normals point to the positive side."""
    nx, ny, nz = f.shape
    inside = f < 0
    # cube index of every sign-changing cube
    corners = [inside[a:nx - 1 + a, b:ny - 1 + b, c:nz - 1 + c] for a in (0, 1) for b in (0, 1) for c in (0, 1)]
    anyin = np.logical_or.reduce(corners)
    allin = np.logical_and.reduce(corners)
    active = anyin & ~allin
    cid = -np.ones(active.shape, np.int64)
    cid[active] = np.arange(int(active.sum()))
    # vertex positions: mean of crossings on the cube's 12 edges
    acc = np.zeros(active.shape + (3,))
    cnt = np.zeros(active.shape)
    offs = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    edges = [(0, 1), (0, 2), (0, 3), (1, 4), (1, 5), (2, 4), (2, 6), (3, 5), (3, 6), (4, 7), (5, 7), (6, 7)]
    sl = lambda o: (slice(o[0], nx - 1 + o[0]), slice(o[1], ny - 1 + o[1]), slice(o[2], nz - 1 + o[2]))  # noqa: E731
    for a, b in edges:
        fa, fb = f[sl(offs[a])], f[sl(offs[b])]
        cross = (fa < 0) != (fb < 0)
        t = np.where(cross, fa / np.where(cross, fa - fb, 1.0), 0.0)
        pa, pb = np.array(offs[a], float), np.array(offs[b], float)
        pos = pa[None, None, None, :] + t[..., None] * (pb - pa)[None, None, None, :]
        acc += np.where(cross[..., None], pos, 0.0)
        cnt += cross
    ii, jj, kk = np.nonzero(active)
    local = acc[active] / cnt[active][:, None]
    verts = origin[None, :] + (np.stack([ii, jj, kk], 1) + local) * h
    faces = []
    # an x-edge (i, j, k)-(i+1, j, k) is shared by cubes (i, j-1..j, k-1..k)
    for axis in range(3):
        a0 = [slice(0, n - 1) if d == axis else slice(1, n - 1) for d, n in enumerate(f.shape)]
        a1 = [slice(1, n) if d == axis else slice(1, n - 1) for d, n in enumerate(f.shape)]
        s0, s1 = inside[tuple(a0)], inside[tuple(a1)]
        change = s0 != s1
        e = np.nonzero(change)
        base = [e[d] + (0 if d == axis else 1) for d in range(3)]
        u, v = [d for d in range(3) if d != axis]

        def cube(du, dv):
            idx = list(base)
            idx[u] = idx[u] - du
            idx[v] = idx[v] - dv
            return cid[idx[0], idx[1], idx[2]]

        c00, c10, c11, c01 = cube(1, 1), cube(0, 1), cube(0, 0), cube(1, 0)
        # (c00, c10, c11, c01) turns counter-clockwise in the (u, v) plane: its
        # normal is +axis when (u, v, axis) is right-handed (axes x and z), -axis
        # for y; the normal must point to the outside (positive) end of the edge
        plus = s0[e]   # inside at the low end: outside along +axis
        flip = ~plus if axis != 1 else plus
        q = np.stack([c00, c10, c11, c01], 1)
        q[flip] = q[flip][:, ::-1]
        ok = (q >= 0).all(1)
        q = q[ok]
        faces.append(np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]]))
    return verts, np.concatenate(faces)


def manikin_shell(seed: int = 0, spacing: float = 6.5, offset: float = 2.0, with_hull: bool = False) -> MeshArrays:
    """Thin open shell, manikin-like: the union surface of 9 seeded
    ellipsoids and capsules (torso ~300 x 200 x 600 mm, hips, chest, neck,
    head, upper and lower arms) triangulated by surface nets at `spacing` mm,
    the bottom and both arm ends cut open, plus an inward copy offset by
    `offset` mm along the vertex normals with reversed winding (the wall).
    spacing 6.5 mm gives ~87k triangles for both sheets together."""
    rng = np.random.default_rng(seed)
    j = lambda s: 1.0 + rng.uniform(-s, s)  # noqa: E731
    ell = [((0, 0, 330), (150 * j(.05), 100 * j(.05), 230 * j(.05))),      # torso
           ((0, 0, 150), (160 * j(.05), 110 * j(.05), 120 * j(.05))),      # hips
           ((0, 15, 430), (140 * j(.05), 95 * j(.05), 90 * j(.05))),       # chest
           ((0, 0, 690), (70 * j(.05), 80 * j(.05), 100 * j(.05)))]        # head
    cap = [((0, 0, 540), (0, 0, 610), 45 * j(.05)),                         # neck
           ((-150, 0, 510), (-250, 0, 330), 45 * j(.05)), ((150, 0, 510), (250, 0, 330), 45 * j(.05)),
           ((-250, 0, 330), (-290, 30, 160), 38 * j(.05)), ((250, 0, 330), (290, 30, 160), 38 * j(.05))]
    lo = np.array([-360.0, -160.0, 0.0])
    hi = np.array([360.0, 160.0, 820.0])
    n = np.ceil((hi - lo) / spacing).astype(int) + 1
    X, Y, Z = np.meshgrid(*[lo[d] + spacing * np.arange(n[d]) for d in range(3)], indexing="ij")
    P = np.stack([X, Y, Z], -1)
    f = np.full(X.shape, np.inf)
    for c, r in ell:
        q = (P - np.array(c)) / np.array(r)
        f = np.minimum(f, (np.linalg.norm(q, axis=-1) - 1.0) * min(r))
    for a, b, r in cap:
        a, b = np.array(a, float), np.array(b, float)
        ab = b - a
        t = np.clip(((P - a) @ ab) / (ab @ ab), 0.0, 1.0)
        f = np.minimum(f, np.linalg.norm(P - (a + t[..., None] * ab), axis=-1) - r)
    v, tri = _surface_nets(f, lo, spacing)
    cen = v[tri].mean(1)
    keep = cen[:, 2] > 70.0                                               # bottom opening
    for a, b, _ in cap[3:]:
        a, b = np.array(a, float), np.array(b, float)
        axis = (b - a) / np.linalg.norm(b - a)
        keep &= ((cen - b) @ axis) < -10.0                                # arm openings at the hands
    tri = tri[keep]
    used = np.unique(tri)
    remap = -np.ones(v.shape[0], np.int64)
    remap[used] = np.arange(used.size)
    v, tri = v[used], remap[tri]
    vn, _, _ = _normals(v.astype(np.float32), tri.astype(np.int32))
    inner = v - offset * vn.astype(np.float64)
    V = np.vstack([v, inner])
    F = np.vstack([tri, tri[:, ::-1] + v.shape[0]])
    return mesh_from_arrays(V, F, f"manikin_s{seed}", with_hull=with_hull)
