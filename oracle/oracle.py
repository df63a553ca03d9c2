"""ctypes front-end of the two parity oracles -- TEST INFRASTRUCTURE ONLY.

``Oracle``    the plain-C restatement (oracle/tomo_oracle.c).
``RefEngine`` the reference INT3 engine compiled from its own sources
              (oracle/_ref/libtomo_ref.so, see oracle/build.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Both expose the same two calls:

* ``sweep(mesh, ypr, opts, grid, threads)`` -> dict with Mo, Mss, Vtc (the
  reference's getMo/getMss/getVtc), VoF/VssF (its float accumulators),
  Vo64/Vss64 (exact int64 totals) and optID;
* ``columns(mesh, ypr, opts, index, grid)`` -> per-column dumps of one
  orientation.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import numpy as np

from . import build as _build

_f32p = ct.POINTER(ct.c_float)
_i32p = ct.POINTER(ct.c_int32)
_i16p = ct.POINTER(ct.c_int16)
_i64p = ct.POINTER(ct.c_int64)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _inputs(mesh, ypr, opts):
    """C-ABI argument arrays; ``opts`` is PrintOptions or a ready (Float32Info, Int32Info) pair."""
    from tomo_shell2026_b200.options import pack_info
    if isinstance(opts, tuple):
        f32, i32 = (np.ascontiguousarray(opts[0], np.float32), np.ascontiguousarray(opts[1], np.int32))
    else:
        f32, i32 = pack_info(opts, mesh, ypr.shape[0])
    return (f32, i32, np.ascontiguousarray(ypr, np.float32), np.ascontiguousarray(mesh.faces, np.int32),
            np.ascontiguousarray(mesh.vertices, np.float32), np.ascontiguousarray(mesh.vertex_normals, np.float32),
            np.ascontiguousarray(mesh.face_normals, np.float32),
            np.ascontiguousarray(mesh.hull_faces, np.int32), np.ascontiguousarray(mesh.hull_vertices, np.float32),
            np.ascontiguousarray(mesh.hull_face_normals, np.float32))


class Oracle:
    """The C restatement."""

    def __init__(self, path: str | os.PathLike | None = None):
        lib_path = Path(path) if path else _build.build_oracle()
        self.lib = ct.CDLL(str(lib_path))
        L = self.lib
        L.tomo_oracle_sweep.restype = ct.c_int
        L.tomo_oracle_sweep.argtypes = [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, ct.c_int, ct.c_int,
                                        _f32p, _f32p, _f32p, _f32p, _f32p, _i64p, _i64p, _i64p, _i64p, _i64p]
        L.tomo_oracle_columns.restype = ct.c_int
        L.tomo_oracle_columns.argtypes = [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, ct.c_int, ct.c_int,
                                          _i32p, _i16p, _i32p, _i16p, _i32p, _i32p, _i32p, _f32p, _f32p]
        L.tomo_oracle_rotation.restype = None
        L.tomo_oracle_rotation.argtypes = [ct.c_float, ct.c_float, ct.c_float, _f32p]
        L.tomo_oracle_threshold.restype = ct.c_float
        L.tomo_oracle_threshold.argtypes = [ct.c_float]
        L.tomo_oracle_vol_to_mass.restype = None
        L.tomo_oracle_vol_to_mass.argtypes = [_f32p, _i32p, _f32p]

    def rotation(self, yaw, pitch, roll) -> np.ndarray:
        out = np.zeros(9, np.float32)
        self.lib.tomo_oracle_rotation(yaw, pitch, roll, _p(out, _f32p))
        return out.reshape(3, 3)

    def threshold(self, theta_c: float) -> np.float32:
        return np.float32(self.lib.tomo_oracle_threshold(theta_c))

    def vol_to_mass(self, f32, i32, vm22) -> np.ndarray:
        vm = np.ascontiguousarray(vm22, np.float32).copy()
        self.lib.tomo_oracle_vol_to_mass(_p(f32, _f32p), _p(i32, _i32p), _p(vm, _f32p))
        return vm

    def sweep(self, mesh, ypr, opts, grid: int = 256, threads: int | None = None) -> dict:
        f32, i32, ypr, tri, vtx, vn, _, _, _, _ = _inputs(mesh, ypr, opts)
        n = ypr.shape[0]
        out = {k: np.zeros(n, np.float32) for k in ("Mo", "Mss", "Vtc", "VoF", "VssF")}
        out.update({k: np.zeros(n, np.int64) for k in ("Vo64", "Vss64", "Vtc64", "entries", "columns")})
        rc = self.lib.tomo_oracle_sweep(
            _p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p), _p(vtx, _f32p), _p(vn, _f32p),
            grid, threads or os.cpu_count() or 1,
            *[_p(out[k], _f32p) for k in ("Mo", "Mss", "Vtc", "VoF", "VssF")],
            *[_p(out[k], _i64p) for k in ("Vo64", "Vss64", "Vtc64", "entries", "columns")])
        if rc < 0:
            raise RuntimeError(f"tomo_oracle_sweep failed: {rc}")
        out["optID"] = rc
        return out

    def columns(self, mesh, ypr, opts, index: int, grid: int = 256) -> dict:
        f32, i32, ypr, tri, vtx, vn, _, _, _, _ = _inputs(mesh, ypr, opts)
        ns = grid * grid
        d = dict(n_vox=np.zeros(ns, np.int32), vox_zn=np.zeros((ns, 64, 2), np.int16),
                 n_fin=np.zeros(ns, np.int32), fin_tzn=np.zeros((ns, 64, 3), np.int16),
                 col_vo=np.zeros(ns, np.int32), col_vss=np.zeros(ns, np.int32), col_vtc=np.zeros(ns, np.int32),
                 vm22=np.zeros(22, np.float32), mat16=np.zeros(16, np.float32))
        rc = self.lib.tomo_oracle_columns(
            _p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p), _p(vtx, _f32p), _p(vn, _f32p),
            index, grid, _p(d["n_vox"], _i32p), _p(d["vox_zn"], _i16p), _p(d["n_fin"], _i32p),
            _p(d["fin_tzn"], _i16p), _p(d["col_vo"], _i32p), _p(d["col_vss"], _i32p), _p(d["col_vtc"], _i32p),
            _p(d["vm22"], _f32p), _p(d["mat16"], _f32p))
        if rc < 0:
            raise RuntimeError(f"tomo_oracle_columns failed: {rc}")
        return d


class RefEngine:
    """The reference INT3 engine (compiled from the reference's own sources)."""

    def __init__(self, path: str | os.PathLike | None = None):
        lib_path = Path(path) if path else _build.build_ref()
        if lib_path is None or not Path(lib_path).exists():
            raise FileNotFoundError("reference engine library not built (oracle/_ref/libtomo_ref.so)")
        self.path = Path(lib_path)
        self.lib = ct.CDLL(str(lib_path))
        L = self.lib
        L.ref_int3_sweep.restype = ct.c_int
        L.ref_int3_sweep.argtypes = [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p,
                                     ct.c_int, ct.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, _i64p, _i64p, _i64p]
        L.ref_int3_columns.restype = ct.c_int
        L.ref_int3_columns.argtypes = [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p,
                                       ct.c_int, ct.c_int, _i32p, _i16p, _i32p, _i16p, _i32p, _i32p, _f32p, _f32p]
        L.ref_int3_pixels.restype = ct.c_int
        L.ref_int3_pixels.argtypes = [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p,
                                      ct.c_int, ct.c_int, _i32p, _i16p, ct.c_int, _f32p, _f32p]
        L.ref_int3_rotation.restype = ct.c_float
        L.ref_int3_rotation.argtypes = [ct.c_float, ct.c_float, ct.c_float, _f32p]

    def rotation(self, yaw, pitch, roll) -> np.ndarray:
        out = np.zeros(16, np.float32)
        self.lib.ref_int3_rotation(yaw, pitch, roll, _p(out, _f32p))
        return out.reshape(4, 4)[:3, :3].copy()

    def pixels(self, mesh, ypr, opts, index: int, grid: int = 256, max_pixels: int = 4_000_000) -> dict:
        """Render pixels, vm_info and mat4x4 of one orientation, as exported
        by the reference after its best-orientation re-run."""
        f32, i32, ypr, tri, vtx, vn, tn, htri, hv, hn = _inputs(mesh, ypr, opts)
        counts = np.zeros(11, np.int32)
        buf = np.zeros((max_pixels, 6), np.int16)
        vm = np.zeros(22, np.float32)
        mat = np.zeros(16, np.float32)
        total = self.lib.ref_int3_pixels(
            _p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p), _p(vtx, _f32p), _p(vn, _f32p),
            _p(tn, _f32p), _p(htri, _i32p), _p(hv, _f32p), _p(hn, _f32p), index, grid,
            _p(counts, _i32p), _p(buf, _i16p), max_pixels, _p(vm, _f32p), _p(mat, _f32p))
        if total > max_pixels:
            raise RuntimeError("pixel buffer too small")
        off = np.concatenate([[0], np.cumsum(counts)])
        return dict(pixels=[buf[off[k]:off[k + 1]].copy() for k in range(11)], vm22=vm, mat16=mat)

    def sweep(self, mesh, ypr, opts, grid: int = 256, threads: int | None = None, exact: bool = True) -> dict:
        args = _inputs(mesh, ypr, opts)
        f32, i32, ypr, tri, vtx, vn, tn, htri, hv, hn = args
        n = ypr.shape[0]
        out = {k: np.zeros(n, np.float32) for k in ("Mo", "Mss", "Vtc", "VoF", "VssF")}
        out.update({k: np.zeros(n, np.int64) for k in ("Vo64", "Vss64", "Vtc64")})
        rc = self.lib.ref_int3_sweep(
            _p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p), _p(vtx, _f32p), _p(vn, _f32p),
            _p(tn, _f32p), _p(htri, _i32p), _p(hv, _f32p), _p(hn, _f32p), grid, threads or os.cpu_count() or 1,
            *[_p(out[k], _f32p) for k in ("Mo", "Mss", "Vtc", "VoF", "VssF")],
            *([_p(out[k], _i64p) for k in ("Vo64", "Vss64", "Vtc64")] if exact else [None, None, None]))
        out["optID"] = rc
        return out

    def columns(self, mesh, ypr, opts, index: int, grid: int = 256) -> dict:
        f32, i32, ypr, tri, vtx, vn, tn, htri, hv, hn = _inputs(mesh, ypr, opts)
        ns = grid * grid
        d = dict(n_vox=np.zeros(ns, np.int32), vox_zn=np.zeros((ns, 64, 2), np.int16),
                 n_fin=np.zeros(ns, np.int32), fin_tzn=np.zeros((ns, 64, 3), np.int16),
                 col_vo=np.zeros(ns, np.int32), col_vss=np.zeros(ns, np.int32),
                 vm22=np.zeros(22, np.float32), mat16=np.zeros(16, np.float32))
        self.lib.ref_int3_columns(
            _p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p), _p(vtx, _f32p), _p(vn, _f32p),
            _p(tn, _f32p), _p(htri, _i32p), _p(hv, _f32p), _p(hn, _f32p), index, grid,
            _p(d["n_vox"], _i32p), _p(d["vox_zn"], _i16p), _p(d["n_fin"], _i32p), _p(d["fin_tzn"], _i16p),
            _p(d["col_vo"], _i32p), _p(d["col_vss"], _i32p), _p(d["vm22"], _f32p), _p(d["mat16"], _f32p))
        return d
