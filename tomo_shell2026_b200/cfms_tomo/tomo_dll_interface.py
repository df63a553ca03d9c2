"""The reference's ctypes front-end of the orientation search
(cfms_tomo/tomo_dll_interface.py:13-135), bound to the B200 library.

Differences from the reference, all at the loading step: the library is a
Linux shared object opened with ``ctypes.CDLL`` (the reference opens a
Windows DLL with ``WinDLL``), and a ``dll_fname`` that names no existing file
(the reference's "Tomo_Shell2026.dll") selects the B200 library built in
this package.  Everything after loading -- argument packing, the YPR grid,
getters, optimum picking, pixel groups -- follows the reference.
"""
from __future__ import annotations

import ctypes as ct
import os
from copy import copy, deepcopy
from typing import Optional

import numpy as np

from .tomo_io import (Cptr1d, Cptr1d_to_np, Cptr1i, Cptr1i_to_np, Cptr1iL, findOptimals, np_to_Cptr1d,
                      np_to_Cptr1iL, toRadian)
from .tomo_object import TomoObject
from .tomo_slicingOptions import (TOMO_PixelVarNames, SlicingOptions, TomoPixels, TOMO_nPixelFormat,
                                  enumPixelType)


def _library_file(dll_fname: str) -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    for cand in (dll_fname, os.path.join(here, dll_fname)):
        if cand and os.path.isfile(cand):
            return cand
    from ..native import library_path
    path = library_path()
    if not path.exists():
        raise FileNotFoundError(f"B200 library not built: {path}")
    return str(path)


class TomoDLLInterface:
    CppDLL = None
    slicing_option = None
    nYPR_Intervals = 1
    (yaw_range, pitch_range, roll_range) = ([], [], [])
    (xx, yy, zz, YPR) = ([], [], [], [])
    (Float32Info, Int32Info) = ([], [])
    (bUseExplicitSS, bUseClosedVolumeVoxel) = (True, False)   # the reference always passes explicit SS

    def __init__(self, dll_fname, s_o: Optional[SlicingOptions], bUseCUDA, bShellMesh):
        self.CppDLL = ct.CDLL(_library_file(dll_fname))
        self.CppFunction = getattr(self.CppDLL, "TomoSh_CUDA" if bUseCUDA else "TomoSh_INT3")
        self.CppFunction.argtypes = (Cptr1d, Cptr1iL, Cptr1d, Cptr1iL, Cptr1d, Cptr1d, Cptr1d, Cptr1iL, Cptr1d, Cptr1d)
        self.CppFunction.restype = ct.c_int32
        self.bShellMesh = bShellMesh
        L = self.CppDLL
        L.getMo.argtypes = (); L.getMo.restype = Cptr1d
        L.getMss.argtypes = (); L.getMss.restype = Cptr1d
        L.getMat4x4.argtypes = (); L.getMat4x4.restype = Cptr1d
        L.getnData2i.argtypes = (ct.c_short,); L.getnData2i.restype = ct.c_int32
        L.getpData2i.argtypes = (ct.c_short,); L.getpData2i.restype = Cptr1i
        L.tomoGetLastErrorString.argtypes = (); L.tomoGetLastErrorString.restype = ct.c_char_p

        S_O = self.slicing_option = copy(s_o)
        self.nYPR_Intervals = int(360 / S_O.theta_YP) + 1
        self.yaw_range = np.linspace(toRadian(0), toRadian(360), num=self.nYPR_Intervals, endpoint=True, dtype=np.float32)
        self.pitch_range = np.linspace(toRadian(0), toRadian(360), num=self.nYPR_Intervals, endpoint=True,
                                       dtype=np.float32)
        self.roll_range = np.zeros(1)
        self.xx, self.yy, self.zz = np.meshgrid(self.yaw_range, self.pitch_range, self.roll_range)
        self.YPR = np.column_stack([self.xx.ravel(), self.yy.ravel(), self.zz.ravel()]).astype(np.float32)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def free(self):
        self.CppDLL.OnDestroy.argtypes = ()
        self.CppDLL.OnDestroy.restype = None
        self.CppDLL.OnDestroy()

    def pack(self, T, n_ypr, bVerbose):
        """Float32Info / Int32Info and the hull arrays of one call (tomo_dll_interface.py:56-82)."""
        S_O = self.slicing_option
        H = T.convex_hull
        H_vtx = np.asarray(H.vertices).astype(np.float32, copy=True)
        H_tri = np.asarray(H.triangles).astype(np.int32, copy=True)   # as in the reference: hull corner coordinates
        H_trinrm = np.asarray(H.face_normals).astype(np.float32, copy=True)
        self.Float32Info = np.array([S_O.dVoxel, S_O.theta_c, T.area, S_O.wall_thickness,
                                     S_O.Fcore, S_O.Fclad, S_O.Fss, S_O.Css,
                                     S_O.PLA_density, S_O.BedType[1], S_O.BedType[2], S_O.BedType[3]]).astype(np.float32)
        self.Int32Info = np.array([bVerbose, self.bUseExplicitSS, self.bShellMesh, S_O.nVoxel,
                                   T.faces.shape[0], T.vertices.shape[0], n_ypr,
                                   H_tri.shape[0], H_vtx.shape[0], S_O.BedType[0],
                                   int(round(S_O.ShellThickness * 1000.0))]).astype(np.int32)
        return H_tri, H_vtx, H_trinrm

    def run_dll(self, cutobject0, bVerbose):
        if bVerbose:
            print("Tomo processing: ", cutobject0.name)
        c_o = deepcopy(cutobject0)
        self.bShellMesh = self.slicing_option.bShellMesh and (not c_o.tmesh.is_watertight)
        T = c_o.tmesh
        vtx = np.asarray(T.vertices).astype(np.float32, copy=True)
        vtx_nrm = np.asarray(T.vertex_normals).astype(np.float32, copy=True)
        tri = np.asarray(T.faces).astype(np.int32, copy=True)
        tri_nrm = np.asarray(T.face_normals).astype(np.float32, copy=True)
        H_tri, H_vtx, H_trinrm = self.pack(T, self.YPR.shape[0], bVerbose)

        self.Cdll_opt_id = self.CppFunction(
            np_to_Cptr1d(self.Float32Info), np_to_Cptr1iL(self.Int32Info), np_to_Cptr1d(self.YPR),
            np_to_Cptr1iL(tri), np_to_Cptr1d(vtx), np_to_Cptr1d(vtx_nrm), np_to_Cptr1d(tri_nrm),
            np_to_Cptr1iL(H_tri), np_to_Cptr1d(H_vtx), np_to_Cptr1d(H_trinrm))
        L = self.CppDLL
        if self.Cdll_opt_id < 0:
            msg = L.tomoGetLastErrorString()
            raise RuntimeError(f"orientation search failed ({self.Cdll_opt_id}): {msg.decode() if msg else ''}")
        return self._collect(c_o, T, bVerbose)

    def run_batch(self, cutobjects, bVerbose):
        """run_dll for every part, all parts swept in one batched graph launch
        (TomoSh_CUDA_Batch); each part's TomoObject equals run_dll's."""
        L = self.CppDLL
        vp = ct.POINTER(ct.c_void_p)
        L.TomoSh_CUDA_Batch.argtypes = (ct.c_int, vp, vp, vp, vp, vp, vp, ct.POINTER(ct.c_int32))
        L.TomoSh_CUDA_Batch.restype = ct.c_int32
        L.tomoBatchExport.argtypes = (ct.c_int,); L.tomoBatchExport.restype = ct.c_int32
        L.tomoBatchRelease.argtypes = (); L.tomoBatchRelease.restype = None
        parts, keep = [], []
        cols = [[] for _ in range(6)]
        for cutobject0 in cutobjects:
            if bVerbose:
                print("Tomo processing: ", cutobject0.name)
            c_o = deepcopy(cutobject0)
            self.bShellMesh = self.slicing_option.bShellMesh and (not c_o.tmesh.is_watertight)
            T = c_o.tmesh
            vtx = np.asarray(T.vertices).astype(np.float32, copy=True)
            vtx_nrm = np.asarray(T.vertex_normals).astype(np.float32, copy=True)
            tri = np.asarray(T.faces).astype(np.int32, copy=True)
            self.pack(T, self.YPR.shape[0], bVerbose)
            arrays = (self.Float32Info.copy(), self.Int32Info.copy(), self.YPR, tri, vtx, vtx_nrm)
            keep.append(arrays)
            for col, a in zip(cols, arrays):
                col.append(a.ctypes.data)
            parts.append((c_o, T))
        n = len(parts)
        ptrs = [(ct.c_void_p * max(n, 1))(*c) for c in cols]
        opt = np.zeros(max(n, 1), np.int32)
        rc = L.TomoSh_CUDA_Batch(n, *[ct.cast(p, vp) for p in ptrs], opt.ctypes.data_as(ct.POINTER(ct.c_int32)))
        if rc < 0:
            msg = L.tomoGetLastErrorString()
            raise RuntimeError(f"batched orientation search failed ({rc}): {msg.decode() if msg else ''}")
        out = []
        try:
            for k, (c_o, T) in enumerate(parts):
                self.Cdll_opt_id = L.tomoBatchExport(k)
                if self.Cdll_opt_id < 0:
                    msg = L.tomoGetLastErrorString()
                    raise RuntimeError(f"export of part {k} failed: {msg.decode() if msg else ''}")
                out.append(self._collect(c_o, T, bVerbose))
        finally:
            L.tomoBatchRelease()
        return out

    def _collect(self, c_o, T, bVerbose):
        """TomoObject of the last call from the getters (tomo_dll_interface.py:103-133)."""
        L = self.CppDLL
        t_o = TomoObject(c_o)

        Mss3D = np.array(Cptr1d_to_np(L.getMss(), self.YPR.shape[0])).astype(np.float32, copy=True)
        if os.environ.get("TOMO_DEBUG_MSS", "0").lower() in ("1", "true", "yes", "on"):
            best_ids = np.argsort(Mss3D)[:8]
            print("TOMO_DEBUG_MSS", "min", float(np.min(Mss3D)), "max", float(np.max(Mss3D)),
                  "sum", float(np.sum(Mss3D)), "best_ids", best_ids.tolist(),
                  "best_vals", [float(Mss3D[i]) for i in best_ids])
        if os.environ.get("TOMO_DEBUG_MSS_FULL", "0").lower() in ("1", "true", "yes", "on"):
            print("TOMO_DEBUG_MSS_FULL", [float(v) for v in Mss3D])
        self.Mss3D = Mss3D

        t_o.best_vminfo, _ = findOptimals(self.YPR, Mss3D, bVerbose)
        t_o.best_vminfo.set_max_length(T)

        for p_type in (enumPixelType.eptSS, enumPixelType.eptBed):
            n_2i = L.getnData2i(p_type)
            if n_2i > 0:
                p_2i = L.getpData2i(p_type)
                pxls = Cptr1i_to_np(p_2i, n_2i * TOMO_nPixelFormat).reshape(n_2i, TOMO_nPixelFormat)
                pxls = np.array(pxls).astype(float)[:, 0:3]
                t_o.pxl_groups.append(TomoPixels(p_type, TOMO_PixelVarNames[p_type], pxls))

        t_o.mat4x4 = np.array(Cptr1d_to_np(L.getMat4x4(), 4 * 4)).astype(np.float32, copy=True).reshape(4, 4)
        return t_o
