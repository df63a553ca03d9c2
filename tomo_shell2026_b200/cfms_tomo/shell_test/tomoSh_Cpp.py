"""``tomoSh_Cpp``: load a mesh file and run one orientation search through the
C-ABI by function name (cfms_tomo/shell_test/tomoSh_Cpp.py:4-120), on the
B200 library.  ``Run('TomoSh_INT3')`` and ``Run('TomoSh_CUDA')`` both reach
the B200 path, whose results are the INT3 results."""
from __future__ import annotations

import ctypes as ct

import numpy as np

from ..tomo_slicingOptions import enumBedType, enumPixelType
from .tomoSh_io import (Cptr1d, Cptr1d_to_np, Cptr1i, Cptr1i_to_np, Cptr1iL, CppDLLFileName, EndTimer, FStr,
                        LoadInputMesh, StartTimer, getBoundary, g_nPixelFormat, g_PixelEnums, g_PixelVarNames,
                        np_to_Cptr1d, np_to_Cptr1iL, toDegree, toRadian)


class tomoSh_Cpp:
    wall_thickness = 1.0
    PLA_density = 0.001121
    Fclad = 1.0
    Fcore = 0.15
    Fss = 0.2
    Css = 1.0
    bVerbose = False
    bUseExplicitSS = False
    bUseClosedVolumeVoxel = False
    bShellMesh = False
    ShellThickness = 0.5
    dVoxel = 1.0
    nVoxel = 256
    theta_c = toRadian(60.0)
    nYPR_Intervals = 0
    BedType = (enumBedType.ebtRaft, 0.0, 0.0, 0.0)

    def __init__(self, filename, nYPR_Intervals, yaw_range, pitch_range, roll_range, bVerbose):
        self.FileName = filename
        (self.mesh0, self.tri, self.vtx, self.vtx_nrm, self.tri_nrm, self.tri_area, self.tri_center,
         self.chull_tri, self.chull_vtx, self.chull_trinrm) = LoadInputMesh(filename)
        self.xx, self.yy, self.zz = np.meshgrid(yaw_range, pitch_range, roll_range)
        self.YPR = np.column_stack([self.xx.ravel(), self.yy.ravel(), self.zz.ravel()]).astype(np.float32)
        self.nYPR_Intervals = nYPR_Intervals
        self.bVerbose = bVerbose
        mn, mx, _ = getBoundary(self.vtx)
        x1, y1, z1 = list(map(int, mx))
        x0, y0, z0 = list(map(int, mn))
        d = max(max(x1 - x0, y1 - y0), z1 - z0)
        self.AABB2D = (0, 0, d, d)
        if self.bVerbose:
            print("vtx=", self.vtx.shape)
            print("tri=", self.tri.shape)
            print("YPR=", toDegree(self.YPR), self.YPR.shape)

    def info_arrays(self):
        f32 = np.array([self.dVoxel, self.theta_c, self.mesh0.area, self.wall_thickness,
                        self.Fcore, self.Fclad, self.Fss, self.Css,
                        self.PLA_density, self.BedType[1], self.BedType[2], self.BedType[3]]).astype(np.float32)
        i32 = np.array([self.bVerbose, self.bUseExplicitSS, self.bShellMesh, self.nVoxel,
                        self.tri.shape[0], self.vtx.shape[0], self.YPR.shape[0],
                        self.chull_tri.shape[0], self.chull_vtx.shape[0], self.BedType[0],
                        int(round(self.ShellThickness * 1000.0))]).astype(np.int32)
        return f32, i32

    def Run(self, cpp_function_name):
        self.Float32Info, self.Int32Info = self.info_arrays()
        time0 = StartTimer()
        self.CppDLL = ct.CDLL(CppDLLFileName())
        self.CppFunction = getattr(self.CppDLL, cpp_function_name)
        self.CppFunction.argtypes = (Cptr1d, Cptr1iL, Cptr1d, Cptr1iL, Cptr1d, Cptr1d, Cptr1d, Cptr1iL, Cptr1d, Cptr1d)
        self.CppFunction.restype = ct.c_int32
        self.Cdll_opt_id = self.CppFunction(
            np_to_Cptr1d(self.Float32Info), np_to_Cptr1iL(self.Int32Info), np_to_Cptr1d(self.YPR),
            np_to_Cptr1iL(self.tri), np_to_Cptr1d(self.vtx), np_to_Cptr1d(self.vtx_nrm), np_to_Cptr1d(self.tri_nrm),
            np_to_Cptr1iL(self.chull_tri), np_to_Cptr1d(self.chull_vtx), np_to_Cptr1d(self.chull_trinrm))
        EndTimer(time0, self.FileName + "    " + cpp_function_name)
        L = self.CppDLL
        if self.Cdll_opt_id < 0:
            L.tomoGetLastErrorString.restype = ct.c_char_p
            msg = L.tomoGetLastErrorString()
            raise RuntimeError(f"{cpp_function_name} failed ({self.Cdll_opt_id}): {msg.decode() if msg else ''}")

        L.getMo.argtypes = (); L.getMo.restype = Cptr1d
        L.getMss.argtypes = (); L.getMss.restype = Cptr1d
        n = self.YPR.shape[0]
        self.Mo3D = np.array(Cptr1d_to_np(L.getMo(), n)).astype(np.float32)
        self.Mss3D = np.array(Cptr1d_to_np(L.getMss(), n)).astype(np.float32)
        self.Mtotal3D = self.Mo3D + self.Mss3D
        L.getVolMassInfo.argtypes = (); L.getVolMassInfo.restype = Cptr1d
        self.vm_info = np.array(Cptr1d_to_np(L.getVolMassInfo(), 21)).astype(np.float32)

        if self.bVerbose:
            k = self.nYPR_Intervals
            if k * k == n:
                print("Mo3D=    ", FStr(self.Mo3D.reshape(k, k), precision=2))
                print("Mss3D=   ", FStr(self.Mss3D.reshape(k, k), precision=2))
                print("Mtotal3D=", FStr(self.Mtotal3D.reshape(k, k), precision=2))
            L.getnData2i.argtypes = (ct.c_short,); L.getnData2i.restype = ct.c_int32
            L.getpData2i.argtypes = (ct.c_short,); L.getpData2i.restype = Cptr1i
            for p_type, p_name in zip(g_PixelEnums, g_PixelVarNames):
                e = getattr(enumPixelType, p_type).value
                n_2i = L.getnData2i(e)
                if n_2i == 0:
                    setattr(self, p_name, np.array([[0, 0, 0, 0, 0, 0]]))
                else:
                    setattr(self, p_name, Cptr1i_to_np(L.getpData2i(e), n_2i * g_nPixelFormat).reshape(n_2i, g_nPixelFormat))

        L.OnDestroy.argtypes = ()
        L.OnDestroy.restype = None
        L.OnDestroy()

    def Print_tabbed(self):
        if self.bVerbose:
            print("Va, Vb, Vtc, Vnv,")
            print(self.vm_info[0], self.vm_info[1], self.vm_info[2], self.vm_info[3], sep=" ")
