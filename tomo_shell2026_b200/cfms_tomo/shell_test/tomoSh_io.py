"""Mesh loading, geometry helpers and optimum picking of the reference's
script front-end (cfms_tomo/shell_test/tomoSh_io_trimesh.py), minus its
plotting (matplotlib / plotly figures are not part of this library).

``LoadInputMesh`` (tomoSh_io_trimesh.py:530-558) loads a mesh file, moves
its AABB centre to the origin and returns the arrays handed to the C-ABI.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from ..meshio import load
from ..tomo_io import (Cptr1d, Cptr1d_to_np, Cptr1i, Cptr1i_to_np, Cptr1iL, Cptr1iL_to_np, EndTimer, FStr,  # noqa: F401
                       StartTimer, np_to_Cptr1d, np_to_Cptr1i, np_to_Cptr1iL, smallestN_indices, toDegree, toRadian)
from ..tomo_slicingOptions import enumBedType, enumPixelType  # noqa: F401

g_PixelEnums = ("eptAl", "eptBe", "eptSSB", "eptSSA", "eptSS", "eptBed", "eptVo", "eptVss", "eptTC", "eptNVB", "eptNVA")
g_PixelVarNames = ("al_pxls", "be_pxls", "SSB_pxls", "SSA_pxls", "SS_pxls", "Bed_pxls", "Vo_pxls", "Vss_pxls",
                   "TC_pxls", "NVB_pxls", "NVA_pxls")
g_nPixelFormat = 6
g_nOptimalsToDisplay = 3
g_fMARGIN = 0.001
g_fNORMALFACTOR = 1000.0
g_mesh0_surface_area = 0.0
g_input_mesh_filename = ""


def CppDLLFileName() -> str:
    from ...native import library_path
    return str(library_path())


def getBoundary(vtx):
    v = np.asarray(vtx)
    mn = np.array([np.min(v[:, 0]), np.min(v[:, 1]), np.min(v[:, 2])])
    mx = np.array([np.max(v[:, 0]), np.max(v[:, 1]), np.max(v[:, 2])])
    return mn, mx, (mn + mx) * 0.5


def Area3D(p1, p2, p3):
    return np.linalg.norm(np.cross(p2 - p1, p3 - p1)) * 0.5


def getMeshTriArea(vtx, tri):
    v = np.asarray(vtx, dtype=np.float64)
    t = np.asarray(tri)
    return 0.5 * np.linalg.norm(np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]]), axis=1)


def LoadInputMesh(filename):
    global g_mesh0_surface_area, g_input_mesh_filename
    if not os.path.isfile(filename):
        print("[ERROR] File Does not Exists: " + filename)
        sys.exit(0)
    if not os.path.isfile(CppDLLFileName()):
        print("[ERROR] C++ Dll Does not Exists: " + CppDLLFileName())
        sys.exit(0)
    mesh0 = load(filename, force="mesh")
    _, _, center = getBoundary(mesh0.vertices)
    mesh0.apply_transform(np.array([[1, 0, 0, -center[0]], [0, 1, 0, -center[1]], [0, 0, 1, -center[2]],
                                    [0, 0, 0, 1]], dtype=np.float64))
    g_mesh0_surface_area = mesh0.area
    vtx = np.asarray(mesh0.vertices).astype(np.float32)
    tri = np.asarray(mesh0.faces).astype(np.int32)
    tri_nrm = np.asarray(mesh0.face_normals).astype(np.float32)
    vtx_nrm = np.asarray(mesh0.vertex_normals).astype(np.float32)
    tri_area = getMeshTriArea(vtx, tri)
    chull = mesh0.convex_hull
    chull_tri = np.asarray(chull.faces).astype(np.int32)
    chull_vtx = np.array(chull.vertices).astype(np.float32)
    chull_trinrm = np.asarray(chull.face_normals).astype(np.float32)
    tr_center = np.average(vtx[tri], axis=1).astype(np.float32)
    g_input_mesh_filename = filename
    return mesh0, tri, vtx, vtx_nrm, tri_nrm, tri_area, tr_center, chull_tri, chull_vtx, chull_trinrm


def paramsYP(yaw_range, pitch_range, theta_c):
    rows = [[yaw, pitch, 0.0, theta_c, k + g_fMARGIN]
            for k, (pitch, yaw) in enumerate((p, y) for p in pitch_range for y in yaw_range)]
    params = np.asarray(rows, dtype=np.float32).reshape(-1, 5)
    return params, np.size(yaw_range), np.size(pitch_range), np.size(yaw_range) * np.size(pitch_range)


def findOptimals(YPR, data, nOptimal):
    """Best / worst nOptimal rows [yaw, pitch, roll, value] (tomoSh_io_trimesh.py:430-452)."""
    best_ids, worst_ids = smallestN_indices(data, nOptimal, maintain_order=True)
    n = min(best_ids.size, nOptimal)
    optimal = np.zeros((n, 4))
    worst = np.zeros((n, 4))
    for i in range(n):
        o, w = best_ids[i], worst_ids[i]
        optimal[i] = np.array([YPR[o, 0], YPR[o, 1], YPR[o, 2], data[o]])
        print(i + 1, "st optimal is at [", FStr(toDegree([YPR[o, 0], YPR[o, 1], YPR[o, 2]])),
              "], Mss=", FStr(data[o], precision=3))
        worst[i] = np.array([YPR[w, 0], YPR[w, 1], YPR[w, 2], data[w]])
        print(i + 1, "st worst is at [", FStr(toDegree([YPR[w, 0], YPR[w, 1], YPR[w, 2]])),
              "], Mss=", FStr(data[w], precision=3))
    return optimal, worst
