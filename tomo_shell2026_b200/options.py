"""Printer options and the order-critical info arrays of the TomoSh_* C-ABI.

``pack_info`` produces the two arrays exactly as the reference Python surface
builds them before every call (cfms_tomo/tomo_dll_interface.py:73-82 and
cfms_tomo/shell_test/tomoSh_Cpp.py:53-62); their layout is what
S3DPrinterInfo::Set reads (Tomo_Shell_vc_src/cpu_src/S3DPrinterInfo.h:42-47,
S3DPrinterInfo.cpp:130-144):

Float32Info[12] = dVoxel, theta_c, surface_area, wall_thickness, Fcore, Fclad,
                  Fss, Css, PLA_density, BedInnerBound, BedOuterBound, BedThickness
Int32Info[11]   = bVerbose, bUseExplicitSS, bShellMesh, nVoxel, nTri, nVtx, nYPR,
                  nHullTri, nHullVtx, BedType, round(ShellThickness*1000)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

F32_INFO_LEN = 12
I32_INFO_LEN = 11

BED_NONE, BED_BRIM, BED_RAFT, BED_SKIRT = 0, 1, 2, 3


@dataclass
class PrintOptions:
    """Defaults follow SlicingOptions (cfms_tomo/tomo_slicingOptions.py:41-58)
    except the bed, which is off unless asked for."""

    dVoxel: float = 1.0
    theta_c: float = float(60.0 * np.pi / 180.0)
    wall_thickness: float = 0.8
    Fcore: float = 0.15
    Fclad: float = 1.0
    Fss: float = 0.2
    Css: float = 1.0
    PLA_density: float = 0.001121
    bed_type: int = BED_NONE
    bed_inner: float = 0.0
    bed_outer: float = 0.0
    bed_thickness: float = 0.0
    explicit_ss: bool = True
    shell_mesh: bool = False
    shell_thickness: float = 0.5
    verbose: bool = False
    n_voxel: int = 256


def pack_info(opts: PrintOptions, mesh, n_ypr: int) -> tuple[np.ndarray, np.ndarray]:
    """Return (Float32Info[12] float32, Int32Info[11] int32)."""
    f32 = np.array([opts.dVoxel, opts.theta_c, mesh.area, opts.wall_thickness,
                    opts.Fcore, opts.Fclad, opts.Fss, opts.Css,
                    opts.PLA_density, opts.bed_inner, opts.bed_outer, opts.bed_thickness],
                   dtype=np.float64).astype(np.float32)
    i32 = np.array([int(bool(opts.verbose)), int(bool(opts.explicit_ss)), int(bool(opts.shell_mesh)),
                    int(opts.n_voxel), mesh.n_tri, mesh.n_vtx, int(n_ypr),
                    int(mesh.hull_faces.shape[0]), int(mesh.hull_vertices.shape[0]), int(opts.bed_type),
                    int(round(opts.shell_thickness * 1000.0))], dtype=np.int32)
    return f32, i32
