"""Printer options, pixel / bed enums and pixel groups of the reference
front-end (cfms_tomo/tomo_slicingOptions.py:1-58).  The enum values are the
C-ABI's pixel type and bed type numbers (Tomo_Shell_vc_src/Tomo_types.h:45-59)."""
from __future__ import annotations

from enum import Enum

from .tomo_io import toRadian


class enumPixelType(int, Enum):
    eptAl = 0
    eptBe = 1
    eptSSB = 2
    eptSSA = 3
    eptSS = 4
    eptBed = 5
    eptVo = 6
    eptVss = 7
    eptTC = 8
    eptNVB = 9
    eptNVA = 10
    eptNumberOfSubPixels = 11


class enumBedType(int, Enum):
    ebtNone = 0
    ebtBrim = 1
    ebtRaft = 2
    ebtSkirt = 3


g_tomo_theta_YP = 10
TOMO_nOptimalsToDisplay = 3
TOMO_nPixelFormat = 6   # x, y, z, nx, ny, nz
TOMO_PixelVarNames = ("al_pxls", "be_pxls", "SSB_pxls", "SSA_pxls", "SS_pxls", "Bed_pxls", "Vo_pxls", "Vss_pxls",
                      "TC_pxls", "NVB_pxls", "NVA_pxls")


class TomoPixels:
    def __init__(self, type: enumPixelType, name, pxls):  # noqa: A002 - reference argument name
        self.type = type
        self.name = name
        self.pxls = pxls.copy()

    def copy(self):
        return TomoPixels(self.type, self.name, self.pxls)


class SlicingOptions:
    """Class-level defaults as in the reference; instances override per attribute."""
    wall_thickness = 0.8        # mm
    PLA_density = 0.001121      # g/mm^3
    Fclad = 1.0
    Fcore = 0.15
    Fss = 0.2
    Css = 1.0
    dVoxel = 1.0
    nVoxel = 256
    theta_c = toRadian(60.0)
    bUseExplicitSS = False
    BedType = (enumBedType.ebtRaft, 0, 2, 0.3 + 0.27 + 2 * 0.2)   # type, inner, outer, thickness
    (Yaw, Pitch, Roll) = (0, 0, 0)
    theta_YP = g_tomo_theta_YP   # degrees
    bVerbose = True
    bUseCUDA = True
    bShellMesh = True
    ShellThickness = 0.5
