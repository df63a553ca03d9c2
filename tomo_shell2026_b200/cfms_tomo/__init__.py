"""Reference-compatible Python surface of the orientation search.

Mirrors the reference package ``cfms_tomo`` (cfms_tomo/__init__.py,
tomo_dll_interface.py, tomo_io.py, tomo_object.py, tomo_result.py,
tomo_slicingOptions.py, shell_test/tomoSh_Cpp.py) over the B200 library, so
callers written against the reference keep working:

    from tomo_shell2026_b200.cfms_tomo import TomoManager, SlicingOptions

``TomoManager.get_best_orientation`` (cfms_tomo/__init__.py:26-30) runs the
search for every part of a group.  Mesh cutting and shell generation
(``get_shells``, cfms_meshcut) are not part of this library.
"""
from __future__ import annotations

from .cut_parts import CutGroup, CutObject
from .meshio import TriMesh, load
from .tomo_dll_interface import TomoDLLInterface
from .tomo_object import TomoObject
from .tomo_result import TomoResult, VolMassData
from .tomo_slicingOptions import SlicingOptions, TomoPixels, enumBedType, enumPixelType

g_bVerbose = True
g_bUseCUDA = False
g_bShellMesh = True
g_tomo_theta_YP = 10


class TomoManager:
    """Runs the orientation search over the parts of a cut group."""

    def __init__(self, s_o: SlicingOptions):
        self.slicing_option = s_o
        self.CppDLL = TomoDLLInterface("Tomo_Shell2026.dll", s_o, s_o.bUseCUDA, s_o.bShellMesh)

    def get_best_orientation(self, C_G: CutGroup):
        self.name = f"{C_G.name}_tomo"
        self.input_gr = C_G
        for c_o in C_G.cutobjects:
            c_o.tomo_object = self.CppDLL.run_dll(c_o, self.slicing_option.bVerbose)

    def get_best_orientation_batched(self, C_G: CutGroup):
        """get_best_orientation with every part swept in one batched launch
        (the parts' results are those of get_best_orientation)."""
        self.name = f"{C_G.name}_tomo"
        self.input_gr = C_G
        for c_o, t_o in zip(C_G.cutobjects, self.CppDLL.run_batch(C_G.cutobjects, self.slicing_option.bVerbose)):
            c_o.tomo_object = t_o

    def get_shells(self, offset_size):
        raise NotImplementedError("shell generation belongs to the mesh-cutting package, not this library")


__all__ = ["TomoManager", "TomoDLLInterface", "SlicingOptions", "TomoObject", "TomoResult", "VolMassData",
           "TomoPixels", "enumPixelType", "enumBedType", "CutObject", "CutGroup", "TriMesh", "load"]
