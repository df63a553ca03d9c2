"""The two containers TomoManager reads from the reference's mesh-cutting
package (cfms_meshcut.cut_object.CutObject / cut_group.CutGroup): a named
part holding a mesh, and a named list of parts.  Only the attributes the
orientation search uses are kept (``name``, ``tmesh``, ``tomo_object``,
``transform``); cutting, offsetting and shells are not part of this library."""
from __future__ import annotations

import numpy as np

from .meshio import TriMesh


class CutObject:
    def __init__(self, name: str, tmesh: TriMesh):
        self.name = name
        self.tmesh = tmesh
        self.tomo_object = None

    def transform(self, mat4x4):
        self.tmesh.apply_transform(np.asarray(mat4x4, dtype=np.float64))


class CutGroup:
    def __init__(self, name: str, cutobjects=None):
        self.name = name
        self.cutobjects = list(cutobjects or [])
