"""Per-part result container (cfms_tomo/tomo_object.py:1-31): the best
orientation, the support and bed pixel groups and the best mat4x4.
Rendering (``add_to``, a polyscope point cloud) is not part of this
library."""
from __future__ import annotations

from copy import copy

import numpy as np

from .tomo_result import TomoResult


class TomoObject:
    def __init__(self, cutobject, pxl_groups=None, best=None, colorspan=None, mat4x4=None):
        self.raw_cutobject = cutobject
        self.pxl_groups = [p.copy() for p in pxl_groups] if pxl_groups else []
        self.best_vminfo = copy(best) if best else TomoResult()
        self.colorspan = copy(colorspan) if colorspan else None
        self.mat4x4 = mat4x4.copy() if mat4x4 is not None else None

    def add_to(self, ps, parent_group_id):
        raise NotImplementedError("rendering is outside the orientation-search library")

    def translate_by(self, vec):
        for p_g in self.pxl_groups:
            p_g.pxls = np.add(np.array(p_g.pxls), vec)

    def copy(self):
        return TomoObject(self.raw_cutobject, self.pxl_groups, self.best_vminfo, self.colorspan, self.mat4x4)
