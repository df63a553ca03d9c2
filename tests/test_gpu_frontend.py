"""The reference-compatible Python surface on the GPU: TomoManager over a
two-part group against the fixture the reference engine produced for the
same packed arrays, and the tomoSh_Cpp script runner on a mesh file."""
from __future__ import annotations

import numpy as np
import pytest

from tests.test_frontend import _write_ply
from tomo_shell2026_b200 import meshgen, native
from tomo_shell2026_b200.cfms_tomo import CutGroup, CutObject, SlicingOptions, TomoManager, TriMesh, enumPixelType
from tomo_shell2026_b200.cfms_tomo.tomo_io import findOptimals, toRadian
from tests.test_frontend import GOLD

pytestmark = pytest.mark.gpu


def test_manager_matches_reference_engine():
    d = np.load(GOLD)
    s_o = SlicingOptions()
    s_o.theta_YP = 30
    s_o.bVerbose = False
    parts = [CutObject(f"part{k}", TriMesh(d[f"p{k}_vertices"].astype(np.float64), d[f"p{k}_faces"],
                                           d[f"p{k}_vertex_normals"], process=False)) for k in range(2)]
    group = CutGroup("pair", parts)
    mgr = TomoManager(s_o)
    for k, c_o in enumerate(group.cutobjects):
        # run part by part to read each part's Mss through the interface
        t_o = mgr.CppDLL.run_dll(c_o, False)
        assert np.array_equal(mgr.CppDLL.Mss3D.view(np.int32), d[f"p{k}_Mss"].view(np.int32)), f"part {k}: Mss differs"
        assert mgr.CppDLL.Cdll_opt_id == int(d[f"p{k}_optID"])
        best, _ = findOptimals(d["YPR"], d[f"p{k}_Mss"])
        assert t_o.best_vminfo.vmData == best.vmData
        groups = {g.type: g.pxls for g in t_o.pxl_groups}
        for p_type, key in ((enumPixelType.eptSS, "SS"), (enumPixelType.eptBed, "Bed")):
            want = d[f"p{k}_{key}"][:, :3].astype(float)
            got = groups.get(p_type, np.zeros((0, 3)))
            assert np.array_equal(got, want), f"part {k}: {key} pixels differ"
        assert np.array_equal(t_o.mat4x4.ravel().view(np.int32), d[f"p{k}_mat16"].view(np.int32))
    mgr.get_best_orientation(group)
    assert mgr.name == "pair_tomo"
    assert all(c.tomo_object is not None for c in group.cutobjects)


def test_script_runner_on_a_mesh_file(tmp_path):
    from tomo_shell2026_b200.cfms_tomo.shell_test.tomoSh_Cpp import tomoSh_Cpp
    m = meshgen.small_solid(4, with_hull=False)
    path = tmp_path / "part.ply"
    _write_ply(path, m.vertices, m.faces, binary=True)
    n = 7
    yaw = np.linspace(toRadian(0), toRadian(360), num=n, endpoint=True, dtype=np.float32)
    pitch = np.linspace(toRadian(0), toRadian(360), num=n, endpoint=True, dtype=np.float32)
    runs = []
    for fn in ("TomoSh_INT3", "TomoSh_CUDA"):
        t = tomoSh_Cpp(str(path), n, yaw, pitch, np.zeros(1), bVerbose=False)
        t.bUseExplicitSS = True
        t.bShellMesh = not t.mesh0.is_watertight
        t.Run(cpp_function_name=fn)
        runs.append(t)
    assert np.array_equal(runs[0].Mss3D, runs[1].Mss3D)
    assert runs[0].Cdll_opt_id == runs[1].Cdll_opt_id
    # the same arrays through the package's own binding
    t = runs[0]
    arrays = t.mesh0.to_arrays()
    from tomo_shell2026_b200.options import PrintOptions
    r = native.sweep(arrays, t.YPR, PrintOptions(dVoxel=1.0, explicit_ss=True, wall_thickness=t.wall_thickness,
                                                   bed_type=int(t.BedType[0]), bed_inner=float(t.BedType[1]),
                                                   bed_outer=float(t.BedType[2]), bed_thickness=float(t.BedType[3])))
    assert np.array_equal(r.Mss, t.Mss3D)


def test_batched_manager_equals_part_by_part():
    d = np.load(GOLD)
    s_o = SlicingOptions()
    s_o.theta_YP = 30
    s_o.bVerbose = False

    def group():
        return CutGroup("pair", [CutObject(f"part{k}", TriMesh(d[f"p{k}_vertices"].astype(np.float64),
                                                               d[f"p{k}_faces"], d[f"p{k}_vertex_normals"],
                                                               process=False)) for k in range(2)])

    g1, g2 = group(), group()
    mgr = TomoManager(s_o)
    mgr.get_best_orientation(g1)
    mgr.get_best_orientation_batched(g2)
    for a, b in zip(g1.cutobjects, g2.cutobjects):
        ta, tb = a.tomo_object, b.tomo_object
        assert ta.best_vminfo.vmData == tb.best_vminfo.vmData
        assert np.array_equal(ta.mat4x4.view(np.int32), tb.mat4x4.view(np.int32))
        assert [p.type for p in ta.pxl_groups] == [p.type for p in tb.pxl_groups]
        for pa, pb in zip(ta.pxl_groups, tb.pxl_groups):
            assert np.array_equal(pa.pxls, pb.pxls)
