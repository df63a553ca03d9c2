"""Edge cases of the C-ABI on the GPU, against the reference engine built from
its own sources (oracle/_ref) where it can run them and the C restatement
otherwise: one and zero orientations, an empty mesh, a mesh wider than the
reference's 256-column grid with a raft, alternating meshes in one process,
and inputs the library must reject."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

from tests.test_gpu_parity import _compare, _same_bits
from tomo_shell2026_b200 import meshgen, native
from tomo_shell2026_b200.options import PrintOptions

pytestmark = pytest.mark.gpu


def test_single_orientation_and_its_export(oracle, ref_engine):
    m = meshgen.small_solid(41)
    ypr = meshgen.ypr_grid([37.0], [23.0])
    opts = PrintOptions(explicit_ss=True, bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    r = native.sweep(m, ypr, opts)
    _compare(r, oracle.sweep(m, ypr, opts), "one orientation")
    assert r.optID == 0
    ex = ref_engine.pixels(m, ypr, opts, 0)
    for k in range(11):
        assert np.array_equal(r.pixels[k], ex["pixels"][k]), f"pixel type {k}"
    assert _same_bits(r.volmass, ex["vm22"])
    assert _same_bits(r.mat4x4.ravel(), ex["mat16"])


def test_zero_orientations():
    m = meshgen.small_solid(42)
    r = native.sweep(m, np.zeros((0, 3), np.float32), PrintOptions())
    assert r.optID == 0 and r.Mss.size == 0
    assert all(p.shape[0] == 0 for p in r.pixels)


def test_empty_mesh(oracle):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    m = meshgen.MeshArrays(v, np.zeros((0, 3), np.int32), np.zeros_like(v), np.zeros((0, 3), np.float32), 0.0)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 90), [0.0, 30.0])
    r = native.sweep(m, ypr, PrintOptions())
    o = oracle.sweep(m, ypr, PrintOptions())
    assert _same_bits(r.Mss, o["Mss"]) and _same_bits(r.Mo, o["Mo"]) and r.optID == o["optID"]


def test_wide_mesh_with_raft_on_a_grown_grid(oracle):
    """A footprint wider than 256 columns grows the slot grid; the raft
    window and its scan order stay the reference's."""
    m = meshgen.perturbed_icosphere(4, 150.0, 43, with_hull=False)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 60), [0.0, 45.0, 90.0])
    opts = PrintOptions(explicit_ss=True, bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    r = native.sweep(m, ypr, opts)
    G = native.stats()["grid"]
    assert G > 256
    _compare(r, oracle.sweep(m, ypr, opts, grid=G), "wide raft")


def test_alternating_meshes_keep_their_results():
    a, b = meshgen.small_solid(44), meshgen.solid_82k(45)
    ya = meshgen.ypr_grid(np.arange(0, 360, 30), np.arange(0, 70, 30))
    yb = meshgen.ypr_grid(np.arange(0, 360, 45), [0.0, 60.0])
    ra1 = native.sweep(a, ya, PrintOptions())
    native.sweep(b, yb, PrintOptions(explicit_ss=False))
    ra2 = native.sweep(a, ya, PrintOptions())
    assert _same_bits(ra1.Mss, ra2.Mss) and np.array_equal(ra1.Vss64, ra2.Vss64) and ra1.optID == ra2.optID
    for k in range(11):
        assert np.array_equal(ra1.pixels[k], ra2.pixels[k])


def test_rejected_inputs():
    m = meshgen.small_solid(46)
    ypr = meshgen.ypr_grid([0.0, 90.0], [0.0])
    bad = meshgen.MeshArrays(m.vertices.copy(), m.faces, m.vertex_normals, m.face_normals, m.area)
    bad.vertices[3, 2] = np.nan
    with pytest.raises(native.TomoError, match="non-finite"):
        native.sweep(bad, ypr, PrintOptions())
    yn = ypr.copy()
    yn[1, 0] = np.inf
    with pytest.raises(native.TomoError, match="non-finite orientation"):
        native.sweep(m, yn, PrintOptions())
    with pytest.raises(native.TomoError, match="bad printer parameters"):
        native.sweep(m, ypr, PrintOptions(bed_outer=-1.0))
    f32 = np.zeros(12, np.float32)
    rc = native.lib().TomoSh_CUDA(f32.ctypes.data_as(ct.POINTER(ct.c_float)), None, None, None, None, None, None,
                                  None, None, None)
    assert rc == -1
    # the library stays usable after every rejection
    r = native.sweep(m, ypr, PrintOptions())
    assert r.Mss.size == 2


def test_read_probe():
    """The library's read-bandwidth probe: a positive figure for an
    L2-resident device buffer, refusals for host memory and misalignment."""
    import torch
    buf = torch.zeros(8 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    gbs = native.read_bandwidth(buf.data_ptr(), buf.numel() * 4, reps=4)
    assert gbs > 100.0
    host = np.zeros(1024, np.float32)
    ms = ct.c_float(0.0)
    L = native.lib()
    assert L.tomoProbeReadBandwidth(ct.c_void_p(host.ctypes.data), host.nbytes, 1, ct.byref(ms)) == -1
    assert L.tomoProbeReadBandwidth(ct.c_void_p(buf.data_ptr() + 4), 1024, 1, ct.byref(ms)) == -1
