"""The C-ABI library on the CPU: it loads, exports every symbol declared in
include/tomo_b200.h, its host-side arithmetic is pinned to the reference,
and without a GPU its entry points fail with an error code instead of
crashing or falling back to the CPU."""
from __future__ import annotations

import ctypes as ct
import re
from pathlib import Path

import numpy as np
import pytest

from tomo_shell2026_b200 import meshgen, native
from tomo_shell2026_b200.options import PrintOptions, pack_info

HEADER = Path(__file__).resolve().parents[1] / "include" / "tomo_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_header_declares_reference_exports():
    names = declared_functions()
    for ref in ("TomoSh_CUDA", "getMss", "getMo", "getVtc", "getVolMassInfo", "getMat4x4", "getnData2i",
                "getpData2i", "OnDestroy"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    lib = ct.CDLL(str(native.library_path()))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    bound = {name for name, _, _ in native.EXPORTS}
    assert set(declared_functions()) <= bound, "native.EXPORTS lacks a declared function"


def test_option_keys_match_the_header():
    """The option keys native.py passes to tomoSetOption are the header's."""
    text = HEADER.read_text()
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(TOMO_\w+)\s+(-?\d+)", text)}
    opts = {k: v for k, v in defines.items() if k.startswith("TOMO_OPT_")}
    assert opts, "no TOMO_OPT_ keys in the header"
    for name, value in opts.items():
        assert getattr(native, name) == value, f"native.{name} != {value}"
    assert len(set(opts.values())) == len(opts), "option keys collide"


def bits(a):
    a = np.asarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a


def test_host_rotation_matches_reference(oracle, ref_engine):
    rng = np.random.default_rng(1)
    grid = np.deg2rad(np.arange(0, 361, 1.0)).astype(np.float32)
    for y in grid:
        for p_ in grid[::15]:
            assert np.array_equal(bits(native.rotation(y, p_, 0.0)), bits(ref_engine.rotation(y, p_, 0.0)))
    for y, p_, r in rng.uniform(-10, 10, (500, 3)).astype(np.float32):
        assert np.array_equal(bits(native.rotation(y, p_, r)), bits(oracle.rotation(y, p_, r)))


def test_host_threshold_and_mass(oracle):
    for deg in (0.0, 30.0, 45.0, 60.0, 72.5, 89.9):
        th = np.float32(deg * np.pi / 180)
        assert bits(native.shadow_threshold(th)) == bits(oracle.threshold(th))
    rng = np.random.default_rng(2)
    m = meshgen.small_solid(0, with_hull=False)
    for explicit in (True, False):
        f32, i32 = pack_info(PrintOptions(explicit_ss=explicit), m, 10)
        for _ in range(200):
            vm = np.zeros(22, np.float32)
            vm[4] = np.float32(rng.choice([0.0, 0.0005, 1.0, rng.uniform(0, 3e7)]))
            vm[8] = np.float32(rng.uniform(0, 5e7))
            vm[11] = np.float32(rng.uniform(0, 1e4))
            assert np.array_equal(bits(native.vol_to_mass(f32, i32, vm)), bits(oracle.vol_to_mass(f32, i32, vm)))


def test_info_layout_matches_reference_order():
    m = meshgen.small_solid(0, with_hull=True)
    opts = PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=0.5, bed_type=2, bed_inner=0.0,
                        bed_outer=2.0, bed_thickness=0.97, verbose=True)
    f32, i32 = pack_info(opts, m, 77)
    assert f32.dtype == np.float32 and f32.shape == (12,)
    assert i32.dtype == np.int32 and i32.shape == (11,)
    assert list(i32) == [1, 1, 1, 256, m.n_tri, m.n_vtx, 77, m.hull_faces.shape[0], m.hull_vertices.shape[0], 2, 500]
    assert f32[2] == np.float32(m.area) and f32[10] == np.float32(2.0) and f32[11] == np.float32(0.97)


def test_ypr_grid_layout():
    ypr = meshgen.ypr_grid([0, 10, 20], [0, 5])
    assert ypr.shape == (6, 3) and ypr.dtype == np.float32
    assert np.allclose(np.rad2deg(ypr[:, 0]), [0, 10, 20, 0, 10, 20], atol=1e-4)   # yaw fastest
    assert np.allclose(np.rad2deg(ypr[:, 1]), [0, 0, 0, 5, 5, 5], atol=1e-4)


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU error path")
def test_sweep_without_gpu_fails_loudly():
    m = meshgen.small_solid(0, with_hull=False)
    ypr = meshgen.ypr_grid([0, 90], [0])
    with pytest.raises(native.TomoError, match="CUDA"):
        native.sweep(m, ypr, PrintOptions())
    assert native.lib().tomoGetLastError() == -2
