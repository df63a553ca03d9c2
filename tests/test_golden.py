"""The oracle restatement against the golden fixtures made by the reference
INT3 engine (tests/golden/make_golden.py).  Bit-exact on every output."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from tomo_shell2026_b200.meshgen import MeshArrays
from tomo_shell2026_b200.options import PrintOptions

# per-case sweep fixtures (manager_*.npz belong to the front-end tests)
GOLDEN_DIR = Path(__file__).parent / "golden"
# the small per-case fixtures (the front-end's and the full-size sweeps' have their own layouts)
GOLDEN = sorted(p for p in GOLDEN_DIR.glob("*.npz")
                if not p.name.startswith(("manager_", "mesh_")) and not p.stem.endswith("_full"))


def load_case(path):
    d = dict(np.load(path))
    mesh = MeshArrays(d["vertices"], d["faces"], d["vertex_normals"], d["face_normals"], float(d["area"]))
    f, i = d["f32info"], d["i32info"]
    opts = PrintOptions(dVoxel=float(f[0]), theta_c=float(f[1]), wall_thickness=float(f[3]), Fcore=float(f[4]),
                        Fclad=float(f[5]), Fss=float(f[6]), Css=float(f[7]), PLA_density=float(f[8]),
                        bed_inner=float(f[9]), bed_outer=float(f[10]), bed_thickness=float(f[11]),
                        explicit_ss=bool(i[1]), shell_mesh=bool(i[2]), shell_thickness=float(i[10]) / 1000.0,
                        bed_type=int(i[9]), n_voxel=int(i[3]))
    return d, mesh, opts


def bits(a):
    a = np.asarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a


def test_fixtures_present():
    assert len(GOLDEN) >= 6


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_golden(oracle, path):
    d, mesh, opts = load_case(path)
    f32, i32 = __import__("tomo_shell2026_b200.options", fromlist=["pack_info"]).pack_info(opts, mesh, d["ypr"].shape[0])
    assert np.array_equal(f32.view(np.int32), d["f32info"].view(np.int32)), "info packing differs"
    out = oracle.sweep(mesh, d["ypr"], opts, grid=256, threads=4)
    for k in ("Mo", "Mss", "Vtc", "VoF", "VssF", "Vo64", "Vss64", "Vtc64"):
        assert np.array_equal(bits(out[k]), bits(d[k])), f"{k} differs"
    assert out["optID"] == int(d["optID"])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_columns_match_golden(oracle, path):
    d, mesh, opts = load_case(path)
    c = oracle.columns(mesh, d["ypr"], opts, int(d["col_index"]), grid=256)
    slots = d["col_slots"]
    assert np.array_equal(np.nonzero(c["n_fin"])[0], slots), "occupied columns differ"
    assert np.array_equal(c["n_vox"][slots], d["col_nvox"])
    assert np.array_equal(c["n_fin"][slots], d["col_nfin"])
    assert np.array_equal(c["col_vo"][slots], d["col_vo"])
    assert np.array_equal(c["col_vss"][slots], d["col_vss"])
    rows = np.concatenate([c["fin_tzn"][s, :n] for s, n in zip(slots, d["col_nfin"])], 0)
    assert np.array_equal(rows, d["col_rows"]), "paired column rows differ"
    assert np.array_equal(bits(c["vm22"]), bits(d["vm22"])), "vm_info differs"
    assert np.array_equal(bits(c["mat16"]), bits(d["mat16"])), "mat4x4 differs"
