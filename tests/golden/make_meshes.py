"""Golden fixtures on the reference's own mesh files.

Each fixture holds the mesh arrays exactly as the engines consume them --
read from the reference checkout's MeshData by the trimesh-free loaders of
tomo_shell2026_b200.cfms_tomo (PLY, STL, glTF), so the GPU host needs no
mesh file -- and the outputs of the reference INT3 engine (compiled from the
reference sources, oracle/_ref/libtomo_ref.so) on the 10-degree grid
(yaw 0..350 x pitch 0..180, 684 orientations) for a few printer setups:
explicit and implicit support, shell mode for the open meshes, and a raft.

Real geometry brings what the seeded solids do not: degenerate and
sub-pixel triangles (centroid fallbacks), open borders, and uneven triangle
sizes.

    python tests/golden/make_meshes.py     # needs the reference checkout
"""
from __future__ import annotations

import json
import os
import sys
from dataclasses import asdict
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from tomo_shell2026_b200 import meshgen  # noqa: E402
from tomo_shell2026_b200.options import PrintOptions  # noqa: E402

OUT = Path(__file__).resolve().parent
YAW = np.arange(0, 360, 10)
PITCH = np.arange(0, 190, 10)

# (fixture name, file under MeshData, scale to millimetres)
MESHES = [
    ("mesh_manikin_ply", "(3)manikin.ply", 1.0),
    ("mesh_bunny_stl", "Bunny_69k.stl", 1.0),
    ("mesh_body_gltf", "SK6th_M20_87k_NoFinger.gltf", 10000.0),
    ("mesh_sphere_ply", "(1)sphere.ply", 1.0),
]


def variants(shell: bool):
    """Printer setups evaluated per mesh (shell mode follows the mesh's
    watertightness, as TomoManager sets it)."""
    yield "explicit", PrintOptions(explicit_ss=True, shell_mesh=shell)
    yield "implicit", PrintOptions(explicit_ss=False, shell_mesh=shell)
    yield "raft", PrintOptions(explicit_ss=True, shell_mesh=shell, bed_type=2, bed_outer=2.0, bed_thickness=0.97)


def load_arrays(ref_root: Path, filename: str, scale: float):
    from tomo_shell2026_b200.cfms_tomo import load
    tm = load(ref_root / "MeshData" / filename)
    m = tm.to_arrays(with_hull=False)
    if scale != 1.0:
        m = meshgen.mesh_from_arrays(m.vertices.astype(np.float64) * scale, m.faces, filename, with_hull=False)
    return m, bool(tm.is_watertight)


def main():
    from oracle.build import REF_ROOT
    from oracle.oracle import RefEngine
    ref = RefEngine()
    threads = os.cpu_count() or 1
    ypr = meshgen.ypr_grid(YAW, PITCH)
    for name, filename, scale in MESHES:
        m, watertight = load_arrays(REF_ROOT, filename, scale)
        out = dict(source=np.array(f"MeshData/{filename} x {scale:g}"), watertight=np.bool_(watertight),
                   vertices=m.vertices, faces=m.faces, vertex_normals=m.vertex_normals,
                   face_normals=m.face_normals, area=np.float64(m.area),
                   yaw_deg=YAW.astype(np.int32), pitch_deg=PITCH.astype(np.int32))
        tags = []
        for tag, opts in variants(shell=not watertight):
            r = ref.sweep(m, ypr, opts, grid=256, threads=threads)
            tags.append(tag)
            out[f"{tag}_options"] = np.array(json.dumps(asdict(opts)))
            for k in ("Vo64", "Vss64", "Vtc64", "VoF", "VssF", "Mo", "Mss", "Vtc"):
                out[f"{tag}_{k}"] = r[k]
            out[f"{tag}_optID"] = np.int32(r["optID"])
        out["variants"] = np.array(tags)
        np.savez_compressed(OUT / f"{name}.npz", **out)
        print(f"{name}: {m.n_tri} triangles, watertight {watertight}, "
              f"{(OUT / (name + '.npz')).stat().st_size / 1024:.0f} KB", flush=True)


if __name__ == "__main__":
    main()
