"""Full-size golden fixtures: whole 1-degree sweeps of the two large workloads.

The reference INT3 engine (oracle/_ref/libtomo_ref.so, compiled from the
reference sources by oracle/build.py) runs every orientation of

* ``solid82k_full``  -- the 81,920-triangle solid (icosphere subdivision 6,
  r = 80 mm, SH degree <= 8 at amplitude 0.25 plus 4 Gaussian bumps/dents),
  0.5 mm voxels, explicit support, yaw 0..359 x pitch 0..60 at 1 degree
  (21,960 orientations);
* ``manikin_full``   -- the manikin-like thin open shell (~88k triangles,
  openings, 2 mm inward wall), shell mode at 0.5 mm shell thickness, 1 mm
  voxels, the same 21,960-orientation grid.

The meshes are not stored: both are regenerated from their seeds by
tomo_shell2026_b200.meshgen, and the fixture keeps a SHA-256 of the exact
arrays handed to the engine so a test can prove it regenerated the same
bytes.  Stored per orientation: the exact int64 Vo / Vss / Vtc, the float32
accumulators VoF / VssF and the exported Mo / Mss / Vtc, plus optID (the
reference's first strict argmin of Mss, Tomo_Shell2026.cpp:89-97).

    python tests/golden/make_fullsize.py [solid82k_full|manikin_full ...]

needs the reference checkout and takes roughly 7 + 17 minutes on 8 host
threads.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from tomo_shell2026_b200 import meshgen  # noqa: E402
from tomo_shell2026_b200.options import PrintOptions  # noqa: E402

OUT = Path(__file__).resolve().parent

YAW = np.arange(0, 360, 1)
PITCH = np.arange(0, 61, 1)


def mesh_sha256(mesh) -> str:
    h = hashlib.sha256()
    for a in (np.ascontiguousarray(mesh.vertices, np.float32), np.ascontiguousarray(mesh.faces, np.int32),
              np.ascontiguousarray(mesh.vertex_normals, np.float32), np.float64(mesh.area)):
        h.update(np.asarray(a).tobytes())
    return h.hexdigest()


def slot_grid(vertices, bed_outer: float = 0.0) -> int:
    """Slot-grid edge the library picks for a mesh: 256 when the rotated mesh
    fits, else its bounding-sphere span plus margins (a grid large enough
    for every orientation changes no result)."""
    v = np.asarray(vertices, np.float32)
    c = ((v.min(0) + v.max(0)).astype(np.float64) * 0.5).astype(np.float32).astype(np.float64)
    r2 = ((v.astype(np.float64) - c) ** 2).sum(1).max()
    span = 2.0 * np.sqrt(r2) * 1.004 + max(0.0, bed_outer) + 6.0
    return 256 if span <= 256.0 else int(span) + int(max(0.0, bed_outer)) + 2


def cases():
    """(name, mesh factory, options, description) of each full-size fixture."""
    yield ("solid82k_full", lambda: meshgen.solid_82k(0, with_hull=False), PrintOptions(explicit_ss=True),
           "solid_82k(0), 0.5 mm (coordinates x2), explicit support, theta_c 60, no bed")
    yield ("manikin_full", lambda: meshgen.manikin_shell(0),
           PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=0.5),
           "manikin_shell(0), 1 mm, shell mode (shell thickness 0.5), explicit support, no bed")


def make(name, factory, opts, desc, ref, threads):
    mesh = factory()
    ypr = meshgen.ypr_grid(YAW, PITCH)
    G = slot_grid(mesh.vertices, opts.bed_outer)
    t0 = time.time()
    out = ref.sweep(mesh, ypr, opts, grid=G, threads=threads)
    dt = time.time() - t0
    np.savez_compressed(
        OUT / f"{name}.npz",
        mesh_sha256=np.array(mesh_sha256(mesh)), description=np.array(desc), grid=np.int32(G),
        yaw_deg=YAW.astype(np.int32), pitch_deg=PITCH.astype(np.int32),
        Vo64=out["Vo64"], Vss64=out["Vss64"], Vtc64=out["Vtc64"], VoF=out["VoF"], VssF=out["VssF"],
        Mo=out["Mo"], Mss=out["Mss"], Vtc=out["Vtc"], optID=np.int32(out["optID"]),
        ref_seconds=np.float64(dt), ref_threads=np.int32(threads))
    print(f"{name}: {ypr.shape[0]} orientations on grid {G}, optID {out['optID']}, {dt:.0f} s on {threads} threads, "
          f"{(OUT / (name + '.npz')).stat().st_size / 1024:.0f} KB", flush=True)


def main(names):
    from oracle.oracle import RefEngine
    ref = RefEngine()
    threads = os.cpu_count() or 1
    for name, factory, opts, desc in cases():
        if names and name not in names:
            continue
        make(name, factory, opts, desc, ref, threads)


if __name__ == "__main__":
    main(sys.argv[1:])
