"""Generate the golden fixtures of the orientation search.

Every fixture is produced by the reference INT3 engine itself -- compiled
from the reference sources into oracle/_ref/libtomo_ref.so by
oracle/build.py -- driven through oracle/oracle.py:RefEngine.  The fixtures
pin both the oracle restatement (tests/test_golden.py, CPU) and the CUDA
path (tests/test_gpu_golden.py).  Inputs are seeded synthetic meshes; the
mesh arrays are stored in the fixture so the fixture alone reproduces the
call.

    python tests/golden/make_golden.py        # needs the reference checkout
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import RefEngine  # noqa: E402
from tomo_shell2026_b200 import meshgen  # noqa: E402
from tomo_shell2026_b200.options import PrintOptions, pack_info  # noqa: E402

OUT = Path(__file__).resolve().parent


def layers_mesh():
    rng = np.random.default_rng(3)
    V, F = [], []
    n = 10
    for L in range(40):
        xs, ys = np.meshgrid(np.linspace(20, 60, n), np.linspace(20, 60, n), indexing="ij")
        zs = 10 + L * 2.3 + 0.8 * np.sin(xs * 0.3 + L) + 0.5 * rng.standard_normal(xs.shape)
        base = len(V)
        V += list(np.stack([xs.ravel(), ys.ravel(), zs.ravel()], 1))
        for i in range(n - 1):
            for j in range(n - 1):
                a = base + i * n + j
                b, c, d = a + 1, a + n, a + n + 1
                F += [(a, c, b), (b, c, d)] if L % 2 else [(a, b, c), (b, d, c)]
    return meshgen.mesh_from_arrays(np.array(V), np.array(F), "layers", with_hull=False)


def cases():
    g10 = meshgen.ypr_grid(np.arange(0, 360, 10), np.arange(0, 190, 10))
    g30 = meshgen.ypr_grid(np.arange(0, 360, 30), np.arange(0, 190, 30))
    g45 = meshgen.ypr_grid(np.arange(0, 360, 45), np.arange(0, 60, 20))
    solid = meshgen.small_solid(0, with_hull=False)
    solid1 = meshgen.small_solid(1, with_hull=False)
    soup = meshgen.random_mesh(1500, 5)
    yield "solid5k_explicit", solid, g10, PrintOptions(explicit_ss=True)
    yield "solid5k_implicit", solid, g10, PrintOptions(explicit_ss=False)
    yield "solid5k_shell_raft", solid1, g30, PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=0.5,
                                                           bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    yield "solid5k_skirt_implicit", solid1, g30, PrintOptions(explicit_ss=False, bed_type=3, bed_inner=1.0,
                                                              bed_outer=3.0, bed_thickness=0.97)
    yield "soup_shell_brim", soup, g30, PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=2.3,
                                                     bed_type=1, bed_outer=2.0, bed_thickness=0.97)
    yield "layers_cap63", layers_mesh(), g45, PrintOptions(explicit_ss=True, shell_mesh=True, bed_type=2,
                                                          bed_outer=2.0, bed_thickness=0.97)


def manager_parts():
    """Two parts for the reference-compatible front-end: a closed solid and
    an open one (its top cap removed), which switches the shell mode on."""
    from tomo_shell2026_b200.cfms_tomo import TriMesh
    a = meshgen.small_solid(2, with_hull=False)
    b = meshgen.small_solid(3, with_hull=False)
    cz = b.vertices[b.faces].mean(1)[:, 2]
    keep = cz < np.quantile(cz, 0.85)
    parts = []
    for name, v, f in (("closed", a.vertices, a.faces), ("open", b.vertices, b.faces[keep])):
        m = meshgen.mesh_from_arrays(v, f, name, with_hull=False)
        parts.append(TriMesh(m.vertices.astype(np.float64), m.faces, vertex_normals=m.vertex_normals,
                             process=False, name=name))
    return parts


def make_manager(ref):
    """TomoManager over the two parts, evaluated by the reference engine with
    exactly the arrays TomoDLLInterface packs (theta_YP = 30: 13 x 13 YPR)."""
    from tomo_shell2026_b200.cfms_tomo import SlicingOptions, TomoDLLInterface
    s_o = SlicingOptions()
    s_o.theta_YP = 30
    s_o.bVerbose = False
    itf = TomoDLLInterface("Tomo_Shell2026.dll", s_o, True, True)
    out = {"YPR": itf.YPR}
    for k, tm in enumerate(manager_parts()):
        itf.bShellMesh = s_o.bShellMesh and not tm.is_watertight
        itf.pack(tm, itf.YPR.shape[0], False)
        info = (itf.Float32Info.copy(), itf.Int32Info.copy())
        arrays = tm.to_arrays(with_hull=True)
        sw = ref.sweep(arrays, itf.YPR, info, grid=256, threads=8)
        ex = ref.pixels(arrays, itf.YPR, info, int(sw["optID"]), grid=256)
        out.update({f"p{k}_vertices": arrays.vertices, f"p{k}_faces": arrays.faces,
                    f"p{k}_vertex_normals": arrays.vertex_normals, f"p{k}_f32info": info[0], f"p{k}_i32info": info[1],
                    f"p{k}_Mss": sw["Mss"], f"p{k}_Mo": sw["Mo"], f"p{k}_optID": np.int32(sw["optID"]),
                    f"p{k}_SS": ex["pixels"][4], f"p{k}_Bed": ex["pixels"][5], f"p{k}_mat16": ex["mat16"]})
    itf.free()
    np.savez_compressed(OUT / "manager_two_parts.npz", **out)
    print(f"manager_two_parts: {itf.YPR.shape[0]} orientations per part, "
          f"{(OUT / 'manager_two_parts.npz').stat().st_size / 1024:.0f} KB")


def main():
    ref = RefEngine()
    make_manager(ref)
    for name, mesh, ypr, opts in cases():
        f32, i32 = pack_info(opts, mesh, ypr.shape[0])
        out = ref.sweep(mesh, ypr, opts, grid=256, threads=8)
        # one orientation's per-column state, compactly: occupied slots only
        idx = int(out["optID"])
        d = ref.columns(mesh, ypr, opts, idx, grid=256)
        occ = np.nonzero(d["n_fin"])[0].astype(np.int32)
        rows = [d["fin_tzn"][s, : d["n_fin"][s]] for s in occ]
        off = np.concatenate([[0], np.cumsum([r.shape[0] for r in rows])]).astype(np.int32)
        ex = ref.pixels(mesh, ypr, opts, idx, grid=256)
        pcount = np.array([px.shape[0] for px in ex["pixels"]], np.int32)
        np.savez_compressed(
            OUT / f"{name}.npz",
            pix_count=pcount, pix_data=np.concatenate(ex["pixels"], 0).astype(np.int16), pix_vm22=ex["vm22"],
            f32info=f32, i32info=i32, ypr=ypr, vertices=mesh.vertices, faces=mesh.faces,
            vertex_normals=mesh.vertex_normals, face_normals=mesh.face_normals, area=np.float64(mesh.area),
            Mo=out["Mo"], Mss=out["Mss"], Vtc=out["Vtc"], VoF=out["VoF"], VssF=out["VssF"],
            Vo64=out["Vo64"], Vss64=out["Vss64"], Vtc64=out["Vtc64"], optID=np.int32(out["optID"]),
            col_index=np.int32(idx), col_slots=occ, col_nvox=d["n_vox"][occ], col_nfin=d["n_fin"][occ],
            col_vo=d["col_vo"][occ], col_vss=d["col_vss"][occ], col_rows=np.concatenate(rows, 0).astype(np.int16),
            col_off=off, vm22=d["vm22"], mat16=d["mat16"])
        print(f"{name}: {ypr.shape[0]} orientations, optID {out['optID']}, "
              f"{(OUT / (name + '.npz')).stat().st_size / 1024:.0f} KB")


if __name__ == "__main__":
    main()
