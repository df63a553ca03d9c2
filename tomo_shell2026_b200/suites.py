"""Workload suites beyond the single-mesh sweep: many uneven meshes in one
batched launch, and the learned-proposal search over many meshes.

``batched_suite`` -- seeded meshes with triangle counts log-uniform in
[t_min, t_max], half from the small-solid generator (r = 50 mm, 1 mm
voxels, spherical harmonics of degree <= 3, amplitude 0.15) and half from
the 82k-solid generator (r = 80 mm, 0.5 mm voxels, degree <= 8, amplitude
0.25, 4 bumps/dents), each on the 1-degree yaw x pitch 0-60 grid.  All
meshes are swept in one captured graph (``native.Batch``) and, for
comparison, one by one (``native.Session``); every mesh's results must be
bit-identical between the two.

``surrogate_suite`` -- small-solid meshes on the 0.5-degree grid
(yaw 0-359.5 x pitch 0-60, 720 x 121 = 87,120 orientations): the exhaustive
device sweep against ``surrogate.search`` (5-degree coarse points, 2.5-degree
proposal blocks).

``shell_suite`` -- the thin open shell (manikin-like union surface, openings,
2 mm inward wall; shell mode, 1 mm voxels) on the 1-degree yaw x pitch 0-60
grid: device orientations/s of the full sweep.

All return plain dicts of aggregate figures (times in seconds, device time
from CUDA events for the sweeps, wall time for the search call).
"""
from __future__ import annotations

import math

import numpy as np

from . import meshgen, native, surrogate
from .options import PrintOptions


def uneven_meshes(n: int, seed: int = 0, t_min: int = 1000, t_max: int = 120000):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        t = int(round(math.exp(rng.uniform(math.log(t_min), math.log(t_max)))))
        if k % 2 == 0:
            m = meshgen.perturbed_sphere(t, 50.0, seed * 1000 + k, with_hull=False)
        else:
            m = meshgen.perturbed_sphere(t, 80.0, seed * 1000 + k, n_harmonics=12, max_degree=8, amplitude=0.25,
                                         n_bumps=4, scale=2.0, with_hull=False)
        out.append(m)
    return out


def batched_suite(n_meshes: int = 64, seed: int = 0, yaw_step: float = 1.0, pitch_max: float = 60.0,
                  t_min: int = 1000, t_max: int = 120000) -> dict:
    meshes = uneven_meshes(n_meshes, seed, t_min, t_max)
    ypr = meshgen.ypr_grid(np.arange(0, 360, yaw_step), np.arange(0, pitch_max + 1e-9, yaw_step))
    opts = PrintOptions(explicit_ss=True)
    plain_s, plain = 0.0, []
    for m in meshes:
        s = native.Session(m, ypr, opts)
        s.run_device()                              # warm (allocations)
        plain_s += s.run_device() / 1000.0
        opt, _, mss, _ = s.finish()
        plain.append((opt, mss.copy(), native.results(ypr.shape[0])["Vss64"].copy()))
    b = native.Batch(meshes, [ypr] * len(meshes), opts, autotune=True)
    b.run(use_graph=True)                           # capture + first replay
    # sweep (graph replay) and the re-runs of flagged orientations, until
    # every mesh is resolved -- the same span Session.run_device times
    batched_s = b.run(use_graph=True) / 1000.0
    exact = 0
    for k, (opt, mss, vss) in enumerate(plain):
        r = b.results(k)
        exact += int(r["optID"] == opt and np.array_equal(r["Mss"].view(np.int32), mss.view(np.int32))
                     and np.array_equal(r["Vss64"], vss))
    st = native.Batch.stats()
    native.Batch.release()
    n_or = len(meshes) * ypr.shape[0]
    tris = [m.n_tri for m in meshes]
    return {"meshes": len(meshes), "orientations": n_or, "triangles_min": int(min(tris)),
            "triangles_max": int(max(tris)), "batched_s": batched_s, "plain_s": plain_s,
            "batched_orientations_per_s": n_or / batched_s, "plain_orientations_per_s": n_or / plain_s,
            "batched_triangle_orientations_per_s": sum(tris) * ypr.shape[0] / batched_s,
            "bit_exact_meshes": exact, "graph_nodes": st["graph_nodes"], "graph_kernels": st["graph_kernels"],
            "size_classes_tuned": st["tuned_total"], "reruns": st["reruns"],
            "rerun_fraction": st["reruns"] / max(n_or, 1), "graph_replay_s": st["graph_us"] / 1e6,
            "timing": "device time on the library stream (CUDA events) from the first kernel until every mesh is "
                      "resolved, re-runs included, on both sides"}


def block_rank(score: np.ndarray, target: int, n_yaw: int, n_pitch: int, cell: int) -> int:
    """Rank (0 = first) of the block holding grid point `target` when blocks
    are ordered by their smallest score."""
    ncy = (n_yaw + cell - 1) // cell
    ids = np.arange(score.size)
    blk = (ids % n_yaw) // cell + ((ids // n_yaw) // cell) * ncy
    bmin = np.full(blk.max() + 1, np.inf)
    np.minimum.at(bmin, blk, score)
    order = np.argsort(bmin, kind="stable")
    return int(np.nonzero(order == blk[target])[0][0])


def coarse_interpolation(vss: np.ndarray, n_yaw: int, n_pitch: int, stride: int) -> np.ndarray:
    """The method without the network: exact Vss of the coarse points,
    bilinearly interpolated onto the grid (yaw periodic)."""
    g = vss.reshape(n_pitch, n_yaw).astype(np.float64)
    cy = np.arange(0, n_yaw, stride)
    cp = np.arange(0, n_pitch, stride)
    c = g[np.ix_(cp, cy)]
    fy = np.arange(n_yaw) / stride
    fp = np.minimum(np.arange(n_pitch) / stride, len(cp) - 1)
    y0 = np.floor(fy).astype(int) % len(cy)
    y1 = (y0 + 1) % len(cy)
    wy = fy - np.floor(fy)
    p0 = np.floor(fp).astype(int)
    p1 = np.minimum(p0 + 1, len(cp) - 1)
    wp = fp - p0
    rows = c[p0][:, y0] * (1 - wy) + c[p0][:, y1] * wy
    rows1 = c[p1][:, y0] * (1 - wy) + c[p1][:, y1] * wy
    return ((1 - wp)[:, None] * rows + wp[:, None] * rows1).ravel()


def surrogate_suite(n_meshes: int = 100, seed0: int = 1000, stride: int = 10, cell: int = 5, top_k: int = 64,
                    steps: int = 300, ratio_target: float = 0.2, margin: float = 1.0, holdout: float = 0.0,
                    lr: float = 3e-3, max_eval: int = -1, log_scale: float = 0.3, ablation: bool = True) -> dict:
    """The learned-proposal search against the exhaustive sweep on the same
    meshes, and (``ablation``) the same search without the network -- blocks
    ranked by a bilinear interpolation of the exact coarse values -- so the
    network's gain is measured on identical inputs.

    Clocks: ``exhaustive_s`` is device time (CUDA events on the library's
    stream around tomoSweepDevice: the whole 0.5-degree sweep, re-runs and
    result fetch, mesh already uploaded); ``search_s`` is host wall-clock time
    around the tomoSurrogateSearch call (upload, coarse sweep, training,
    prediction, refinement rounds, result fetch)."""
    ypr = meshgen.ypr_grid(np.arange(0, 360, 0.5), np.arange(0, 60.5, 0.5))
    n_yaw, n_pitch = 720, 121
    opts = PrintOptions(explicit_ss=True)
    kw = dict(stride=stride, cell=cell, top_k=top_k, steps=steps, margin=margin, holdout=holdout, lr=lr,
              max_eval=max_eval, log_scale=log_scale)
    kinds = ("network", "interpolation") if ablation else ("network",)
    rows = []
    # one untimed search of each kind first: first-call costs (allocations, kernel loading)
    warm = meshgen.small_solid(seed0 - 1, with_hull=False)
    for kind in kinds:
        surrogate.search(warm, ypr, n_yaw, n_pitch, opts, proposal=kind, **kw)
    for k in range(n_meshes):
        m = meshgen.small_solid(seed0 + k, with_hull=False)
        s = native.Session(m, ypr, opts)
        s.run_device()
        ex_s = s.run_device() / 1000.0
        opt, _, mss, _ = s.finish()
        row = dict(exhaustive_s=ex_s)
        for kind in kinds:
            r = surrogate.search(m, ypr, n_yaw, n_pitch, opts, seed=k, proposal=kind, **kw)
            row[kind] = dict(same_value=bool(np.float32(r.Mss[r.optID]) == mss[opt]), same_index=r.optID == opt,
                             ratio=r.seconds / ex_s, search_s=r.seconds, evaluated=r.evaluated,
                             fallback=r.fallback, rel_error=r.rel_error, max_abs_error=r.max_abs_error,
                             rank=block_rank(r.pred_vss, opt, n_yaw, n_pitch, cell))
        rows.append(row)

    def summary(kind):
        xs = [r[kind] for r in rows]
        ok = [x["same_value"] and x["ratio"] <= ratio_target for x in xs]
        return {"optimum_recall": float(np.mean([x["same_value"] for x in xs])),
                "same_index": float(np.mean([x["same_index"] for x in xs])),
                "fallbacks": int(sum(x["fallback"] for x in xs)),
                "meshes_at_target": float(np.mean(ok)),
                "median_time_ratio": float(np.median([x["ratio"] for x in xs])),
                "p95_time_ratio": float(np.percentile([x["ratio"] for x in xs], 95)),
                "median_search_s": float(np.median([x["search_s"] for x in xs])),
                "median_evaluated": float(np.median([x["evaluated"] for x in xs])),
                "mean_evaluated": float(np.mean([x["evaluated"] for x in xs])),
                "median_rel_error": float(np.median([x["rel_error"] for x in xs])),
                "median_max_abs_error": float(np.median([x["max_abs_error"] for x in xs])),
                "optimum_block_in_top_k": float(np.mean([x["rank"] < top_k for x in xs])),
                "median_optimum_block_rank": float(np.median([x["rank"] for x in xs])),
                "mean_optimum_block_rank": float(np.mean([x["rank"] for x in xs]))}

    out = {"meshes": n_meshes, "grid": [n_yaw, n_pitch], "orientations": int(ypr.shape[0]),
           "coarse_deg": stride * 0.5, "cell_deg": cell * 0.5, "margin": margin, "holdout": holdout,
           "train_steps": steps, "learning_rate": lr, "max_eval": max_eval, "log_scale": log_scale,
           "ratio_target": ratio_target,
           "median_exhaustive_s": float(np.median([r["exhaustive_s"] for r in rows])),
           "clocks": {"exhaustive": "device time, CUDA events around tomoSweepDevice (sweep, re-runs, result fetch)",
                      "search": "host wall clock around tomoSurrogateSearch (everything from upload to results)"}}
    out.update(summary("network"))
    if ablation:
        out["without_network"] = summary("interpolation")
        ev_net = np.array([r["network"]["evaluated"] for r in rows], np.float64)
        ev_wo = np.array([r["interpolation"]["evaluated"] for r in rows], np.float64)
        out["network_gain"] = {
            "evaluations_saved_mean": float(np.mean(ev_wo - ev_net)),
            "evaluations_ratio_median": float(np.median(ev_net / np.maximum(ev_wo, 1))),
            "meshes_fewer_evaluations": float(np.mean(ev_net < ev_wo)),
            "time_ratio_median": float(np.median([r["network"]["search_s"] / r["interpolation"]["search_s"]
                                                  for r in rows]))}
    return out


def shell_suite(seed: int = 0) -> dict:
    m = meshgen.manikin_shell(seed)
    ypr = meshgen.ypr_grid(np.arange(0, 360), np.arange(0, 61))
    opts = PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=0.5)
    s = native.Session(m, ypr, opts)
    s.run_device()
    sec = s.run_device() / 1000.0
    opt, _, _, _ = s.finish()
    st = native.stats()
    r = native.results(ypr.shape[0])
    return {"mesh": "manikin-like open shell, union of 9 ellipsoids/capsules, 2 mm wall", "triangles": m.n_tri,
            "orientations": int(ypr.shape[0]), "seconds": sec, "orientations_per_s": ypr.shape[0] / sec,
            "triangle_orientations_per_s": m.n_tri * ypr.shape[0] / sec, "slot_grid": st["grid"],
            "strip_h": st["strip_h"], "entries_per_orientation": float(r["entries"].mean()),
            "overflow_reruns": st["overflow_reruns"], "safe_reruns": st["safe_reruns"], "optID": int(opt)}
