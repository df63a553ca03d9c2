#!/usr/bin/env python
"""Throughput of the exhaustive orientation search on B200.

Workload (one "step" = one full sweep): the 82k-triangle solid -- icosphere
subdivision 6 (81,920 triangles), r = 80 mm, radial spherical-harmonic
perturbation (degree <= 8, amplitude 0.25) plus 4 Gaussian bumps/dents
(sigma 10 mm, +-20 mm), seeded -- at 0.5 mm voxels (coordinates x2), over
yaw 0..359 x pitch 0..60 at 1 degree (21,960 orientations), explicit support
shadows, theta_c = 60 degrees, no bed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value`` is orientations/s of the device
sweep with mesh and orientations resident in device memory (CUDA events on
the engine's stream); ``e2e`` is the same metric through the reference
C-ABI call TomoSh_CUDA with host buffers; ``roofline`` rates the dominant
kernel (k_strip) against the measured HBM copy bandwidth; ``cpu_baseline``
is the reference INT3 engine (built from the reference sources) on the
host cores over a bounded sample of the same orientations.  With N > 1
(torchrun) the ranks split the one headline sweep into contiguous
orientation shards (strong scaling: the total work is the same at every N)
and combine the optimum with one MIN all-reduce; nothing else crosses ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "orientations/s & time-to-exact-optimum, 82k-tri mesh 1deg grid, batched vs plain"
UNIT = "orientations/s"
YAW = np.arange(0, 360, 1)
PITCH = np.arange(0, 61, 1)
L2_BYTES = 126 * 1024 * 1024


def workload(seed: int, max_orientations: int = 0):
    from tomo_shell2026_b200 import meshgen
    from tomo_shell2026_b200.options import PrintOptions
    mesh = meshgen.solid_82k(seed)
    ypr = meshgen.ypr_grid(YAW, PITCH)
    if max_orientations > 0:
        ypr = np.ascontiguousarray(ypr[:max_orientations])
    opts = PrintOptions(explicit_ss=True)
    return mesh, ypr, opts


def config(mesh, ypr, grid=None, extra=None):
    c = {"workload": "solid82k_1deg", "mesh": f"icosphere s6 {mesh.n_tri} tris, SH deg<=8 amp 0.25 + 4 bumps",
         "orientations": int(ypr.shape[0]), "grid_yaw_pitch": "yaw 0..359 x pitch 0..60 step 1 deg",
         "voxel_mm": 0.5, "shadow": "explicit", "theta_c_deg": 60, "bed": "none",
         "l2": "per-step working set (GBs of column lists and fold values) exceeds the 126 MB L2; "
               "a 256 MB buffer is also written between timed steps"}
    if grid is not None:
        c["slot_grid"] = int(grid)
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        mhz, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not mhz:
            return None
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(mhz)}


# ------------------------------------------------------------------ CPU baseline

def cpu_baseline(mesh, ypr, opts, grid, budget_s: float, gpu_vss=None, threads: int | None = None,
                 n: int | None = None, gpu_mss=None):
    """The reference INT3 engine (oracle/_ref, built from the reference sources)
    -- or, if that library is absent, the oracle's C restatement -- on an
    evenly strided sample of the workload's orientations, all host threads."""
    from oracle import build as ob
    from oracle.oracle import Oracle, RefEngine
    threads = threads or os.cpu_count() or 1
    # every reference worker owns a grid x grid x 64 x 3 int16 slot buffer
    # (cpu_src/STomoVoxelSpaceInfo.cpp:137-150); keep them within half the RAM
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
        per_thread = grid * grid * 64 * 3 * 2 + 64 * 1024 * 1024
        threads = max(1, min(threads, int(0.5 * avail // per_thread)))
    except (ValueError, OSError):
        pass
    kind = "reference"
    try:
        eng = RefEngine(ob.REF_LIB) if ob.REF_LIB.exists() else None
    except OSError:
        eng = None
    if eng is None:
        eng, kind = Oracle(), "port"
    n_all = ypr.shape[0]
    # grow a strided sample until one call takes at least half the budget
    # (a call's fixed cost -- threads and their slot buffers -- makes small
    # samples look slow, so the size is re-estimated from each larger call)
    fixed = n is not None
    n = min(n_all, n if fixed else max(threads, 8))
    while True:
        idx = np.linspace(0, n_all - 1, n).astype(np.int64)
        t0 = time.perf_counter()
        out = eng.sweep(mesh, ypr[idx], opts, grid=grid, threads=threads)
        dt = time.perf_counter() - t0
        if fixed or dt >= 0.5 * budget_s or n >= n_all:
            break
        n = int(min(n_all, max(2 * n, n * budget_s / max(dt, 1e-6))))
        n = min(n_all, max(threads, (n // threads) * threads))
    res = {"value": n / dt, "unit": UNIT, "cores": int(threads), "kind": kind, "n": n,
           "sample": f"{n} of the {n_all} orientations, evenly strided, one call, {dt:.1f} s"}
    if gpu_vss is not None and "Vss64" in out:
        res["sample_vss_bit_identical"] = bool(np.array_equal(out["Vss64"], gpu_vss[idx]))
    if gpu_mss is not None and "Mss" in out:
        res["sample_mss_bit_identical"] = bool(np.array_equal(np.asarray(out["Mss"], np.float32).view(np.int32),
                                                              np.asarray(gpu_mss, np.float32)[idx].view(np.int32)))
    return res


# ------------------------------------------------------------------ arms

def run_reference(args, rank):
    if rank != 0:
        return 0
    mesh, ypr, opts = workload(0, args.max_orientations)
    from tomo_shell2026_b200.meshgen import MeshArrays  # noqa: F401
    grid = _grid_for(mesh)
    # the first warm-up step sizes the sample (about ref_step_s of CPU work);
    # every later step evaluates that same sample
    n = None
    for _ in range(max(1, args.warmup)):
        n = cpu_baseline(mesh, ypr, opts, grid, budget_s=args.ref_step_s, n=n)["n"]
    vals = []
    last = None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        last = cpu_baseline(mesh, ypr, opts, grid, budget_s=args.ref_step_s, n=n)
        vals.append(last["value"])
    wall = time.perf_counter() - t0
    v = float(statistics.median(vals))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall * 1000 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "impl": "reference", "config": config(mesh, ypr, grid),
            "cpu_baseline": {k: last[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _grid_for(mesh):
    """Slot grid edge the engine picks for this mesh (host-side rule, same as the library)."""
    v = mesh.vertices
    mn, mx = v.min(0), v.max(0)
    c = ((mn + mx).astype(np.float32) * np.float32(0.5)).astype(np.float64)
    r = np.sqrt(((v.astype(np.float64) - c) ** 2).sum(1).max())
    span = 2.0 * r * 1.004 + 6.0
    return 256 if span <= 256.0 else int(span) + 2


def run_ours(args, rank, world, local_rank):
    import torch
    from tomo_shell2026_b200 import native

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    from tomo_shell2026_b200 import sharding
    mesh, ypr_all, opts = workload(0, args.max_orientations)
    n = ypr_all.shape[0]
    b, e = sharding.shard_range(n, rank, world)
    ypr = np.ascontiguousarray(ypr_all[b:e])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    sess = native.Session(mesh, ypr, opts)
    grid = sess.grid()
    for _ in range(args.warmup):
        sess.run_device()
        flush.zero_()
    torch.cuda.synchronize()

    # ---- value: device sweep, inputs resident
    native.profile(True, reset=True)
    phys = _physical_gpu(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = []
    with ClockSampler(phys) as clk:
        for _ in range(args.steps):
            step_ms.append(sess.run_device())
            flush.zero_()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    klog = native.kernel_log()
    native.profile(False, reset=False)
    res = native.results(e - b)
    opt, Mo, Mss, Vtc = sess.finish()
    if dist:
        opt = sharding.global_first_optimal(Mss, b, n)
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = args.steps * n / (total_ms / 1000.0)

    # ---- e2e: reference C-ABI with host buffers (H2D + D2H inside); with
    # N > 1 each rank's TomoSh_CUDA call sweeps its shard and the optimum is
    # combined across ranks inside the timed region
    for _ in range(args.warmup):
        sharding.sweep_shard(mesh, ypr_all, opts)
    e2e_s = []
    for _ in range(max(1, args.steps)):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = sharding.sweep_shard(mesh, ypr_all, opts)
        torch.cuda.synchronize()
        e2e_s.append(time.perf_counter() - t0)
        assert r.optID == opt and np.array_equal(r.shard.Vss64, res["Vss64"]), "e2e run differs from the device run"
    e2e_total = float(sum(e2e_s))
    if dist:
        t = torch.tensor([e2e_total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = len(e2e_s) * n / e2e_total
    h2d = mesh.n_vtx * 16 * 2 + mesh.n_tri * 16 + (e - b) * (9 * 4 + 4)
    d2h = (e - b) * (5 * 8 + 5 * 4)

    # ---- L2 read bandwidth from the library's probe (no L2 figure in the measured peaks)
    l2_gbs = None
    try:
        probe = torch.zeros(48 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        l2_gbs = native.read_bandwidth(probe.data_ptr(), probe.numel() * 4, reps=40)
        del probe
    except Exception as exc:   # a measurement aid: never costs the bench line
        print(f"read probe skipped: {exc}", file=sys.stderr)

    # ---- roofline of the dominant kernel (k_strip), live event timing
    peaks = _peaks()
    strip = klog["k_strip"]
    algo_bytes_per_orient = 24 * mesh.n_vtx + 12 * mesh.n_tri + 16 * res["entries"].astype(np.float64) + 16
    algo_bytes = float(algo_bytes_per_orient.sum()) * args.steps
    strip_ms = strip["ms"] if strip["timed"] else float("nan")
    achieved = algo_bytes / (strip_ms / 1000.0) / 1e9 if strip["timed"] else None
    launches_per_step = {k: v["launches"] / args.steps for k, v in klog.items()}
    roof = {"bound": "hbm", "kernel": "k_strip", "achieved": achieved, "peak": peaks[0], "unit": "GB/s",
            "frac": (achieved / peaks[0]) if achieved else None, "peak_source": peaks[1],
            "traffic": _traffic(mesh, res, strip["launches"] / args.steps),
            "avg_launch_ms": strip_ms / max(strip["timed"], 1),
            "bytes_per_launch": algo_bytes / max(strip["launches"], 1),
            "l2_read_gbs": l2_gbs, "frac_of_l2": (achieved / l2_gbs) if (achieved and l2_gbs) else None,
            "l2_source": "the library's read probe over a 48 MB buffer, 40 passes after one untimed pass",
            # Event spans per kernel kind and step, each on its launching stream.  These are stream spans,
            # not kernel times: the binning kernels of batch k+1 run on their own stream beside batch k's
            # strips, so their spans include time spent waiting for SMs and for the other stream.  The
            # per-kernel breakdown is the serialised ncu launch list summarised under profiles/.
            "stream_spans_ms_per_step": {k: v["ms"] / args.steps for k, v in klog.items() if v["timed"]}}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": config(mesh, ypr_all, grid, {"parallelism": f"orientation shards x{world}",
                                                "batch_orientations": native.stats()["batch"],
                                                "strip_h": native.stats()["strip_h"]}),
            "time_to_exact_optimum_s": total_ms / args.steps / 1000.0,
            "triangle_orientations_per_s": value * mesh.n_tri,
            "optID": int(opt),
            "reruns_per_step": {"overflow": native.stats()["overflow_reruns"], "safe": native.stats()["safe_reruns"]},
            "roofline": roof,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(sum(v["launches"] for v in klog.values())),
            "launches_per_step": launches_per_step,
            "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(mesh, ypr, opts, grid, budget_s=args.cpu_budget_s,
                                            gpu_vss=res["Vss64"], gpu_mss=Mss)
        # the same engine on one host thread, on a smaller sample
        one = cpu_baseline(mesh, ypr, opts, grid, budget_s=args.cpu_budget_s / 2, gpu_vss=res["Vss64"], threads=1)
        line["cpu_baseline"]["single_thread"] = {k: one[k] for k in ("value", "unit", "cores", "kind", "sample")
                                                 if k in one}
        line["cpu_baseline"]["single_thread"]["sample_vss_bit_identical"] = one.get("sample_vss_bit_identical")
    if world == 1 and not args.no_extras:
        line["plain"] = plain_rate(mesh, ypr, opts)
        from tomo_shell2026_b200 import suites
        line["batched"] = suites.batched_suite(n_meshes=args.batched_meshes)
        line["surrogate"] = suites.surrogate_suite(n_meshes=args.surrogate_meshes)
        line["shell"] = suites.shell_suite()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def plain_rate(mesh, ypr, opts, n: int = 256) -> dict:
    """The same sweep launched one orientation at a time (every kernel of the
    pipeline per orientation, as a per-orientation engine does), on an evenly
    strided sample of the grid: device orientations/s."""
    from tomo_shell2026_b200 import native
    sub = np.ascontiguousarray(ypr[np.linspace(0, ypr.shape[0] - 1, n).astype(np.int64)])
    native.set_option(native.TOMO_OPT_BATCH, 1)
    try:
        s = native.Session(mesh, sub, opts)
        s.run_device()
        ms = s.run_device()
    finally:
        native.set_option(native.TOMO_OPT_BATCH, 256)
    return {"orientations": n, "orientations_per_s": n / (ms / 1000.0), "orientations_per_launch": 1}


def run_suite(args) -> int:
    """Full-size suites, one JSON line each (not part of the default run)."""
    import torch
    from tomo_shell2026_b200 import suites
    torch.cuda.set_device(0)
    if args.suite == "batched":
        r = suites.batched_suite(n_meshes=64)
        line = {"metric": "aggregate orientations/s, 64 uneven meshes (1k-120k tris), 1deg grid, one graph launch",
                "value": r["batched_orientations_per_s"], "unit": "orientations/s", "higher_is_better": True,
                "suite": r}
    elif args.suite == "shell":
        r = suites.shell_suite()
        line = {"metric": "orientations/s, 87k-tri thin open shell (manikin-like, 2 mm wall), 1deg grid, shell mode",
                "value": r["orientations_per_s"], "unit": "orientations/s", "higher_is_better": True, "suite": r}
    else:
        r = suites.surrogate_suite(n_meshes=100)
        line = {"metric": "learned-proposal search: meshes reaching the exhaustive optimum in <= 1/5 of its time",
                "value": r["meshes_at_target"], "unit": "fraction of 100 meshes", "higher_is_better": True,
                "suite": r}
    print(json.dumps(line), flush=True)
    return 0


def _physical_gpu(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
        except (ValueError, KeyError):
            pass
    return 6650.0, "fallback"


def _traffic(mesh, res, launches_per_step):
    """DRAM bytes per k_strip launch from the committed ncu summary, when
    present, scaled from its launch size to this run's orientations per launch."""
    p = ROOT / "profiles" / "k_strip_traffic.json"
    if not p.exists() or not launches_per_step:
        return None
    try:
        d = json.loads(p.read_text())
        per_orientation = float(d["dram_bytes_per_launch"]) / float(d["orientations_per_launch"])
        return per_orientation * (len(res["Vss64"]) / launches_per_step)
    except (ValueError, KeyError, ZeroDivisionError):
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cpu-budget-s", type=float, default=15.0)
    ap.add_argument("--ref-step-s", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the plain-launch, batched and surrogate figures added to the line")
    ap.add_argument("--batched-meshes", type=int, default=16)
    ap.add_argument("--surrogate-meshes", type=int, default=100)
    ap.add_argument("--suite", choices=("none", "batched", "surrogate", "shell"), default="none",
                    help="run a full-size suite instead (64 uneven meshes / 100 searched meshes)")
    ap.add_argument("--max-orientations", type=int, default=0,
                    help="keep only the first N orientations (small profiling cases; 0 = the whole grid)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.suite != "none":
        return run_suite(args) if rank == 0 else 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            rc = run_ours(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
        return rc
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
