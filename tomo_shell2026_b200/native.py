"""ctypes binding of libtomo_b200.so (declarations in include/tomo_b200.h).

There is no CPU fallback: if the CUDA library is missing or cannot be
loaded, :func:`lib` raises.  ``sweep`` is the one-call form used by the
reference-compatible Python surface; ``Session`` exposes the split
prepare / device-sweep / finish form used for timing.
"""
from __future__ import annotations

import ctypes as ct
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .build import LIB

_f32p = ct.POINTER(ct.c_float)
_i32p = ct.POINTER(ct.c_int32)
_i16p = ct.POINTER(ct.c_int16)
_u32p = ct.POINTER(ct.c_uint32)
_i64p = ct.POINTER(ct.c_int64)

TOMO_OPT_BATCH, TOMO_OPT_STRIP_H, TOMO_OPT_FORCE_SAFE, TOMO_OPT_NORMAL_SMEM, TOMO_OPT_EXPORT = 1, 2, 3, 4, 5
TOMO_OPT_ADAPTIVE = 6
TOMO_OPT_PROPOSAL = 7
TOMO_OPT_FOLD_LIMIT = 8

# (name, restype, argtypes) for every export of include/tomo_b200.h
EXPORTS = [
    ("TomoSh_CUDA", ct.c_int32, [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p]),
    ("TomoSh_INT3", ct.c_int32, [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p]),
    ("getMss", _f32p, []),
    ("getMo", _f32p, []),
    ("getVtc", _f32p, []),
    ("getVolMassInfo", _f32p, []),
    ("getMat4x4", _f32p, []),
    ("getnData2i", ct.c_int32, [ct.c_short]),
    ("getpData2i", _i16p, [ct.c_short]),
    ("OnDestroy", None, []),
    ("getVo64", _i64p, []),
    ("getVss64", _i64p, []),
    ("getVtc64", _i64p, []),
    ("tomoGetLastError", ct.c_int, []),
    ("tomoGetLastErrorString", ct.c_char_p, []),
    ("tomoRotation", None, [ct.c_float, ct.c_float, ct.c_float, _f32p]),
    ("tomoShadowThreshold", ct.c_float, [ct.c_float]),
    ("tomoVolToMass", None, [_f32p, _i32p, _f32p]),
    ("tomoSetOption", ct.c_int, [ct.c_int, ct.c_int]),
    ("tomoGetStats", ct.c_int, [_i64p, ct.c_int]),
    ("tomoGetResults", ct.c_int, [_i64p, _i64p, _i64p, _f32p, _f32p, _f32p, _i32p, _i32p, _i64p, _i64p]),
    ("tomoPrepare", ct.c_int, [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p]),
    ("tomoSweepDevice", ct.c_int, [ct.c_void_p, ct.c_void_p, _f32p]),
    ("tomoFinish", ct.c_int, [_f32p, _f32p, _f32p]),
    ("tomoGridSize", ct.c_int, []),
    ("tomoProfile", ct.c_int, [ct.c_int, ct.c_int]),
    ("tomoProbeReadBandwidth", ct.c_int, [ct.c_void_p, ct.c_longlong, ct.c_int, ct.POINTER(ct.c_float)]),
    ("tomoGetKernelLog", ct.c_int, [_i64p, ct.POINTER(ct.c_double), _i64p, ct.c_int]),
    ("tomoColumnDump", ct.c_int, [ct.c_int, ct.c_int, _i32p, _u32p, _i16p]),
    ("tomoSweepStatic", ct.c_int, [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, _f32p, _f32p, _f32p, ct.c_void_p]),
    ("tomoBatchPrepare", ct.c_int, [ct.c_int] + [ct.POINTER(ct.c_void_p)] * 6),
    ("tomoBatchRun", ct.c_int, [ct.c_int, _f32p]),
    ("tomoBatchResults", ct.c_int, [ct.c_int, _f32p, _f32p, _f32p, _i64p, _i64p, _i64p]),
    ("TomoSh_CUDA_Batch", ct.c_int, [ct.c_int] + [ct.POINTER(ct.c_void_p)] * 6 + [_i32p]),
    ("tomoBatchStats", ct.c_int, [_i64p, ct.c_int]),
    ("tomoBatchConfig", ct.c_int, [ct.c_int, _i32p]),
    ("tomoBatchSetOption", ct.c_int, [ct.c_int, ct.c_int]),
    ("tomoBatchRelease", None, []),
    ("tomoBatchExport", ct.c_int, [ct.c_int]),
    ("tomoMlpInit", ct.c_int, [ct.c_int]),
    ("tomoMlpParams", ct.c_int, [_f32p, _f32p]),
    ("tomoMlpGrad", ct.c_int, [_f32p, _f32p, ct.c_int, _f32p, _f32p]),
    ("tomoMlpAdam", ct.c_int, [ct.c_float]),
    ("tomoMlpFit", ct.c_int, [_f32p, _f32p, ct.c_int, ct.c_int, ct.c_float, _f32p]),
    ("tomoMlpPredict", ct.c_int, [_f32p, ct.c_int, _f32p]),
    ("tomoSurrogateSearch", ct.c_int, [_f32p, _i32p, _f32p, _i32p, _f32p, _f32p, ct.c_int, ct.c_int, _i32p, _f32p,
                                       _f32p, _f32p, ct.POINTER(ct.c_double)]),
]

_LIB: ct.CDLL | None = None


def library_path() -> Path:
    return Path(os.environ.get("TOMO_B200_LIB", str(LIB)))


def lib() -> ct.CDLL:
    """Load (once) and return the CUDA library; raises if it is not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists():
        raise RuntimeError(f"libtomo_b200.so not found at {path}; run tomo_shell2026_b200/build.py")
    L = ct.CDLL(str(path))
    for name, res, args in EXPORTS:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class TomoError(RuntimeError):
    pass


def _check(rc: int) -> int:
    if rc < 0:
        L = lib()
        msg = L.tomoGetLastErrorString()
        raise TomoError(f"libtomo_b200 error {rc}: {msg.decode() if msg else ''}")
    return rc


def rotation(yaw: float, pitch: float, roll: float) -> np.ndarray:
    out = np.zeros(9, np.float32)
    lib().tomoRotation(yaw, pitch, roll, _p(out, _f32p))
    return out.reshape(3, 3)


def shadow_threshold(theta_c: float) -> np.float32:
    return np.float32(lib().tomoShadowThreshold(theta_c))


def vol_to_mass(f32info, i32info, vm22) -> np.ndarray:
    vm = np.ascontiguousarray(vm22, np.float32).copy()
    lib().tomoVolToMass(_p(f32info, _f32p), _p(i32info, _i32p), _p(vm, _f32p))
    return vm


KERNEL_KINDS = ("k_reset", "k_rotate", "k_bin_count", "k_bin_scan", "k_bin_fill", "k_strip", "k_bed", "k_fold",
                "k_strip_redo")


def profile(enable: bool, reset: bool = True) -> None:
    """Per-launch CUDA-event timing inside the engine (events on each kernel's own stream)."""
    lib().tomoProfile(1 if enable else 0, 1 if reset else 0)


def kernel_log() -> dict:
    n = len(KERNEL_KINDS)
    launches = np.zeros(n, np.int64)
    ms = np.zeros(n, np.float64)
    timed = np.zeros(n, np.int64)
    lib().tomoGetKernelLog(_p(launches, _i64p), ms.ctypes.data_as(ct.POINTER(ct.c_double)), _p(timed, _i64p), n)
    return {k: dict(launches=int(launches[i]), ms=float(ms[i]), timed=int(timed[i])) for i, k in enumerate(KERNEL_KINDS)}


def read_bandwidth(dev_ptr: int, nbytes: int, reps: int = 40) -> float:
    """GB/s of the library's read probe over a device buffer (tomoProbeReadBandwidth)."""
    ms = ct.c_float(0.0)
    _check(lib().tomoProbeReadBandwidth(ct.c_void_p(dev_ptr), nbytes, reps, ct.byref(ms)))
    return nbytes * reps / (ms.value * 1e6) if ms.value > 0 else float("nan")


def set_option(key: int, value: int) -> None:
    if lib().tomoSetOption(key, value) != 0:
        raise TomoError(f"bad option {key}={value}")


def stats() -> dict:
    """Strip plan and re-run counts of the last sweep (``static_*``: of the
    last tomoSweepStatic call)."""
    out = np.zeros(12, np.int64)
    _check(lib().tomoGetStats(_p(out, _i64p), 12))
    return dict(grid=int(out[0]), strip_h=int(out[1]), strips=int(out[2]), ent_cap=int(out[3]),
                overflow_reruns=int(out[4]), n_ypr=int(out[5]), batch=int(out[6]), safe_reruns=int(out[7]),
                prio_reruns=int(out[8]), static_overflow_reruns=int(out[9]), static_prio_reruns=int(out[10]),
                static_safe_reruns=int(out[11]))


@dataclass
class SweepResult:
    optID: int
    Mo: np.ndarray
    Mss: np.ndarray
    Vtc: np.ndarray
    Vo64: np.ndarray
    Vss64: np.ndarray
    Vtc64: np.ndarray
    VoF: np.ndarray
    VssF: np.ndarray
    VtcF: np.ndarray
    n_bed: np.ndarray
    flags: np.ndarray
    entries: np.ndarray
    columns: np.ndarray
    volmass: np.ndarray
    mat4x4: np.ndarray
    pixels: list  # 11 arrays of (n, 6) int16 records x,y,z,nx,ny,nz, one per pixel type


def pixels() -> list:
    """getnData2i/getpData2i of the last sweep, one (n, 6) int16 array per type."""
    L = lib()
    out = []
    for k in range(11):
        n = int(L.getnData2i(k))
        p = L.getpData2i(k)
        out.append(np.ctypeslib.as_array(p, shape=(n, 6)).copy() if n and p else np.zeros((0, 6), np.int16))
    return out


def _arrays(mesh, ypr):
    return (np.ascontiguousarray(ypr, np.float32), np.ascontiguousarray(mesh.faces, np.int32),
            np.ascontiguousarray(mesh.vertices, np.float32), np.ascontiguousarray(mesh.vertex_normals, np.float32),
            np.ascontiguousarray(mesh.face_normals, np.float32), np.ascontiguousarray(mesh.hull_faces, np.int32),
            np.ascontiguousarray(mesh.hull_vertices, np.float32),
            np.ascontiguousarray(mesh.hull_face_normals, np.float32))


def results(n: int) -> dict:
    out = {k: np.zeros(n, np.int64) for k in ("Vo64", "Vss64", "Vtc64", "entries", "columns")}
    out.update({k: np.zeros(n, np.float32) for k in ("VoF", "VssF", "VtcF")})
    out.update({k: np.zeros(n, np.int32) for k in ("n_bed", "flags")})
    _check(lib().tomoGetResults(_p(out["Vo64"], _i64p), _p(out["Vss64"], _i64p), _p(out["Vtc64"], _i64p),
                                _p(out["VoF"], _f32p), _p(out["VssF"], _f32p), _p(out["VtcF"], _f32p),
                                _p(out["n_bed"], _i32p), _p(out["flags"], _i32p), _p(out["entries"], _i64p),
                                _p(out["columns"], _i64p)))
    return out


def sweep(mesh, ypr, opts) -> SweepResult:
    """One TomoSh_CUDA call (the reference C-ABI) plus the exact side outputs."""
    from .options import pack_info
    L = lib()
    f32, i32 = pack_info(opts, mesh, ypr.shape[0])
    ypr, tri, vtx, vn, tn, ht, hv, hn = _arrays(mesh, ypr)
    opt = _check(L.TomoSh_CUDA(_p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p), _p(vtx, _f32p),
                               _p(vn, _f32p), _p(tn, _f32p), _p(ht, _i32p), _p(hv, _f32p), _p(hn, _f32p)))
    n = ypr.shape[0]
    get = lambda fn: np.ctypeslib.as_array(fn(), shape=(n,)).copy() if n else np.zeros(0, np.float32)
    r = results(n)
    return SweepResult(opt, get(L.getMo), get(L.getMss), get(L.getVtc), r["Vo64"], r["Vss64"], r["Vtc64"],
                       r["VoF"], r["VssF"], r["VtcF"], r["n_bed"], r["flags"], r["entries"], r["columns"],
                       np.ctypeslib.as_array(L.getVolMassInfo(), shape=(22,)).copy(),
                       np.ctypeslib.as_array(L.getMat4x4(), shape=(16,)).copy().reshape(4, 4), pixels())


class Batch:
    """Many meshes, one graph launch (tomoBatchPrepare / tomoBatchRun)."""

    def __init__(self, meshes, yprs, opts, autotune: bool = True, tune_sample: int = 512):
        from .options import pack_info
        if not isinstance(opts, (list, tuple)):
            opts = [opts] * len(meshes)
        self.n = [int(y.shape[0]) for y in yprs]
        self._keep = []
        cols = [[] for _ in range(6)]
        for m, y, o in zip(meshes, yprs, opts):
            f32, i32 = pack_info(o, m, y.shape[0])
            y, tri, vtx, vn, *_ = _arrays(m, y)
            self._keep += [f32, i32, y, tri, vtx, vn]
            for c, a in zip(cols, (f32, i32, y, tri, vtx, vn)):
                c.append(a.ctypes.data)
        self._ptrs = [(ct.c_void_p * max(len(meshes), 1))(*c) for c in cols]
        L = lib()
        _check(L.tomoBatchSetOption(1, 1 if autotune else 0))
        _check(L.tomoBatchSetOption(2, int(tune_sample)))
        _check(L.tomoBatchPrepare(len(meshes), *self.pointer_args()))

    def pointer_args(self):
        return [ct.cast(p, ct.POINTER(ct.c_void_p)) for p in self._ptrs]

    def run(self, use_graph: bool = True) -> float:
        ms = ct.c_float(0.0)
        _check(lib().tomoBatchRun(1 if use_graph else 0, ct.byref(ms)))
        return float(ms.value)

    def results(self, m: int) -> dict:
        n = self.n[m]
        out = {k: np.zeros(n, np.float32) for k in ("Mo", "Mss", "Vtc")}
        out.update({k: np.zeros(n, np.int64) for k in ("Vo64", "Vss64", "Vtc64")})
        out["optID"] = _check(lib().tomoBatchResults(m, *[_p(out[k], _f32p) for k in ("Mo", "Mss", "Vtc")],
                                                       *[_p(out[k], _i64p) for k in ("Vo64", "Vss64", "Vtc64")]))
        return out

    def config(self, m: int) -> dict:
        c = np.zeros(4, np.int32)
        _check(lib().tomoBatchConfig(m, _p(c, _i32p)))
        return dict(batch=int(c[0]), normal_smem=int(c[1]), strip_h=int(c[2]), grid=int(c[3]))

    @staticmethod
    def stats() -> dict:
        out = np.zeros(9, np.int64)
        _check(lib().tomoBatchStats(_p(out, _i64p), 9))
        keys = ("meshes", "orientations", "graph_nodes", "graph_kernels", "tuned_now", "tuned_total", "reruns",
                "device_us", "graph_us")
        return {k: int(v) for k, v in zip(keys, out)}

    @staticmethod
    def release() -> None:
        lib().tomoBatchRelease()


def sweep_static(mesh, ypr, opts, stream: int | None = None) -> tuple[int, np.ndarray, np.ndarray, np.ndarray]:
    """tomoSweepStatic: (optID, Mo, Mss, Vtc) without any allocation by the library."""
    from .options import pack_info
    f32, i32 = pack_info(opts, mesh, ypr.shape[0])
    ypr, tri, vtx, vn, *_ = _arrays(mesh, ypr)
    n = ypr.shape[0]
    Mo, Mss, Vtc = (np.zeros(n, np.float32) for _ in range(3))
    opt = _check(lib().tomoSweepStatic(_p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p),
                                       _p(vtx, _f32p), _p(vn, _f32p), _p(Mo, _f32p), _p(Mss, _f32p),
                                       _p(Vtc, _f32p), stream))
    return opt, Mo, Mss, Vtc


class Session:
    """Split form: upload once, sweep on the device repeatedly, finish on the host."""

    def __init__(self, mesh, ypr, opts):
        from .options import pack_info
        self.n = ypr.shape[0]
        self.f32, self.i32 = pack_info(opts, mesh, self.n)
        self.ypr, self.tri, self.vtx, self.vn, *_ = _arrays(mesh, ypr)
        _check(lib().tomoPrepare(_p(self.f32, _f32p), _p(self.i32, _i32p), _p(self.ypr, _f32p),
                                 _p(self.tri, _i32p), _p(self.vtx, _f32p), _p(self.vn, _f32p)))

    def run_device(self, ev_start=None, ev_stop=None) -> float:
        ms = ct.c_float(0.0)
        _check(lib().tomoSweepDevice(ev_start, ev_stop, ct.byref(ms)))
        return float(ms.value)

    def finish(self) -> tuple[int, np.ndarray, np.ndarray, np.ndarray]:
        Mo = np.zeros(self.n, np.float32)
        Mss = np.zeros(self.n, np.float32)
        Vtc = np.zeros(self.n, np.float32)
        opt = _check(lib().tomoFinish(_p(Mo, _f32p), _p(Mss, _f32p), _p(Vtc, _f32p)))
        return opt, Mo, Mss, Vtc

    def grid(self) -> int:
        return int(lib().tomoGridSize())

    def columns(self, index: int, safe: bool = False) -> dict:
        G = self.grid()
        cols = np.zeros((G * G, 8), np.int32)
        keys = np.zeros((G * G, 64), np.uint32)
        types = np.zeros((G * G, 64), np.int16)
        fl = _check(lib().tomoColumnDump(index, 1 if safe else 0, _p(cols, _i32p), _p(keys, _u32p), _p(types, _i16p)))
        return dict(G=G, cols=cols, keys=keys, types=types, flags=fl)
