"""Learned-proposal orientation search and its MLP (libtomo_b200.so).

``search`` runs the whole coarse -> train -> propose -> refine -> gate
pipeline of ``tomoSurrogateSearch`` on one mesh: the exact kernels evaluate
the coarse grid points, the MLP (hand-written CUDA forward, backward and
Adam kernels) is trained on their exact Vss, proposes the most promising
cells of the fine grid, the exact kernels evaluate those, and the search
falls back to the exhaustive sweep when the network's observed error says
it cannot be trusted.  The ``mlp_*`` functions expose the network itself
(gradient checks, standalone fitting).
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import numpy as np

from .native import _check, _f32p, _i32p, _p, _arrays, lib

_f64p = ct.POINTER(ct.c_double)


def _lib():
    return lib()


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def mlp_init(seed: int = 0) -> int:
    return _check(_lib().tomoMlpInit(int(seed)))


def mlp_params(set_to=None) -> np.ndarray:
    L = _lib()
    n = _check(L.tomoMlpParams(None, None))
    out = np.zeros(n, np.float32)
    _check(L.tomoMlpParams(_p(out, _f32p), _p(_f32(set_to), _f32p) if set_to is not None else None))
    return out


def mlp_grad(x, y) -> tuple[float, np.ndarray]:
    x, y = _f32(x), _f32(y)
    g = np.zeros(mlp_params().size, np.float32)
    loss = np.zeros(1, np.float32)
    _check(_lib().tomoMlpGrad(_p(x, _f32p), _p(y, _f32p), y.size, _p(g, _f32p), _p(loss, _f32p)))
    return float(loss[0]), g


def mlp_adam(lr: float) -> None:
    _check(_lib().tomoMlpAdam(float(lr)))


def mlp_fit(x, y, steps: int, lr: float) -> float:
    x, y = _f32(x), _f32(y)
    loss = np.zeros(1, np.float32)
    _check(_lib().tomoMlpFit(_p(x, _f32p), _p(y, _f32p), y.size, int(steps), float(lr), _p(loss, _f32p)))
    return float(loss[0])


def mlp_predict(x) -> np.ndarray:
    x = _f32(x)
    out = np.zeros(x.shape[0], np.float32)
    _check(_lib().tomoMlpPredict(_p(x, _f32p), x.shape[0], _p(out, _f32p)))
    return out


@dataclass
class SearchResult:
    optID: int
    Mss: np.ndarray         # exact Mss of the evaluated orientations, NaN elsewhere
    pred_vss: np.ndarray    # the network's Vss on every orientation
    evaluated: int
    fallback: bool
    rel_error: float
    max_abs_error: float
    train_loss: float
    seconds: float
    seconds_exact: float
    seconds_train: float
    seconds_predict: float
    cells_refined: int
    rounds: int
    coarse: int


def search(mesh, ypr, n_yaw: int, n_pitch: int, opts, stride: int = 10, cell: int = 5, top_k: int = 64,
           steps: int = 300, lr: float = 3e-3, seed: int = 0, max_eval: int = -1, gate: float = 0.5,
           margin: float = 1.0, holdout: float = 0.0, log_scale: float = 0.3,
           proposal: str = "network") -> SearchResult:
    """Learned-proposal search over ypr = grid [n_pitch][n_yaw] (yaw fastest):
    coarse training points every `stride` grid steps, refinement in blocks of
    cell x cell grid points, fallback past max_eval evaluated orientations
    (default: an eighth of the grid); see tomoSurrogateSearch.  The defaults
    are the setting measured on the 0.5-degree grid with 5-degree coarse
    points: 64 proposed 2.5-degree blocks, log-scaled targets, margin 1.

    ``proposal="interpolation"`` runs the same search without the network:
    the blocks are ranked by a bilinear interpolation of the exact coarse
    values and the error gate uses that interpolation's observed error;
    ``proposal="mean"`` ranks by the mean of the network and that
    interpolation."""
    from .native import TOMO_OPT_PROPOSAL
    from .options import pack_info
    modes = {"network": 0, "interpolation": 1, "mean": 2}
    if proposal not in modes:
        raise ValueError("proposal must be 'network', 'interpolation' or 'mean'")
    f32, i32 = pack_info(opts, mesh, ypr.shape[0])
    ypr, tri, vtx, vn, *_ = _arrays(mesh, ypr)
    n = ypr.shape[0]
    if max_eval < 0:
        max_eval = max(1, n // 8)
    ip = np.array([stride, cell, top_k, steps, seed, max_eval], np.int32)
    fp = np.array([lr, gate, margin, holdout, log_scale], np.float32)
    mss = np.zeros(n, np.float32)
    pred = np.zeros(n, np.float32)
    st = np.zeros(12, np.float64)
    _check(_lib().tomoSetOption(TOMO_OPT_PROPOSAL, modes[proposal]))
    try:
        opt = _check(_lib().tomoSurrogateSearch(_p(f32, _f32p), _p(i32, _i32p), _p(ypr, _f32p), _p(tri, _i32p),
                                                _p(vtx, _f32p), _p(vn, _f32p), int(n_yaw), int(n_pitch),
                                                _p(ip, _i32p), _p(fp, _f32p), _p(mss, _f32p), _p(pred, _f32p),
                                                st.ctypes.data_as(_f64p)))
    finally:
        _lib().tomoSetOption(TOMO_OPT_PROPOSAL, 0)
    return SearchResult(opt, mss, pred, int(st[0]), bool(st[1]), float(st[2]), float(st[3]), float(st[4]),
                        float(st[5]), float(st[6]), float(st[7]), float(st[8]), int(st[9]), int(st[10]), int(st[11]))
