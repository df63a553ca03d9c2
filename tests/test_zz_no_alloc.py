"""tomoSweepStatic, the allocation-free form of TomoSh_CUDA, against
TomoSh_CUDA itself: two calls in a row must each return the same optID and
bit-identical Mo / Mss / Vtc, and the second call must leave the device's
free memory unchanged.  Collected last (file name) so that it also runs
after every other GPU test has used the library."""
from __future__ import annotations

import numpy as np
import pytest

from tests.test_golden import GOLDEN, GOLDEN_DIR, bits, load_case
from tomo_shell2026_b200 import meshgen, native
from tomo_shell2026_b200.options import PrintOptions

pytestmark = pytest.mark.gpu


def _defaults():
    native.set_option(native.TOMO_OPT_BATCH, 128)
    native.set_option(native.TOMO_OPT_STRIP_H, 0)
    native.set_option(native.TOMO_OPT_FORCE_SAFE, 0)
    native.set_option(native.TOMO_OPT_NORMAL_SMEM, 0)


def _same(ref, got):
    opt, Mo, Mss, Vtc = got
    assert opt == ref.optID
    assert np.array_equal(bits(Mo), bits(ref.Mo)), "Mo differs"
    assert np.array_equal(bits(Mss), bits(ref.Mss)), "Mss differs"
    assert np.array_equal(bits(Vtc), bits(ref.Vtc)), "Vtc differs"


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_static_matches_tomosh_cuda_twice(path):
    import torch
    _defaults()
    d, mesh, opts = load_case(path)
    ref = native.sweep(mesh, d["ypr"], opts)
    _same(ref, native.sweep_static(mesh, d["ypr"], opts))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _same(ref, native.sweep_static(mesh, d["ypr"], opts))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_static_ragged_batch_and_stream():
    """Seven orientations (a partial last batch of four), on a torch stream."""
    import torch
    _defaults()
    d, mesh, opts = load_case(GOLDEN[0])
    ypr = np.ascontiguousarray(d["ypr"][5:12])
    ref = native.sweep(mesh, ypr, opts)
    s = torch.cuda.Stream()
    for _ in range(2):
        _same(ref, native.sweep_static(mesh, ypr, opts, stream=s.cuda_stream))


def test_static_rejects_beyond_limits():
    ypr = meshgen.ypr_grid(np.arange(0, 360, 90), np.arange(0, 60, 30))
    v, f = meshgen.icosphere(6)   # 81920 triangles
    big = meshgen.mesh_from_arrays(v * 40.0, f, "big", with_hull=False)
    with pytest.raises(native.TomoError, match="static limit of 16384"):
        native.sweep_static(big, ypr, PrintOptions())
    small = meshgen.small_solid(0, with_hull=False)
    wide = meshgen.mesh_from_arrays(small.vertices * 3.0, small.faces, "wide", with_hull=False)
    with pytest.raises(native.TomoError, match="static limit of 256"):
        native.sweep_static(wide, ypr, PrintOptions())


def _static_reruns():
    st = native.stats()
    return st["static_overflow_reruns"], st["static_prio_reruns"], st["static_safe_reruns"]


def test_static_rerun_ladder_first_come_cap():
    """Columns past the 63-pixel cap (the stacked-layers mesh): the flagged
    orientations are re-run with first-come priorities, as TomoSh_CUDA does,
    and the results still equal TomoSh_CUDA's, twice."""
    _defaults()
    d, mesh, opts = load_case(GOLDEN_DIR / "layers_cap63.npz")
    ref = native.sweep(mesh, d["ypr"], opts)
    for _ in range(2):
        _same(ref, native.sweep_static(mesh, d["ypr"], opts))
        assert _static_reruns()[1] > 0, "no orientation took the priority re-run"


def _wide_layers(n_layers=20, n=20, seed=4):
    """Stacked wavy sheets across most of the 256-column grid: about twenty
    pixels in every column, far more entries per strip than a default strip
    holds."""
    rng = np.random.default_rng(seed)
    V, F = [], []
    for L in range(n_layers):
        xs, ys = np.meshgrid(np.linspace(20, 170, n), np.linspace(20, 170, n), indexing="ij")
        zs = 10 + L * 2.3 + 0.8 * np.sin(xs * 0.3 + L) + 0.5 * rng.standard_normal(xs.shape)
        base = len(V)
        V += list(np.stack([xs.ravel(), ys.ravel(), zs.ravel()], 1))
        for i in range(n - 1):
            for j in range(n - 1):
                a = base + i * n + j
                b, c, d = a + 1, a + n, a + n + 1
                F += [(a, c, b), (b, c, d)] if L % 2 else [(a, b, c), (b, d, c)]
    return meshgen.mesh_from_arrays(np.array(V), np.array(F), "wide_layers", with_hull=False)


def test_static_rerun_ladder_overflowing_strips():
    """Strips whose pixel lists overflow the default shared-memory budget are
    re-run with the large budget (and beyond that in safe mode), as
    TomoSh_CUDA does; results equal TomoSh_CUDA's, twice."""
    _defaults()
    mesh = _wide_layers()
    assert mesh.n_tri <= 16384
    ypr = meshgen.ypr_grid(np.arange(0, 360, 90), np.arange(0, 61, 30))
    opts = PrintOptions()
    ref = native.sweep(mesh, ypr, opts)
    for _ in range(2):
        _same(ref, native.sweep_static(mesh, ypr, opts))
        big, prio, safe = _static_reruns()
        assert big + safe > 0, "no strip overflowed"
