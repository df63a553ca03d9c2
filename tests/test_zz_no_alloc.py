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


def test_static_rerun_ladder_dense_mesh():
    """A dense 16k-triangle sphere (about one triangle per voxel face): strip
    lists and silhouette columns force re-runs; results equal TomoSh_CUDA's."""
    _defaults()
    mesh = meshgen.perturbed_sphere(16000, 30.0, 7, with_hull=False)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 45), np.arange(0, 61, 30))
    opts = PrintOptions()
    ref = native.sweep(mesh, ypr, opts)
    for _ in range(2):
        _same(ref, native.sweep_static(mesh, ypr, opts))
    assert sum(_static_reruns()) > 0, "the dense mesh re-ran nothing"
