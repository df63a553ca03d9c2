"""Multi-mesh batch (tomoBatchPrepare / tomoBatchRun / TomoSh_CUDA_Batch):
uneven meshes, options and orientation lists in one graph launch must give
every mesh exactly what TomoSh_CUDA gives it alone -- with the graph, on a
graph replay, and without the graph."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

from tests.test_golden import bits
from tomo_shell2026_b200 import meshgen, native
from tomo_shell2026_b200.options import PrintOptions

pytestmark = pytest.mark.gpu


def _defaults():
    native.set_option(native.TOMO_OPT_BATCH, 256)
    native.set_option(native.TOMO_OPT_STRIP_H, 0)
    native.set_option(native.TOMO_OPT_FORCE_SAFE, 0)
    native.set_option(native.TOMO_OPT_NORMAL_SMEM, 0)


def _cases():
    g10 = meshgen.ypr_grid(np.arange(0, 360, 10), np.arange(0, 70, 10))       # 252
    g30 = meshgen.ypr_grid(np.arange(0, 360, 30), np.arange(0, 190, 30))      # 84
    g7 = np.ascontiguousarray(meshgen.ypr_grid(np.arange(0, 360, 45), np.arange(0, 60, 20))[:7])
    return [
        (meshgen.perturbed_icosphere(2, 30.0, 11, with_hull=False), g30, PrintOptions()),
        (meshgen.perturbed_icosphere(5, 60.0, 12, n_bumps=2, with_hull=False), g10, PrintOptions(explicit_ss=False)),
        (meshgen.small_solid(13, with_hull=False), g30,
         PrintOptions(shell_mesh=True, shell_thickness=0.5, bed_type=2, bed_outer=2.0, bed_thickness=0.97)),
        (meshgen.random_mesh(900, 14), g7, PrintOptions(bed_type=1, bed_outer=2.0, bed_thickness=0.97)),
        (meshgen.perturbed_icosphere(3, 20.0, 15, with_hull=False), g10, PrintOptions()),
    ]


def _same(ref, got, m):
    assert got["optID"] == ref.optID, f"mesh {m}: optID"
    for k in ("Mo", "Mss", "Vtc"):
        assert np.array_equal(bits(got[k]), bits(getattr(ref, k))), f"mesh {m}: {k} differs"
    for k in ("Vo64", "Vss64", "Vtc64"):
        assert np.array_equal(got[k], getattr(ref, k)), f"mesh {m}: {k} differs"


def test_batch_matches_single_mesh_calls():
    _defaults()
    cases = _cases()
    refs = [native.sweep(m, y, o) for m, y, o in cases]
    b = native.Batch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases], autotune=True,
                     tune_sample=64)
    for use_graph in (True, True, False):
        b.run(use_graph=use_graph)
        for m, ref in enumerate(refs):
            _same(ref, b.results(m), m)
    st = native.Batch.stats()
    assert st["meshes"] == len(cases) and st["orientations"] == sum(c[1].shape[0] for c in cases)
    assert st["graph_nodes"] > 0 and st["graph_kernels"] > 0
    for m in range(len(cases)):
        c = b.config(m)
        assert c["batch"] in (64, 128, 256) and c["normal_smem"] in (0, 73728, 101376)   # 0: four strip CTAs per SM
    native.Batch.release()


def test_one_call_batch_export():
    _defaults()
    cases = _cases()[:3]
    refs = [native.sweep(m, y, o) for m, y, o in cases]
    b = native.Batch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases], autotune=False)
    opt = np.full(len(cases), -1, np.int32)
    rc = native.lib().TomoSh_CUDA_Batch(len(cases), *b.pointer_args(), opt.ctypes.data_as(ct.POINTER(ct.c_int32)))
    assert rc == 0
    assert [int(x) for x in opt] == [r.optID for r in refs]
    native.Batch.release()
