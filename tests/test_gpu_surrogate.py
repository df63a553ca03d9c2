"""Learned-proposal search on the GPU: the network's forward pass, gradients
and Adam step against the CPU oracle (oracle/mlp_oracle.py), training, and
the whole search against the exhaustive sweep of the same grid."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp_oracle as mo
from tomo_shell2026_b200 import meshgen, native, surrogate
from tomo_shell2026_b200.options import PrintOptions

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    ypr = np.column_stack([rng.uniform(0, 2 * np.pi, n), rng.uniform(0, 1.05, n), np.zeros(n)]).astype(np.float32)
    x = mo.features(ypr)
    y = (np.sin(3 * ypr[:, 0]) * np.cos(2 * ypr[:, 1]) + 0.3 * ypr[:, 1]).astype(np.float32)
    return x, y


def test_forward_matches_oracle():
    surrogate.mlp_init(3)
    rng = np.random.default_rng(1)
    theta = rng.normal(0, 0.15, mo.layout()[1]).astype(np.float32)
    surrogate.mlp_params(set_to=theta)
    x, _ = _data(1000, 2)
    got = surrogate.mlp_predict(x)
    want = mo.forward(theta.astype(np.float64), x.astype(np.float64))[-1][:, 0]
    assert np.max(np.abs(got - want)) <= 1e-5 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("n", [7, 936])
def test_gradient_matches_oracle(n):
    surrogate.mlp_init(4)
    theta = surrogate.mlp_params().astype(np.float64)
    x, y = _data(n, 5)
    loss, g = surrogate.mlp_grad(x, y)
    ref_loss, ref_g = mo.loss_and_grad(theta, x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-5 * max(1.0, ref_loss)
    # float32 accumulation over n samples: relative error of the whole gradient, and per element
    assert np.linalg.norm(g - ref_g) <= 1e-4 * np.linalg.norm(ref_g)
    assert np.allclose(g, ref_g, rtol=1e-3, atol=1e-5 * np.max(np.abs(ref_g)))


def test_adam_step_matches_oracle():
    surrogate.mlp_init(6)
    theta = surrogate.mlp_params().astype(np.float64)
    x, y = _data(300, 7)
    _, g = surrogate.mlp_grad(x, y)
    surrogate.mlp_adam(1e-3)
    got = surrogate.mlp_params().astype(np.float64)
    want, _, _ = mo.adam_step(theta, g.astype(np.float64), np.zeros_like(theta), np.zeros_like(theta), 1, 1e-3)
    assert np.max(np.abs(got - want)) <= 1e-6


def test_training_fits_a_smooth_target():
    surrogate.mlp_init(8)
    x, y = _data(936, 9)
    first = surrogate.mlp_grad(x, y)[0]
    last = surrogate.mlp_fit(x, y, 400, 3e-3)
    assert last < 0.05 * first
    pred = surrogate.mlp_predict(x)
    assert np.sqrt(np.mean((pred - y) ** 2)) < 0.1


@pytest.mark.parametrize("seed", [21, 22])
def test_search_reaches_the_exhaustive_optimum(seed):
    """1-degree grid (yaw 0-359 x pitch 0-60), 5-degree cells: the search must
    find the exhaustive sweep's optimal Mss while evaluating a fraction of
    the grid (the gain over the method without the network, which evaluates
    every orientation)."""
    mesh = meshgen.small_solid(seed, with_hull=False)
    n_yaw, n_pitch = 360, 61
    ypr = meshgen.ypr_grid(np.arange(0, 360), np.arange(0, 61))
    opts = PrintOptions(explicit_ss=True)
    ex = native.sweep(mesh, ypr, opts)
    r = surrogate.search(mesh, ypr, n_yaw, n_pitch, opts, stride=5, cell=5, top_k=16, seed=seed)
    assert np.float32(r.Mss[r.optID]) == ex.Mss[ex.optID], "optimum value differs from the exhaustive sweep"
    done = ~np.isnan(r.Mss)
    assert np.array_equal(r.Mss[done].view(np.int32), ex.Mss[done].view(np.int32)), "evaluated Mss not exact"
    if not r.fallback:
        assert r.evaluated < 0.25 * ypr.shape[0]
    print(f"seed {seed}: evaluated {r.evaluated}/{ypr.shape[0]}, fallback {r.fallback}, rel err {r.rel_error:.3f}, "
          f"same index {r.optID == ex.optID}, {r.seconds * 1e3:.1f} ms")


def test_bed_falls_back_to_exhaustive():
    mesh = meshgen.small_solid(23, with_hull=False)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 10), np.arange(0, 70, 10))
    opts = PrintOptions(bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    ex = native.sweep(mesh, ypr, opts)
    r = surrogate.search(mesh, ypr, 36, 7, opts, stride=2, cell=2)
    assert r.fallback and r.evaluated == ypr.shape[0]
    assert r.optID == ex.optID and np.array_equal(r.Mss.view(np.int32), ex.Mss.view(np.int32))


@pytest.mark.parametrize("seed", [31, 32, 33])
def test_search_with_and_without_the_network(seed):
    """The ablation: the same coarse-to-fine search with blocks ranked by the
    trained network, by a bilinear interpolation of the exact coarse values
    (no network), and by the mean of the two.  Each must reach the exhaustive
    sweep's optimal Mss with exact values wherever it evaluated, while
    evaluating a small fraction of the grid; the evaluation counts of the
    three are printed side by side (the suite in bench.py reports them over
    100 meshes)."""
    mesh = meshgen.small_solid(seed, with_hull=False)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 0.5), np.arange(0, 60.5, 0.5))
    opts = PrintOptions(explicit_ss=True)
    ex = native.sweep(mesh, ypr, opts)
    counts = {}
    for kind in ("network", "interpolation", "mean"):
        r = surrogate.search(mesh, ypr, 720, 121, opts, seed=seed, proposal=kind)
        assert np.float32(r.Mss[r.optID]) == ex.Mss[ex.optID], f"{kind}: optimum value differs from the exhaustive sweep"
        done = ~np.isnan(r.Mss)
        assert np.array_equal(r.Mss[done].view(np.int32), ex.Mss[done].view(np.int32)), f"{kind}: evaluated Mss not exact"
        assert r.evaluated < 0.1 * ypr.shape[0], f"{kind}: evaluated {r.evaluated} of {ypr.shape[0]}"
        counts[kind] = (r.evaluated, round(r.seconds * 1e3, 1), round(r.max_abs_error, 1))
    print(f"seed {seed}: (evaluated, ms, max abs error) {counts}")
