"""CUDA path vs the oracle, through the C-ABI (TomoSh_CUDA and the split
entry points).  Integer outputs and the reference's float32 outputs are
compared bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from tomo_shell2026_b200 import meshgen, native
from tomo_shell2026_b200.options import PrintOptions

pytestmark = pytest.mark.gpu

FLOAT_KEYS = ("Mo", "Mss", "Vtc")


def _same_bits(a, b):
    a = np.asarray(a); b = np.asarray(b)
    if a.dtype == np.float32:
        return np.array_equal(a.view(np.int32), b.view(np.int32))
    return np.array_equal(a, b)


def _compare(res, ora, label=""):
    assert _same_bits(res.Vo64, ora["Vo64"]), f"{label} Vo64 differs at {np.nonzero(res.Vo64 != ora['Vo64'])[0][:10]}"
    assert _same_bits(res.Vss64, ora["Vss64"]), f"{label} Vss64 differs at {np.nonzero(res.Vss64 != ora['Vss64'])[0][:10]}"
    assert _same_bits(res.Vtc64, ora["Vtc64"]), f"{label} Vtc64 differs"
    assert _same_bits(res.VoF, ora["VoF"]), f"{label} VoF differs"
    assert _same_bits(res.VssF, ora["VssF"]), f"{label} VssF differs"
    for k in FLOAT_KEYS:
        assert _same_bits(getattr(res, k), ora[k]), f"{label} {k} differs at {np.nonzero(getattr(res, k) != ora[k])[0][:10]}"
    assert res.optID == ora["optID"], f"{label} optID {res.optID} != {ora['optID']}"
    assert np.array_equal(res.entries, ora["entries"]), f"{label} entry counts differ"
    assert np.array_equal(res.columns, ora["columns"]), f"{label} occupied-column counts differ"


GRID_SMALL = meshgen.ypr_grid(np.arange(0, 360, 30), np.arange(0, 190, 30))


@pytest.mark.parametrize("explicit_ss", [True, False])
def test_small_solid_sweep(oracle, explicit_ss):
    m = meshgen.small_solid(0)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 10), np.arange(0, 190, 10))
    opts = PrintOptions(explicit_ss=explicit_ss)
    _compare(native.sweep(m, ypr, opts), oracle.sweep(m, ypr, opts), "small solid")


@pytest.mark.parametrize("bed", [(1, 0.0, 2.0, 0.97), (2, 0.0, 2.0, 0.97), (3, 1.0, 3.0, 0.97), (2, 0.0, 5.5, 1.3)])
@pytest.mark.parametrize("explicit_ss", [True, False])
def test_bed_types(oracle, bed, explicit_ss):
    m = meshgen.small_solid(1)
    bt, bi, bo, th = bed
    opts = PrintOptions(explicit_ss=explicit_ss, bed_type=bt, bed_inner=bi, bed_outer=bo, bed_thickness=th)
    _compare(native.sweep(m, GRID_SMALL, opts), oracle.sweep(m, GRID_SMALL, opts), f"bed {bed}")


@pytest.mark.parametrize("thickness", [0.5, 2.3])
def test_shell_mode(oracle, thickness):
    m = meshgen.small_solid(2)
    opts = PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=thickness, bed_type=2, bed_outer=2.0,
                        bed_thickness=0.97)
    _compare(native.sweep(m, GRID_SMALL, opts), oracle.sweep(m, GRID_SMALL, opts), "shell")


@pytest.mark.parametrize("explicit_ss", [True, False])
def test_triangle_soup_slivers(oracle, explicit_ss):
    s = meshgen.random_mesh(3000, 5)
    opts = PrintOptions(explicit_ss=explicit_ss, shell_mesh=True, bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    _compare(native.sweep(s, GRID_SMALL, opts), oracle.sweep(s, GRID_SMALL, opts), "soup")


def _layers(n_layers=45, n=12, seed=3):
    rng = np.random.default_rng(seed)
    V, F = [], []
    for L in range(n_layers):
        xs, ys = np.meshgrid(np.linspace(20, 80, n), np.linspace(20, 80, n), indexing="ij")
        zs = 10 + L * 2.3 + 0.8 * np.sin(xs * 0.3 + L) + 0.5 * rng.standard_normal(xs.shape)
        base = len(V)
        V += list(np.stack([xs.ravel(), ys.ravel(), zs.ravel()], 1))
        for i in range(n - 1):
            for j in range(n - 1):
                a = base + i * n + j
                b, c, d = a + 1, a + n, a + n + 1
                F += [(a, c, b), (b, c, d)] if L % 2 else [(a, b, c), (b, d, c)]
    return meshgen.mesh_from_arrays(np.array(V), np.array(F), "layers")


@pytest.mark.parametrize("shell", [False, True])
def test_slot_cap_truncation(oracle, shell):
    m = _layers()
    ypr = meshgen.ypr_grid(np.arange(0, 360, 45), np.arange(0, 60, 20))
    opts = PrintOptions(explicit_ss=True, shell_mesh=shell, bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    _compare(native.sweep(m, ypr, opts), oracle.sweep(m, ypr, opts), "layers")


@pytest.mark.parametrize("h", [1, 2, 4, 8])
def test_strip_heights_agree(oracle, h):
    m = meshgen.small_solid(3)
    opts = PrintOptions(explicit_ss=True, bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    native.set_option(native.TOMO_OPT_STRIP_H, h)
    try:
        res = native.sweep(m, GRID_SMALL, opts)
    finally:
        native.set_option(native.TOMO_OPT_STRIP_H, 0)
    _compare(res, oracle.sweep(m, GRID_SMALL, opts), f"H={h}")


def test_safe_mode_agrees(oracle):
    m = meshgen.small_solid(4)
    opts = PrintOptions(explicit_ss=False, shell_mesh=True, bed_type=1, bed_outer=2.0, bed_thickness=0.97)
    native.set_option(native.TOMO_OPT_FORCE_SAFE, 1)
    try:
        res = native.sweep(m, GRID_SMALL, opts)
    finally:
        native.set_option(native.TOMO_OPT_FORCE_SAFE, 0)
    _compare(res, oracle.sweep(m, GRID_SMALL, opts), "safe")


def test_columns_match_oracle(oracle):
    m = meshgen.small_solid(0)
    ypr = GRID_SMALL
    opts = PrintOptions(explicit_ss=True, shell_mesh=True, bed_type=2, bed_outer=2.0, bed_thickness=0.97)
    sess = native.Session(m, ypr, opts)
    G = sess.grid()
    assert G == 256
    for idx in (0, 7, 40):
        for safe in (False, True):
            d = sess.columns(idx, safe=safe)
            o = oracle.columns(m, ypr, opts, idx, grid=G)
            nd = d["cols"][:, 0]
            # distinct pixel count after voxelization, per column
            assert np.array_equal(nd, np.minimum(o["n_vox"], 63)), f"n_vox differs (idx {idx}, safe {safe})"
            # pixel count after pairing (floor sentinels)
            occ = nd > 0
            bed_free = o["n_fin"].copy()
            assert np.array_equal(d["cols"][occ, 2], o["col_vo"][occ]), "per-column Vo differs"
            assert np.array_equal(d["cols"][occ, 3], o["col_vss"][occ]), "per-column Vss differs"
            # kept keys in column order against the oracle's sorted rows
            for s in np.nonzero(nd > 1)[0][:2000]:
                n = nd[s]
                z = (d["keys"][s, :n] >> 16).astype(np.int64) - 32768
                nz = (d["keys"][s, :n] & 0xFFFF).astype(np.int64) - 32768
                oz = o["fin_tzn"][s, :n, 1]
                onz = o["fin_tzn"][s, :n, 2]
                assert np.array_equal(z, oz) and np.array_equal(nz, onz), f"column {s} keys differ"
                ot = o["fin_tzn"][s, :n, 0] & ~32  # bed bit is added after pairing
                assert np.array_equal(d["types"][s, :n], ot), f"column {s} types differ"
            del bed_free


def test_repeat_runs_identical():
    m = meshgen.small_solid(5)
    opts = PrintOptions(explicit_ss=True, shell_mesh=True)
    a = native.sweep(m, GRID_SMALL, opts)
    b = native.sweep(m, GRID_SMALL, opts)
    assert _same_bits(a.Mss, b.Mss) and np.array_equal(a.Vss64, b.Vss64) and a.optID == b.optID


def test_large_grid_solid(oracle):
    m = meshgen.solid_82k(0)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 90), np.arange(0, 61, 30))
    opts = PrintOptions(explicit_ss=True)
    res = native.sweep(m, ypr, opts)
    st = native.stats()
    assert st["grid"] > 256
    _compare(res, oracle.sweep(m, ypr, opts, grid=st["grid"]), "82k")


@pytest.mark.parametrize("explicit_ss", [True, False])
def test_fold_escape_table(oracle, explicit_ss):
    """Fold records hold a column's (vo, vss, tc) as 16-bit values; a column
    whose values do not fit goes through the batch's escape table.  Lowering
    the record range so that a few hundred columns of one orientation escape
    must leave every output bit unchanged (the 82k solid's Vo passes 2^24, so
    its float fold is replayed column by column and reads those escapes); a
    range of 1 overflows the table and must be an error, not a wrong sum."""
    m = meshgen.solid_82k(0)
    ypr = meshgen.ypr_grid(np.array([30.0]), np.array([40.0]))
    opts = PrintOptions(explicit_ss=explicit_ss)
    sess = native.Session(m, ypr, opts)
    G = sess.grid()
    cols = sess.columns(0)["cols"]
    mag = np.sort(np.abs(cols[cols[:, 0] > 0, 2:5]).max(axis=1))[::-1]
    lim = int(mag[600])
    assert 1 <= lim < int(mag[0]) and np.count_nonzero(mag > lim) <= 600
    want = oracle.sweep(m, ypr, opts, grid=G)
    assert int(want["Vo64"][0]) > (1 << 24)
    for bad in (0, -5, 32768):
        with pytest.raises(native.TomoError):
            native.set_option(native.TOMO_OPT_FOLD_LIMIT, bad)
    try:
        native.set_option(native.TOMO_OPT_FOLD_LIMIT, lim)
        res = native.sweep(m, ypr, opts)
        _compare(res, want, f"limit {lim}")
        native.set_option(native.TOMO_OPT_FOLD_LIMIT, 1)
        with pytest.raises(native.TomoError, match="escape table"):
            native.sweep(m, ypr, opts)
    finally:
        native.set_option(native.TOMO_OPT_FOLD_LIMIT, 32767)
    _compare(native.sweep(m, ypr, opts), want, "default range")


def test_bad_index_is_an_error():
    m = meshgen.small_solid(0)
    bad = meshgen.MeshArrays(m.vertices, m.faces.copy(), m.vertex_normals, m.face_normals, m.area)
    bad.faces[5, 1] = m.n_vtx + 10
    with pytest.raises(native.TomoError):
        native.sweep(bad, GRID_SMALL, PrintOptions())


def test_manikin_open_shell(oracle):
    """The thin open shell workload (87k-triangle manikin union surface with
    openings and a 2 mm inward wall, shell mode, a ~1000-column slot grid) on
    a few orientations of its 1-degree grid."""
    m = meshgen.manikin_shell(0)
    ypr = np.ascontiguousarray(meshgen.ypr_grid(np.arange(0, 360, 1), np.arange(0, 61, 1))[::3989])
    opts = PrintOptions(explicit_ss=True, shell_mesh=True, shell_thickness=0.5)
    res = native.sweep(m, ypr, opts)
    G = native.stats()["grid"]
    assert G > 256
    _compare(res, oracle.sweep(m, ypr, opts, grid=G, threads=2), "manikin")


@pytest.mark.parametrize("adaptive", [0, 1])
def test_overflow_ladder_and_adaptive_budget(oracle, adaptive):
    """A strip budget far too small for the mesh: with adaptation off every
    orientation overflows and is re-run with the large budget; with it on,
    the sweep raises its budget after the first batches.  Both exact."""
    m = meshgen.perturbed_icosphere(5, 60.0, 31, with_hull=False)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 15), np.arange(0, 70, 10))
    opts = PrintOptions()
    native.set_option(native.TOMO_OPT_ADAPTIVE, adaptive)
    native.set_option(native.TOMO_OPT_NORMAL_SMEM, 19456)   # ~100 entries per one-row strip
    native.set_option(native.TOMO_OPT_BATCH, 32)
    try:
        res = native.sweep(m, ypr, opts)
        st = native.stats()
    finally:
        native.set_option(native.TOMO_OPT_ADAPTIVE, 1)
        native.set_option(native.TOMO_OPT_NORMAL_SMEM, 0)
        native.set_option(native.TOMO_OPT_BATCH, 256)
    _compare(res, oracle.sweep(m, ypr, opts), f"adaptive={adaptive}")
    if adaptive:
        assert st["overflow_reruns"] < ypr.shape[0] // 2
    else:
        assert st["overflow_reruns"] > 0


def test_dense_mesh_first_come_priorities(oracle):
    """A 100k-triangle solid at 1 mm: columns along the silhouette pass the
    63-pixel cap, so which keys survive depends on first-come order; those
    orientations are re-run with priorities carried in the normal strips."""
    m = meshgen.perturbed_sphere(100000, 50.0, 7, with_hull=False)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 45), np.arange(0, 61, 30))
    opts = PrintOptions()
    res = native.sweep(m, ypr, opts)
    st = native.stats()
    _compare(res, oracle.sweep(m, ypr, opts), "dense")
    assert st["prio_reruns"] > 0


@pytest.mark.parametrize("explicit_ss", [True, False])
def test_arbitrary_yaw_pitch_roll(oracle, explicit_ss):
    """Orientations off the yaw/pitch grid: random angles in radians with a
    non-zero roll, negative and beyond a full turn, over several batches."""
    rng = np.random.default_rng(22)
    m = meshgen.small_solid(22)
    ypr = rng.uniform(-7.0, 7.0, (300, 3)).astype(np.float32)
    opts = PrintOptions(explicit_ss=explicit_ss, shell_mesh=True, shell_thickness=0.5, bed_type=2, bed_outer=2.0,
                        bed_thickness=0.97)
    native.set_option(native.TOMO_OPT_BATCH, 64)
    try:
        res = native.sweep(m, ypr, opts)
    finally:
        native.set_option(native.TOMO_OPT_BATCH, 256)
    _compare(res, oracle.sweep(m, ypr, opts), "yaw/pitch/roll")


@pytest.mark.parametrize("dvoxel,theta_deg", [(0.5, 30.0), (1.0, 45.0), (2.0, 75.0)])
@pytest.mark.parametrize("explicit_ss", [True, False])
def test_voxel_size_and_critical_angle(oracle, dvoxel, theta_deg, explicit_ss):
    """Printer parameters off their defaults (voxel size, critical angle)."""
    m = meshgen.small_solid(23)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 15), np.arange(0, 190, 15))
    opts = PrintOptions(dVoxel=dvoxel, theta_c=float(np.deg2rad(theta_deg)), explicit_ss=explicit_ss, bed_type=1,
                        bed_outer=2.0, bed_thickness=0.97)
    _compare(native.sweep(m, ypr, opts), oracle.sweep(m, ypr, opts), f"dVoxel {dvoxel}, theta_c {theta_deg}")


@pytest.mark.parametrize("case", [
    dict(wall_thickness=0.4, Fcore=0.3, Fclad=0.9, Fss=0.1, Css=1.5, PLA_density=0.00124),
    dict(wall_thickness=1.2, Fcore=0.05, Fclad=1.0, Fss=0.35, Css=0.8, PLA_density=0.001121),
])
@pytest.mark.parametrize("shell_thickness", [0.5, 1.7, 3.0])
def test_mass_model_and_shell_offset(oracle, case, shell_thickness):
    """The library's own VolToMass restatement at mass-model parameters off
    their defaults (wall, infill fractions, density) and at three shell twin
    offsets, with a skirt and both shadow models: Mo / Mss / Vtc bits and
    optID against the oracle (itself pinned against the reference engine at
    the same parameters)."""
    m = meshgen.small_solid(24)
    ypr = meshgen.ypr_grid(np.arange(0, 360, 45), np.arange(0, 190, 45))
    for explicit_ss in (True, False):
        opts = PrintOptions(explicit_ss=explicit_ss, shell_mesh=True, shell_thickness=shell_thickness, bed_type=3,
                            bed_inner=1.0, bed_outer=3.0, bed_thickness=0.97, **case)
        _compare(native.sweep(m, ypr, opts), oracle.sweep(m, ypr, opts), f"mass model {case}, explicit {explicit_ss}")
