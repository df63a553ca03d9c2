"""Workload generators and suite helpers (CPU only): geodesic spheres of any
size, the thin open shell, and the block ranking used to compare the
network's proposals with the coarse-interpolation baseline."""
from __future__ import annotations

import numpy as np
import pytest

from tomo_shell2026_b200 import meshgen
from tomo_shell2026_b200.suites import block_rank, coarse_interpolation, uneven_meshes


@pytest.mark.parametrize("freq", [1, 3, 7, 20])
def test_geodesic_sphere_closed_outward(freq):
    v, f = meshgen.geodesic_sphere(freq)
    assert f.shape[0] == 20 * freq * freq
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
    m = meshgen.mesh_from_arrays(v * 40.0, f, with_hull=False)
    assert m.is_watertight
    out = np.einsum("ij,ij->i", m.face_normals, m.vertices[m.faces].mean(1))
    assert np.all(out > 0)
    assert set(np.bincount(f.ravel())) <= {5, 6}


def test_uneven_meshes_span_sizes():
    ms = uneven_meshes(6, seed=3, t_min=1000, t_max=20000)
    t = [m.n_tri for m in ms]
    assert min(t) >= 900 and max(t) <= 22000 and len(set(t)) > 1
    assert all(m.is_watertight for m in ms)


def test_manikin_shell_is_open_thin_wall():
    m = meshgen.manikin_shell(0, spacing=16.0)
    assert not m.is_watertight
    half = m.n_tri // 2
    outer, inner = m.faces[:half], m.faces[half:] - m.n_vtx // 2
    assert np.array_equal(outer[:, ::-1], inner)          # inner wall: same triangles, reversed winding
    d = np.linalg.norm(m.vertices[: m.n_vtx // 2] - m.vertices[m.n_vtx // 2:], axis=1)
    assert np.allclose(d, 2.0, atol=1e-3)
    top = m.vertices[outer].mean(1)[:, 2] > m.vertices[:, 2].max() - 20
    assert np.mean(m.face_normals[:half][top][:, 2] > 0) > 0.9    # outer sheet faces outward


def test_block_rank_and_interpolation():
    n_yaw, n_pitch = 72, 13
    yy, pp = np.meshgrid(np.arange(n_yaw), np.arange(n_pitch))
    f = ((yy - 30) ** 2 + (pp - 7) ** 2).ravel().astype(float)
    assert block_rank(f, int(np.argmin(f)), n_yaw, n_pitch, 4) == 0
    ci = coarse_interpolation(f, n_yaw, n_pitch, 4)
    on = ((yy % 4 == 0) & (pp % 4 == 0)).ravel()
    assert np.allclose(ci[on], f[on])
