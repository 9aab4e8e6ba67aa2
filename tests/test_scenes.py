"""Synthetic workload generators: sizes of the benchmark configurations."""
import numpy as np

from oracle import oracle as O
from rtcollisiondetection_b200 import scenes


def test_discrete_small_sizes():
    m = scenes.discrete_small()
    assert m.n_tris == 5264 and m.n_obstacles == 28
    assert len(O.unique_edges(m.tris)) == 7896


def test_sweep_scene_sizes():
    m = scenes.sweep_scene()
    assert m.n_tris == 49744 and m.n_obstacles == 167
    assert len(O.unique_edges(m.tris)) == 74616


def test_dense_scene_sizes():
    m = scenes.discrete_dense()
    assert m.n_obstacles == 321
    assert 420_000 < m.n_tris < 440_000
    assert 100_000 <= m.n_tris - 64 * 12 - 256 * 1280 < 101_000
    m2 = scenes.discrete_dense(ico_level=2)
    assert 180_000 < m2.n_tris < 185_000


def test_generators_are_deterministic(panda):
    assert np.array_equal(scenes.discrete_small().verts, scenes.discrete_small().verts)
    assert np.array_equal(scenes.uniform_poses(panda, 10), scenes.uniform_poses(panda, 10))
    q, off = scenes.random_walk_trajectories(panda, 5, 32)
    assert q.shape == (160, 7) and off[-1] == 160
    assert np.all(q >= panda['lower']) and np.all(q <= panda['upper'])


def test_uneven_waypoint_counts():
    n = scenes.log_uniform_counts(4096, 8, 64)
    assert n.min() >= 8 and n.max() <= 64
    assert [scenes.quad_ctrl_count(k) for k in (3, 8, 9, 64)] == [3, 4, 5, 32]


def test_synthetic_spheres(panda):
    c, r, l = scenes.synth_spheres(panda)
    assert len(r) == 64 and np.all((r >= 0.02) & (r <= 0.08))
    assert np.bincount(l).tolist() == [8] * 8


def test_icosphere_is_closed():
    v, t = scenes.icosphere(2)
    assert len(t) == 320 and len(v) == 162
    e = O.unique_edges(t)
    assert len(e) == 480
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
