"""Seed producers and file formats of the reference pipeline (CPU)."""
import os

import numpy as np

from caustic_b200 import problems, seeds


def test_picture_orientation_round_trip(tmp_path):
    """read_pic_txt_to_array: data[y*m + x] = matrix[m-1-x][y]."""
    m, n = 3, 4
    mat = np.arange(m * n, dtype=float).reshape(m, n)
    data, size = seeds.picture_from_matrix(mat)
    assert size == (m, n)
    for y in range(n):
        for x in range(m):
            assert data[y * m + x] == mat[m - 1 - x][y]
    p = tmp_path / "pic.txt"
    seeds.write_picture_txt(str(p), data, size)
    d2, s2 = seeds.read_picture_txt(str(p))
    assert s2 == size and np.array_equal(d2, data)


def test_proj_corner_rules():
    pd = [0.0, 160.0, -60.0, 100.0]
    # sites touching every side push the box out by 1 (main.cu:165-187)
    xy = np.array([[0.0, -60.0], [160.0, 100.0], [80.0, 20.0]])
    assert list(seeds.proj_corner(xy, pd)) == [-1.0, 161.0, -61.0, 101.0]
    # sites strictly inside leave the domain as the box
    xy = np.array([[1.0, -50.0], [150.0, 90.0]])
    assert list(seeds.proj_corner(xy, pd)) == pd


def test_boundary_points_are_hull_sites_near_the_sides():
    pts = seeds.initial_xy_point(400, [0.0, 4.0, 0.0, 4.0])
    tri, left, right, bottom, top = seeds.find_boundary_points(pts, 400, [0.0, 4.0, 0.0, 4.0])
    assert np.allclose(pts[left, 0], 0.0) and np.allclose(pts[right, 0], 4.0)
    assert np.allclose(pts[bottom, 1], 0.0) and np.allclose(pts[top, 1], 4.0)
    assert len(left) > 5 and len(bottom) > 5


def test_six_digit_writers(tmp_path):
    p = tmp_path / "w" / "final_proj_point_weights.txt"
    seeds.write_weights(str(p), [2083.3312, -512.43412, 1e-7, 0.0])
    assert p.read_text().split() == ["2083.33", "-512.434", "1e-07", "0"]
    q = tmp_path / "out.txt"
    seeds.write_points(str(q), np.array([[28.38521, -26.948912], [1.0, 2.0]]), keep=[True, False])
    assert q.read_text() == "28.3852 -26.9489\n"


def test_synthetic_generators_are_seeded_and_normalised():
    a = problems.make(1, g=16, res=32)
    b = problems.make(1, g=16, res=32)
    assert np.array_equal(a.xy, b.xy) and np.array_equal(a.picture, b.picture)
    assert abs(a.picture.sum() - 1) < 1e-12 and abs(a.nu.sum() - 1) < 1e-12
    assert a.picture.min() > 0
    c = problems.make(2, g=16, res=32)
    assert c.nu.max() / c.nu.min() > 5   # beam masses
    assert np.all((c.xy > 0) & (c.xy < 1))


def test_define_parameter_layout(tmp_path):
    pts = seeds.initial_xy_point(100, [0, 4, 0, 4])
    proj = seeds.initial_proj_point(pts, [0, 4, 0, 4], [0, 16, -6, 10])
    _, l, r, b, t = seeds.find_boundary_points(pts, 100, [0, 4, 0, 4])
    d = tmp_path / "seed"
    seeds.define_parameter(str(d), pts, proj, l, r, b, t)
    for f in ("points.txt", "proj_xy.txt", "left_idx.txt", "right_idx.txt", "bottom_idx.txt", "top_idx.txt"):
        assert os.path.exists(d / f)
    assert np.allclose(seeds.read_points(str(d / "proj_xy.txt")), proj, atol=1e-6)
    assert np.array_equal(seeds.read_ints(str(d / "left_idx.txt")), l)
