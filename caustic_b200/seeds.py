"""Seed producers and file formats of the reference pipeline.

The reference's Python driver builds the solver inputs (spline_irra.py:32-41)
and the solver executable reads and writes text files (main.cu:89-334).  This
module restates both sides so the solver can be fed exactly what the
reference feeds it:

* ``initial_xy_point``      data_utils.py:374-411  triangular source lattice
* ``initial_proj_point``    data_utils.py:413-435  similarity map into proj_domain
* ``find_boundary_points``  data_utils.py:437-491  hull sites near the bbox sides
* ``proj_corner``           main.cu:149-187        mirror box
* ``picture_from_matrix``   basic_function.cuh:145-204  picture txt -> density
* ``matrix_from_picture``   basic_function.cuh:205-248  density -> picture txt
* readers / writers of points, index lists, weights and centroid files
  (basic_function.cuh:96-143, main.cu:291-334, basic_function.py:774-780)
"""
from __future__ import annotations

import os

import numpy as np


def initial_xy_point(point_num, sample_domain, sample_type="triangle"):
    """Triangular lattice: rows alternate full and half-shifted, with the
    half-shifted rows padded by sites on both side edges."""
    if sample_type != "triangle":
        raise ValueError(f"Unknown sample_type: {sample_type}.")
    sd = [float(v) for v in sample_domain]
    xs_, ys_ = sd[1] - sd[0], sd[3] - sd[2]
    n = float(point_num)
    nxs = np.sqrt(np.sqrt(3) / 2 * n * xs_ / ys_)
    nys = nxs * 2 / np.sqrt(3) * ys_ / xs_
    nxs = int(nxs) + 1
    nys = int(nys) + 1
    if nys % 2 == 0:
        nys += 1
    xstep = xs_ / float(nxs - 1)
    ystep = ys_ / float(nys - 1)
    pts = []
    for i in range(nys):
        y = i * ystep
        if i % 2 == 0:
            for j in range(nxs):
                pts.append([j * xstep, y])
        else:
            pts.append([0.0, y])
            for j in range(nxs - 1):
                pts.append([j * xstep + xstep / 2.0, y])
            pts.append([xs_, y])
    return np.array(pts, dtype=float)


def initial_proj_point(points, sample_domain, proj_domain):
    sx0, sx1, sy0, sy1 = [float(v) for v in sample_domain]
    px0, px1, py0, py1 = [float(v) for v in proj_domain]
    scale = min((px1 - px0) / (sx1 - sx0), (py1 - py0) / (sy1 - sy0))
    scx, scy = (sx0 + sx1) / 2, (sy0 + sy1) / 2
    pcx, pcy = (px0 + px1) / 2, (py0 + py1) / 2
    out = np.empty_like(points, dtype=float)
    out[:, 0] = (points[:, 0] - scx) * scale + pcx
    out[:, 1] = (points[:, 1] - scy) * scale + pcy
    return out


def find_boundary_points(points, point_num, sample_domain):
    """Delaunay-hull vertices within tol = 0.1*sqrt(area/point_num) of the
    bounding-box sides: (triangles, left, right, bottom, top)."""
    from scipy.spatial import Delaunay

    tri = Delaunay(points).simplices
    sd = [float(v) for v in sample_domain]
    tol = 0.1 * np.sqrt((sd[1] - sd[0]) * (sd[3] - sd[2]) / point_num)
    x, y = points[:, 0], points[:, 1]
    masks = [np.isclose(x, x.min(), atol=tol), np.isclose(x, x.max(), atol=tol),
             np.isclose(y, y.min(), atol=tol), np.isclose(y, y.max(), atol=tol)]
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e.sort(axis=1)
    uniq, cnt = np.unique(e, axis=0, return_counts=True)
    bnd = np.zeros(len(points), dtype=bool)
    bnd[uniq[cnt == 1].ravel()] = True
    return (tri,) + tuple(np.where(m & bnd)[0] for m in masks)


def proj_corner(proj_xy, proj_domain):
    """Box the mirror sites are reflected across: bbox of the sites and the
    domain, pushed out by 1 on a side where a site is extremal."""
    xy = np.asarray(proj_xy, dtype=float).reshape(-1, 2)
    pd = [float(v) for v in proj_domain]
    xmn, xmx = xy[:, 0].min(), xy[:, 0].max()
    ymn, ymx = xy[:, 1].min(), xy[:, 1].max()
    c = [min(xmn, pd[0]), max(xmx, pd[1]), min(ymn, pd[2]), max(ymx, pd[3])]
    if c[0] == xmn:
        c[0] -= 1
    if c[1] == xmx:
        c[1] += 1
    if c[2] == ymn:
        c[2] -= 1
    if c[3] == ymx:
        c[3] += 1
    return np.array(c)


def picture_from_matrix(mat):
    """Text matrix (m rows, n columns) -> density[ix + iy*m], size (m, n):
    data[y*m + x] = matrix[m-1-x][y]."""
    mat = np.asarray(mat, dtype=float)
    m, n = mat.shape
    return np.ascontiguousarray(mat[::-1, :].T).reshape(-1), (m, n)


def matrix_from_picture(data, size):
    m, n = int(size[0]), int(size[1])
    return np.asarray(data, dtype=float).reshape(n, m).T[::-1, :]


def read_picture_txt(path):
    """read_pic_txt_to_array: whitespace matrix, rows of equal length."""
    rows = []
    with open(path) as f:
        for line in f:
            v = line.split()
            if not v:
                continue
            if rows and len(v) != len(rows[0]):
                raise ValueError(f"{path}: rows of different length")
            rows.append([float(t) for t in v])
    if not rows:
        raise ValueError(f"{path}: empty")
    return picture_from_matrix(np.array(rows))


def write_picture_txt(path, data, size):
    """save_array_to_txt: fixed, 6 decimals."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    mat = matrix_from_picture(data, size)
    with open(path, "w") as f:
        for row in mat:
            f.write(" ".join(f"{v:.6f}" for v in row) + "\n")


def read_points(path):
    """readPointsFlat: 'x y' pairs."""
    v = np.loadtxt(path, dtype=float, ndmin=2)
    return v.reshape(-1, 2)


def read_ints(path):
    if os.path.getsize(path) == 0:
        return np.zeros(0, dtype=np.int64)
    return np.atleast_1d(np.loadtxt(path, dtype=np.int64))


def read_weights(path):
    return np.atleast_1d(np.loadtxt(path, dtype=float))


def fmt6(v):
    """A double as std::ostream prints it by default (6 significant digits)."""
    return f"{v:.6g}"


def write_weights(path, w):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        for v in w:
            f.write(fmt6(v) + "\n")


def write_points(path, xy, keep=None):
    """in.txt / out.txt: 'x y' of the cells that exist."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        for i, (x, y) in enumerate(np.asarray(xy).reshape(-1, 2)):
            if keep is None or keep[i]:
                f.write(f"{fmt6(x)} {fmt6(y)}\n")


def define_parameter(seed_dir, points, proj_points, left, right, bottom, top):
    """basic_function.py:774-780: the seed files the solver reads."""
    os.makedirs(seed_dir, exist_ok=True)
    np.savetxt(os.path.join(seed_dir, "points.txt"), points, fmt="%f")
    np.savetxt(os.path.join(seed_dir, "proj_xy.txt"), proj_points, fmt="%f")
    for name, idx in (("left", left), ("right", right), ("bottom", bottom), ("top", top)):
        np.savetxt(os.path.join(seed_dir, f"{name}_idx.txt"), idx, fmt="%d")
