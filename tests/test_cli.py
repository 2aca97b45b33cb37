"""The caustic_GPU shim: the reference executable's argv + file contract
(main.cu:51-342) over the C ABI, run in a directory tree laid out like the
reference repository."""
import json
import os
import subprocess

import numpy as np
import pytest

from caustic_b200 import build, seeds
from oracle import oracle as O

XIUSHI = "tiny_tri_standard_sp_parallel_light_rl"


def make_tree(root, total_iter=2000, tol=0.01):
    """Reference layout: Optimal_Transport_rl/build is the working directory."""
    sd = [0.0, 4.0, 0.0, 4.0]
    pd = [0.0, 16.0, -6.0, 10.0]
    pts = seeds.initial_xy_point(400, sd)
    proj = seeds.initial_proj_point(pts, sd, pd)
    _, l, r, b, t = seeds.find_boundary_points(pts, 400, sd)
    ot = os.path.join(root, "Optimal_Transport_rl")
    build_dir = os.path.join(ot, "build")
    os.makedirs(build_dir)
    seed_dir = os.path.join(ot, "seed_point", XIUSHI)
    seeds.define_parameter(seed_dir, pts, proj, l, r, b, t)
    n = len(pts)
    ins = np.tile([0.0, 0.0, 1.0], (n, 1))
    np.savetxt(os.path.join(seed_dir, "inside_light_direct.txt"), ins, fmt="%.6f")
    rng = np.random.default_rng(0)
    for k in (0, 1):
        os.makedirs(os.path.join(seed_dir, str(k)))
        np.savetxt(os.path.join(seed_dir, str(k), "height.txt"), rng.uniform(10, 12, n), fmt="%.6f")
    yy, xx = np.mgrid[0:24, 0:24]
    pic = 20 + 200 * np.exp(-((xx - 9.0) ** 2 + (yy - 14.0) ** 2) / 40.0)
    os.makedirs(os.path.join(root, "data", "pic_data"))
    np.savetxt(os.path.join(root, "data", "pic_data", "tiny.txt"), pic, fmt="%.6f")
    cfg = {
        "test_num": "sp_parallel_light_rl",
        "picture_para": {"name": "tiny"},
        "sample_point_para": {"point_num": 400, "data_name": "tiny_tri_standard", "sample_domain": sd,
                              "total_iter": total_iter, "convergence_tolerance": tol, "history_size": 7,
                              "initial_step": 1, "if_aa_op_initial": True, "aa_history_size": 7,
                              "aa_fixed_para": -2},
        "len_para": {"z_of_len": 0, "z_of_receiver": 160.0, "proj_domain": pd, "refraction_index": 1.5},
        "light_para": {"light_type": "parallel_light", "point_light_coordinate": [20.0, 20.0, -20.0]},
    }
    jdir = os.path.join(ot, "set_json", XIUSHI)
    os.makedirs(jdir)
    with open(os.path.join(jdir, "_py_sp_settings.json"), "w") as f:
        json.dump(cfg, f, indent=1)
    return build_dir, pts, proj, pic, sd, pd


@pytest.fixture(scope="module")
def cli():
    build.build_lib()
    exe = build.build_cli()
    assert exe and os.path.exists(exe)
    return exe


def test_usage_and_json_errors(cli, tmp_path):
    r = subprocess.run([cli], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "Need one input number" in r.stderr
    r = subprocess.run([cli, "0", "missing"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 255
    build_dir, *_ = make_tree(str(tmp_path / "ref"))
    jpath = os.path.join(build_dir, "..", "set_json", XIUSHI, "_py_sp_settings.json")
    with open(jpath) as f:
        cfg = json.load(f)
    del cfg["sample_point_para"]["history_size"]
    with open(jpath, "w") as f:
        json.dump(cfg, f)
    r = subprocess.run([cli, "0", XIUSHI], cwd=build_dir, capture_output=True, text=True)
    assert r.returncode == 3 and "history_size" in r.stderr


def test_missing_height_file(cli, tmp_path):
    build_dir, *_ = make_tree(str(tmp_path / "ref"))
    os.remove(os.path.join(build_dir, "..", "seed_point", XIUSHI, "0", "height.txt"))
    r = subprocess.run([cli, "0", XIUSHI], cwd=build_dir, capture_output=True, text=True)
    assert r.returncode == 2 and "height.txt" in r.stderr


@pytest.mark.gpu
def test_file_contract_first_and_second_outer_iteration(gpu, cli, tmp_path):
    root = str(tmp_path / "ref")
    build_dir, pts, proj, pic, sd, pd = make_tree(root)
    r = subprocess.run([cli, "0", XIUSHI], cwd=build_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    wfile = os.path.join(root, "data", "weights", XIUSHI, "0", "final_proj_point_weights.txt")
    w = seeds.read_weights(wfile)
    assert len(w) == len(pts)
    # the written (6-digit) weights solve the problem the reference poses
    nu = O.source_masses(pts, sd)
    dens, size = seeds.picture_from_matrix(pic)
    prob = O.Problem(proj, nu, O.normalize_picture(dens, sd), size, pd)
    e = O.evaluate(prob, w, keep_cells=True)
    assert np.linalg.norm(e.g) < 0.05
    out = seeds.read_points(os.path.join(root, "data", "point_data", XIUSHI, "0", "out.txt"))
    inn = seeds.read_points(os.path.join(root, "data", "point_data", XIUSHI, "in.txt"))
    assert out.shape == inn.shape
    c, ex = O.centers(e.cells, O.normalize_picture(dens, sd), size, pd)
    assert np.abs(out - c[ex]).max() < 0.05
    assert os.path.exists(os.path.join(root, "data", "point_data", XIUSHI, "0", "_py_sp_settings.json"))
    # diagnostics beside the build directory (ot_op.cuh:214-219, 281-286, 510-535)
    ot = os.path.join(root, "Optimal_Transport_rl")
    img = np.loadtxt(os.path.join(ot, "render_result", XIUSHI, "0", "render_initial.txt"))
    assert img.shape == pic.shape and abs(img.sum() - pic.sum()) < 1e-3 * pic.sum()
    with open(os.path.join(ot, "mesh_output", XIUSHI, "0", "mesh_initial.obj")) as f:
        faces = [ln for ln in f if ln.startswith("f ")]
    assert len(faces) == len(pts)
    # periodic files of iteration 0 and the files of the converged iteration
    # (ot_op.cuh:484-535): weights_<it>, render_<it>, mesh_<it>.obj
    wnames = os.listdir(os.path.join(ot, "weights", XIUSHI, "0"))
    assert "weights_0.txt" in wnames
    assert os.path.exists(os.path.join(ot, "render_result", XIUSHI, "0", "render_0.txt"))
    last = max(int(fn[len("weights_"):-4]) for fn in wnames)
    assert last > 0
    assert os.path.exists(os.path.join(ot, "mesh_output", XIUSHI, "0", f"mesh_{last}.obj"))
    assert os.path.exists(os.path.join(ot, "render_result", XIUSHI, "0", f"render_{last}.txt"))
    wl = seeds.read_weights(os.path.join(ot, "weights", XIUSHI, "0", f"weights_{last}.txt"))
    assert np.array_equal(wl, w)   # the converged iterate is the final one
    # second outer iteration: warm start + Fresnel-reweighted Anderson solve
    r = subprocess.run([cli, "1", XIUSHI], cwd=build_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    w1 = seeds.read_weights(os.path.join(root, "data", "weights", XIUSHI, "1", "final_proj_point_weights.txt"))
    assert len(w1) == len(pts) and np.isfinite(w1).all()
    assert os.path.exists(os.path.join(root, "data", "point_data", XIUSHI, "1", "out.txt"))
    # pre-pass files (ot_op.cuh:1020-1074) and the Anderson loop's, tagged
    # with the outer iteration (ot_op.cuh:1270-1321)
    wn1 = os.listdir(os.path.join(ot, "weights", XIUSHI, "1"))
    assert "pre_weights_0.txt" in wn1 and "1_weights_0.txt" in wn1
    assert os.path.exists(os.path.join(ot, "render_result", XIUSHI, "1", "1_render_0.txt"))
    assert os.path.exists(os.path.join(ot, "render_result", XIUSHI, "1", "pre_render_initial.txt"))
