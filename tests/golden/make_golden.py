"""Generate the golden fixtures of the reference run (run once, where the
reference tree is available; the fixtures are committed beside this script).

The reference repository commits the outputs of one real solve of its
pipeline (configs/_py_sp_settings.json: 160,000-point triangular lattice on
[0,40]^2, image ustc_centerL 640x640, proj_domain [0,160]x[-60,100]):

  data/pic_data/ustc_centerL.txt                                 target image
  data/point_data/<xiushi>/in.txt                                source sites
  data/weights/<xiushi>/0/final_proj_point_weights.txt           converged w
  data/point_data/<xiushi>/0/out.txt                             centroids

Fixtures written here:
  ustc_centerL.npz        image as uint8 (all values are integers 0..200)
  weights0.txt.gz         the converged weights, verbatim text (6 digits)
  out0_sub.txt.gz         every 16th centroid line, verbatim, with its index
  in_sub.txt.gz           every 64th source-site line, verbatim, with its index
  run.json                the solver parameters of that run
"""
import gzip
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
XIUSHI = "ustc_centerL_tri_standard_sp_parallel_light_rl"


def main(REF):
    pic = np.loadtxt(os.path.join(REF, "data/pic_data/ustc_centerL.txt"))
    assert np.all(pic == np.round(pic)) and pic.min() >= 0 and pic.max() <= 255
    np.savez_compressed(os.path.join(HERE, "ustc_centerL.npz"), picture=pic.astype(np.uint8))

    with open(os.path.join(REF, f"data/weights/{XIUSHI}/0/final_proj_point_weights.txt")) as f:
        wtxt = f.read()
    with gzip.open(os.path.join(HERE, "weights0.txt.gz"), "wt") as f:
        f.write(wtxt)

    with open(os.path.join(REF, f"data/point_data/{XIUSHI}/0/out.txt")) as f:
        out_lines = f.read().splitlines()
    with gzip.open(os.path.join(HERE, "out0_sub.txt.gz"), "wt") as f:
        f.write(f"# n={len(out_lines)}\n")
        for i in range(0, len(out_lines), 16):
            f.write(f"{i} {out_lines[i]}\n")

    with open(os.path.join(REF, f"data/point_data/{XIUSHI}/in.txt")) as f:
        in_lines = f.read().splitlines()
    with gzip.open(os.path.join(HERE, "in_sub.txt.gz"), "wt") as f:
        f.write(f"# n={len(in_lines)}\n")
        for i in range(0, len(in_lines), 64):
            f.write(f"{i} {in_lines[i]}\n")

    with open(os.path.join(REF, "configs/_py_sp_settings.json")) as f:
        cfg = json.load(f)
    run = {
        "point_num": cfg["sample_point_para"]["point_num"],
        "type": cfg["sample_point_para"]["type"],
        "sample_domain": cfg["sample_point_para"]["sample_domain"],
        "proj_domain": cfg["len_para"]["proj_domain"],
        "total_iter": cfg["sample_point_para"]["total_iter"],
        "convergence_tolerance": cfg["sample_point_para"]["convergence_tolerance"],
        "history_size": cfg["sample_point_para"]["history_size"],
        "initial_step": cfg["sample_point_para"]["initial_step"],
        "light_type": cfg["light_para"]["light_type"],
        "picture": cfg["picture_para"]["name"],
        "n_sites": len(in_lines),
    }
    with open(os.path.join(HERE, "run.json"), "w") as f:
        json.dump(run, f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the reference repository checkout>")
    main(sys.argv[1])
