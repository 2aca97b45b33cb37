// caustic_GPU -- the reference executable's process + file contract over the
// C ABI (include/causticot.h).
//
// Reference: Optimal_Transport_rl/main.cu:51-342, run by
// utils/basic_function.py:14-34 as `caustic_GPU <ot_time> <xiushi>` with the
// working directory Optimal_Transport_rl/build.  Inputs and outputs are the
// same files at the same relative paths:
//   ../set_json/<xiushi>/_py_sp_settings.json
//   ../../data/pic_data/<picture_para.name>.txt
//   ../seed_point/<xiushi>/{points,proj_xy,left_idx,right_idx,bottom_idx,top_idx}.txt
//   ../seed_point/<xiushi>/inside_light_direct.txt, ../seed_point/<xiushi>/<k>/height.txt
//   ../../data/weights/<xiushi>/<k-1>/final_proj_point_weights.txt   (k > 0)
// ->
//   ../../data/weights/<xiushi>/<k>/final_proj_point_weights.txt
//   ../../data/point_data/<xiushi>/<k>/out.txt (+ a copy of the JSON)
//   ../../data/point_data/<xiushi>/in.txt      (k == 0)
//
// Exit status: 0 done (also when the iteration cap is reached, as the
// reference); 1 usage (as the reference); 255 unreadable JSON (the
// reference's `return -1`); 2 a light/height file is missing; 3 a key is
// missing or of the wrong type; 4 unknown light type; 5 an input file is
// malformed; 6 the solver failed (CUDA error, bad problem).
#include "causticot.h"
#include "json_min.hpp"

#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace fs = std::filesystem;

static bool read_pairs(const std::string &path, std::vector<double> &v)
{
    std::ifstream f(path);
    if (!f) {
        std::cerr << "cannot open file: " << path << std::endl;
        return false;
    }
    double x, y;
    while (f >> x >> y) {
        v.push_back(x);
        v.push_back(y);
    }
    return true;
}

static bool read_ints(const std::string &path, std::vector<int> &v)
{
    std::ifstream f(path);
    if (!f) {
        std::cerr << "cannot open file: " << path << std::endl;
        return false;
    }
    int a;
    while (f >> a) v.push_back(a);
    return true;
}

// read_pic_txt_to_array (basic_function.cuh:145-204): data[y*m + x] = row m-1-x, column y.
static bool read_picture(const std::string &path, std::vector<double> &data, int &m, int &n)
{
    std::ifstream f(path);
    if (!f) {
        std::cerr << "cannot open file: " << path << std::endl;
        return false;
    }
    std::vector<std::vector<double>> rows;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::vector<double> r;
        double v;
        while (is >> v) r.push_back(v);
        if (r.empty()) continue;
        if (!rows.empty() && r.size() != rows[0].size()) {
            std::cerr << "picture rows have different lengths: " << path << std::endl;
            return false;
        }
        rows.push_back(std::move(r));
    }
    if (rows.empty()) {
        std::cerr << "picture is empty: " << path << std::endl;
        return false;
    }
    m = (int)rows.size();
    n = (int)rows[0].size();
    data.assign((size_t)m * n, 0.0);
    for (int y = 0; y < n; y++)
        for (int x = 0; x < m; x++) data[(size_t)y * m + x] = rows[m - 1 - x][y];
    return true;
}

static void ensure_parent(const std::string &p) { fs::create_directories(fs::path(p).parent_path()); }

// writeOBJ (basic_function.cuh:15-59): one face per cell with >= 3 vertices
// (the rings here are the cells inside proj_domain)
static bool write_obj(cot_handle *h, const std::vector<double> &w, const std::string &path)
{
    const int n = (int)w.size();
    std::vector<int> off(n + 1);
    int cap = 16 * n + 64;
    std::vector<double> xy;
    std::vector<int> nb;
    for (int tries = 0; tries < 6; tries++) {
        xy.resize(2 * (size_t)cap);
        nb.resize(cap);
        int rc = cot_cells(h, w.data(), off.data(), xy.data(), nb.data(), cap);
        if (rc == COT_OK) break;
        if (rc != COT_ECAPACITY) return false;
        cap *= 2;
    }
    ensure_parent(path);
    std::ofstream f(path);
    if (!f) return false;
    int g = 1;
    for (int i = 0; i < n; i++) {
        int a = off[i], b = off[i + 1];
        if (b - a < 3) continue;
        for (int k = a; k < b; k++) f << "v " << xy[2 * k] << " " << xy[2 * k + 1] << " 0.0\n";
        f << "f ";
        for (int k = a; k < b; k++) f << g++ << " ";
        f << "\n";
    }
    return true;
}

// save_array_to_txt (basic_function.cuh:205-248): fixed, 6 decimals, rows of x from the top
static bool write_render(cot_handle *h, const std::vector<double> &w, double gray, int m, int nn, const std::string &path)
{
    std::vector<double> img((size_t)m * nn);
    if (cot_render(h, w.data(), gray, img.data()) != COT_OK) return false;
    ensure_parent(path);
    std::ofstream f(path);
    if (!f) return false;
    char buf[64];
    for (int row = 0; row < m; row++) {
        for (int col = 0; col < nn; col++) {
            std::snprintf(buf, sizeof buf, "%.6f", img[(size_t)col * m + (m - 1 - row)]);
            f << buf;
            if (col != nn - 1) f << " ";
        }
        f << "\n";
    }
    return true;
}

static void write_weights_file(const std::vector<double> &w, const std::string &path)
{
    ensure_parent(path);
    std::ofstream f(path);
    for (double v : w) f << v << std::endl;
}

// Diagnostics written during a solve through the progress callback, on the
// reference's schedule and names:
//   starting points (iteration -1): render_initial + mesh_initial.obj of
//     direct_ot (ot_op.cuh:214-219, 285-286); pre_render_initial +
//     pre_initial_mesh.obj at the re-weighted warm start and render_initial
//     after the pre-pass of aarl_direct_ot (ot_op.cuh:797-820, 1094-1099);
//   direct_ot (ot_op.cuh:478-535): every 500 iterations weights_<it> and
//     render_<it>; on convergence weights_, mesh_<it>.obj and render_;
//   pre-pass of aarl_direct_ot (ot_op.cuh:1014-1074): the same with "pre_";
//   Anderson loop (ot_op.cuh:1270-1321): <t>_weights_<it> every 200,
//     <t>_render_<it> every 500, and all three on convergence.
struct Diagnostics {
    cot_handle *h = nullptr;
    double gray = 1.0;
    int pm = 0, pn = 0;
    std::string render_dir, mesh_dir, wdir, ot_time;
};

static int on_progress(void *user, int phase, int iteration, int status, const double *w, const double *nu, int n,
                       double grad_norm, double max_rel_err)
{
    (void)nu;
    Diagnostics &D = *static_cast<Diagnostics *>(user);
    const std::vector<double> wv(w, w + n);
    if (iteration < 0) {
        bool ok = true;
        if (phase == COT_PHASE_LBFGS)
            ok = write_render(D.h, wv, D.gray, D.pm, D.pn, D.render_dir + "render_initial.txt") &&
                 write_obj(D.h, wv, D.mesh_dir + "mesh_initial.obj");
        else if (phase == COT_PHASE_PREPASS)
            ok = write_render(D.h, wv, D.gray, D.pm, D.pn, D.render_dir + "pre_render_initial.txt") &&
                 write_obj(D.h, wv, D.mesh_dir + "pre_initial_mesh.obj");
        else
            ok = write_render(D.h, wv, D.gray, D.pm, D.pn, D.render_dir + "render_initial.txt");
        if (!ok) std::cerr << "could not write the initial diagnostics" << std::endl;
        return 0;
    }
    const std::string it = std::to_string(iteration);
    std::string tag;
    int weights_every = 500;
    if (phase == COT_PHASE_PREPASS) tag = "pre_";
    if (phase == COT_PHASE_ANDERSON) {
        tag = D.ot_time + "_";
        weights_every = 200;
    }
    if (iteration % 100 == 0 || status != 0)
        std::cout << (phase == COT_PHASE_ANDERSON ? "aa " : phase == COT_PHASE_PREPASS ? "pre " : "") << iteration
                  << ": |g| " << grad_norm << ", max rel " << max_rel_err << std::endl;
    bool ok = true;
    if (iteration % weights_every == 0 || status == 1) write_weights_file(wv, D.wdir + tag + "weights_" + it + ".txt");
    if (iteration % 500 == 0 || status == 1)
        ok = write_render(D.h, wv, D.gray, D.pm, D.pn, D.render_dir + tag + "render_" + it + ".txt");
    if (status == 1) ok = write_obj(D.h, wv, D.mesh_dir + tag + "mesh_" + it + ".obj") && ok;
    if (!ok) std::cerr << "could not write the diagnostics of iteration " << iteration << std::endl;
    return 0;
}

static int solver_error(cot_handle *h, const char *what)
{
    char buf[512];
    cot_last_error(h, buf, sizeof buf);
    std::cerr << what << ": " << buf << std::endl;
    if (h) cot_destroy(h);
    return 6;
}

int main(int argc, char *argv[])
{
    if (argc < 3) {
        std::cerr << "Need one input number\n";
        return 1;
    }
    const std::string ot_time = argv[1];
    const std::string xiushi = argv[2];
    const std::string json_path = "../set_json/" + xiushi + "/_py_sp_settings.json";
    jmin::Handler J;
    std::string jerr;
    if (!J.loadFromFile(json_path, &jerr)) {
        std::cout << "cannot read the solver JSON: " << jerr << std::endl;
        return 255;
    }
    std::string picture_name, light_type;
    int total_iter = 0, history_size = 0, aa_history_size = 0;
    double tol = 0, initial_step = 1, aa_fixed_para = 0, z_of_len = 0, z_of_receiver = 0, refraction_index = 1;
    bool if_aa_op_initial = false;
    std::vector<double> sample_domain, proj_domain, point_light;
    try {
        jmin::Handler sp = J.object("sample_point_para");
        jmin::Handler lp = J.object("len_para");
        jmin::Handler li = J.object("light_para");
        (void)J.string("test_num");
        (void)sp.string("data_name");
        picture_name = J.object("picture_para").string("name");
        total_iter = sp.integer("total_iter");
        tol = sp.number("convergence_tolerance");
        history_size = sp.integer("history_size");
        aa_history_size = sp.integer("aa_history_size");
        aa_fixed_para = sp.number("aa_fixed_para");
        if_aa_op_initial = sp.boolean("if_aa_op_initial");
        initial_step = sp.number("initial_step");
        z_of_len = lp.number("z_of_len");
        z_of_receiver = lp.number("z_of_receiver");
        refraction_index = lp.number("refraction_index");
        light_type = li.string("light_type");
        point_light = li.numbers("point_light_coordinate");
        sample_domain = sp.numbers("sample_domain");
        proj_domain = lp.numbers("proj_domain");
        if (point_light.size() < 3 || sample_domain.size() < 4 || proj_domain.size() < 4)
            throw std::runtime_error("point_light_coordinate needs 3 values, the domains 4");
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return 3;
    }

    std::vector<double> picture;
    int pm = 0, pn = 0;
    if (!read_picture("../../data/pic_data/" + picture_name + ".txt", picture, pm, pn)) return 5;
    const std::string seed = "../seed_point/" + xiushi + "/";
    std::vector<double> points, proj_xy;
    std::vector<int> idx[4];
    if (!read_pairs(seed + "points.txt", points) || !read_pairs(seed + "proj_xy.txt", proj_xy)) return 5;
    const char *idx_names[4] = {"left_idx.txt", "right_idx.txt", "bottom_idx.txt", "top_idx.txt"};
    // read for the reference's input checks only: cells are built inside
    // proj_domain directly, so no mirror sites are needed
    for (int k = 0; k < 4; k++) read_ints(seed + idx_names[k], idx[k]);
    const int n = (int)(points.size() / 2);
    if (n <= 0 || proj_xy.size() != points.size()) {
        std::cerr << "points.txt and proj_xy.txt must hold the same number of sites" << std::endl;
        return 5;
    }
    for (int k = 0; k < 4; k++)
        for (int i : idx[k])
            if (i < 0 || i >= n) {
                std::cerr << idx_names[k] << ": index " << i << " out of range" << std::endl;
                return 5;
            }

    // warm start from the previous outer iteration (main.cu:193-198)
    std::vector<double> w(n, 0.0);
    if (ot_time != "0") {
        int prev = std::stoi(ot_time) - 1;
        std::string wp = "../../data/weights/" + xiushi + "/" + std::to_string(prev) + "/final_proj_point_weights.txt";
        std::ifstream f(wp);
        if (!f) {
            std::cerr << "cannot open file: " << wp << std::endl;  // the reference keeps w = 0 then
        } else {
            std::vector<double> v;
            double x;
            while (f >> x) v.push_back(x);
            for (int i = 0; i < n && i < (int)v.size(); i++) w[i] = v[i];
        }
    }

    // light directions, refracted directions and heights (main.cu:204-272)
    std::vector<double> input_light(3 * (size_t)n), inside_light(3 * (size_t)n), height(n);
    if (light_type == "parallel_light") {
        for (int i = 0; i < n; i++) {
            input_light[3 * i] = 0;
            input_light[3 * i + 1] = 0;
            input_light[3 * i + 2] = 1;
        }
    } else if (light_type == "point_light") {
        for (int i = 0; i < n; i++) {
            double d[3] = {points[2 * i] - point_light[0], points[2 * i + 1] - point_light[1], z_of_len - point_light[2]};
            double l = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (int c = 0; c < 3; c++) input_light[3 * i + c] = d[c] / l;
        }
    } else {
        std::cerr << "Unknown light_type: " << light_type << std::endl;
        return 4;
    }
    {
        std::string p = seed + "inside_light_direct.txt";
        std::ifstream f(p);
        if (!f) {
            std::cerr << "Failed to open file: " << p << std::endl;
            return 2;
        }
        for (int i = 0; i < n; i++) {
            double d[3];
            if (!(f >> d[0] >> d[1] >> d[2])) {
                std::cerr << "Error reading direction for point " << i << std::endl;
                break;
            }
            double l = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (int c = 0; c < 3; c++) inside_light[3 * i + c] = l > 0 ? d[c] / l : 0.0;
        }
    }
    {
        std::string p = seed + ot_time + "/height.txt";
        std::ifstream f(p);
        if (!f) {
            std::cerr << "Failed to open file: " << p << std::endl;
            return 2;
        }
        for (int i = 0; i < n; i++) {
            if (!(f >> height[i])) {
                std::cerr << "Error reading height for point " << i << std::endl;
                break;
            }
        }
    }
    cot_config cfg{};
    cot_handle *h = nullptr;
    if (cot_create(&cfg, &h) != COT_OK) return solver_error(nullptr, "cot_create");
    std::vector<double> nu(n);
    if (light_type == "parallel_light") {
        if (cot_source_masses(h, points.data(), n, sample_domain.data(), nu.data()) != COT_OK)
            return solver_error(h, "cot_source_masses");
    } else if (cot_source_masses_point_light(h, points.data(), n, sample_domain.data(), point_light.data(), z_of_len,
                                             nu.data()) != COT_OK) {
        return solver_error(h, "cot_source_masses_point_light");
    }
    if (cot_set_problem(h, proj_xy.data(), nu.data(), n, picture.data(), pm, pn, proj_domain.data(), COT_MEM_HOST) != COT_OK)
        return solver_error(h, "cot_set_problem");

    // diagnostics of the reference, written from the solve's progress reports
    double raw_sum = 0;
    for (double v : picture) raw_sum += v;
    const double area_scalar = (sample_domain[1] - sample_domain[0]) * (sample_domain[3] - sample_domain[2]);
    const double gray = raw_sum / area_scalar;
    const std::string render_dir = "../render_result/" + xiushi + "/" + ot_time + "/";
    const std::string mesh_dir = "../mesh_output/" + xiushi + "/" + ot_time + "/";
    const std::string wdir = "../weights/" + xiushi + "/" + ot_time + "/";

    Diagnostics diag;
    diag.h = h;
    diag.gray = gray;
    diag.pm = pm;
    diag.pn = pn;
    diag.render_dir = render_dir;
    diag.mesh_dir = mesh_dir;
    diag.wdir = wdir;
    diag.ot_time = ot_time;
    if (cot_set_progress(h, on_progress, &diag, 100) != COT_OK) return solver_error(h, "cot_set_progress");

    cot_solve_opts o{};
    o.mode = COT_SOLVE_REFERENCE;
    o.history = history_size;
    o.max_iter = total_iter;
    o.tol = tol;
    o.initial_step = initial_step;
    cot_solve_stats st{};
    int rc;
    if (ot_time == "0") {
        rc = cot_solve(h, w.data(), &o, &st, COT_MEM_HOST);
    } else {
        cot_aarl_inputs ai{};
        ai.points_xy = points.data();
        ai.input_light = input_light.data();
        ai.inside_light = inside_light.data();
        ai.height = height.data();
        ai.z_of_len = z_of_len;
        ai.z_of_receiver = z_of_receiver;
        ai.refraction_index = refraction_index;
        ai.sample_domain[0] = sample_domain[0];
        ai.sample_domain[1] = sample_domain[1];
        ai.sample_domain[2] = sample_domain[2];
        ai.sample_domain[3] = sample_domain[3];
        ai.aa_history = aa_history_size;
        ai.aa_fixed_para = aa_fixed_para;
        ai.lbfgs_prepass = if_aa_op_initial ? 1 : 0;
        rc = cot_solve_aarl(h, w.data(), &ai, &o, &st);
    }
    if (rc != COT_OK && rc != COT_ENOTCONV) return solver_error(h, "solve");
    std::cout << "iterations " << st.iterations << ", evaluations " << st.evaluations << ", |g| " << st.grad_norm
              << ", max rel " << st.max_rel_err << ", converged " << st.converged << ", " << st.ms << " ms" << std::endl;
    std::vector<double> cen(2 * (size_t)n);
    std::vector<unsigned char> ex(n);
    if (cot_centroids(h, w.data(), cen.data(), ex.data(), 1, COT_MEM_HOST) != COT_OK) return solver_error(h, "cot_centroids");
    cot_destroy(h);

    // writers (main.cu:291-334): default ostream formatting, 6 significant digits
    std::string wfile = "../../data/weights/" + xiushi + "/" + ot_time + "/final_proj_point_weights.txt";
    ensure_parent(wfile);
    {
        std::ofstream f(wfile);
        for (int i = 0; i < n; i++) f << w[i] << std::endl;
    }
    std::string out_dir = "../../data/point_data/" + xiushi + "/" + ot_time + "/";
    fs::create_directories(out_dir);
    try {
        fs::copy_file(json_path, fs::path(out_dir) / "_py_sp_settings.json", fs::copy_options::overwrite_existing);
    } catch (const fs::filesystem_error &e) {
        std::cerr << "Copy failed: " << e.what() << std::endl;
    }
    if (ot_time == "0") {
        std::ofstream f("../../data/point_data/" + xiushi + "/in.txt");
        for (int i = 0; i < n; i++)
            if (ex[i]) f << points[2 * i] << " " << points[2 * i + 1] << std::endl;
    }
    {
        std::ofstream f(out_dir + "out.txt");
        for (int i = 0; i < n; i++)
            if (ex[i]) f << cen[2 * i] << " " << cen[2 * i + 1] << std::endl;
    }
    return 0;
}
