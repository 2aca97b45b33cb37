/*
 * causticot.h -- C ABI of the B200 semi-discrete optimal-transport solver.
 *
 * Replaces the first stage of the caustic pipeline: the `caustic_GPU`
 * executable built from Optimal_Transport_rl/ in rmk523/caustic.  That
 * executable is reached through a process + file contract
 * (utils/basic_function.py:14-34 runs it; main.cu:51-342 reads the JSON and
 * seed files and writes the weights and centroids).  These entry points are
 * the in-process form of the same stages; each comment names the reference
 * code it replaces.  The `caustic_GPU` shim in this package keeps the
 * process + file contract on top of them.
 *
 * Conventions
 *  - every function returns COT_OK (0) or a negative COT_E* code and never
 *    aborts; cot_last_error() gives the message of the last failure;
 *  - coordinates are doubles, sites interleaved xy[2*i], xy[2*i+1];
 *  - domains are {xmin, xmax, ymin, ymax} (the reference's sample_domain /
 *    proj_domain order, main.cu:81-83);
 *  - the density image is density[ix + iy*nx] with nx pixels along x (the
 *    reference's d_picture[i_x + i_y*size[0]], basic_function.cuh:805);
 *  - pointer arguments are caller-owned and live in host memory unless
 *    `mem` says COT_MEM_DEVICE (then they are device pointers on the
 *    handle's device); the library owns its workspace;
 *  - one handle per stream; a handle is not shared between host threads.
 */
#ifndef CAUSTICOT_H_
#define CAUSTICOT_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define COT_API __attribute__((visibility("default")))
#else
#define COT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define COT_VERSION_MAJOR 0
#define COT_VERSION_MINOR 1
#define COT_VERSION_PATCH 0

enum {
    COT_OK = 0,
    COT_EINVAL = -1,       /* bad argument */
    COT_ECUDA = -2,        /* CUDA runtime error */
    COT_ENOPROBLEM = -3,   /* cot_set_problem has not been called */
    COT_ECAPACITY = -4,    /* caller buffer too small */
    COT_ERING = -5,        /* a cell exceeded the vertex capacity */
    COT_ENOTCONV = -6,     /* solver stopped before the tolerance */
    COT_ETIMEOUT = -7,     /* a bounded device wait gave up */
    COT_ENOMEM = -8,       /* allocation failed */
    COT_ECANCELLED = -9    /* the progress callback asked the solve to stop */
};

enum { COT_MEM_HOST = 0, COT_MEM_DEVICE = 1 };

/* Solver flavours.
 * COT_SOLVE_REFERENCE: direct_ot's loop (ot_op.cuh:289-537): backtracking
 *   with simple decrease from initial_step, reject when a ring is too
 *   complex, restart at step <= 1e-4*initial_step, stop when the gradient
 *   norm taken at the start of the iteration is below `tol` and no cell is
 *   empty.
 * COT_SOLVE_WOLFE: L-BFGS with a strong-Wolfe line search (bracket by
 *   doubling, zoom by bisection), stop when max_i |mu_i - nu_i| / nu_i <= tol.
 */
enum { COT_SOLVE_REFERENCE = 0, COT_SOLVE_WOLFE = 1 };

typedef struct cot_handle cot_handle;

typedef struct {
    int device;          /* CUDA device ordinal */
    int bucket_size;     /* target sites per neighbour bucket (0: default 16) */
    int cells_per_warp;  /* cells one warp works at once in the solve's cell
                            kernel: 1 (32 lanes a cell), 2 (16 lanes a cell,
                            rings above 16 vertices redone on 32) or 4 (8
                            lanes a cell, rings above 8 redone on 32); 0:
                            default (1) */
    int max_ring;        /* ring-complexity reject threshold (0: 200, as
                            ot_op.cuh:376 max_edge_num/2) */
    int profile;         /* 1: time every cell-kernel launch with CUDA events
                            recorded on the launching stream */
} cot_config;

/* Kernel accounting of a handle (no reference counterpart: measurement). */
typedef struct {
    long long launches;       /* kernels this library launched */
    long long cell_launches;  /* launches of the fused cell kernel */
    double cell_ms;           /* their summed device time (profile=1) */
    long long evaluations;    /* objective evaluations */
} cot_kernel_stats;

typedef struct {
    int mode;            /* COT_SOLVE_* */
    int history;         /* L-BFGS memory (reference: history_size) */
    int max_iter;        /* reference: total_iter */
    double tol;          /* see the mode */
    double initial_step; /* reference: initial_step */
    double c1, c2;       /* Wolfe constants (0: 1e-4, 0.9) */
    int max_ls;          /* line-search trials per iteration (0: 30) */
    int use_graph;       /* >= 0 (default): the trial loop runs on the device
                            as one CUDA graph (a WHILE node, one line-search
                            trial per pass; the host looks only when it stops),
                            or the host-driven loop if the handle's stream
                            cannot be captured (the legacy default stream);
                            -1: the host-driven loop, one 64-byte control-block
                            read per trial */
} cot_solve_opts;

typedef struct {
    int iterations;
    int evaluations;     /* objective evaluations incl. every trial */
    int restarts;
    int converged;
    double f;            /* final objective */
    double max_rel_err;  /* max_i |mu_i - nu_i| / nu_i at exit */
    double grad_norm;    /* ||mu - nu||_2 at exit */
    int empty_cells;     /* cells with mu_i == 0 at exit */
    int ring_overflows;  /* trials rejected as too complex */
    double ms;           /* device time of the solve */
} cot_solve_stats;

/* Library version. */
COT_API int cot_version(int *major, int *minor, int *patch);

/* Handle life cycle (replaces the cudaMalloc/cudaFree blocks of
 * ot_op.cuh:121-152, 548-583). */
COT_API int cot_create(const cot_config *cfg, cot_handle **out);
COT_API int cot_destroy(cot_handle *h);

/* Stream used by every call on the handle (NULL: the handle's own stream). */
COT_API int cot_set_stream(cot_handle *h, void *cuda_stream);

/* Problem definition: sites, target masses, target density, domain.
 * Replaces main.cu:130-198 (reading proj_xy and the picture) plus the
 * density normalisation of ot_op.cuh:81-88,154: the density is scaled so
 * that it sums to sum(nu), which is the reference's area_scalar.
 * Mirror sites (power_diagram.cpp:26-49) are not needed: a mirror never
 * wins over its own site inside proj_domain, so every cell restricted to
 * proj_domain is the same with or without them. */
COT_API int cot_set_problem(cot_handle *h, const double *sites_xy, const double *nu, int n,
                    const double *density, int nx, int ny, const double proj_domain[4],
                    int mem);

/* One objective + gradient evaluation at weights w (caller order).
 * Replaces polygons_in_VD + compute_inte + compute_subtract + compute_f
 * (ot_op.cuh:208-278, 364-403).  Outputs may be NULL.
 *   f_total = sum_i f_i; mu[i]; g[i] = mu_i - nu_i; f_cell[i] = f_i. */
COT_API int cot_eval(cot_handle *h, const double *w, double *f_total, double *mu, double *g,
             double *f_cell, int mem);

/* Cells at weights w, restricted to proj_domain: CCW rings and, for every
 * ring edge, the index of the neighbouring site (-1..-4 for the domain
 * sides bottom, right, top, left).  Replaces the polygons / start_num /
 * length arrays of polygons_in_VD (power_diagram.cpp:8-134) after the
 * domain clip of basic_function.cuh:763.  ring_offsets has n+1 entries;
 * capacity is the size of ring_xy in vertices.  Host memory only. */
COT_API int cot_cells(cot_handle *h, const double *w, int *ring_offsets, double *ring_xy,
              int *ring_nbr, int capacity);

/* Solve for the weights from w_inout (caller order).  Replaces the solver
 * loop of direct_ot (ot_op.cuh:289-537). */
COT_API int cot_solve(cot_handle *h, double *w_inout, const cot_solve_opts *opts,
              cot_solve_stats *stats, int mem);

/* Solve count independent problems, one per handle (all on one device,
 * each handle at most once), in a single CUDA graph launch on the first
 * handle's stream (which must not be the legacy default stream): handle k's
 * solve is one branch of the graph -- its first evaluation, then its own
 * device-driven trial loop -- and the branches run concurrently, so many
 * small instances share the GPU instead of queueing.  w_inout[k]: host array
 * of handle k's n weights (start in, result out).  stats (nullable): count
 * entries; their ms is the time of the whole batch.  Progress callbacks are
 * not called.  COT_ENOTCONV when some solve stopped before the tolerance
 * (its stats say which).  Errors are reported on the first handle.  Replaces
 * running the reference's caustic_GPU once per instance. */
COT_API int cot_solve_batch(cot_handle *const *handles, int count, double *const *w_inout,
                            const cot_solve_opts *opts, cot_solve_stats *stats);

/* Options of the damped Newton solve (0 selects the default in brackets). */
typedef struct {
    double tol;          /* stop when max_i |mu_i - nu_i| / nu_i <= tol */
    int max_iter;        /* Newton steps [100] */
    double cg_rtol;      /* relative residual of each step's linear solve [0.1] */
    int cg_max_iter;     /* conjugate-gradient iterations per step [2000] */
    int lbfgs_chunk;     /* while a cell is empty the L-BFGS runs, stopping as */
    int lbfgs_rounds;    /* soon as none is, for at most lbfgs_chunk x
                            lbfgs_rounds iterations [10 x 50] */
    int history;         /* L-BFGS memory of those rounds and of the fall-back [10] */
    int shrink_steps;    /* when the start leaves a cell empty: try the start
                            scaled by 1/2, 1/4, ... (this many times) and keep
                            the first that empties none, before any L-BFGS;
                            the weights w = 0 never empty a cell [0: off] */
} cot_newton_opts;

typedef struct {
    int newton_iterations;  /* accepted Newton steps */
    int lbfgs_iterations;   /* L-BFGS iterations (empty-cell rounds and fall-back) */
    int evaluations;        /* objective evaluations of both */
    int cg_iterations;      /* conjugate-gradient iterations, summed over the steps */
    int converged;
    int fallback;           /* 1: the Newton steps stalled and the L-BFGS finished */
    double max_rel_err;     /* at exit */
    double grad_norm;       /* ||mu - nu||_2 at exit */
    int empty_cells;
    double ms;              /* device time */
} cot_newton_stats;

/* Damped Newton solve of the same problem to max_i |mu_i - nu_i| / nu_i <=
 * tol.  No counterpart in the reference (its solvers are first-order:
 * direct_ot's L-BFGS, ot_op.cuh:289-537, and aarl_direct_ot's Anderson
 * acceleration).  The masses' Jacobian dmu/dw is a weighted graph Laplacian
 * over the cells' shared edges: entry (i, j) is -(integral of the density
 * along the edge) / (2 |s_i - s_j|).  Each step solves dmu/dw d = nu - mu by
 * Jacobi-preconditioned conjugate gradients (one cooperative kernel) and
 * halves the step until every mass stays above half its starting minimum and
 * |mu - nu| falls by the factor (1 - tau/2) (Kitagawa, Merigot and Thibert,
 * J. Eur. Math. Soc. 2019).  A cell that is empty has no row, so while some
 * cell is empty the solve first runs this library's L-BFGS
 * (COT_SOLVE_WOLFE) until every cell has mass; if the Newton steps stall
 * the L-BFGS finishes from the last point (stats->fallback).  w_inout in
 * caller order (mem: COT_MEM_HOST or COT_MEM_DEVICE).  COT_ENOTCONV when the
 * tolerance was not reached. */
COT_API int cot_solve_newton(cot_handle *h, double *w_inout, const cot_newton_opts *opts,
                             cot_newton_stats *stats, int mem);

/* The masses' Jacobian dmu/dw at weights w (caller order; w host or device
 * per mem) as CSR in host memory: row i lists (j, dmu_i/dw_j) for j = i and
 * every site j that shares an edge with cell i, columns ascending.
 * row_offsets has n+1 entries; *nnz receives the entry count.  With cols or
 * vals NULL only row_offsets and *nnz are filled (a size query); else
 * capacity must be at least *nnz (COT_ECAPACITY).  No counterpart in the
 * reference (the matrix of cot_solve_newton's steps). */
COT_API int cot_mass_jacobian(cot_handle *h, const double *w, int mem, int *row_offsets, int *cols, double *vals,
                              int capacity, int *nnz);

/* Inputs of the Fresnel-reweighted solve (host arrays, caller order). */
typedef struct {
    const double *points_xy;     /* source (lens) sites, 2n */
    const double *input_light;   /* incoming direction per site, 3n */
    const double *inside_light;  /* refracted direction per site, 3n, unit */
    const double *height;        /* lens thickness along inside_light, n */
    double z_of_len, z_of_receiver, refraction_index;
    double sample_domain[4];
    int aa_history;              /* Anderson memory (aa_history_size) */
    double aa_fixed_para;        /* step of the fixed-point map (aa_fixed_para) */
    int lbfgs_prepass;           /* if_aa_op_initial: L-BFGS first, nu fixed */
} cot_aarl_inputs;

/* Solve of the later outer iterations: aarl_direct_ot (ot_op.cuh:591-1385).
 * The target masses are the problem's masses (the source masses lambda)
 * re-weighted by the Fresnel transmittance of each cell's light path
 * (compute_energy_remain_rate, basic_function.cuh:437-494), evaluated at the
 * plain cell centroids and renormalised to the same total; they change with
 * the weights.  Optional L-BFGS pre-pass with the masses fixed (opts: the
 * reference's history_size, total_iter, convergence_tolerance,
 * initial_step), then Anderson acceleration of w <- w + aa_fixed_para * g,
 * stopped when ||mu - nu||_2 < tol (empty cells checked every tenth
 * iteration, as the reference).  On return the problem's masses are the
 * re-weighted ones.  w_inout in host memory. */
COT_API int cot_solve_aarl(cot_handle *h, double *w_inout, const cot_aarl_inputs *in,
                           const cot_solve_opts *opts, cot_solve_stats *stats);

/* Progress of a solve.  The phases are the reference's three loops:
 * COT_PHASE_LBFGS (direct_ot, ot_op.cuh:289-537, i.e. cot_solve),
 * COT_PHASE_PREPASS (the L-BFGS pre-pass of aarl_direct_ot,
 * ot_op.cuh:823-1074) and COT_PHASE_ANDERSON (its Anderson loop,
 * ot_op.cuh:1135-1323). */
enum { COT_PHASE_LBFGS = 0, COT_PHASE_PREPASS = 1, COT_PHASE_ANDERSON = 2 };

/* Called at the start of each phase (iteration = -1: the starting point,
 * after the masses of that phase are set), after every iteration whose
 * 0-based index (the reference's `iter`) is a multiple of `every`, and after
 * the last iteration of each phase.  cot_solve_aarl reports the start of the
 * pre-pass phase even when the pre-pass is off.
 * status: 0 the phase goes on, 1 it has just converged, 2 it has stopped
 * without converging (iteration limit or line-search failure).  w: the
 * weights after that iteration; nu: the target masses in force (re-weighted
 * ones in the Anderson phase); both host arrays of n doubles in caller order,
 * valid during the call only.  grad_norm = ||mu - nu||_2 and max_rel_err at
 * w.  The callback may call cot_eval, cot_cells, cot_centroids and
 * cot_render on the same handle: those stage their weights apart from the
 * solve's iterate and leave its state alone.  It must not call
 * cot_set_problem or start another solve on the handle.  A non-zero return
 * stops the solve with COT_ECANCELLED (w_inout then holds the last iterate).
 * This is how the caustic_GPU shim writes the reference's periodic and final
 * weights_<iter>.txt, render_<iter>.txt and mesh_<iter>.obj
 * (ot_op.cuh:484-535, 1020-1074, 1270-1321). */
typedef int (*cot_progress_fn)(void *user, int phase, int iteration, int status, const double *w,
                               const double *nu, int n, double grad_norm, double max_rel_err);

/* Install (fn != NULL, every >= 1) or remove (fn == NULL) the progress
 * callback of a handle. */
COT_API int cot_set_progress(cot_handle *h, cot_progress_fn fn, void *user, int every);

/* Density-weighted (weighted=1) or plain centroids of the cells at w and
 * the exist flags.  Replaces compute_center (basic_function.cuh:1056-1191,
 * ot_op.cuh:539-546). */
COT_API int cot_centroids(cot_handle *h, const double *w, double *xy, unsigned char *exist,
                  int weighted, int mem);

/* Source masses of parallel light: areas of the unweighted cells of the
 * source points inside sample_domain, normalised to total area_scalar.
 * Replaces compute_clip_area + the normalisation of ot_op.cuh:90-92,158,
 * 199-206.  Independent of the problem set on the handle. */
COT_API int cot_source_masses(cot_handle *h, const double *points_xy, int n,
                      const double sample_domain[4], double *nu_out);

/* Source masses of a point light at light[3]: solid angle each unweighted
 * source cell (inside sample_domain, in the plane z_of_len) subtends from the
 * light, normalised to total area_scalar.  Replaces solid_angle /
 * len_solid_angle + the normalisation (basic_function.cuh:558-588,635-658;
 * ot_op.cuh:160-206). */
COT_API int cot_source_masses_point_light(cot_handle *h, const double *points_xy, int n,
                                          const double sample_domain[4], const double light[3],
                                          double z_of_len, double *nu_out);

/* Diagnostic splat of nu over the pixels, nu_i * area(cell_i ∩ pixel) /
 * area(cell_i) (render, basic_function.cuh:660-741), scaled by the
 * reference's gray_multiple = sum(raw density) / area_scalar
 * (ot_op.cuh:215).  out has nx*ny entries (host memory). */
COT_API int cot_render(cot_handle *h, const double *w, double gray_multiple, double *out);

/* Allocation-free evaluation summary.  No counterpart in the reference (its
 * host code copies the per-cell arrays back and sums them on the CPU).
 * For callers that may not call cudaMalloc where they need these numbers:
 * code recording a CUDA stream capture (an allocation there breaks the
 * capture) and hosts that give the library a fixed memory budget with no
 * allocations after start-up.  Reduces per-cell results already on the
 * device -- mu, f_cell, nu (n doubles each, device pointers, e.g. the outputs
 * of cot_eval with COT_MEM_DEVICE) -- to out[0..3] (device) =
 * {sum f_cell, max |mu - nu| / nu, sum (mu - nu)^2, count(mu == 0)};
 * a NaN mass makes out[1] +inf, so that it never passes a tolerance.
 * Allocates nothing: its scratch is one fixed array per device
 * (COT_NOALLOC_MAX_BLOCKS x 4 doubles + a counter, about 32 KB) that every
 * GPU loading the library holds until exit; n above COT_NOALLOC_MAX_N is
 * rejected with COT_EINVAL.  All calls share that array: calls that overlap
 * on the GPU race, so order them on one stream.  The first call on a device
 * looks the array's address up; make it before any stream capture starts.
 * Errors are read with cot_last_error(NULL, ...). */
#define COT_NOALLOC_BLOCK_ELEMS 2048
#define COT_NOALLOC_MAX_BLOCKS 1024
#define COT_NOALLOC_MAX_N (COT_NOALLOC_BLOCK_ELEMS * COT_NOALLOC_MAX_BLOCKS)
#define COT_NOALLOC_MAX_DEVICES 64
COT_API int cot_eval_summary_noalloc(const double *mu, const double *f_cell, const double *nu, int n,
                                     double *out, void *cuda_stream);

/* Kernel accounting since the last reset; waits for the handle's stream.
 * reset=1 clears the counters after reading. */
COT_API int cot_get_kernel_stats(cot_handle *h, cot_kernel_stats *out, int reset);

/* Which slow paths the last evaluation of this handle took (diagnostics;
 * no counterpart in the reference): out[0] rings above 32 vertices (the
 * large-ring pass), out[1] cells whose certificate walk overflowed and was
 * finished by a block of warps, out[2] cells integrated first because of a
 * large pixel box, out[3] cells whose integration was shared by several
 * warps.  Waits for the handle's stream; valid until the next evaluation. */
COT_API int cot_eval_counters(cot_handle *h, int *out4);

/* Message of the last failure on this handle (or of the last failed
 * cot_create when h is NULL). */
COT_API int cot_last_error(cot_handle *h, char *buf, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* CAUSTICOT_H_ */
