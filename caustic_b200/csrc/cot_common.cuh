// Internal types shared by the solver's CUDA translation units.
//
// Data layout in HBM (one problem per handle):
//   sites     double2 xy[n]      sorted by neighbour bucket, then input index
//   masses    double  nu[n]      same order
//   buckets   int     bstart[nb+1]  CSR into the sorted sites, row-major
//             (bucket (u,v) = u + v*bx) over the sites' bounding box
//   tree      double4 tstat[nodes] {box centre x, y, half width, half height} (static; empty: half width -1)
//             double4 tdyn[nodes]  {ax, ay, B, 0} weight bound (per evaluation)
//             level 0 = the buckets, each higher level merges 2x2 nodes
//   density   double  rho[nx*ny] density per unit area, rho[ix + iy*nx]
//
// Every per-site vector the solver keeps (w, mu, L-BFGS history) is in the
// sorted order; the C ABI permutes at the boundary.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define COT_MAX_LEVELS 24
#define COT_MAX_HIST 32
#define COT_BASIS (2 * COT_MAX_HIST + 1)
#define COT_NBC 16  // cached neighbours per cell
#ifndef COT_BLEAF
#define COT_BLEAF 64 // leaf buckets listed per bucket by the bucket walk (<= the frontier)
#endif

// Static geometry, passed by value to the kernels.
struct CotGeo {
    int n;                 // sites
    const double2 *xy;     // sorted sites
    const double *nu;      // sorted masses
    const int *bstart;     // bucket CSR, nb + 1 entries
    const int *sbucket;    // bucket of each sorted site
    int bx, by;            // bucket grid
    double ox, oy;         // bucket grid origin
    double ihx, ihy;       // inverse bucket extent
    int nlev;              // tree levels (level 0 = buckets)
    int lev_off[COT_MAX_LEVELS];
    int lev_w[COT_MAX_LEVELS];
    int lev_h[COT_MAX_LEVELS];
    const double4 *tstat;  // {box centre x, y, half width, half height}; empty: half width < 0
    double4 *tdyn;         // {ax, ay, B, 0}: w_j/2 <= a.s_j + B over the node
    const double *rho;     // density per unit area
    int nx, ny;            // pixels along x, along y
    double pd[4];          // proj_domain {xmin, xmax, ymin, ymax}
    double xs, ys;         // pixel extent (reference x_step, y_step)
    double ixs, iys;       // their reciprocals
    double margin;         // safety margin of the bound-tree exclusion test
};

// Per-evaluation scalar results (written by the reduction's last block).
struct CotEvalOut {
    double f;          // sum_i f_i
    double gtd;        // sum_i (mu_i - nu_i) d_i   (0 without a direction)
    double maxrel;     // max_i |mu_i - nu_i| / nu_i
    double gnorm2;     // sum_i (mu_i - nu_i)^2
    int empty;         // cells with mu_i == 0
    int overflow;      // cells above the ring capacity / threshold
    int maxnv;         // largest ring
    int pad;
};

// Solver state kept on the device; every control decision is taken by one
// device thread so that the loop can run without host round trips.
struct CotSolver {
    // control block: the host reads these first 16 ints after each trial
    int ls_active;       // 1 while line-search trials remain
    int accepted;        // 1 when the last trial was accepted
    int done;
    int converged;
    int failed;
    int iter, evals, restarts, ring_rejects;
    int k;               // stored pairs (loop_iter of the reference)
    int restart;         // reference's restart flag
    int trials;
    int final_eval;      // Wolfe: the pending trial re-evaluates lo
    int need_begin;      // 1 at an iteration boundary (set by accept / reject)
    int eval_mark;       // evals when the iteration began (direction pending while equal)
    int pause_iter;      // graph solve: the device loop stops when iter reaches this
    // options
    int mode;            // COT_SOLVE_*
    int m;               // history
    int max_ls;
    int max_iter;
    int max_ring;
    int stop_nonempty;   // 1: the solve also stops (unconverged) once no cell is empty
    double c1, c2, t0, tol;
    double H0;
    double rho[COT_MAX_HIST];
    double alpha[COT_MAX_HIST];
    double delta[COT_BASIS];            // direction = sum delta_j * basis_j
    double G[COT_BASIS * COT_BASIS];    // Gram matrix of the basis
    // current point
    double f, gd;
    double maxrel, gnorm2;
    int empty;
    int empty_stale;
    double gnorm_stale;  // ||g|| taken at the start of the iteration
    // line search
    double t, lo, hi, f_lo;
    // last trial
    CotEvalOut last;
};

#define COT_CUDA_TRY(expr)                                                                 \
    do {                                                                                   \
        cudaError_t e__ = (expr);                                                          \
        if (e__ != cudaSuccess) return cot::fail(h, COT_ECUDA, #expr, cudaGetErrorString(e__)); \
    } while (0)

namespace cot {

// Launch context: the stream plus the kernel accounting of the handle.
struct CotCtx {
    cudaStream_t s = nullptr;
    long long launches = 0;
    long long cell_launches = 0;
    long long evaluations = 0;
    bool profile = false;
    cudaEvent_t *ev = nullptr;  // pool of event pairs (profile)
    int ev_cap = 0;
    int ev_used = 0;
};

// Launchers implemented in cot_cells.cu.
struct CellsArgs {
    const double *w;       // weights (base point)
    const double *d;       // direction (nullable)
    const double *tptr;    // device scalar step (nullable => 0)
    double *wt;            // trial weights out
    double *wbar;          // per bucket mean w/2 (scratch)
    double *mu;            // per cell mass out
    double *fc;            // per cell objective out, without its -w_i nu_i term
    int *nv;               // per cell ring size out
    int *ovf_list;         // cells whose ring outgrew the first pass
    int *ovf_list2;        // cells whose ring outgrew the second pass
    int *ovf_count;        // device counters: [0] ovf_list size, [1] first-pass
                           // fetch, [2] large-ring fetch over ovf_list, [3]
                           // ovf_list2 size, [4] second-pass fetch, [5]
                           // large-ring fetch over ovf_list2, [6] integration
                           // fetch, [7] unused, [8] the certificate
                           // kernel's fetch, [9] the bucket walk's fetch
    int *nbc;              // cached neighbours, COT_NBC per cell (nullable)
    int *nbn;              // their count per cell (0: none)
    double *cen;           // centroids (nullable)
    unsigned char *exist;  // exist flags (nullable)
    int weighted;          // centroid flavour
    double *solid;         // solid angle of each cell from a point light (nullable)
    double solid_z;        // plane of the cells
    double solid_light[3]; // light position
    double *splat;         // render output, nx*ny (nullable)
    double splat_scale;    // gray_multiple of the render
    double2 *rbuf;         // ring vertices of the solve's path, 32 per cell
    int *lbuf;             // their edge generators between k_cells_first and k_cells_walk
    int *cstate;           // per cell: ring size (+ cached flag) after phase 1, -1 = finished
    double *ring_xy;       // optional fixed-stride ring dump (nullable)
    int *ring_lab;
    int ring_cap;
    // Newton solve only (zero elsewhere): the mass Jacobian's rows
    int keep_labels;       // 1: the final ring's edge generators stay in lbuf
    double *hbig_val;      // rows of rings above COT_RCAP vertices, COT_HBIG_W entries a slot (nullable)
    int *hbig_col;
    int hbig_cap;          // slots
    int *hcnt;             // per cell: row length (ELL), or -(slot + 1) for a big row
    double *hdiag;         // per cell: dmu_i/dw_i
    int *herr;             // set when a big row found no slot
    // the leaf buckets that can reach any ring of a bucket, rebuilt by each
    // evaluation on the two-kernel path (nullable): COT_BLEAF per bucket in
    // walk order, the count (-1: too many)
    int *blist;
    int *bcnt;
    // cells whose integration covers a large pixel box, listed by the
    // certificate kernel so that the integration kernel starts them first
    // (two-kernel path only; nullable)
    int *hlist;
    // cells whose certificate walk overflowed its frontier, finished by
    // k_cells_heavy a block each (two-kernel path only; nullable)
    int *wlist;
    // cells whose integration is shared by several warps (two-kernel path;
    // nullable): their list (hsplit_cap at most), the parts' raw sums and a
    // ticket per slot (0 between evaluations)
    int *hsplit;
    double *hpart;
    unsigned int *hticket;
    int hsplit_cap;
};

#define COT_HBIG_W 256  // entries of a big Jacobian row (the large-ring pass's capacity)
#define COT_SPLIT 8          // warps that share the integration of a cell with a very large pixel box
#define COT_HSPLIT_CAP 2048  // such cells per evaluation (the rest are integrated whole, first)

void launch_eval(const CotGeo &g, const CellsArgs &a, int cells_per_warp, int num_sms,
                 CotCtx &c);
void launch_reduce(const CotGeo &g, const double *mu, const double *fc, const int *nv,
                   const double *wt, const double *d, int max_ring, double *partials,
                   unsigned int *ticket, CotEvalOut *out, CotSolver *solver, CotCtx &c);
int reduce_blocks(int n);

// Launchers implemented in cot_solver.cu.
void launch_begin_iteration(CotSolver *S, CotCtx &c);
void launch_direction(const CotGeo &g, const CotSolver *S, const double *Sv, const double *Yv,
                      const double *mu, double *d, CotCtx &c);
void launch_accept(const CotGeo &g, CotSolver *S, double *Sv, double *Yv, double *w,
                   const double *wt, double *mu, const double *mut, const double *d,
                   double *partials, unsigned int *ticket, int initial, CotCtx &c);
void launch_reject(CotSolver *S, CotCtx &c);
void launch_loop_cond(cudaGraphConditionalHandle hc, const CotSolver *S, CotCtx &c);
void launch_reject_cond(cudaGraphConditionalHandle hc, CotSolver *S, CotCtx &c);
void launch_init_from_eval(CotSolver *S, const CotEvalOut *out, CotCtx &c);
void configure_cells_kernels();

// Problem set-up on the device (cot_build.cu).  build_stats writes a
// {xmin, xmax, ymin, ymax, sum nu, first bad site, first bad mass} record to
// site_out and {sum, first bad pixel} to dens_out; build_sort with temp ==
// nullptr only sets *temp_bytes.
cudaError_t build_stats(int n, const double *xy, const double *nu, long long npix, const double *dens,
                        double *partials, unsigned int *ticket, void *site_out, void *dens_out, cudaStream_t s);
size_t build_partials_doubles();
cudaError_t build_sort(int n, const double *xy, const double *nu, double ox, double oy, double ihx, double ihy,
                       int bx, int by, int *keys, int *idx, int *keys2, int *idx2, void *temp, size_t *temp_bytes,
                       double2 *sxy, double *snu, int *sbucket, int *perm, int *bstart, cudaStream_t s);
cudaError_t build_tree(int nb, const int *bstart, const double2 *sxy, double L, int nlev, const int *off,
                       const int *lw, const int *lh, double4 *tstat, cudaStream_t s);
cudaError_t build_density(long long npix, const double *in, double gray, double ga, double *rho, cudaStream_t s);

// Launchers implemented in cot_newton.cu (the Newton solve's kernels).
struct NewtonEvalStats {
    double gnorm2;   // sum (mu - nu)^2
    double minmu;    // min mu
    double maxrel;   // max |mu - nu| / nu (+inf with a NaN)
    int empty;       // cells with mu == 0
    int maxnv;       // largest ring
};
struct PcgState {
    int iterations;
    int error;       // a grid barrier gave up waiting
    double rr0, rr;  // squared residual norms at the start and the end
    unsigned int bar_count, bar_gen;
};
void launch_hessian(const CotGeo &g, const double2 *rbuf, const int *lbuf, const int *nv, double *hval, int *hcol,
                    int *hcnt, double *hdiag, CotCtx &c);
void launch_newton_stats(int n, const double *mu, const double *nu, const int *nv, double *partials,
                         unsigned int *ticket, NewtonEvalStats *out, CotCtx &c);
int pcg_max_blocks(int n, int num_sms);
cudaError_t launch_pcg(int n, const double *hval, const int *hcol, const int *hcnt, const double *hbig_val,
                       const int *hbig_col, const double *hdiag, const double *b, double *x, double *r, double *z,
                       double *pa, double *pb, double *q, double *partials, PcgState *st, double rtol, int max_it,
                       int blocks, CotCtx &c);
void launch_fcell_full(int n, const double *fc, const double *wt, const double *nu, double *out, CotCtx &c);
void launch_fresnel_nu(int n, const double *cen, const double *src, const double *inl, const double *insl,
                       const double *hgt, const double *lam, double zl, double zr, double eta, double total,
                       double *energy, double *partials, double *nu, CotCtx &c);
void launch_aa_store_gram(int n, const double *w, const double *mu, const double *nu, double alpha, double *G,
                          double *F, int h, int cnt, double *partials, unsigned int *ticket, double *row, CotCtx &c);
void launch_aa_combine(int n, const double *F, const double *coef, int cnt, const double *w, double *d, CotCtx &c);

}  // namespace cot
