// C ABI of the solver (declarations and reference mapping: include/causticot.h).
//
// Host side of a handle: the one-time problem set-up (bucket counting sort,
// bound-tree statistics, density scaling), the permutations between the
// caller's site order and the bucket order used on the device, and the solve
// loop that launches the device kernels and reads one control block per
// line-search trial.
#include "../../include/causticot.h"
#include "cot_common.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <climits>
#include <string>
#include <vector>

struct CotProblemDev {
    int n = 0;
    int nb = 0;
    int nodes = 0;
    size_t cap_n = 0, cap_nb = 0, cap_nodes = 0, cap_pix = 0;  // allocated sizes (grow only)
    // set-up scratch: partial sums, their tickets, the input statistics,
    // the sort's temporary storage
    double *bpart = nullptr;
    unsigned int *bticket = nullptr;
    unsigned char *bstat = nullptr;
    void *cubtmp = nullptr;
    size_t cubtmp_bytes = 0;
    unsigned long long gen = 0;  // changes whenever the problem or its buffers change
    double2 *xy = nullptr;
    double *nu = nullptr;
    int *bstart = nullptr;
    int *sbucket = nullptr;
    double4 *tstat = nullptr;
    double4 *tdyn = nullptr;
    double *rho = nullptr;
    int *perm = nullptr;   // sorted -> caller index
    std::vector<int> hperm;
    CotGeo geo{};
    // per evaluation
    double *w = nullptr, *wt = nullptr, *d = nullptr, *mu = nullptr, *mut = nullptr, *fc = nullptr;
    double *wq = nullptr;  // weights of the query entry points, apart from a solve's iterate w
    double *wbar = nullptr;
    int *blist = nullptr, *bcnt = nullptr;  // the bucket walk's leaf lists (solves only)
    double2 *rbuf = nullptr;  // ring vertices between the cell and integration kernels
    int *lbuf = nullptr;      // ring generators between the two ring-building kernels
    int *cstate = nullptr;    // per-cell state between them
    int *nv = nullptr, *ovf_list = nullptr, *ovf_list2 = nullptr, *ovf_count = nullptr;
    int *wlist = nullptr;  // cells whose certificate walk overflowed (finished a block each)
    int *hsplit = nullptr;           // cells whose integration is shared by several warps
    double *hpart = nullptr;         // their parts' raw sums
    unsigned int *hticket = nullptr; // a ticket per slot, 0 between evaluations
    int *nbc = nullptr, *nbn = nullptr;        // neighbour cache of the solves
    int *nbc_q = nullptr, *nbn_q = nullptr;    // and of the query entry points
    double *partials = nullptr;
    unsigned int *ticket = nullptr;
    CotEvalOut *out = nullptr;
    double *tmp = nullptr;  // caller-order staging (2n doubles)
    // solver
    CotSolver *S = nullptr;
    double *Sv = nullptr, *Yv = nullptr;
    int hist_alloc = 0;
    // Newton solve (allocated by its first call): the Jacobian rows (ELL,
    // entry k of cell i at [k * n + i]), the rows of rings above 32
    // vertices, the conjugate-gradient vectors and the step
    double *hval = nullptr, *hdiag = nullptr, *hbig_val = nullptr;
    int *hcol = nullptr, *hcnt = nullptr, *hbig_col = nullptr, *herr = nullptr;
    int hbig_cap = 0;
    double *nb_b = nullptr, *nb_r = nullptr, *nb_z = nullptr, *nb_pa = nullptr, *nb_pb = nullptr, *nb_q = nullptr;
    double *nb_part = nullptr, *nb_tau = nullptr;
    cot::PcgState *pcg = nullptr;
    cot::NewtonEvalStats *nst = nullptr;
    unsigned int *nticket = nullptr;
};

struct cot_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cot_config cfg{};
    int num_sms = 148;
    std::string err;
    CotProblemDev P;
    bool has_problem = false;
    CotSolver *hS = nullptr;  // pinned mirror of the control block
    cot::NewtonEvalStats *hN = nullptr;  // pinned copies of the Newton solve's trial statistics
    cot::PcgState *hP = nullptr;         // and of its inner solve's state
    unsigned char *hB = nullptr;         // pinned copy of the set-up's input statistics
    // the device-driven trial loop's graph, kept while the problem, its
    // buffers and the stream stay the same (instantiating it costs more than
    // a short solve of a small problem)
    cudaGraphExec_t trial_exec = nullptr;
    cudaStream_t trial_stream = nullptr;
    unsigned long long trial_gen = 0;
    long long trial_counts[3] = {0, 0, 0};
    cot::CotCtx ctx;
    // progress callback (cot_set_progress) and its caller-order buffers
    cot_progress_fn prog_fn = nullptr;
    void *prog_user = nullptr;
    int prog_every = 1;
    std::vector<double> prog_w, prog_nu;
    cot::CotCtx &c()
    {
        ctx.s = stream;
        return ctx;
    }
};

static std::string g_create_err;
static std::atomic<unsigned long long> g_problem_gen{0};  // problem generations (any handle, any host thread)

namespace cot {

int fail(cot_handle *h, int code, const char *what, const char *detail)
{
    std::string m = std::string(what) + (detail ? std::string(": ") + detail : std::string());
    if (h) h->err = m;
    else g_create_err = m;
    return code;
}

static int failf(cot_handle *h, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return fail(h, code, buf, nullptr);
}

// ---- small device helpers --------------------------------------------------
__global__ void k_gather(int n, const int *__restrict__ perm, const double *__restrict__ src, double *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}
__global__ void k_scatter(int n, const int *__restrict__ perm, const double *__restrict__ src, double *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[perm[i]] = src[i];
}
__global__ void k_scatter2(int n, const int *__restrict__ perm, const double *__restrict__ src, double *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        dst[2 * perm[i]] = src[2 * i];
        dst[2 * perm[i] + 1] = src[2 * i + 1];
    }
}
__global__ void k_scatter_u8(int n, const int *__restrict__ perm, const unsigned char *__restrict__ src,
                             unsigned char *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[perm[i]] = src[i];
}
__global__ void k_grad(int n, const double *__restrict__ mu, const double *__restrict__ nu, double *__restrict__ g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g[i] = mu[i] - nu[i];
}

static inline int nblk(int n) { return (n + 255) / 256; }

}  // namespace cot

using namespace cot;

// The buffers sized by the sites and pixels (with the Newton buffers and
// the L-BFGS history, which are sized by the sites too).
static void free_sized_by_sites(CotProblemDev &P)
{
    void *ptrs[] = {P.xy, P.nu, P.sbucket, P.rho, P.perm, P.w, P.wt, P.d, P.mu, P.mut, P.wq, P.fc, P.rbuf, P.lbuf,
                    P.cstate, P.nv, P.ovf_list, P.ovf_list2, P.ovf_count, P.wlist, P.hsplit, P.hpart, P.hticket, P.nbc, P.nbn, P.nbc_q, P.nbn_q, P.partials,
                    P.ticket, P.out, P.tmp, P.S, P.Sv, P.Yv, P.hval, P.hdiag, P.hbig_val, P.hcol, P.hcnt,
                    P.hbig_col, P.herr, P.nb_b, P.nb_r, P.nb_z, P.nb_pa, P.nb_pb, P.nb_q, P.nb_part, P.nb_tau, P.pcg,
                    P.nst, P.nticket, P.bpart, P.bticket, P.bstat, P.cubtmp};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    P.xy = nullptr; P.nu = nullptr; P.sbucket = nullptr; P.rho = nullptr; P.perm = nullptr;
    P.w = P.wt = P.d = P.mu = P.mut = P.wq = P.fc = nullptr;
    P.rbuf = nullptr; P.lbuf = P.cstate = P.nv = P.ovf_list = P.ovf_list2 = P.ovf_count = P.wlist = nullptr;
    P.hsplit = nullptr; P.hpart = nullptr; P.hticket = nullptr;
    P.nbc = P.nbn = P.nbc_q = P.nbn_q = nullptr;
    P.partials = nullptr; P.ticket = nullptr; P.out = nullptr; P.tmp = nullptr; P.S = nullptr;
    P.Sv = P.Yv = nullptr; P.hist_alloc = 0;
    P.hval = P.hdiag = P.hbig_val = nullptr; P.hcol = P.hcnt = P.hbig_col = P.herr = nullptr; P.hbig_cap = 0;
    P.nb_b = P.nb_r = P.nb_z = P.nb_pa = P.nb_pb = P.nb_q = P.nb_part = P.nb_tau = nullptr;
    P.pcg = nullptr; P.nst = nullptr; P.nticket = nullptr;
    P.bpart = nullptr; P.bticket = nullptr; P.bstat = nullptr; P.cubtmp = nullptr; P.cubtmp_bytes = 0;
    P.cap_n = P.cap_pix = 0;
}

// The buffers sized by the bucket grid and the tree.
static void free_sized_by_grid(CotProblemDev &P)
{
    void *ptrs[] = {P.bstart, P.tstat, P.tdyn, P.wbar, P.blist, P.bcnt};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    P.bstart = nullptr; P.tstat = P.tdyn = nullptr; P.wbar = nullptr; P.blist = P.bcnt = nullptr;
    P.cap_nb = P.cap_nodes = 0;
}

static void free_problem(CotProblemDev &P)
{
    free_sized_by_sites(P);
    free_sized_by_grid(P);
    P = CotProblemDev();
}

extern "C" int cot_version(int *major, int *minor, int *patch)
{
    if (major) *major = COT_VERSION_MAJOR;
    if (minor) *minor = COT_VERSION_MINOR;
    if (patch) *patch = COT_VERSION_PATCH;
    return COT_OK;
}

extern "C" int cot_create(const cot_config *cfg, cot_handle **out)
{
    if (!out) return fail(nullptr, COT_EINVAL, "cot_create: out is NULL", nullptr);
    *out = nullptr;
    cot_handle *h = new (std::nothrow) cot_handle();
    if (!h) return fail(nullptr, COT_ENOMEM, "cot_create: out of host memory", nullptr);
    if (cfg) h->cfg = *cfg;
    if (h->cfg.bucket_size <= 0) h->cfg.bucket_size = 16;
    if (h->cfg.cells_per_warp <= 0) h->cfg.cells_per_warp = 1;
    if (h->cfg.cells_per_warp != 1 && h->cfg.cells_per_warp != 2 && h->cfg.cells_per_warp != 4) {
        delete h;
        return failf(nullptr, COT_EINVAL, "cot_create: cells_per_warp must be 1, 2 or 4");
    }
    if (h->cfg.max_ring <= 0) h->cfg.max_ring = 200;
    h->device = h->cfg.device;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        delete h;
        return fail(nullptr, COT_ECUDA, "cot_create: no CUDA device", e != cudaSuccess ? cudaGetErrorString(e) : nullptr);
    }
    if (h->device < 0 || h->device >= ndev) {
        delete h;
        return fail(nullptr, COT_EINVAL, "cot_create: bad device ordinal", nullptr);
    }
    e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hS, sizeof(CotSolver));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hN, sizeof(NewtonEvalStats));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hP, sizeof(PcgState));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hB, 256);
    if (e != cudaSuccess) {
        if (h->hS) cudaFreeHost(h->hS);
        if (h->hN) cudaFreeHost(h->hN);
        if (h->own_stream) cudaStreamDestroy(h->own_stream);
        delete h;
        return fail(nullptr, COT_ECUDA, "cot_create", cudaGetErrorString(e));
    }
    configure_cells_kernels();
    h->stream = h->own_stream;
    if (h->cfg.profile) {
        const int cap = 1 << 16;
        h->ctx.ev = new (std::nothrow) cudaEvent_t[cap];
        if (h->ctx.ev) {
            for (int k = 0; k < cap; k++) {
                if (cudaEventCreate(&h->ctx.ev[k]) != cudaSuccess) break;
                h->ctx.ev_cap = k + 1;
            }
            h->ctx.ev_cap &= ~1;
        }
        h->ctx.profile = true;
    }
    *out = h;
    return COT_OK;
}

extern "C" int cot_destroy(cot_handle *h)
{
    if (!h) return COT_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_problem(h->P);
    if (h->ctx.ev) {
        for (int k = 0; k < h->ctx.ev_cap; k++) cudaEventDestroy(h->ctx.ev[k]);
        delete[] h->ctx.ev;
    }
    if (h->trial_exec) cudaGraphExecDestroy(h->trial_exec);
    if (h->hS) cudaFreeHost(h->hS);
    if (h->hN) cudaFreeHost(h->hN);
    if (h->hP) cudaFreeHost(h->hP);
    if (h->hB) cudaFreeHost(h->hB);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return COT_OK;
}

extern "C" int cot_set_stream(cot_handle *h, void *s)
{
    if (!h) return COT_EINVAL;
    h->stream = s ? (cudaStream_t)s : h->own_stream;
    return COT_OK;
}

extern "C" int cot_set_progress(cot_handle *h, cot_progress_fn fn, void *user, int every)
{
    if (!h) return COT_EINVAL;
    if (fn && every < 1) return fail(h, COT_EINVAL, "cot_set_progress: every must be >= 1", nullptr);
    h->prog_fn = fn;
    h->prog_user = fn ? user : nullptr;
    h->prog_every = fn ? every : 1;
    return COT_OK;
}

extern "C" int cot_get_kernel_stats(cot_handle *h, cot_kernel_stats *out, int reset)
{
    if (!h || !out) return COT_EINVAL;
    COT_CUDA_TRY(cudaSetDevice(h->device));
    COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    CotCtx &c = h->ctx;
    double ms = 0.0;
    for (int k = 0; k + 1 < c.ev_used; k += 2) {
        float t = 0.0f;
        COT_CUDA_TRY(cudaEventElapsedTime(&t, c.ev[k], c.ev[k + 1]));
        ms += t;
    }
    out->launches = c.launches;
    out->cell_launches = c.cell_launches;
    out->cell_ms = ms;
    out->evaluations = c.evaluations;
    if (reset) {
        c.launches = c.cell_launches = c.evaluations = 0;
        c.ev_used = 0;
    }
    return COT_OK;
}

extern "C" int cot_eval_counters(cot_handle *h, int *out4)
{
    if (!h || !out4) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_eval_counters: no problem set", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    int c[16];
    COT_CUDA_TRY(cudaMemcpyAsync(c, h->P.ovf_count, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    // the counters that the cell kernels fill (cot_cells.cu: launch_eval)
    out4[0] = c[0];
    out4[1] = c[11];
    out4[2] = c[10];
    out4[3] = std::min(c[13], COT_HSPLIT_CAP);
    return COT_OK;
}

extern "C" int cot_last_error(cot_handle *h, char *buf, size_t n)
{
    const std::string &m = h ? h->err : g_create_err;
    if (!buf || n == 0) return COT_EINVAL;
    std::snprintf(buf, n, "%s", m.c_str());
    return COT_OK;
}


// Build the device problem (the kernels are in cot_build.cu): input checks
// and sums, the bucket grid over the sites' box, the stable sort of the
// sites by bucket (then caller index), the static bound tree, and the
// density scaled to sum(nu) per unit area.  The host reads only the box and
// the sums.  Inputs are host arrays (copied in first) or device arrays
// (read in place) per mem.
static int build_problem(cot_handle *h, CotProblemDev &P, const double *xy_in, const double *nu_in,
                         const double *dens_in, int n, int nx, int ny, const double pd[4], int mem)
{
    cudaStream_t s = h->stream;
    const size_t npix = (size_t)nx * ny;
    // ---- buffers sized by the sites and pixels (grow only) ---------------
    if (!(P.xy != nullptr && (size_t)n <= P.cap_n && npix <= P.cap_pix)) {
        free_sized_by_sites(P);
        P.cap_n = (size_t)n;
        P.cap_pix = npix;
        const size_t N = P.cap_n;
        cudaError_t e = cudaSuccess;
        auto A = [&](void **p, size_t bytes) {
            if (e == cudaSuccess) e = cudaMalloc(p, bytes > 0 ? bytes : 16);
        };
        A((void **)&P.xy, N * sizeof(double2));
        A((void **)&P.nu, N * 8);
        A((void **)&P.sbucket, N * sizeof(int));
        A((void **)&P.rho, P.cap_pix * 8);
        A((void **)&P.perm, N * sizeof(int));
        A((void **)&P.w, N * 8);
        A((void **)&P.wt, N * 8);
        A((void **)&P.wq, N * 8);
        A((void **)&P.rbuf, N * 32 * sizeof(double2));
        A((void **)&P.lbuf, N * 32 * sizeof(int));
        A((void **)&P.cstate, N * sizeof(int));
        A((void **)&P.d, N * 8);
        A((void **)&P.mu, N * 8);
        A((void **)&P.mut, N * 8);
        A((void **)&P.fc, N * 8);
        A((void **)&P.nv, N * sizeof(int));
        A((void **)&P.ovf_list, N * sizeof(int));
        A((void **)&P.ovf_list2, N * sizeof(int));
        A((void **)&P.ovf_count, 16 * sizeof(int));
        A((void **)&P.wlist, N * sizeof(int));
        A((void **)&P.hsplit, COT_HSPLIT_CAP * sizeof(int));
        A((void **)&P.hpart, (size_t)COT_HSPLIT_CAP * COT_SPLIT * 4 * sizeof(double));
        A((void **)&P.hticket, COT_HSPLIT_CAP * sizeof(unsigned int));
        A((void **)&P.nbc, N * COT_NBC * sizeof(int));
        A((void **)&P.nbn, N * sizeof(int));
        A((void **)&P.nbc_q, N * COT_NBC * sizeof(int));
        A((void **)&P.nbn_q, N * sizeof(int));
        A((void **)&P.partials, (size_t)reduce_blocks((int)N) * (5 * COT_MAX_HIST + 8) * 8);
        A((void **)&P.ticket, sizeof(unsigned int));
        A((void **)&P.out, sizeof(CotEvalOut));
        A((void **)&P.tmp, 2 * N * 8);
        A((void **)&P.S, sizeof(CotSolver));
        A((void **)&P.bpart, build_partials_doubles() * 8);
        A((void **)&P.bticket, 2 * sizeof(unsigned int));
        A((void **)&P.bstat, 256);
        if (e == cudaSuccess) e = cudaMemsetAsync(P.bticket, 0, 2 * sizeof(unsigned int), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(P.hticket, 0, COT_HSPLIT_CAP * sizeof(unsigned int), s);
        if (e != cudaSuccess) {
            free_sized_by_sites(P);
            return fail(h, COT_ENOMEM, "cot_set_problem: device allocation", cudaGetErrorString(e));
        }
    }
    // ---- inputs on the device ------------------------------------------
    const double *dxy = xy_in, *dnu = nu_in, *dd = dens_in;
    if (mem == COT_MEM_HOST) {
        // staging: raw sites in tmp, raw masses in mut, the raw density in
        // rho (scaled there in place below)
        COT_CUDA_TRY(cudaMemcpyAsync(P.tmp, xy_in, 2 * (size_t)n * 8, cudaMemcpyHostToDevice, s));
        COT_CUDA_TRY(cudaMemcpyAsync(P.mut, nu_in, (size_t)n * 8, cudaMemcpyHostToDevice, s));
        COT_CUDA_TRY(cudaMemcpyAsync(P.rho, dens_in, npix * 8, cudaMemcpyHostToDevice, s));
        dxy = P.tmp;
        dnu = P.mut;
        dd = P.rho;
    }
    // ---- checks, box and sums (one read back) ----------------------------
    COT_CUDA_TRY(build_stats(n, dxy, dnu, (long long)npix, dd, P.bpart, P.bticket, P.bstat, P.bstat + 128, s));
    COT_CUDA_TRY(cudaMemcpyAsync(h->hB, P.bstat, 256, cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaStreamSynchronize(s));
    struct SiteStatsH {
        double xmin, xmax, ymin, ymax, nusum;
        long long bad_xy, bad_nu;
    } ss;
    struct DensStatsH {
        double sum;
        long long bad;
    } ds;
    std::memcpy(&ss, h->hB, sizeof ss);
    std::memcpy(&ds, h->hB + 128, sizeof ds);
    if (ss.bad_xy >= 0) return failf(h, COT_EINVAL, "site %lld is not finite", ss.bad_xy);
    if (ss.bad_nu >= 0) return failf(h, COT_EINVAL, "cot_set_problem: nu[%lld] must be positive", ss.bad_nu);
    if (ds.bad >= 0) return failf(h, COT_EINVAL, "density pixel %lld is negative or not finite", ds.bad);
    if (!(ds.sum > 0)) return failf(h, COT_EINVAL, "density sums to zero");
    // ---- the bucket grid and the tree's levels -----------------------------
    const double xmin = ss.xmin, xmax = ss.xmax, ymin = ss.ymin, ymax = ss.ymax;
    double L = std::max({pd[1] - pd[0], pd[3] - pd[2], xmax - xmin, ymax - ymin,
                         std::fabs(pd[0]), std::fabs(pd[1]), std::fabs(pd[2]), std::fabs(pd[3])});
    if (!(L > 0)) L = 1.0;
    double wx = std::max(xmax - xmin, 1e-9 * L), wy = std::max(ymax - ymin, 1e-9 * L);
    wx *= 1.0 + 1e-12;
    wy *= 1.0 + 1e-12;
    const int bs = h->cfg.bucket_size;
    const double nbt = std::max(1.0, (double)n / bs);
    int bx = std::max(1, (int)std::llround(std::sqrt(nbt * wx / wy)));
    int by = std::max(1, (int)std::llround(nbt / bx));
    bx = std::min(bx, 1 << 15);
    by = std::min(by, 1 << 15);
    const int nb = bx * by;
    const double hx = wx / bx, hy = wy / by;
    const double ihx = 1.0 / hx, ihy = 1.0 / hy;
    std::vector<int> off, lw, lh;
    int W = bx, H = by, total = 0;
    while (true) {
        off.push_back(total);
        lw.push_back(W);
        lh.push_back(H);
        total += W * H;
        if (W == 1 && H == 1) break;
        W = (W + 1) / 2;
        H = (H + 1) / 2;
        if ((int)off.size() >= COT_MAX_LEVELS) return failf(h, COT_EINVAL, "too many tree levels");
    }
    const int nlev = (int)off.size();
    if (!(P.bstart != nullptr && (size_t)nb <= P.cap_nb && (size_t)total <= P.cap_nodes)) {
        free_sized_by_grid(P);
        P.cap_nb = (size_t)nb;
        P.cap_nodes = (size_t)total;
        cudaError_t e = cudaMalloc(&P.bstart, (P.cap_nb + 1) * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&P.tstat, P.cap_nodes * sizeof(double4));
        if (e == cudaSuccess) e = cudaMalloc(&P.tdyn, P.cap_nodes * sizeof(double4));
        if (e == cudaSuccess) e = cudaMalloc(&P.wbar, P.cap_nb * 8);
        if (e == cudaSuccess) e = cudaMalloc(&P.blist, P.cap_nb * COT_BLEAF * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&P.bcnt, P.cap_nb * sizeof(int));
        if (e != cudaSuccess) {
            free_sized_by_grid(P);
            return fail(h, COT_ENOMEM, "cot_set_problem: device allocation", cudaGetErrorString(e));
        }
    }
    P.n = n;
    P.nb = nb;
    P.nodes = total;
    P.gen = ++g_problem_gen;
    // ---- the sort by bucket, the tree, the density -------------------------
    size_t need = 0;
    COT_CUDA_TRY(build_sort(n, dxy, dnu, xmin, ymin, ihx, ihy, bx, by, P.nv, P.ovf_list, P.ovf_list2, P.cstate,
                            nullptr, &need, P.xy, P.nu, P.sbucket, P.perm, P.bstart, s));
    if (need > P.cubtmp_bytes) {
        if (P.cubtmp) cudaFree(P.cubtmp);
        P.cubtmp = nullptr;
        P.cubtmp_bytes = 0;
        COT_CUDA_TRY(cudaMalloc(&P.cubtmp, need));
        P.cubtmp_bytes = need;
    }
    need = P.cubtmp_bytes;
    COT_CUDA_TRY(build_sort(n, dxy, dnu, xmin, ymin, ihx, ihy, bx, by, P.nv, P.ovf_list, P.ovf_list2, P.cstate,
                            P.cubtmp, &need, P.xy, P.nu, P.sbucket, P.perm, P.bstart, s));
    COT_CUDA_TRY(build_tree(nb, P.bstart, P.xy, L, nlev, off.data(), lw.data(), lh.data(), P.tstat, s));
    const double xs = (pd[1] - pd[0]) / (double)nx, ys = (pd[3] - pd[2]) / (double)ny;
    const double ga = xs * ys;
    const double gray = ds.sum / ss.nusum;
    COT_CUDA_TRY(build_density((long long)npix, dd, gray, ga, P.rho, s));
    COT_CUDA_TRY(cudaMemsetAsync(P.ticket, 0, sizeof(unsigned int), s));
    COT_CUDA_TRY(cudaMemsetAsync(P.ovf_count, 0, 16 * sizeof(int), s));
    COT_CUDA_TRY(cudaMemsetAsync(P.nbn, 0, P.cap_n * sizeof(int), s));
    COT_CUDA_TRY(cudaMemsetAsync(P.nbn_q, 0, P.cap_n * sizeof(int), s));
    COT_CUDA_TRY(cudaMemsetAsync(P.bcnt, 0xff, P.cap_nb * sizeof(int), s));     // no bucket list yet
    if (P.hcnt) COT_CUDA_TRY(cudaMemsetAsync(P.hcnt, 0, P.cap_n * sizeof(int), s));
    P.hperm.resize(n);
    COT_CUDA_TRY(cudaMemcpyAsync(P.hperm.data(), P.perm, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaStreamSynchronize(s));

    CotGeo &g = P.geo;
    g = CotGeo{};
    g.n = n;
    g.xy = P.xy;
    g.nu = P.nu;
    g.bstart = P.bstart;
    g.sbucket = P.sbucket;
    g.bx = bx;
    g.by = by;
    g.ox = xmin;
    g.oy = ymin;
    g.ihx = ihx;
    g.ihy = ihy;
    g.nlev = nlev;
    for (int l = 0; l < nlev; l++) {
        g.lev_off[l] = off[l];
        g.lev_w[l] = lw[l];
        g.lev_h[l] = lh[l];
    }
    g.tstat = P.tstat;
    g.tdyn = P.tdyn;
    g.rho = P.rho;
    g.nx = nx;
    g.ny = ny;
    for (int k = 0; k < 4; k++) g.pd[k] = pd[k];
    g.xs = xs;
    g.ys = ys;
    g.ixs = 1.0 / xs;
    g.iys = 1.0 / ys;
    g.margin = 1e-11 * L * L;
    return COT_OK;
}

extern "C" int cot_set_problem(cot_handle *h, const double *sites_xy, const double *nu, int n,
                               const double *density, int nx, int ny, const double proj_domain[4], int mem)
{
    if (!h) return COT_EINVAL;
    if (n <= 0 || !sites_xy || !nu || !density || nx <= 0 || ny <= 0 || !proj_domain)
        return fail(h, COT_EINVAL, "cot_set_problem: bad argument", nullptr);
    if (mem != COT_MEM_HOST && mem != COT_MEM_DEVICE) return fail(h, COT_EINVAL, "cot_set_problem: bad mem flag", nullptr);
    const double *pd = proj_domain;
    if (!(pd[1] > pd[0]) || !(pd[3] > pd[2]) || !std::isfinite(pd[0]) || !std::isfinite(pd[1]) ||
        !std::isfinite(pd[2]) || !std::isfinite(pd[3]))
        return fail(h, COT_EINVAL, "cot_set_problem: empty or non-finite proj_domain", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    h->has_problem = false;
    const int r = build_problem(h, h->P, sites_xy, nu, density, n, nx, ny, pd, mem);
    if (r != COT_OK) return r;
    h->has_problem = true;
    return COT_OK;
}

// Caller-order vector -> sorted device vector.
static int upload_sorted(cot_handle *h, const double *src, int mem, double *dst)
{
    CotProblemDev &P = h->P;
    size_t N = (size_t)P.n;
    if (mem == COT_MEM_DEVICE) {
        k_gather<<<nblk(P.n), 256, 0, h->stream>>>(P.n, P.perm, src, dst);
        h->ctx.launches++;
    } else {
        COT_CUDA_TRY(cudaMemcpyAsync(P.tmp, src, N * 8, cudaMemcpyHostToDevice, h->stream));
        k_gather<<<nblk(P.n), 256, 0, h->stream>>>(P.n, P.perm, P.tmp, dst);
        h->ctx.launches++;
    }
    COT_CUDA_TRY(cudaGetLastError());
    return COT_OK;
}

// Sorted device vector -> caller-order vector.
static int download_sorted(cot_handle *h, const double *src, double *dst, int mem)
{
    CotProblemDev &P = h->P;
    size_t N = (size_t)P.n;
    if (mem == COT_MEM_DEVICE) {
        k_scatter<<<nblk(P.n), 256, 0, h->stream>>>(P.n, P.perm, src, dst);
        h->ctx.launches++;
    } else {
        k_scatter<<<nblk(P.n), 256, 0, h->stream>>>(P.n, P.perm, src, P.tmp);
        h->ctx.launches++;
        COT_CUDA_TRY(cudaMemcpyAsync(dst, P.tmp, N * 8, cudaMemcpyDeviceToHost, h->stream));
    }
    COT_CUDA_TRY(cudaGetLastError());
    return COT_OK;
}

static CellsArgs cells_args(CotProblemDev &P, const double *w, const double *d, const double *tptr)
{
    CellsArgs a{};
    a.w = w;
    a.d = d;
    a.tptr = tptr;
    a.wt = P.wt;
    a.wbar = P.wbar;
    a.rbuf = P.rbuf;
    a.lbuf = P.lbuf;
    a.cstate = P.cstate;
    a.mu = P.mut;
    a.fc = P.fc;
    a.nv = P.nv;
    a.ovf_list = P.ovf_list;
    a.ovf_list2 = P.ovf_list2;
    a.ovf_count = P.ovf_count;
    a.wlist = P.wlist;
    a.hsplit = P.hsplit;
    a.hpart = P.hpart;
    a.hticket = P.hticket;
    a.hsplit_cap = COT_HSPLIT_CAP;
    // the query entry points (weights in P.wq) keep their own neighbour cache
    // so that a query made during a solve does not change the solve's clip
    // order
    const bool query = (w == P.wq);
    a.nbc = query ? P.nbc_q : P.nbc;
    a.nbn = query ? P.nbn_q : P.nbn;
    // scratch of the bucket walk (rebuilt by every evaluation that uses it)
    a.blist = P.blist;
    a.bcnt = P.bcnt;
    return a;
}

extern "C" int cot_eval(cot_handle *h, const double *w, double *f_total, double *mu, double *g, double *f_cell,
                        int mem)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_eval: no problem set", nullptr);
    if (!w) return fail(h, COT_EINVAL, "cot_eval: w is NULL", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    int r;
    if ((r = upload_sorted(h, w, mem, P.wq)) != COT_OK) return r;
    CellsArgs a = cells_args(P, P.wq, nullptr, nullptr);
    launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
    launch_reduce(P.geo, P.mut, P.fc, P.nv, P.wt, nullptr, h->cfg.max_ring, P.partials, P.ticket, P.out, nullptr, h->c());
    COT_CUDA_TRY(cudaGetLastError());
    CotEvalOut o;
    COT_CUDA_TRY(cudaMemcpyAsync(&o, P.out, sizeof o, cudaMemcpyDeviceToHost, s));
    if (mu && (r = download_sorted(h, P.mut, mu, mem)) != COT_OK) return r;
    // per-cell results staged in the second half of P.tmp (the first half
    // is the scatter's staging); the solve's vectors stay untouched
    double *stage = P.tmp + P.n;
    if (f_cell) {
        launch_fcell_full(P.n, P.fc, P.wt, P.nu, stage, h->c());
        if ((r = download_sorted(h, stage, f_cell, mem)) != COT_OK) return r;
    }
    if (g) {
        k_grad<<<nblk(P.n), 256, 0, s>>>(P.n, P.mut, P.nu, stage);
        if ((r = download_sorted(h, stage, g, mem)) != COT_OK) return r;
    }
    COT_CUDA_TRY(cudaStreamSynchronize(s));
    if (f_total) *f_total = o.f;
    if (o.maxnv > 256) return failf(h, COT_ERING, "cot_eval: a cell has more than 256 vertices");
    return COT_OK;
}

extern "C" int cot_cells(cot_handle *h, const double *w, int *ring_offsets, double *ring_xy, int *ring_nbr,
                         int capacity)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_cells: no problem set", nullptr);
    if (!w || !ring_offsets) return fail(h, COT_EINVAL, "cot_cells: NULL argument", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    const int cap = 256;
    size_t N = (size_t)P.n;
    double *rxy = nullptr;
    int *rlab = nullptr;
    COT_CUDA_TRY(cudaMalloc(&rxy, N * cap * 2 * 8));
    cudaError_t e = cudaMalloc(&rlab, N * cap * sizeof(int));
    if (e != cudaSuccess) {
        cudaFree(rxy);
        return fail(h, COT_ENOMEM, "cot_cells: device allocation", cudaGetErrorString(e));
    }
    int r = upload_sorted(h, w, COT_MEM_HOST, P.wq);
    std::vector<double> hxy;
    std::vector<int> hlab, hnv(N);
    if (r == COT_OK) {
        CellsArgs a = cells_args(P, P.wq, nullptr, nullptr);
        a.ring_xy = rxy;
        a.ring_lab = rlab;
        a.ring_cap = cap;
        launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
        hxy.resize(N * cap * 2);
        hlab.resize(N * cap);
        e = cudaMemcpyAsync(hxy.data(), rxy, N * cap * 2 * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hlab.data(), rlab, N * cap * sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hnv.data(), P.nv, N * sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) r = fail(h, COT_ECUDA, "cot_cells", cudaGetErrorString(e));
    }
    cudaFree(rxy);
    cudaFree(rlab);
    if (r != COT_OK) return r;
    // caller order, CSR
    std::vector<int> byc(N);
    for (size_t p = 0; p < N; p++) byc[P.hperm[p]] = (int)p;
    int o = 0;
    for (size_t i = 0; i < N; i++) {
        int p = byc[i];
        int m = hnv[p];
        if (m > cap) return failf(h, COT_ERING, "cot_cells: cell %zu has more than %d vertices", i, cap);
        ring_offsets[i] = o;
        if (o + m > capacity) return failf(h, COT_ECAPACITY, "cot_cells: capacity %d too small", capacity);
        for (int k = 0; k < m; k++) {
            if (ring_xy) {
                ring_xy[2 * (o + k)] = hxy[2 * ((size_t)p * cap + k)];
                ring_xy[2 * (o + k) + 1] = hxy[2 * ((size_t)p * cap + k) + 1];
            }
            if (ring_nbr) {
                int l = hlab[(size_t)p * cap + k];
                ring_nbr[o + k] = l >= 0 ? P.hperm[l] : l;
            }
        }
        o += m;
    }
    ring_offsets[N] = o;
    return COT_OK;
}

extern "C" int cot_centroids(cot_handle *h, const double *w, double *xy, unsigned char *exist, int weighted, int mem)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_centroids: no problem set", nullptr);
    if (!w || !xy || !exist) return fail(h, COT_EINVAL, "cot_centroids: NULL argument", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    size_t N = (size_t)P.n;
    int r;
    if ((r = upload_sorted(h, w, mem, P.wq)) != COT_OK) return r;
    double *cen = nullptr;
    unsigned char *ex = nullptr, *ex2 = nullptr;
    COT_CUDA_TRY(cudaMalloc(&cen, N * 2 * 8 * 2));
    cudaError_t e = cudaMalloc(&ex, N * 2);
    if (e != cudaSuccess) {
        cudaFree(cen);
        return fail(h, COT_ENOMEM, "cot_centroids: device allocation", cudaGetErrorString(e));
    }
    ex2 = ex + N;
    CellsArgs a = cells_args(P, P.wq, nullptr, nullptr);
    a.cen = cen;
    a.exist = ex;
    a.weighted = weighted ? 1 : 0;
    launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
    double *cen2 = cen + 2 * N;
    k_scatter2<<<nblk(P.n), 256, 0, s>>>(P.n, P.perm, cen, cen2);
    k_scatter_u8<<<nblk(P.n), 256, 0, s>>>(P.n, P.perm, ex, ex2);
    cudaMemcpyKind k = mem == COT_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    e = cudaMemcpyAsync(xy, cen2, N * 2 * 8, k, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(exist, ex2, N, k, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(cen);
    cudaFree(ex);
    if (e != cudaSuccess) return fail(h, COT_ECUDA, "cot_centroids", cudaGetErrorString(e));
    return COT_OK;
}

// Source masses of the reference (ot_op.cuh:90-92,156-206): cells of the
// source points (weights 0) inside the sample domain; parallel light weighs
// them by area (compute_clip_area), a point light by the solid angle they
// subtend from the light (solid_angle, basic_function.cuh:635-650);
// normalised to total area_scalar.
static int source_masses_impl(cot_handle *h, const double *points_xy, int n, const double *sd, const double *light,
                              double z, double *nu_out)
{
    COT_CUDA_TRY(cudaSetDevice(h->device));
    // unweighted cells inside the sample domain, one "pixel" of unit density
    std::vector<double> one(n, 1.0), dens(1, 1.0);
    CotProblemDev Q;
    int r = build_problem(h, Q, points_xy, one.data(), dens.data(), n, 1, 1, sd, COT_MEM_HOST);
    if (r != COT_OK) free_problem(Q);
    if (r != COT_OK) return r;
    cudaStream_t s = h->stream;
    std::vector<double> val(n), sorted(n);
    double *solid = nullptr;
    cudaError_t e = cudaMemsetAsync(Q.w, 0, (size_t)n * 8, s);
    if (e == cudaSuccess && light) e = cudaMalloc(&solid, (size_t)n * 8);
    if (e == cudaSuccess) {
        CellsArgs a = cells_args(Q, Q.w, nullptr, nullptr);
        if (light) {
            a.solid = solid;
            a.solid_z = z;
            for (int c = 0; c < 3; c++) a.solid_light[c] = light[c];
        }
        launch_eval(Q.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
        e = cudaMemcpyAsync(sorted.data(), light ? solid : Q.mut, (size_t)n * 8, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (solid) cudaFree(solid);
    std::vector<int> perm = Q.hperm;
    free_problem(Q);
    if (e != cudaSuccess) return fail(h, COT_ECUDA, "cot_source_masses", cudaGetErrorString(e));
    const double dom = (sd[1] - sd[0]) * (sd[3] - sd[2]);
    // parallel light: the unit "pixel" integrates to n over the domain, so
    // mu = n * area / dom; a point light: the solid angles themselves
    for (int p = 0; p < n; p++) val[perm[p]] = light ? sorted[p] : sorted[p] * dom / (double)n;
    double tot = 0;
    for (int i = 0; i < n; i++) tot += val[i];
    if (!(tot > 0)) return fail(h, COT_EINVAL, "cot_source_masses: zero total", nullptr);
    for (int i = 0; i < n; i++) nu_out[i] = val[i] / tot * dom;
    return COT_OK;
}

extern "C" int cot_source_masses(cot_handle *h, const double *points_xy, int n, const double sample_domain[4],
                                 double *nu_out)
{
    if (!h) return COT_EINVAL;
    if (!points_xy || n <= 0 || !sample_domain || !nu_out) return fail(h, COT_EINVAL, "cot_source_masses: bad argument", nullptr);
    const double *sd = sample_domain;
    if (!(sd[1] > sd[0]) || !(sd[3] > sd[2])) return fail(h, COT_EINVAL, "cot_source_masses: empty sample_domain", nullptr);
    return source_masses_impl(h, points_xy, n, sd, nullptr, 0.0, nu_out);
}

extern "C" int cot_source_masses_point_light(cot_handle *h, const double *points_xy, int n,
                                             const double sample_domain[4], const double light[3], double z_of_len,
                                             double *nu_out)
{
    if (!h) return COT_EINVAL;
    if (!points_xy || n <= 0 || !sample_domain || !light || !nu_out)
        return fail(h, COT_EINVAL, "cot_source_masses_point_light: bad argument", nullptr);
    const double *sd = sample_domain;
    if (!(sd[1] > sd[0]) || !(sd[3] > sd[2])) return fail(h, COT_EINVAL, "cot_source_masses_point_light: empty sample_domain", nullptr);
    return source_masses_impl(h, points_xy, n, sd, light, z_of_len, nu_out);
}

extern "C" int cot_render(cot_handle *h, const double *w, double gray_multiple, double *out)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_render: no problem set", nullptr);
    if (!w || !out) return fail(h, COT_EINVAL, "cot_render: NULL argument", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    const size_t npx = (size_t)P.geo.nx * P.geo.ny;
    double *img = nullptr;
    COT_CUDA_TRY(cudaMalloc(&img, npx * 8));
    int r = upload_sorted(h, w, COT_MEM_HOST, P.wq);
    cudaError_t e = cudaMemsetAsync(img, 0, npx * 8, s);
    if (r == COT_OK && e == cudaSuccess) {
        CellsArgs a = cells_args(P, P.wq, nullptr, nullptr);
        a.splat = img;
        a.splat_scale = gray_multiple;
        launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
        e = cudaMemcpyAsync(out, img, npx * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFree(img);
    if (r != COT_OK) return r;
    if (e != cudaSuccess) return fail(h, COT_ECUDA, "cot_render", cudaGetErrorString(e));
    return COT_OK;
}

// ---------------------------------------------------------------------------
// solve
// ---------------------------------------------------------------------------
// Options check shared by the solve entry points.
static int check_opts(cot_handle *h, cot_solve_opts &o)
{
    if (o.mode != COT_SOLVE_REFERENCE && o.mode != COT_SOLVE_WOLFE) return fail(h, COT_EINVAL, "solve: bad mode", nullptr);
    if (o.history <= 0 || o.history > COT_MAX_HIST) return failf(h, COT_EINVAL, "solve: history must be in 1..%d", COT_MAX_HIST);
    if (o.max_iter < 0) return fail(h, COT_EINVAL, "solve: max_iter < 0", nullptr);
    if (!(o.initial_step > 0)) o.initial_step = 1.0;
    if (!(o.c1 > 0)) o.c1 = 1e-4;
    if (!(o.c2 > 0)) o.c2 = 0.9;
    if (o.max_ls <= 0) o.max_ls = 30;
    return COT_OK;
}

// Device L-BFGS from the weights in P.w (sorted order).  On return P.w holds
// the last accepted point, P.mu its masses, and *out the control block.
// Progress report: the solve's iterate (sorted w on the device) and the
// masses in force, in caller order, handed to the callback.  Returns
// COT_ECANCELLED when the callback asks to stop.
static int report_progress(cot_handle *h, int phase, int iteration, int status, double grad_norm,
                           double max_rel_err)
{
    CotProblemDev &P = h->P;
    h->prog_w.resize(P.n);
    h->prog_nu.resize(P.n);
    int r;
    if ((r = download_sorted(h, P.w, h->prog_w.data(), COT_MEM_HOST)) != COT_OK) return r;
    COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if ((r = download_sorted(h, P.nu, h->prog_nu.data(), COT_MEM_HOST)) != COT_OK) return r;
    COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->prog_fn(h->prog_user, phase, iteration, status, h->prog_w.data(), h->prog_nu.data(), P.n, grad_norm,
                   max_rel_err))
        return failf(h, COT_ECANCELLED, "solve stopped by the progress callback after iteration %d", iteration);
    return COT_OK;
}

// One pass of the device-driven trial loop (the body of its WHILE node).
static void launch_trial_body(cot_handle *h, cudaGraphConditionalHandle hc, double *tptr, CotCtx &c)
{
    CotProblemDev &P = h->P;
    launch_begin_iteration(P.S, c);
    launch_direction(P.geo, P.S, P.Sv, P.Yv, P.mu, P.d, c);
    CellsArgs a = cells_args(P, P.w, P.d, tptr);
    launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, c);
    launch_reduce(P.geo, P.mut, P.fc, P.nv, P.wt, P.d, h->cfg.max_ring, P.partials, P.ticket, P.out, P.S, c);
    launch_accept(P.geo, P.S, P.Sv, P.Yv, P.w, P.wt, P.mu, P.mut, P.d, P.partials, P.ticket, 0, c);
    launch_reject_cond(hc, P.S, c);
}

// The first point of a solve: its evaluation becomes the current point.
static void launch_first_point(cot_handle *h, CotCtx &c)
{
    CotProblemDev &P = h->P;
    CellsArgs a = cells_args(P, P.w, nullptr, nullptr);
    launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, c);
    launch_reduce(P.geo, P.mut, P.fc, P.nv, P.wt, nullptr, h->cfg.max_ring, P.partials, P.ticket, P.out, nullptr, c);
    launch_init_from_eval(P.S, P.out, c);
    launch_accept(P.geo, P.S, P.Sv, P.Yv, P.w, P.wt, P.mu, P.mut, P.d, P.partials, P.ticket, 1, c);
}

static double *step_ptr(CotProblemDev &P)
{
    return reinterpret_cast<double *>(reinterpret_cast<char *>(P.S) + offsetof(CotSolver, t));
}

// Counters that one body of the trial graph adds per execution.
struct BodyCounts {
    long long launches = 0, cell_launches = 0, evaluations = 0;
};

// The trial loop as one CUDA graph: a WHILE node whose body is one line-search
// trial -- begin + direction (no-ops inside a line search), the evaluation,
// the reduction with its line-search decision, accept / reject (no-ops unless
// the line search just ended) and the loop condition.  The whole solve then
// runs on the device without a host round trip per trial; the host looks
// again only when the loop stops (done, or a progress report is due).
// Returns COT_OK with *exec set, or an error (the caller then runs the
// host-driven loop).
static int build_trial_graph(cot_handle *h, double *tptr, cudaGraphExec_t *exec, BodyCounts *bc)
{
    cudaStream_t s = h->stream;
    *exec = nullptr;
    if (s == nullptr || s == cudaStreamLegacy) return COT_EINVAL;  // the legacy stream cannot be captured
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return COT_ECUDA;
    cudaGraphConditionalHandle hc;
    cudaError_t e = cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node;
    if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hc;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    }
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                            cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        cudaGetLastError();
        return COT_ECUDA;
    }
    // counters and per-launch event timing stay out of the captured body
    CotCtx &c = h->c();
    const CotCtx saved = c;
    c.profile = false;
    launch_trial_body(h, hc, tptr, c);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s, &captured);
    bc->launches = c.launches - saved.launches;
    bc->cell_launches = c.cell_launches - saved.cell_launches;
    bc->evaluations = c.evaluations - saved.evaluations;
    c = saved;
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *exec = nullptr;
        cudaGetLastError();
        return COT_ECUDA;
    }
    return COT_OK;
}

// History buffers and the device control block of a solve from the weights
// in P.w, on the handle's stream.
static int solve_prepare(cot_handle *h, const cot_solve_opts &o, int stop_nonempty = 0)
{
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    const int n = P.n;
    const int m = o.history;
    if (P.hist_alloc < m) {
        if (P.Sv) cudaFree(P.Sv);
        if (P.Yv) cudaFree(P.Yv);
        P.Sv = P.Yv = nullptr;
        P.hist_alloc = 0;
        // sized for the buffers' capacity: a later problem that fits them reuses these
        cudaError_t e = cudaMalloc(&P.Sv, (size_t)m * P.cap_n * 8);
        if (e == cudaSuccess) e = cudaMalloc(&P.Yv, (size_t)m * P.cap_n * 8);
        if (e != cudaSuccess) return fail(h, COT_ENOMEM, "solve: history allocation", cudaGetErrorString(e));
        P.hist_alloc = m;
        P.gen = ++g_problem_gen;  // a graph that captured the old history buffers is stale
    }
    COT_CUDA_TRY(cudaMemsetAsync(P.Sv, 0, (size_t)m * n * 8, s));
    COT_CUDA_TRY(cudaMemsetAsync(P.Yv, 0, (size_t)m * n * 8, s));
    CotSolver &hs = *h->hS;
    std::memset(&hs, 0, sizeof hs);
    hs.mode = o.mode;
    hs.m = m;
    hs.max_ls = o.max_ls;
    hs.max_iter = o.max_iter;
    hs.max_ring = h->cfg.max_ring;
    hs.c1 = o.c1;
    hs.c2 = o.c2;
    hs.t0 = o.initial_step;
    hs.tol = o.tol;
    hs.H0 = 1.0;
    hs.f = INFINITY;
    hs.need_begin = 1;
    hs.pause_iter = INT_MAX;
    hs.stop_nonempty = stop_nonempty;
    if (o.max_iter == 0) hs.done = 1;
    COT_CUDA_TRY(cudaMemcpyAsync(P.S, &hs, sizeof(CotSolver), cudaMemcpyHostToDevice, s));
    return COT_OK;
}

static int solve_device(cot_handle *h, const cot_solve_opts &o, CotSolver &out, float *ms, int phase,
                        bool report_start, int stop_nonempty = 0)
{
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    CotSolver &hs = *h->hS;
    int rp;
    if ((rp = solve_prepare(h, o, stop_nonempty)) != COT_OK) return rp;
    cudaEvent_t e0, e1;
    COT_CUDA_TRY(cudaEventCreate(&e0));
    COT_CUDA_TRY(cudaEventCreate(&e1));
    COT_CUDA_TRY(cudaEventRecord(e0, s));
    launch_first_point(h, h->c());
    if (h->prog_fn && report_start) {
        // the starting point (iteration -1)
        COT_CUDA_TRY(cudaMemcpyAsync(h->hS, P.S, sizeof(CotSolver), cudaMemcpyDeviceToHost, s));
        COT_CUDA_TRY(cudaStreamSynchronize(s));
        const CotSolver snap = hs;
        int r = report_progress(h, phase, -1, 0, std::sqrt(snap.gnorm2), snap.maxrel);
        hs = snap;
        if (r != COT_OK) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            out = hs;
            if (ms) *ms = 0.0f;
            return r;
        }
    }
    const size_t ctl = 16 * sizeof(int);
    int reported = 0;
    double *tptr = step_ptr(P);
    // progress report at an iteration boundary (hs holds the control block)
    auto boundary_report = [&]() -> int {
        if (!(h->prog_fn && hs.iter > 0 && hs.iter != reported && ((hs.iter - 1) % h->prog_every == 0 || hs.done)))
            return COT_OK;
        // iteration hs.iter - 1 is complete; the whole control block carries
        // its |g| and max-rel figures
        reported = hs.iter;
        COT_CUDA_TRY(cudaMemcpyAsync(h->hS, P.S, sizeof(CotSolver), cudaMemcpyDeviceToHost, s));
        COT_CUDA_TRY(cudaStreamSynchronize(s));
        const CotSolver snap = hs;
        const int status = !snap.done ? 0 : (snap.converged ? 1 : 2);
        int r = report_progress(h, phase, snap.iter - 1, status, std::sqrt(snap.gnorm2), snap.maxrel);
        hs = snap;
        return r;
    };
    auto stop = [&](int r) -> int {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        out = hs;
        if (ms) *ms = 0.0f;
        return r;
    };
    cudaGraphExec_t exec = nullptr;
    BodyCounts bc;
    if (o.use_graph >= 0) {
        if (h->trial_exec && h->trial_stream == s && h->trial_gen == P.gen) {
            exec = h->trial_exec;
            bc.launches = h->trial_counts[0];
            bc.cell_launches = h->trial_counts[1];
            bc.evaluations = h->trial_counts[2];
        } else {
            if (h->trial_exec) cudaGraphExecDestroy(h->trial_exec);
            h->trial_exec = nullptr;
            if (build_trial_graph(h, tptr, &exec, &bc) == COT_OK) {
                h->trial_exec = exec;
                h->trial_stream = s;
                h->trial_gen = P.gen;
                h->trial_counts[0] = bc.launches;
                h->trial_counts[1] = bc.cell_launches;
                h->trial_counts[2] = bc.evaluations;
            }
        }
    }
    if (exec != nullptr) {
        // device-driven loop: one graph launch runs trials until the solve is
        // done or the next progress report is due
        COT_CUDA_TRY(cudaMemcpyAsync(h->hS, P.S, ctl, cudaMemcpyDeviceToHost, s));
        COT_CUDA_TRY(cudaStreamSynchronize(s));
        const int evals0 = hs.evals;
        int r = COT_OK;
        while (!hs.done && r == COT_OK) {
            int pause = INT_MAX;
            if (h->prog_fn) {
                // iteration k (k a multiple of every) completes at iter k+1
                const int every = h->prog_every;
                pause = ((hs.iter + every - 1) / every) * every + 1;
            }
            hs.pause_iter = pause;
            cudaError_t e = cudaMemcpyAsync(reinterpret_cast<char *>(P.S) + offsetof(CotSolver, pause_iter),
                                            &hs.pause_iter, sizeof(int), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h->hS, P.S, ctl, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                r = fail(h, COT_ECUDA, "solve: trial graph", cudaGetErrorString(e));
                break;
            }
            r = boundary_report();
        }
        const long long bodies = hs.evals - evals0;
        h->ctx.launches += bodies * bc.launches;
        h->ctx.cell_launches += bodies * bc.cell_launches;
        h->ctx.evaluations += bodies * bc.evaluations;
        if (r != COT_OK) return stop(r);
    } else {
        // host-driven loop: one control-block read per trial
        while (true) {
            launch_begin_iteration(P.S, h->c());
            launch_direction(P.geo, P.S, P.Sv, P.Yv, P.mu, P.d, h->c());
            COT_CUDA_TRY(cudaMemcpyAsync(h->hS, P.S, ctl, cudaMemcpyDeviceToHost, s));
            COT_CUDA_TRY(cudaStreamSynchronize(s));
            int r = boundary_report();
            if (r != COT_OK) return stop(r);
            if (hs.done) break;
            while (true) {
                CellsArgs a = cells_args(P, P.w, P.d, tptr);
                launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
                launch_reduce(P.geo, P.mut, P.fc, P.nv, P.wt, P.d, h->cfg.max_ring, P.partials, P.ticket, P.out, P.S,
                              h->c());
                COT_CUDA_TRY(cudaMemcpyAsync(h->hS, P.S, ctl, cudaMemcpyDeviceToHost, s));
                COT_CUDA_TRY(cudaStreamSynchronize(s));
                if (!hs.ls_active) break;
            }
            if (hs.accepted)
                launch_accept(P.geo, P.S, P.Sv, P.Yv, P.w, P.wt, P.mu, P.mut, P.d, P.partials, P.ticket, 0, h->c());
            else
                launch_reject(P.S, h->c());
            COT_CUDA_TRY(cudaGetLastError());
        }
    }
    COT_CUDA_TRY(cudaEventRecord(e1, s));
    COT_CUDA_TRY(cudaMemcpyAsync(h->hS, P.S, sizeof(CotSolver), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaStreamSynchronize(s));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t;
    out = hs;
    return COT_OK;
}

static void fill_stats(const CotSolver &hs, float ms, cot_solve_stats *stats)
{
    if (!stats) return;
    stats->iterations = hs.iter;
    stats->evaluations = hs.evals;
    stats->restarts = hs.restarts;
    stats->converged = hs.converged;
    stats->f = hs.f;
    stats->max_rel_err = hs.maxrel;
    stats->grad_norm = std::sqrt(hs.gnorm2);
    stats->empty_cells = hs.empty;
    stats->ring_overflows = hs.ring_rejects;
    stats->ms = ms;
}

extern "C" int cot_solve(cot_handle *h, double *w_inout, const cot_solve_opts *opts, cot_solve_stats *stats, int mem)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_solve: no problem set", nullptr);
    if (!w_inout || !opts) return fail(h, COT_EINVAL, "cot_solve: NULL argument", nullptr);
    cot_solve_opts o = *opts;
    int r;
    if ((r = check_opts(h, o)) != COT_OK) return r;
    COT_CUDA_TRY(cudaSetDevice(h->device));
    if ((r = upload_sorted(h, w_inout, mem, h->P.w)) != COT_OK) return r;
    CotSolver hs;
    float ms = 0;
    const int rs = solve_device(h, o, hs, &ms, COT_PHASE_LBFGS, true);
    if (rs == COT_ECANCELLED) {
        // the last iterate goes back to the caller
        if ((r = download_sorted(h, h->P.w, w_inout, mem)) != COT_OK) return r;
        COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
        fill_stats(hs, ms, stats);
        return rs;
    }
    if (rs != COT_OK) return rs;
    if ((r = download_sorted(h, h->P.w, w_inout, mem)) != COT_OK) return r;
    COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    fill_stats(hs, ms, stats);
    if (!hs.converged) return failf(h, COT_ENOTCONV, "cot_solve: stopped after %d iterations (max rel err %.3e)", hs.iter, hs.maxrel);
    return COT_OK;
}

// Many independent solves in one graph launch: handle k's solve is one
// branch (its first evaluation, then its own WHILE node over the trial
// body), so the branches run concurrently and small instances overlap.
extern "C" int cot_solve_batch(cot_handle *const *hs_in, int count, double *const *w_inout,
                               const cot_solve_opts *opts, cot_solve_stats *stats)
{
    if (!hs_in || count <= 0 || !hs_in[0]) return COT_EINVAL;
    cot_handle *h0 = hs_in[0];
    if (!w_inout || !opts) return fail(h0, COT_EINVAL, "cot_solve_batch: NULL argument", nullptr);
    for (int k = 0; k < count; k++) {
        cot_handle *h = hs_in[k];
        if (!h || !w_inout[k]) return failf(h0, COT_EINVAL, "cot_solve_batch: entry %d is NULL", k);
        if (!h->has_problem) return failf(h0, COT_ENOPROBLEM, "cot_solve_batch: handle %d has no problem", k);
        if (h->device != h0->device) return failf(h0, COT_EINVAL, "cot_solve_batch: handle %d is on another device", k);
        for (int j = 0; j < k; j++)
            if (hs_in[j] == h) return failf(h0, COT_EINVAL, "cot_solve_batch: handle %d appears twice", k);
    }
    cot_solve_opts o = *opts;
    int r;
    if ((r = check_opts(h0, o)) != COT_OK) return r;
    {
        const cudaError_t ed = cudaSetDevice(h0->device);
        if (ed != cudaSuccess) return fail(h0, COT_ECUDA, "cot_solve_batch: cudaSetDevice", cudaGetErrorString(ed));
    }
    cudaStream_t s = h0->stream;
    if (s == nullptr || s == cudaStreamLegacy)
        return fail(h0, COT_EINVAL, "cot_solve_batch: the first handle's stream cannot be captured (legacy default stream)",
                    nullptr);
    // every handle works on the batch stream for the set-up and the capture
    std::vector<cudaStream_t> saved(count);
    for (int k = 0; k < count; k++) {
        saved[k] = hs_in[k]->stream;
        hs_in[k]->stream = s;
    }
    auto restore = [&]() {
        for (int k = 0; k < count; k++) hs_in[k]->stream = saved[k];
    };
    auto bail = [&](int code) {
        restore();
        return code;
    };
    for (int k = 0; k < count; k++) {
        if ((r = upload_sorted(hs_in[k], w_inout[k], COT_MEM_HOST, hs_in[k]->P.w)) != COT_OK) return bail(r);
        if ((r = solve_prepare(hs_in[k], o)) != COT_OK) return bail(r);
    }
    cudaGraph_t G = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<BodyCounts> first(count), body(count);
    cudaError_t e = cudaGraphCreate(&G, 0);
    for (int k = 0; k < count && e == cudaSuccess; k++) {
        cot_handle *h = hs_in[k];
        CotCtx &c = h->c();
        const CotCtx keep = c;
        c.profile = false;
        cudaGraph_t child = nullptr;
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            launch_first_point(h, c);
            e = cudaStreamEndCapture(s, &child);
        }
        first[k].launches = c.launches - keep.launches;
        first[k].cell_launches = c.cell_launches - keep.cell_launches;
        first[k].evaluations = c.evaluations - keep.evaluations;
        cudaGraphNode_t n1 = nullptr, cn = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&n1, G, nullptr, 0, child);
        if (child) cudaGraphDestroy(child);
        cudaGraphConditionalHandle hc;
        cudaGraphNodeParams cp = {};
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hc, G, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = hc;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&cn, G, &n1, 1, &cp);
        }
        if (e == cudaSuccess)
            e = cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal);
        const long long l0 = c.launches, cl0 = c.cell_launches, ev0 = c.evaluations;
        if (e == cudaSuccess) {
            launch_trial_body(h, hc, step_ptr(h->P), c);
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(s, &captured);
        }
        body[k].launches = c.launches - l0;
        body[k].cell_launches = c.cell_launches - cl0;
        body[k].evaluations = c.evaluations - ev0;
        c = keep;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, G, 0);
    if (G) cudaGraphDestroy(G);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bail(fail(h0, COT_ECUDA, "cot_solve_batch: graph", cudaGetErrorString(e)));
    }
    cudaEvent_t e0, e1;
    e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    if (e != cudaSuccess) return bail(fail(h0, COT_ECUDA, "cot_solve_batch: launch", cudaGetErrorString(e)));
    int unconverged = 0;
    for (int k = 0; k < count; k++) {
        cot_handle *h = hs_in[k];
        CotSolver &hs = *h->hS;
        e = cudaMemcpyAsync(h->hS, h->P.S, sizeof(CotSolver), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && (r = download_sorted(h, h->P.w, w_inout[k], COT_MEM_HOST)) != COT_OK) return bail(r);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return bail(fail(h0, COT_ECUDA, "cot_solve_batch: results", cudaGetErrorString(e)));
        const long long bodies = hs.evals > 0 ? hs.evals - 1 : 0;
        h->ctx.launches += first[k].launches + bodies * body[k].launches;
        h->ctx.cell_launches += first[k].cell_launches + bodies * body[k].cell_launches;
        h->ctx.evaluations += first[k].evaluations + bodies * body[k].evaluations;
        if (stats) fill_stats(hs, ms, &stats[k]);
        if (!hs.converged) unconverged++;
    }
    restore();
    if (unconverged)
        return failf(h0, COT_ENOTCONV, "cot_solve_batch: %d of %d solves stopped before the tolerance", unconverged,
                     count);
    return COT_OK;
}

// Small symmetric positive system A a = 1 by LDL^T (A n x n, n <= 32).
static bool ldlt_solve_ones(std::vector<double> A, int n, std::vector<double> &x)
{
    std::vector<double> L((size_t)n * n, 0.0), D(n, 0.0);
    for (int j = 0; j < n; j++) {
        double d = A[(size_t)j * n + j];
        for (int k = 0; k < j; k++) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k] * D[k];
        if (!(d != 0.0) || !std::isfinite(d)) return false;
        D[j] = d;
        L[(size_t)j * n + j] = 1.0;
        for (int i = j + 1; i < n; i++) {
            double v = A[(size_t)i * n + j];
            for (int k = 0; k < j; k++) v -= L[(size_t)i * n + k] * L[(size_t)j * n + k] * D[k];
            L[(size_t)i * n + j] = v / d;
        }
    }
    x.assign(n, 1.0);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < i; k++) x[i] -= L[(size_t)i * n + k] * x[k];
    for (int i = 0; i < n; i++) x[i] /= D[i];
    for (int i = n - 1; i >= 0; i--)
        for (int k = i + 1; k < n; k++) x[i] -= L[(size_t)k * n + i] * x[k];
    for (double v : x)
        if (!std::isfinite(v)) return false;
    return true;
}

// Fresnel-reweighted Anderson solve: aarl_direct_ot (ot_op.cuh:591-1385).
extern "C" int cot_solve_aarl(cot_handle *h, double *w_inout, const cot_aarl_inputs *in, const cot_solve_opts *opts,
                              cot_solve_stats *stats)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_solve_aarl: no problem set", nullptr);
    if (!w_inout || !in || !opts || !in->points_xy || !in->input_light || !in->inside_light || !in->height)
        return fail(h, COT_EINVAL, "cot_solve_aarl: NULL argument", nullptr);
    cot_solve_opts o = *opts;
    o.mode = COT_SOLVE_REFERENCE;
    int r;
    if ((r = check_opts(h, o)) != COT_OK) return r;
    const int M = in->aa_history;
    if (M <= 0 || M > COT_MAX_HIST) return failf(h, COT_EINVAL, "cot_solve_aarl: aa_history must be in 1..%d", COT_MAX_HIST);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    const int n = P.n;
    const size_t N = (size_t)n;
    // sorted copies of the per-site inputs
    const std::vector<int> &perm = P.hperm;
    std::vector<double> src(2 * N), inl(3 * N), insl(3 * N), hgt(N);
    for (size_t p = 0; p < N; p++) {
        int i = perm[p];
        src[2 * p] = in->points_xy[2 * (size_t)i];
        src[2 * p + 1] = in->points_xy[2 * (size_t)i + 1];
        for (int c = 0; c < 3; c++) {
            inl[3 * p + c] = in->input_light[3 * (size_t)i + c];
            insl[3 * p + c] = in->inside_light[3 * (size_t)i + c];
        }
        hgt[p] = in->height[i];
    }
    // device workspace of this call
    double *dsrc = nullptr, *dinl = nullptr, *dinsl = nullptr, *dhgt = nullptr, *lam = nullptr, *energy = nullptr;
    double *cen = nullptr, *G = nullptr, *F = nullptr, *row = nullptr, *coef = nullptr, *step = nullptr;
    unsigned char *ex = nullptr;
    auto release = [&]() {
        void *ps[] = {dsrc, dinl, dinsl, dhgt, lam, energy, cen, G, F, row, coef, step, ex};
        for (void *q : ps)
            if (q) cudaFree(q);
    };
    cudaError_t e = cudaMalloc(&dsrc, 2 * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&dinl, 3 * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&dinsl, 3 * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&dhgt, N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&lam, N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&energy, N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&cen, 2 * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&ex, N);
    if (e == cudaSuccess) e = cudaMalloc(&G, (size_t)M * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&F, (size_t)M * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&row, COT_MAX_HIST * 8);
    if (e == cudaSuccess) e = cudaMalloc(&coef, COT_MAX_HIST * 8);
    if (e == cudaSuccess) e = cudaMalloc(&step, 8);
    if (e != cudaSuccess) {
        release();
        return fail(h, COT_ENOMEM, "cot_solve_aarl: device allocation", cudaGetErrorString(e));
    }
    auto cuda_fail = [&](const char *what, cudaError_t err) {
        release();
        return fail(h, COT_ECUDA, what, cudaGetErrorString(err));
    };
#define AARL_TRY(expr)                                  \
    do {                                                \
        cudaError_t e__ = (expr);                       \
        if (e__ != cudaSuccess) return cuda_fail(#expr, e__); \
    } while (0)
    AARL_TRY(cudaMemcpyAsync(dsrc, src.data(), 2 * N * 8, cudaMemcpyHostToDevice, s));
    AARL_TRY(cudaMemcpyAsync(dinl, inl.data(), 3 * N * 8, cudaMemcpyHostToDevice, s));
    AARL_TRY(cudaMemcpyAsync(dinsl, insl.data(), 3 * N * 8, cudaMemcpyHostToDevice, s));
    AARL_TRY(cudaMemcpyAsync(dhgt, hgt.data(), N * 8, cudaMemcpyHostToDevice, s));
    // the problem's masses are the source masses lambda; they sum to area_scalar
    AARL_TRY(cudaMemcpyAsync(lam, P.nu, N * 8, cudaMemcpyDeviceToDevice, s));
    std::vector<double> hl(N);
    AARL_TRY(cudaMemcpyAsync(hl.data(), lam, N * 8, cudaMemcpyDeviceToHost, s));
    AARL_TRY(cudaStreamSynchronize(s));
    double area_scalar = 0;
    for (double v : hl) area_scalar += v;
    if ((r = upload_sorted(h, w_inout, COT_MEM_HOST, P.w)) != COT_OK) {
        release();
        return r;
    }
    cudaEvent_t e0, e1;
    AARL_TRY(cudaEventCreate(&e0));
    AARL_TRY(cudaEventCreate(&e1));
    AARL_TRY(cudaEventRecord(e0, s));
    CotEvalOut ho{};
    int evals = 0, iters = 0, restarts = 0, ring_rejects = 0;
    // plain centroids at P.w + t*d -> Fresnel-weighted nu (ot_op.cuh:779-795, 1082-1092, 1212-1224);
    // fills P.mut / P.fc / P.nv / P.wt for that point and reduces with the new nu
    auto eval_with_nu = [&](const double *d, const double *tptr, bool update_nu) -> int {
        CellsArgs a = cells_args(P, P.w, d, tptr);
        a.cen = cen;
        a.exist = ex;
        a.weighted = 0;
        launch_eval(P.geo, a, h->cfg.cells_per_warp, h->num_sms, h->c());
        evals++;
        // ring check first (polygons_in_VD + the max_edge_num/2 test)
        launch_reduce(P.geo, P.mut, P.fc, P.nv, P.wt, nullptr, h->cfg.max_ring, P.partials, P.ticket, P.out, nullptr, h->c());
        cudaError_t err = cudaMemcpyAsync(&ho, P.out, sizeof ho, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) return -1;
        if (ho.overflow > 0) return 1;
        if (update_nu) {
            launch_fresnel_nu(n, cen, dsrc, dinl, dinsl, dhgt, lam, in->z_of_len, in->z_of_receiver,
                              in->refraction_index, area_scalar, energy, P.partials, P.nu, h->c());
            launch_reduce(P.geo, P.mut, P.fc, P.nv, P.wt, nullptr, h->cfg.max_ring, P.partials, P.ticket, P.out, nullptr, h->c());
            err = cudaMemcpyAsync(&ho, P.out, sizeof ho, cudaMemcpyDeviceToHost, s);
            if (err == cudaSuccess) err = cudaStreamSynchronize(s);
            if (err != cudaSuccess) return -1;
        }
        return 0;
    };
    // 1. nu from the centroids at the warm start
    if (eval_with_nu(nullptr, nullptr, true) < 0) return cuda_fail("cot_solve_aarl: first evaluation", cudaGetLastError());
    // masses of the current point kept in P.mu: a progress callback may
    // evaluate on the handle, which reuses the trial buffers
    AARL_TRY(cudaMemcpyAsync(P.mu, P.mut, N * 8, cudaMemcpyDeviceToDevice, s));
    // start of the pre-pass phase (reported whether or not the pre-pass runs)
    auto report_start = [&](int phase) -> int {
        if (!h->prog_fn) return COT_OK;
        int rr = report_progress(h, phase, -1, 0, std::sqrt(ho.gnorm2), ho.maxrel);
        if (rr != COT_OK) {
            if (rr == COT_ECANCELLED && download_sorted(h, P.w, w_inout, COT_MEM_HOST) == COT_OK) {
                cudaStreamSynchronize(s);
                if (stats) *stats = cot_solve_stats{};
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            release();
        }
        return rr;
    };
    if ((r = report_start(COT_PHASE_PREPASS)) != COT_OK) return r;
    // 2. optional L-BFGS pre-pass with nu fixed (ot_op.cuh:823-1074)
    CotSolver pre{};
    if (in->lbfgs_prepass) {
        float pms = 0;
        if ((r = solve_device(h, o, pre, &pms, COT_PHASE_PREPASS, false)) != COT_OK) {
            if (r == COT_ECANCELLED && download_sorted(h, P.w, w_inout, COT_MEM_HOST) == COT_OK) {
                cudaStreamSynchronize(s);
                fill_stats(pre, 0.0f, stats);
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            release();
            return r;
        }
        evals += pre.evals;
        // 3. nu again from the centroids at the pre-pass result
        if (eval_with_nu(nullptr, nullptr, true) < 0) return cuda_fail("cot_solve_aarl: evaluation", cudaGetLastError());
        AARL_TRY(cudaMemcpyAsync(P.mu, P.mut, N * 8, cudaMemcpyDeviceToDevice, s));
    }
    // current point: P.w, masses P.mu, nu in P.nu
    if ((r = report_start(COT_PHASE_ANDERSON)) != COT_OK) return r;
    double f = ho.f, gnorm = std::sqrt(ho.gnorm2), maxrel = ho.maxrel;
    int empty = ho.empty;
    // 4. Anderson acceleration on w <- w + alpha g (ot_op.cuh:1112-1323)
    std::vector<double> A((size_t)M * M, 0.0), hrow(M), a;
    int aa_loop = 0;
    bool converged = false;
    for (int it = 0; it < o.max_iter; it++) {
        iters = it + 1;
        const int cnt = std::min(aa_loop + 1, M);
        const int hidx = aa_loop % M;
        const int empty_start = empty;
        launch_aa_store_gram(n, P.w, P.mu, P.nu, in->aa_fixed_para, G, F, hidx, cnt, P.partials, P.ticket, row, h->c());
        AARL_TRY(cudaMemcpyAsync(hrow.data(), row, cnt * 8, cudaMemcpyDeviceToHost, s));
        AARL_TRY(cudaStreamSynchronize(s));
        for (int j = 0; j < cnt; j++) A[(size_t)hidx * M + j] = A[(size_t)j * M + hidx] = hrow[j];
        std::vector<double> As((size_t)cnt * cnt);
        for (int i = 0; i < cnt; i++)
            for (int j = 0; j < cnt; j++) As[(size_t)i * cnt + j] = A[(size_t)i * M + j] + (i == j ? 1e-10 : 0.0);
        if (!ldlt_solve_ones(As, cnt, a)) {
            release();
            return fail(h, COT_ENOTCONV, "cot_solve_aarl: singular Anderson system", nullptr);
        }
        double sa = 0;
        for (double v : a) sa += v;
        for (double &v : a) v /= sa;
        AARL_TRY(cudaMemcpyAsync(coef, a.data(), cnt * 8, cudaMemcpyHostToDevice, s));
        launch_aa_combine(n, F, coef, cnt, P.w, P.d, h->c());
        double t = 1.0;
        bool accepted = false;
        while (true) {
            AARL_TRY(cudaMemcpyAsync(step, &t, 8, cudaMemcpyHostToDevice, s));
            int rc = eval_with_nu(P.d, step, true);
            if (rc < 0) return cuda_fail("cot_solve_aarl: evaluation", cudaGetLastError());
            if (rc == 1) {
                ring_rejects++;
                t *= 0.5;
            } else {
                // accept unconditionally (ot_op.cuh:1206-1241)
                AARL_TRY(cudaMemcpyAsync(P.w, P.wt, N * 8, cudaMemcpyDeviceToDevice, s));
                AARL_TRY(cudaMemcpyAsync(P.mu, P.mut, N * 8, cudaMemcpyDeviceToDevice, s));
                f = ho.f;
                gnorm = std::sqrt(ho.gnorm2);
                maxrel = ho.maxrel;
                empty = ho.empty;
                aa_loop++;
                accepted = true;
                break;
            }
            if (t <= 1e-4 * o.initial_step) break;
        }
        if (!accepted) {
            aa_loop = 0;
            restarts++;
        }
        // the reference counts empty cells (of the masses at the start of the
        // iteration) only on every tenth iteration (ot_op.cuh:1256-1268)
        const int check_degenerate = (it % 10 == 0) ? empty_start : 0;
        const bool conv_now = gnorm < o.tol && check_degenerate == 0;
        const bool last_it = conv_now || it + 1 == o.max_iter;
        if (h->prog_fn && (it % h->prog_every == 0 || last_it)) {
            const int status = conv_now ? 1 : (last_it ? 2 : 0);
            if ((r = report_progress(h, COT_PHASE_ANDERSON, it, status, gnorm, maxrel)) != COT_OK) {
                if (r == COT_ECANCELLED && download_sorted(h, P.w, w_inout, COT_MEM_HOST) == COT_OK) {
                    cudaStreamSynchronize(s);
                    if (stats) {
                        *stats = cot_solve_stats{};
                        stats->iterations = iters;
                        stats->evaluations = evals;
                        stats->restarts = restarts;
                        stats->f = f;
                        stats->max_rel_err = maxrel;
                        stats->grad_norm = gnorm;
                        stats->empty_cells = empty;
                        stats->ring_overflows = ring_rejects;
                    }
                }
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                release();
                return r;
            }
        }
        if (conv_now) {
            converged = true;
            break;
        }
    }
    AARL_TRY(cudaEventRecord(e1, s));
    if ((r = download_sorted(h, P.w, w_inout, COT_MEM_HOST)) != COT_OK) {
        release();
        return r;
    }
    AARL_TRY(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release();
#undef AARL_TRY
    if (stats) {
        stats->iterations = iters;
        stats->evaluations = evals;
        stats->restarts = restarts;
        stats->converged = converged ? 1 : 0;
        stats->f = f;
        stats->max_rel_err = maxrel;
        stats->grad_norm = gnorm;
        stats->empty_cells = empty;
        stats->ring_overflows = ring_rejects;
        stats->ms = ms;
    }
    if (!converged) return failf(h, COT_ENOTCONV, "cot_solve_aarl: stopped after %d iterations (|g| %.3e)", iters, gnorm);
    return COT_OK;
}

// ---------------------------------------------------------------------------
// damped Newton solve and the masses' Jacobian (no counterpart in the
// reference)
// ---------------------------------------------------------------------------
namespace cot {
__global__ void k_rhs(int n, const double *__restrict__ nu, const double *__restrict__ mu, double *__restrict__ b)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = nu[i] - mu[i];
}
}  // namespace cot

static int newton_alloc(cot_handle *h)
{
    CotProblemDev &P = h->P;
    if (P.hval) return COT_OK;
    // sized for the buffers' capacity: a later problem that fits them reuses these
    const size_t N = P.cap_n;
    const int pcg_blocks = pcg_max_blocks((int)N, h->num_sms);
    P.hbig_cap = std::max(16, std::min((int)N, 4096));
    cudaError_t e = cudaSuccess;
    auto A = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes > 0 ? bytes : 16);
    };
    A((void **)&P.hval, 32 * N * sizeof(double));
    A((void **)&P.hcol, 32 * N * sizeof(int));
    A((void **)&P.hcnt, N * sizeof(int));
    A((void **)&P.hdiag, N * sizeof(double));
    A((void **)&P.hbig_val, (size_t)P.hbig_cap * COT_HBIG_W * sizeof(double));
    A((void **)&P.hbig_col, (size_t)P.hbig_cap * COT_HBIG_W * sizeof(int));
    A((void **)&P.herr, sizeof(int));
    A((void **)&P.nb_b, N * 8);
    A((void **)&P.nb_r, N * 8);
    A((void **)&P.nb_z, N * 8);
    A((void **)&P.nb_pa, N * 8);
    A((void **)&P.nb_pb, N * 8);
    A((void **)&P.nb_q, N * 8);
    A((void **)&P.nb_part, (size_t)std::max(4 * pcg_blocks, 256 * 5) * 8);
    A((void **)&P.nb_tau, 8);
    A((void **)&P.pcg, sizeof(PcgState));
    A((void **)&P.nst, sizeof(NewtonEvalStats));
    A((void **)&P.nticket, sizeof(unsigned int));
    if (e != cudaSuccess) {
        void *ptrs[] = {P.hval, P.hcol, P.hcnt, P.hdiag, P.hbig_val, P.hbig_col, P.herr, P.nb_b, P.nb_r, P.nb_z,
                        P.nb_pa, P.nb_pb, P.nb_q, P.nb_part, P.nb_tau, P.pcg, P.nst, P.nticket};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        P.hval = P.hdiag = P.hbig_val = P.nb_b = P.nb_r = P.nb_z = P.nb_pa = P.nb_pb = P.nb_q = P.nb_part = P.nb_tau = nullptr;
        P.hcol = P.hcnt = P.hbig_col = P.herr = nullptr;
        P.pcg = nullptr;
        P.nst = nullptr;
        P.nticket = nullptr;
        return fail(h, COT_ENOMEM, "cot_solve_newton: device allocation", cudaGetErrorString(e));
    }
    COT_CUDA_TRY(cudaMemsetAsync(P.nticket, 0, sizeof(unsigned int), h->stream));
    COT_CUDA_TRY(cudaMemsetAsync(P.hcnt, 0, N * sizeof(int), h->stream));  // no row refers to a slot yet
    return COT_OK;
}

// CellsArgs of an evaluation that keeps what the Jacobian needs: the final
// rings' generators and the long rings' rows.
static CellsArgs jacobian_args(CotProblemDev &P, const double *w, const double *d, const double *tptr)
{
    CellsArgs a = cells_args(P, w, d, tptr);
    a.keep_labels = 1;
    a.hbig_val = P.hbig_val;
    a.hbig_col = P.hbig_col;
    a.hbig_cap = P.hbig_cap;
    a.hcnt = P.hcnt;
    a.hdiag = P.hdiag;
    a.herr = P.herr;
    return a;
}

// One evaluation for the Newton solve at w + tau d (d == nullptr: at w),
// then its statistics into *h->hN.
static int newton_eval(cot_handle *h, const double *d)
{
    CotProblemDev &P = h->P;
    CellsArgs a = jacobian_args(P, P.w, d, d ? P.nb_tau : nullptr);
    COT_CUDA_TRY(cudaMemsetAsync(P.herr, 0, sizeof(int), h->stream));
    launch_eval(P.geo, a, 1, h->num_sms, h->c());
    launch_newton_stats(P.n, P.mut, P.nu, P.nv, P.nb_part, P.nticket, P.nst, h->c());
    COT_CUDA_TRY(cudaGetLastError());
    COT_CUDA_TRY(cudaMemcpyAsync(h->hN, P.nst, sizeof(NewtonEvalStats), cudaMemcpyDeviceToHost, h->stream));
    COT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return COT_OK;
}

extern "C" int cot_mass_jacobian(cot_handle *h, const double *w, int mem, int *row_offsets, int *cols, double *vals,
                                 int capacity, int *nnz)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_mass_jacobian: no problem set", nullptr);
    if (!w || !row_offsets || !nnz) return fail(h, COT_EINVAL, "cot_mass_jacobian: NULL argument", nullptr);
    if (mem != COT_MEM_HOST && mem != COT_MEM_DEVICE) return fail(h, COT_EINVAL, "cot_mass_jacobian: bad mem flag", nullptr);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    int r;
    if ((r = newton_alloc(h)) != COT_OK) return r;
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    if ((r = upload_sorted(h, w, mem, P.wq)) != COT_OK) return r;
    CellsArgs a = jacobian_args(P, P.wq, nullptr, nullptr);
    COT_CUDA_TRY(cudaMemsetAsync(P.herr, 0, sizeof(int), s));
    launch_eval(P.geo, a, 1, h->num_sms, h->c());
    launch_hessian(P.geo, P.rbuf, P.lbuf, P.nv, P.hval, P.hcol, P.hcnt, P.hdiag, h->c());
    COT_CUDA_TRY(cudaGetLastError());
    const size_t N = (size_t)P.n;
    std::vector<int> cnt(N), nv(N), hcol(32 * N);
    std::vector<double> diag(N), hval(32 * N);
    int herr = 0, nbig = 0;
    COT_CUDA_TRY(cudaMemcpyAsync(cnt.data(), P.hcnt, N * sizeof(int), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaMemcpyAsync(nv.data(), P.nv, N * sizeof(int), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaMemcpyAsync(diag.data(), P.hdiag, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaMemcpyAsync(hcol.data(), P.hcol, 32 * N * sizeof(int), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaMemcpyAsync(hval.data(), P.hval, 32 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaMemcpyAsync(&herr, P.herr, sizeof(int), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaMemcpyAsync(&nbig, P.ovf_count + 7, sizeof(int), cudaMemcpyDeviceToHost, s));
    COT_CUDA_TRY(cudaStreamSynchronize(s));
    for (size_t i = 0; i < N; i++)
        if (nv[i] > 256) return failf(h, COT_ERING, "cot_mass_jacobian: a cell has more than 256 vertices");
    if (herr) return failf(h, COT_ECAPACITY, "cot_mass_jacobian: more than %d cells above 32 vertices", P.hbig_cap);
    nbig = std::min(nbig, P.hbig_cap);
    std::vector<int> bcol((size_t)nbig * COT_HBIG_W);
    std::vector<double> bval((size_t)nbig * COT_HBIG_W);
    if (nbig > 0) {
        COT_CUDA_TRY(cudaMemcpyAsync(bcol.data(), P.hbig_col, bcol.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
        COT_CUDA_TRY(cudaMemcpyAsync(bval.data(), P.hbig_val, bval.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        COT_CUDA_TRY(cudaStreamSynchronize(s));
    }
    // rows in caller order, columns sorted, the diagonal included
    std::vector<std::vector<std::pair<int, double>>> rows(N);
    const std::vector<int> &perm = P.hperm;
    for (size_t i = 0; i < N; i++) {
        auto &row = rows[perm[i]];
        row.emplace_back(perm[i], diag[i]);
        if (cnt[i] >= 0) {
            for (int k = 0; k < cnt[i]; k++) row.emplace_back(perm[hcol[k * N + i]], -hval[k * N + i]);
        } else {
            const size_t base = (size_t)(-cnt[i] - 1) * COT_HBIG_W;
            if (base / COT_HBIG_W >= (size_t)nbig) return failf(h, COT_ECUDA, "cot_mass_jacobian: stale long-ring row");
            for (int k = 0; k < COT_HBIG_W && bcol[base + k] >= 0; k++)
                row.emplace_back(perm[bcol[base + k]], -bval[base + k]);
        }
        std::sort(row.begin(), row.end());
    }
    long long total = 0;
    row_offsets[0] = 0;
    for (size_t i = 0; i < N; i++) {
        total += (long long)rows[i].size();
        row_offsets[i + 1] = (int)std::min<long long>(total, INT_MAX);
    }
    *nnz = (int)std::min<long long>(total, INT_MAX);
    if (!cols || !vals) return COT_OK;  // size query
    if (total > capacity) return failf(h, COT_ECAPACITY, "cot_mass_jacobian: %lld entries, capacity %d", total, capacity);
    size_t q = 0;
    for (size_t i = 0; i < N; i++)
        for (auto &e : rows[i]) {
            cols[q] = e.first;
            vals[q] = e.second;
            q++;
        }
    return COT_OK;
}

extern "C" int cot_solve_newton(cot_handle *h, double *w_inout, const cot_newton_opts *opts,
                                cot_newton_stats *stats, int mem)
{
    if (!h) return COT_EINVAL;
    if (!h->has_problem) return fail(h, COT_ENOPROBLEM, "cot_solve_newton: no problem set", nullptr);
    if (!w_inout || !opts) return fail(h, COT_EINVAL, "cot_solve_newton: NULL argument", nullptr);
    if (mem != COT_MEM_HOST && mem != COT_MEM_DEVICE) return fail(h, COT_EINVAL, "cot_solve_newton: bad mem flag", nullptr);
    cot_newton_opts o = *opts;
    if (!(o.tol > 0)) return fail(h, COT_EINVAL, "cot_solve_newton: tol must be positive", nullptr);
    if (o.max_iter <= 0) o.max_iter = 100;
    if (!(o.cg_rtol > 0) || o.cg_rtol >= 1.0) o.cg_rtol = 0.1;
    if (o.cg_max_iter <= 0) o.cg_max_iter = 2000;
    if (o.lbfgs_chunk <= 0) o.lbfgs_chunk = 10;
    if (o.lbfgs_rounds <= 0) o.lbfgs_rounds = 50;
    if (o.history <= 0) o.history = 10;
    if (o.history > COT_MAX_HIST) return failf(h, COT_EINVAL, "cot_solve_newton: history must be in 1..%d", COT_MAX_HIST);
    o.shrink_steps = std::min(std::max(o.shrink_steps, 0), 30);
    COT_CUDA_TRY(cudaSetDevice(h->device));
    int r;
    if ((r = newton_alloc(h)) != COT_OK) return r;
    CotProblemDev &P = h->P;
    cudaStream_t s = h->stream;
    cot_newton_stats st{};
    if ((r = upload_sorted(h, w_inout, mem, P.w)) != COT_OK) return r;
    cudaEvent_t e0, e1;
    COT_CUDA_TRY(cudaEventCreate(&e0));
    COT_CUDA_TRY(cudaEventCreate(&e1));
    COT_CUDA_TRY(cudaEventRecord(e0, s));
    auto finish = [&](int rc) -> int {
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        st.ms = t;
        if (stats) *stats = st;
        return rc;
    };
    // this library's L-BFGS, for the rounds with empty cells and the fall-back
    cot_solve_opts lo{};
    lo.mode = COT_SOLVE_WOLFE;
    lo.history = o.history;
    lo.tol = o.tol;
    int rc = check_opts(h, lo);
    if (rc != COT_OK) return finish(rc);
    auto lbfgs = [&](int max_iter, int stop_nonempty) -> int {
        lo.max_iter = max_iter;
        CotSolver hs;
        const int rr = solve_device(h, lo, hs, nullptr, COT_PHASE_LBFGS, false, stop_nonempty);
        if (rr != COT_OK) return rr;
        st.lbfgs_iterations += hs.iter;
        st.evaluations += hs.evals;
        st.converged = hs.converged;
        st.max_rel_err = hs.maxrel;
        st.grad_norm = std::sqrt(hs.gnorm2);
        st.empty_cells = hs.empty;
        return COT_OK;
    };
    // 1. L-BFGS while some cell is empty (the Jacobian has no row for an
    //    empty cell): one run that stops as soon as every cell has mass, at
    //    most lbfgs_chunk x lbfgs_rounds iterations (a run that ends early,
    //    e.g. a failed line search, is started again)
    NewtonEvalStats cur{};
    bool ready = false;
    if (o.shrink_steps > 0) {
        // the start scaled towards w = 0 (a power diagram at w = 0 is the
        // Voronoi diagram, which empties no cell inside the density's
        // support): the largest of 1/2, 1/4, ... that empties none.  The
        // trial weights w + tau w with tau = s - 1 are exactly s w.
        if ((rc = newton_eval(h, nullptr)) != COT_OK) return finish(rc);
        st.evaluations++;
        if (h->hN->empty > 0 && h->hN->maxrel > o.tol) {
            double sc = 1.0;
            for (int k = 0; k < o.shrink_steps; k++) {
                sc *= 0.5;
                double *ptau = reinterpret_cast<double *>(h->hB + 208);
                *ptau = sc - 1.0;
                COT_CUDA_TRY(cudaMemcpyAsync(P.nb_tau, ptau, sizeof(double), cudaMemcpyHostToDevice, s));
                if ((rc = newton_eval(h, P.w)) != COT_OK) return finish(rc);
                st.evaluations++;
                if (h->hN->empty == 0) {
                    COT_CUDA_TRY(cudaMemcpyAsync(P.w, P.wt, (size_t)P.n * 8, cudaMemcpyDeviceToDevice, s));
                    break;
                }
            }
        }
    }
    for (int round = 0; round <= o.lbfgs_rounds; round++) {
        if ((rc = newton_eval(h, nullptr)) != COT_OK) return finish(rc);
        st.evaluations++;
        cur = *h->hN;
        st.max_rel_err = cur.maxrel;
        st.grad_norm = std::sqrt(cur.gnorm2);
        st.empty_cells = cur.empty;
        if (cur.maxrel <= o.tol) {
            st.converged = 1;
            break;
        }
        if (cur.empty == 0) {
            ready = true;
            break;
        }
        const int left = o.lbfgs_chunk * o.lbfgs_rounds - st.lbfgs_iterations;
        if (round == o.lbfgs_rounds || left <= 0) break;
        if ((rc = lbfgs(left, 1)) != COT_OK) return finish(rc);
        if (st.converged) break;
    }
    // 2. damped Newton steps (Kitagawa, Merigot and Thibert 2019, Alg. 1):
    //    solve dmu/dw d = nu - mu, then halve tau from 1 until every mass
    //    stays above eps and |g(w + tau d)| <= (1 - tau / 2) |g(w)|
    if (ready && !st.converged) {
        double nu_min = INFINITY;
        {
            std::vector<double> hnu(P.n);
            COT_CUDA_TRY(cudaMemcpyAsync(hnu.data(), P.nu, (size_t)P.n * 8, cudaMemcpyDeviceToHost, s));
            COT_CUDA_TRY(cudaStreamSynchronize(s));
            for (double v : hnu) nu_min = std::min(nu_min, v);
        }
        const double eps = 0.5 * std::min(nu_min, cur.minmu);
        const int pcg_blocks = pcg_max_blocks(P.n, h->num_sms);
        for (int it = 0; it < o.max_iter; it++) {
            if (cur.maxrel <= o.tol) {
                st.converged = 1;
                break;
            }
            // the rings of the current point are the last evaluation's; one
            // read back (pinned) for the long-row flag and the solve's state
            int *herr = reinterpret_cast<int *>(h->hB + 200);
            COT_CUDA_TRY(cudaMemcpyAsync(herr, P.herr, sizeof(int), cudaMemcpyDeviceToHost, s));
            launch_hessian(P.geo, P.rbuf, P.lbuf, P.nv, P.hval, P.hcol, P.hcnt, P.hdiag, h->c());
            k_rhs<<<nblk(P.n), 256, 0, s>>>(P.n, P.nu, P.mut, P.nb_b);
            h->ctx.launches++;
            COT_CUDA_TRY(cudaMemsetAsync(P.pcg, 0, sizeof(PcgState), s));
            COT_CUDA_TRY(launch_pcg(P.n, P.hval, P.hcol, P.hcnt, P.hbig_val, P.hbig_col, P.hdiag, P.nb_b, P.d, P.nb_r,
                                    P.nb_z, P.nb_pa, P.nb_pb, P.nb_q, P.nb_part, P.pcg, o.cg_rtol, o.cg_max_iter,
                                    pcg_blocks, h->c()));
            COT_CUDA_TRY(cudaMemcpyAsync(h->hP, P.pcg, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
            COT_CUDA_TRY(cudaStreamSynchronize(s));
            st.cg_iterations += h->hP->iterations;
            if (*herr != 0 || h->hP->error != 0) break;  // the fall-back below finishes
            const double gn = std::sqrt(cur.gnorm2);
            double tau = 1.0;
            bool accepted = false;
            double *ptau = reinterpret_cast<double *>(h->hB + 208);   // pinned: an asynchronous copy
            for (int ls = 0; ls < 30; ls++) {
                *ptau = tau;
                COT_CUDA_TRY(cudaMemcpyAsync(P.nb_tau, ptau, sizeof(double), cudaMemcpyHostToDevice, s));
                if ((rc = newton_eval(h, P.d)) != COT_OK) return finish(rc);
                st.evaluations++;
                const NewtonEvalStats t = *h->hN;
                if (t.minmu >= eps && std::sqrt(t.gnorm2) <= (1.0 - 0.5 * tau) * gn) {
                    cur = t;
                    accepted = true;
                    break;
                }
                tau *= 0.5;
            }
            if (!accepted) break;  // the damped step stalled: the fall-back below finishes
            // the accepted trial becomes the current point (its rings are in
            // the buffers)
            COT_CUDA_TRY(cudaMemcpyAsync(P.w, P.wt, (size_t)P.n * 8, cudaMemcpyDeviceToDevice, s));
            st.newton_iterations++;
            st.max_rel_err = cur.maxrel;
            st.grad_norm = std::sqrt(cur.gnorm2);
            st.empty_cells = cur.empty;
        }
        if (cur.maxrel <= o.tol) st.converged = 1;
    }
    // 3. fall-back: the L-BFGS from the last accepted point
    if (!st.converged) {
        st.fallback = 1;
        if ((rc = lbfgs(INT_MAX / 2, 0)) != COT_OK) return finish(rc);
    }
    if ((r = download_sorted(h, P.w, w_inout, mem)) != COT_OK) return finish(r);
    COT_CUDA_TRY(cudaStreamSynchronize(s));
    rc = finish(COT_OK);
    if (!st.converged)
        return failf(h, COT_ENOTCONV, "cot_solve_newton: stopped at max rel err %.3e", st.max_rel_err);
    return rc;
}
