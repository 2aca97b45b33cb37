// Power cells and their pixel integrals, one warp per cell.
//
// Replaces, per objective evaluation, the CPU power diagram of the reference
// (polygons_in_VD, power_diagram.cpp:8-134) and its per-cell CUDA kernels
// compute_inte / compute_f / compute_center (basic_function.cuh:743-1191).
//
// Cell i is built as   proj_domain ∩ { x : |x-s_i|^2 - w_i <= |x-s_j|^2 - w_j }
// over the sites j that can reach it.  Working relative to s_i (x = s_i + x')
// the half-plane of neighbour j is   e.x' <= (|e|^2 - (w_j - w_i)) / 2,
// e = s_j - s_i.  Candidates come from the 3x3 neighbour buckets around s_i;
// completeness is certified with a bound tree: writing phi_j = (|s_j|^2-w_j)/2
// and P_j(x) = x.s_j - phi_j (cell i = where P_i is the largest), every tree
// node holds its sites' box and a weight bound {a, B} with w_j/2 <= a.s_j + B,
// so that  P_j(x) <= (|x+a|^2 - dist(x+a, box)^2)/2 + B  for all its sites.
// a is the local slope of the weights, so the bound stays tight when cells
// sit far from their sites.  A node whose bound is below P_i at every vertex
// of the current polygon cannot cut the cell (a convex bound minus a linear
// function peaks at a vertex).
//
// The integration clips nothing: for each pixel of the cell's bounding box the
// exact integrals of 1, x, y and |x-s_i|^2 over cell ∩ pixel are boundary sums
// (Green's theorem in the x-dy form): the polygon edges clipped to the pixel,
// plus the pixel's two vertical sides where they lie inside the cell.  Fully
// covered pixels take a closed form.
#include "cot_common.cuh"
#include "cot_edge.cuh"
#include <math.h>
#include <algorithm>
#include <climits>

namespace cot {

#define FULLMASK 0xffffffffu
#define COT_FRMAX 96
#define COT_REFINE_PASSES 3  // ring refinements before a walk that overflows scans every bucket
#define COT_REFINE_ROUNDS 4  // point-location rounds of one refinement
#define COT_DEFERRED (-3)    // ring size of a cell handed to k_cells_heavy
#ifndef COT_DEFER_LEAVES
#define COT_DEFER_LEAVES 24  // surviving leaf buckets above which a walk is handed to k_cells_heavy
#endif
#ifndef COT_DEFER_PASS
#define COT_DEFER_PASS 1  // refinement passes before a walk is handed to k_cells_heavy (1, 2, 3 measured 134.9, 134.8, 134.3 M cell-evals/s: 65,536 sites, 1024² target)
#endif
static_assert(COT_BLEAF <= COT_FRMAX && COT_BLEAF % 32 == 0, "a bucket list fits a frontier");

#ifdef COT_PHASE_STATS
// Measurement build only: per-phase cycle and event counters, kept per warp
// in shared memory and added to the global totals once when the warp exits.
__device__ unsigned long long cot_phase_stats[16];
// (per segment of LPC lanes: LPC must be a constant in scope where they are used)
__shared__ unsigned long long cot_pst[16][16];
#define PSTAT_ADD(k, v) do { if ((threadIdx.x & (LPC - 1)) == 0) cot_pst[threadIdx.x / LPC][k] += (unsigned long long)(v); } while (0)
#define PSTAT_CLOCK(var) long long var = clock64()
#define PSTAT_INIT() do { if ((threadIdx.x & (LPC - 1)) == 0) for (int q_ = 0; q_ < 16; q_++) cot_pst[threadIdx.x / LPC][q_] = 0; } while (0)
#define PSTAT_FLUSH() do { if ((threadIdx.x & (LPC - 1)) == 0) for (int q_ = 0; q_ < 16; q_++) atomicAdd(&cot_phase_stats[q_], cot_pst[threadIdx.x / LPC][q_]); } while (0)
#define PSTAT_LPC32 constexpr int LPC = 32
#else
#define PSTAT_INIT() do { } while (0)
#define PSTAT_FLUSH() do { } while (0)
#define PSTAT_ADD(k, v) do { } while (0)
#define PSTAT_CLOCK(var) do { } while (0)
#define PSTAT_LPC32 do { } while (0)
#endif
#define COT_WIN 1  // window radius in buckets
// neighbour cache count nbn[i]: +m an ordered ring of m generators, -m an
// unordered list of m sites, -(COT_NB_HIDDEN + m) the m sites that hid the
// cell at the last evaluation
#define COT_NB_HIDDEN 100
#define COT_RCAP 32  // ring buffer vertices per cell (the split integration)
// pixel box above which a cell is integrated first, and above which by
// COT_SPLIT warps (measured at 65,536 sites on a 1024^2 target, M cell-evals/s:
// 512/4096 144.6, 1024/4096 142.5, 512/2048 142.0, 1024/8192 140.8,
// 1024/16384 139.6, 2048/8192 139.3)
#ifndef COT_HEAVY_PIX
#define COT_HEAVY_PIX 512
#endif
#ifndef COT_SPLIT_PIX
#define COT_SPLIT_PIX 4096
#endif
#define CST_HEAVY (-2)      // cstate of a cell on the heavy integration list

// ---------------------------------------------------------------------------
// bucket and tree weight bounds (per evaluation)
// ---------------------------------------------------------------------------

// w_j at the trial point w + t d, explicitly rounded so that every thread
// that needs a bucket's mean computes the same bits.
__device__ __forceinline__ double trial_weight(const double *__restrict__ w, const double *__restrict__ d, double t,
                                               int j)
{
    // no contraction: the trial point is w + t*d exactly as written
    return d != nullptr ? __dadd_rn(w[j], __dmul_rn(t, d[j])) : w[j];
}

// The bucket kernels work one bucket per 16-lane segment (a half warp):
// the segment's lanes take the bucket's sites in turn.
#define BSEG 16
__device__ __forceinline__ unsigned bseg_mask() { return 0xffffu << (threadIdx.x & 16); }
__device__ __forceinline__ double bseg_sum(double v, unsigned m)
{
#pragma unroll
    for (int o = BSEG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o, BSEG);
    return v;
}
__device__ __forceinline__ double bseg_max(double v, unsigned m)
{
#pragma unroll
    for (int o = BSEG / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(m, v, o, BSEG));
    return v;
}

// Trial weights of bucket b's sites and their mean phi (0 for an empty
// bucket).  Block 0 also clears the cell kernels' counters.
__global__ void k_bucket_phi(CotGeo g, const double *__restrict__ w, const double *__restrict__ d,
                             const double *__restrict__ tptr, double *__restrict__ wt,
                             double *__restrict__ wbar, int *counters, int ncounters)
{
    if (blockIdx.x == 0 && (int)threadIdx.x < ncounters) counters[threadIdx.x] = 0;
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) / BSEG;
    const int sl = threadIdx.x & (BSEG - 1);
    if (b >= g.bx * g.by) return;  // whole segments leave together
    const unsigned m = bseg_mask();
    const double t = (d != nullptr && tptr != nullptr) ? *tptr : 0.0;
    const int s0 = g.bstart[b], s1 = g.bstart[b + 1];
    double acc = 0.0;
    for (int j = s0 + sl; j < s1; j += BSEG) {
        const double wj = trial_weight(w, d, t, j);
        wt[j] = wj;
        acc = __dadd_rn(acc, wj);
    }
    acc = bseg_sum(acc, m);
    if (sl == 0) wbar[b] = (s1 > s0) ? 0.5 * acc / (double)(s1 - s0) : 0.0;
}

// Weight bound of bucket b: a_b = slope of w/2 across the neighbouring
// buckets (central difference of their mean w/2 over their box centres,
// one-sided at the grid edges), B_b = max_j w_j/2 - a_b.s_j.  Called by a
// whole segment (mask msk); every lane returns the bound.
__device__ __forceinline__ double4 bucket_bound(const CotGeo &g, const double *__restrict__ wt,
                                                const double *__restrict__ wbar, int b, int sl, unsigned msk)
{
    const double4 st = g.tstat[b];
    if (st.z < 0.0) return make_double4(0.0, 0.0, -INFINITY, 0.0);
    const int u = b % g.bx, v = b / g.bx;
    const double pb = wbar[b];
    double c[2];
    for (int ax = 0; ax < 2; ax++) {
        int bp = -1, bm = -1;
        if (ax == 0) {
            if (u + 1 < g.bx && g.tstat[b + 1].z >= 0.0) bp = b + 1;
            if (u > 0 && g.tstat[b - 1].z >= 0.0) bm = b - 1;
        } else {
            if (v + 1 < g.by && g.tstat[b + g.bx].z >= 0.0) bp = b + g.bx;
            if (v > 0 && g.tstat[b - g.bx].z >= 0.0) bm = b - g.bx;
        }
        const double mb = ax == 0 ? st.x : st.y;
        double val;
        if (bp >= 0 && bm >= 0) {
            const double mp = ax == 0 ? g.tstat[bp].x : g.tstat[bp].y;
            const double mm = ax == 0 ? g.tstat[bm].x : g.tstat[bm].y;
            val = (wbar[bp] - wbar[bm]) / (mp - mm);
        } else if (bp >= 0) {
            const double mp = ax == 0 ? g.tstat[bp].x : g.tstat[bp].y;
            val = (wbar[bp] - pb) / (mp - mb);
        } else if (bm >= 0) {
            const double mm = ax == 0 ? g.tstat[bm].x : g.tstat[bm].y;
            val = (pb - wbar[bm]) / (mb - mm);
        } else {
            val = 0.0;
        }
        if (!isfinite(val)) val = 0.0;
        c[ax] = val;
    }
    double B = -INFINITY;
    const int s0 = g.bstart[b], s1 = g.bstart[b + 1];
    for (int j = s0 + sl; j < s1; j += BSEG) {
        const double2 s = g.xy[j];
        B = fmax(B, 0.5 * wt[j] - (c[0] * s.x + c[1] * s.y));
    }
    B = bseg_max(B, msk);
    return make_double4(c[0], c[1], B, 0.0);
}

// Bucket weight bounds, one bucket per segment.
#define TREE_THREADS 256
__global__ void __launch_bounds__(TREE_THREADS) k_tree_build(CotGeo g, const double *__restrict__ wt,
                                                            const double *__restrict__ wbar)
{
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) / BSEG;
    const int sl = threadIdx.x & (BSEG - 1);
    if (b >= g.bx * g.by) return;  // whole segments leave together
    const double4 bd = bucket_bound(g, wt, wbar, b, sl, bseg_mask());
    if (sl == 0) g.tdyn[b] = bd;
}

// Fixed-order block sum and max over TREE_THREADS threads (every thread
// gets the result).
__device__ __forceinline__ double tree_block_sum(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    for (int k = 0; k < TREE_THREADS / 32; k++) r += sh[k];
    return r;
}
__device__ __forceinline__ double tree_block_max(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULLMASK, v, o));
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = -INFINITY;
    for (int k = 0; k < TREE_THREADS / 32; k++) r = fmax(r, sh[k]);
    return r;
}

// Tree levels 1..lmax (the levels a certificate walk can start from; the
// ones above are never read), one block per node, each straight from the
// buckets and sites under it: a = the mean weight slope of its non-empty
// buckets, B = max_j w_j/2 - a.s_j over its sites, the exact value for that
// a.  No level waits for the one below, and no bound is a bound of bounds.
__global__ void __launch_bounds__(TREE_THREADS) k_tree_levels(CotGeo g, const double *__restrict__ wt)
{
    __shared__ double sh[TREE_THREADS / 32];
    // the highest levels (the most sites a node) first, so that they do not
    // trail the many small nodes of level 1
    const int node = g.lev_off[1] + (int)(gridDim.x - 1 - blockIdx.x);
    int L = 1;
    while (L + 1 < g.nlev && g.lev_off[L + 1] <= node) L++;
    const int q = node - g.lev_off[L], W = g.lev_w[L];
    if (g.tstat[node].z < 0.0) {
        if (threadIdx.x == 0) g.tdyn[node] = make_double4(0.0, 0.0, -INFINITY, 0.0);
        return;
    }
    // the node's buckets: a rectangle of the bucket grid
    const int u0 = (q % W) << L, v0 = (q / W) << L;
    const int u1 = min(u0 + (1 << L), g.bx), v1 = min(v0 + (1 << L), g.by);
    const int rw = u1 - u0, nbk = rw * (v1 - v0);
    double sx = 0.0, sy = 0.0, sc = 0.0;
    for (int k = threadIdx.x; k < nbk; k += TREE_THREADS) {
        const int b = u0 + k % rw + (v0 + k / rw) * g.bx;
        if (g.tstat[b].z < 0.0) continue;
        const double4 d = g.tdyn[b];
        sx += d.x;
        sy += d.y;
        sc += 1.0;
    }
    sx = tree_block_sum(sx, sh);
    sy = tree_block_sum(sy, sh);
    sc = tree_block_sum(sc, sh);
    const double cx = sx / sc, cy = sy / sc;
    double B = -INFINITY;
    for (int v = v0; v < v1; v++) {
        // the rectangle's buckets in one row hold consecutive sites
        const int j0 = g.bstart[u0 + v * g.bx], j1 = g.bstart[u1 + v * g.bx];
        for (int j = j0 + threadIdx.x; j < j1; j += TREE_THREADS) {
            const double2 s2 = g.xy[j];
            B = fmax(B, 0.5 * wt[j] - (cx * s2.x + cy * s2.y));
        }
    }
    B = tree_block_max(B, sh);
    if (threadIdx.x == 0) g.tdyn[node] = make_double4(cx, cy, B, 0.0);
}

// ---------------------------------------------------------------------------
// warp helpers
// ---------------------------------------------------------------------------

// Side of a point w.r.t. a * x + b * y <= c (> 0 means outside).  One explicit
// fused form so that every lane evaluating the same vertex gets the same bits.
__device__ __forceinline__ double side(double a, double b, double c, double x, double y)
{
    return __fma_rn(a, x, __fma_rn(b, y, -c));
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULLMASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
    return v;
}

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(FULLMASK, v, o));
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULLMASK, v, o));
    return v;
}

// A segment of LPC lanes working on one cell (LPC = 32: the whole warp).  A
// warp holds 32 / LPC cells; each segment synchronises, shuffles and votes
// within its own lanes only.
template <int LPC>
struct Seg {
    static_assert(LPC == 32 || LPC == 16 || LPC == 8, "lanes per cell: 32, 16 or 8");
    static constexpr unsigned low = LPC == 32 ? FULLMASK : ((1u << (LPC & 31)) - 1u);
    unsigned mask;  // the segment's lanes in the warp
    int base;       // its first lane
    int sl;         // this lane's index in the segment
    __device__ __forceinline__ Seg()
    {
        const int lane = threadIdx.x & 31;
        base = lane & ~(LPC - 1);
        sl = lane & (LPC - 1);
        mask = low << base;
    }
    __device__ __forceinline__ unsigned ballot(bool p) const { return (__ballot_sync(mask, p) >> base) & low; }
    __device__ __forceinline__ bool any(bool p) const { return ballot(p) != 0u; }
    __device__ __forceinline__ bool all(bool p) const { return ballot(p) == low; }
    template <class T>
    __device__ __forceinline__ T shfl(T v, int src) const { return __shfl_sync(mask, v, src, LPC); }
    template <class T>
    __device__ __forceinline__ T shfl_xor(T v, int o) const { return __shfl_xor_sync(mask, v, o, LPC); }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ unsigned below(int n) const { return n >= LPC ? low : ((1u << n) - 1u); }
    __device__ __forceinline__ int incl_scan(int v) const
    {
#pragma unroll
        for (int o = 1; o < LPC; o <<= 1) {
            int t = __shfl_up_sync(mask, v, o, LPC);
            if (sl >= o) v += t;
        }
        return v;
    }
    // butterfly reductions: for LPC = 32 the same order as the warp versions
    __device__ __forceinline__ double sum(double v) const
    {
#pragma unroll
        for (int o = LPC / 2; o > 0; o >>= 1) v += shfl_xor(v, o);
        return v;
    }
    __device__ __forceinline__ double min(double v) const
    {
#pragma unroll
        for (int o = LPC / 2; o > 0; o >>= 1) v = fmin(v, shfl_xor(v, o));
        return v;
    }
    __device__ __forceinline__ double max(double v) const
    {
#pragma unroll
        for (int o = LPC / 2; o > 0; o >>= 1) v = fmax(v, shfl_xor(v, o));
        return v;
    }
    __device__ __forceinline__ int imin(int v) const
    {
#pragma unroll
        for (int o = LPC / 2; o > 0; o >>= 1) v = ::min(v, shfl_xor(v, o));
        return v;
    }
};


// Intersection of lines a1 x + b1 y = c1 and a2 x + b2 y = c2.  Axis-aligned
// lines are solved directly so that vertices on the domain sides sit exactly on
// them.  Returns false for (near) parallel lines.
__device__ __forceinline__ bool line_meet(double a1, double b1, double c1, double a2, double b2,
                                          double c2, double &x, double &y)
{
    // an axis-parallel line (a domain side) gives one coordinate directly;
    // explicit roundings keep the other the same whichever line came first
    if (b1 == 0.0 && a1 != 0.0) {
        x = __ddiv_rn(c1, a1);
        if (b2 == 0.0) return false;
        y = __ddiv_rn(__dsub_rn(c2, __dmul_rn(a2, x)), b2);
        return true;
    }
    if (a1 == 0.0 && b1 != 0.0) {
        y = __ddiv_rn(c1, b1);
        if (a2 == 0.0) return false;
        x = __ddiv_rn(__dsub_rn(c2, __dmul_rn(b2, y)), a2);
        return true;
    }
    if (b2 == 0.0 && a2 != 0.0) {
        x = __ddiv_rn(c2, a2);
        y = __ddiv_rn(__dsub_rn(c1, __dmul_rn(a1, x)), b1);
        return true;
    }
    if (a2 == 0.0 && b2 != 0.0) {
        y = __ddiv_rn(c2, b2);
        x = __ddiv_rn(__dsub_rn(c1, __dmul_rn(b1, y)), a1);
        return true;
    }
    // uncontracted products: swapping the two lines negates numerator and
    // denominator exactly, so a vertex does not depend on which line clipped
    // which
    double det = __dsub_rn(__dmul_rn(a1, b2), __dmul_rn(a2, b1));
    double sc = (fabs(a1) + fabs(b1)) * (fabs(a2) + fabs(b2));
    if (!(fabs(det) > 1e-13 * sc)) return false;
    x = __ddiv_rn(__dsub_rn(__dmul_rn(c1, b2), __dmul_rn(c2, b1)), det);
    y = __ddiv_rn(__dsub_rn(__dmul_rn(a1, c2), __dmul_rn(a2, c1)), det);
    return true;
}

// Half-plane of site j in the frame of site i: e.x <= (|e|^2 - (w_j - w_i))/2
// with e = s_j - s_i.  One explicitly rounded form for every path that
// builds a ring, so that the same pair of lines always meets in the same bits.
__device__ __forceinline__ void site_line(double2 sj, double2 si, double wj, double wi, double &a, double &b,
                                          double &c, double &key)
{
    a = __dsub_rn(sj.x, si.x);
    b = __dsub_rn(sj.y, si.y);
    key = __fma_rn(a, a, __dmul_rn(b, b));
    c = __dmul_rn(0.5, __dsub_rn(key, __dsub_rn(wj, wi)));
}

// Domain side k (0 bottom, 1 right, 2 top, 3 left; generator -(k+1)) in the
// site's frame, box = {x0, x1, y0, y1} = domain - site: the line of the
// starting rectangle's edge k.
__device__ __forceinline__ void side_line(int k, double4 box, double &a, double &b, double &c)
{
    const double x0 = box.x, x1 = box.y, y0 = box.z, y1 = box.w;
    a = k == 1 ? 1.0 : (k == 3 ? -1.0 : 0.0);
    b = k == 0 ? -1.0 : (k == 2 ? 1.0 : 0.0);
    c = k == 0 ? -y0 : (k == 1 ? x1 : (k == 2 ? y1 : -x0));
}

// Shared scratch of one warp for the large-ring path (rings up to MAXV).
template <int MAXV>
struct WarpPoly {
    double X[MAXV], Y[MAXV];          // vertices, relative to the site
    double A[MAXV], B[MAXV], C[MAXV]; // line of the edge leaving each vertex
    int L[MAXV];                      // its generator (site, or -1..-4)
    double EIX[MAXV], EIY[MAXV], ESL[MAXV];  // per edge: 1/dx, 1/dy, dy/dx
    int fr[2][COT_FRMAX];             // tree traversal lists
    double elo[33], ehi[33];          // section of the cell at column lines
    double slo[32], shi[32];          // y-range of the cell in each column strip
    unsigned char lv[33], rv[33];     // left / right limit of the section valid
};

// Clip the polygon by a x + b y <= c (generator lab).  Returns the new vertex
// count, or -1 when it would exceed MAXV.
template <int MAXV>
__device__ int clip_poly(WarpPoly<MAXV> &P, int nv, double a, double b, double c, int lab, int lane)
{
    constexpr int SPL = MAXV / 32;
    double x[SPL], y[SPL], la[SPL], lb[SPL], lc[SPL], ix[SPL], iy[SPL];
    int ll[SPL], cnt[SPL], pos[SPL];
    bool in[SPL], inn[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) {
        int k = lane + 32 * q;
        cnt[q] = 0;
        in[q] = inn[q] = false;
        if (k < nv) {
            int kn = (k + 1 == nv) ? 0 : k + 1;
            x[q] = P.X[k];
            y[q] = P.Y[k];
            double xn = P.X[kn], yn = P.Y[kn];
            double d0 = side(a, b, c, x[q], y[q]);
            double d1 = side(a, b, c, xn, yn);
            in[q] = d0 <= 0.0;
            inn[q] = d1 <= 0.0;
            la[q] = P.A[k];
            lb[q] = P.B[k];
            lc[q] = P.C[k];
            ll[q] = P.L[k];
            cnt[q] = (in[q] ? 1 : 0) + ((in[q] != inn[q]) ? 1 : 0);
            if (in[q] != inn[q]) {
                if (!line_meet(la[q], lb[q], lc[q], a, b, c, ix[q], iy[q])) {
                    double t = d0 / (d0 - d1);
                    ix[q] = x[q] + t * (xn - x[q]);
                    iy[q] = y[q] + t * (yn - y[q]);
                }
            }
        }
    }
    int base = 0;
#pragma unroll
    for (int q = 0; q < SPL; q++) {
        int inc = warp_incl_scan(cnt[q], lane);
        pos[q] = base + inc - cnt[q];
        base += __shfl_sync(FULLMASK, inc, 31);
    }
    if (base > MAXV) return -1;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < SPL; q++) {
        int k = lane + 32 * q;
        if (k < nv) {
            int p = pos[q];
            if (in[q]) {
                P.X[p] = x[q]; P.Y[p] = y[q];
                P.A[p] = la[q]; P.B[p] = lb[q]; P.C[p] = lc[q]; P.L[p] = ll[q];
                p++;
            }
            if (in[q] != inn[q]) {
                P.X[p] = ix[q]; P.Y[p] = iy[q];
                if (in[q]) { P.A[p] = a; P.B[p] = b; P.C[p] = c; P.L[p] = lab; }
                else { P.A[p] = la[q]; P.B[p] = lb[q]; P.C[p] = lc[q]; P.L[p] = ll[q]; }
            }
        }
    }
    __syncwarp();
    return base;
}

// Clip by every candidate of the chunk (one per lane, j < 0 = none) that cuts
// the polygon, nearest site first.  A candidate that does not cut the polygon
// can never cut a later (smaller) one and is dropped for good.
template <int MAXV>
__device__ int clip_chunk(WarpPoly<MAXV> &P, int nv, int j, const CotGeo &g, double2 si, double wi,
                          const double *__restrict__ wt, int lane, int &status, bool check_dup)
{
    PSTAT_LPC32;
    bool act = j >= 0;
    if (act && check_dup) {
        // a site whose line already bounds the polygon must not clip again
        for (int k = 0; k < nv; k++)
            if (P.L[k] == j) { act = false; break; }
    }
    double a = 0.0, b = 0.0, c = 0.0, key = INFINITY;
    if (act) site_line(g.xy[j], si, wt[j], wi, a, b, c, key);
    while (true) {
        bool cut = false;
        if (act) {
            for (int k = 0; k < nv; k++) {
                if (side(a, b, c, P.X[k], P.Y[k]) > 0.0) { cut = true; break; }
            }
            if (!cut) act = false;
        }
        unsigned mask = __ballot_sync(FULLMASK, cut);
        PSTAT_ADD(4, 1);
        if (mask == 0u) break;
        PSTAT_ADD(3, 1);
        double kk = cut ? key : INFINITY;
        int bl = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ok = __shfl_xor_sync(FULLMASK, kk, o);
            int ol = __shfl_xor_sync(FULLMASK, bl, o);
            if (ok < kk || (ok == kk && ol < bl)) { kk = ok; bl = ol; }
        }
        double A = __shfl_sync(FULLMASK, a, bl);
        double B = __shfl_sync(FULLMASK, b, bl);
        double Cc = __shfl_sync(FULLMASK, c, bl);
        int J = __shfl_sync(FULLMASK, j, bl);
        int r = clip_poly<MAXV>(P, nv, A, B, Cc, J, lane);
        if (r < 0) { status = 1; return nv; }
        nv = r;
        if (lane == bl) act = false;
        if (nv == 0) return 0;
    }
    return nv;
}

// Can no site of `node` beat site i anywhere on the current polygon?  With
// P_j(x) = x.s_j - phi_j, phi_j = (|s_j|^2 - w_j)/2, and the node's weight
// bound (a, B: w_j/2 <= a.s_j + B for each of its sites j),
//     P_j(x) = (x + a).s_j - |s_j|^2/2 + (w_j/2 - a.s_j) <= F(x + a) + B,
//     F(y) = max over the node's site box of y.s - |s|^2/2
//          = (|y|^2 - dist(y, box)^2) / 2,
// F being convex (a maximum of affine functions of y).  The node is excluded
// when F(x + a) + B + margin <= P_i(x) at every vertex x of the polygon: a
// convex function minus an affine one peaks at a vertex.  With x = s_i + v
// (v in the site's frame) and t = v + a the condition reads
//     |t|^2 + 2 (s_i.a + B + margin) - w_i <= dist(s_i + t, box)^2.
// The quadratic is exact where a plane bound of phi would lose h^2/2 for a
// node of half width h.
template <class SP>
__device__ __forceinline__ bool node_excluded(const SP &P, int nv, const CotGeo &g, int node,
                                              double2 si, double wi)
{
    const double4 st = g.tstat[node];
    if (st.z < 0.0) return true;
    const double4 dy = g.tdyn[node];
    const double px = si.x - st.x + dy.x, py = si.y - st.y + dy.y;
    const double C = 2.0 * (si.x * dy.x + si.y * dy.y + dy.z + g.margin) - wi;
    for (int k = 0; k < nv; k++) {
        const double tx = P.X[k] + dy.x, ty = P.Y[k] + dy.y;
        const double ex = fmax(fabs(P.X[k] + px) - st.z, 0.0);
        const double ey = fmax(fabs(P.Y[k] + py) - st.w, 0.0);
        if (!(__fma_rn(tx, tx, __fma_rn(ty, ty, C)) <= __fma_rn(ex, ex, ey * ey))) return false;
    }
    return true;
}

// Green terms of one directed segment in pixel-local coordinates.
struct Mom { double A, Ia, Ib, I2; };

__device__ __forceinline__ void seg_terms(double a0, double b0, double a1, double b1, Mom &m)
{
    double db = b1 - b0;
    m.A += db * (a0 + a1) * 0.5;
    m.Ia += db * (a0 * a0 + a0 * a1 + a1 * a1) * (1.0 / 6.0);
    m.Ib += db * (2.0 * a0 * b0 + a0 * b1 + a1 * b0 + 2.0 * a1 * b1) * (1.0 / 6.0);
    double c3 = (a0 * a0 * a0 + a0 * a0 * a1 + a0 * a1 * a1 + a1 * a1 * a1) * (1.0 / 12.0);
    double cb = (a0 * (3.0 * b0 * b0 + 2.0 * b0 * b1 + b1 * b1) + a1 * (b0 * b0 + 2.0 * b0 * b1 + 3.0 * b1 * b1)) *
                (1.0 / 12.0);
    m.I2 += db * (c3 + cb);
}

// Vertical segment at a from b0 to b1.
__device__ __forceinline__ void vside_terms(double a, double b0, double b1, Mom &m)
{
    double db = b1 - b0;
    m.A += a * db;
    m.Ia += 0.5 * a * a * db;
    m.Ib += 0.5 * a * (b1 * b1 - b0 * b0);
    m.I2 += a * a * a * (1.0 / 3.0) * db + a * (b1 * b1 * b1 - b0 * b0 * b0) * (1.0 / 3.0);
}

// Section [lo, hi] of the polygon at the vertical line x (lo > hi: empty).
template <class SP>
__device__ __forceinline__ void section_at(const SP &P, int nv, double x, double &lo, double &hi)
{
    lo = INFINITY;
    hi = -INFINITY;
    for (int k = 0; k < nv; k++) {
        int kn = (k + 1 == nv) ? 0 : k + 1;
        double px = P.X[k], py = P.Y[k], qx = P.X[kn], qy = P.Y[kn];
        if (px == qx) {
            if (px == x) {
                lo = fmin(lo, fmin(py, qy));
                hi = fmax(hi, fmax(py, qy));
            }
            continue;
        }
        double mn = fmin(px, qx), mx = fmax(px, qx);
        if (x < mn || x > mx) continue;
        double yy = (x == px) ? py : (x == qx) ? qy : py + (x - px) * P.ESL[k];
        lo = fmin(lo, yy);
        hi = fmax(hi, yy);
    }
}

struct CellAcc { double mu, S, Mt, Mx, My; };

// The part of the geometry the pixel integration needs, passed by value.
struct PixGeo {
    const double *rho;
    double pd0, pd2, xs, ys, ixs, iys;
    int nx, ny;
    double *splat;   // render: out[pix] += splat_w * area(cell ∩ pix) (nullable)
    double splat_w;
};

__device__ __forceinline__ PixGeo pix_geo(const CotGeo &g)
{
    PixGeo p;
    p.rho = g.rho;
    p.pd0 = g.pd[0];
    p.pd2 = g.pd[2];
    p.xs = g.xs;
    p.ys = g.ys;
    p.ixs = g.ixs;
    p.iys = g.iys;
    p.nx = g.nx;
    p.ny = g.ny;
    p.splat = nullptr;
    p.splat_w = 0.0;
    return p;
}

// render (basic_function.cuh:660-741): the cell's carried mass spread over
// the pixels in proportion to area; the weight is nu_i * gray / area(cell).
template <class SP>
__device__ PixGeo splat_geo(const CotGeo &g, const CellsArgs &a, const SP &P, int nv, int i, int lane)
{
    PixGeo p = pix_geo(g);
    if (a.splat == nullptr) return p;
    double ar = 0.0;
    for (int k = lane; k < nv; k += 32) {
        int kn = (k + 1 == nv) ? 0 : k + 1;
        ar += P.X[k] * P.Y[kn] - P.X[kn] * P.Y[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ar += __shfl_xor_sync(0xffffffffu, ar, o);
    ar = 0.5 * fabs(ar);
    if (ar != 0.0) {
        p.splat = a.splat;
        p.splat_w = g.nu[i] * a.splat_scale / ar;
    }
    return p;
}

// Integrate the density over the cell (polygon relative to site si).
template <class SP>
__device__ __noinline__ CellAcc integrate_cell(SP &P, int nv, const PixGeo g, double2 si, int lane)
{
    PSTAT_LPC32;
    CellAcc acc = {0.0, 0.0, 0.0, 0.0, 0.0};
    // per-edge reciprocals and slopes: no divisions in the pixel loop
    for (int k = lane; k < nv; k += 32) {
        int kn = (k + 1 == nv) ? 0 : k + 1;
        double dx = P.X[kn] - P.X[k], dy = P.Y[kn] - P.Y[k];
        P.EIX[k] = dx != 0.0 ? 1.0 / dx : 0.0;
        P.EIY[k] = dy != 0.0 ? 1.0 / dy : 0.0;
        P.ESL[k] = dx != 0.0 ? dy / dx : 0.0;
    }
    __syncwarp();
    double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
    for (int k = lane; k < nv; k += 32) {
        mnx = fmin(mnx, P.X[k]); mxx = fmax(mxx, P.X[k]);
        mny = fmin(mny, P.Y[k]); mxy = fmax(mxy, P.Y[k]);
    }
    mnx = warp_min(mnx); mxx = warp_max(mxx); mny = warp_min(mny); mxy = warp_max(mxy);
    // pixel range of the bounding box (basic_function.cuh:791-799)
    // the reference's floor((min - d0) / step) .. floor((max - d0) / step) + 1
    // (basic_function.cuh:791-794), widened by one pixel on each side so that
    // the reciprocal's rounding can never drop a covered pixel; pixels outside
    // the cell are skipped by the strip test below
    int lx = (int)floor((si.x + mnx - g.pd0) * g.ixs) - 1;
    int ly = (int)floor((si.y + mny - g.pd2) * g.iys) - 1;
    int hx = (int)floor((si.x + mxx - g.pd0) * g.ixs) + 2;
    int hy = (int)floor((si.y + mxy - g.pd2) * g.iys) + 2;
    lx = lx > 0 ? lx : 0;
    ly = ly > 0 ? ly : 0;
    hx = hx < g.nx ? hx : g.nx;
    hy = hy < g.ny ? hy : g.ny;
    if (hx <= lx || hy <= ly) return acc;
    PSTAT_ADD(6, (hx - lx) * (hy - ly));
    const double pminx = mnx, pmaxx = mxx;
    double mu = 0.0, S = 0.0, Mt = 0.0, Mx = 0.0, My = 0.0;
    for (int cx0 = lx; cx0 < hx; cx0 += 32) {
        int cw = min(32, hx - cx0);
        // column lines cx0 .. cx0+cw
        for (int c = lane; c <= cw; c += 32) {
            double xl = (double)(cx0 + c) * g.xs + g.pd0 - si.x;
            double lo, hi;
            section_at(P, nv, xl, lo, hi);
            P.elo[c] = lo;
            P.ehi[c] = hi;
            P.rv[c] = (pminx <= xl && xl < pmaxx) ? 1 : 0;  // right limit (left side of a pixel)
            P.lv[c] = (pminx < xl && xl <= pmaxx) ? 1 : 0;  // left limit (right side of a pixel)
        }
        __syncwarp();
        // y-range of the cell inside each column strip
        for (int c = lane; c < cw; c += 32) {
            double xl = (double)(cx0 + c) * g.xs + g.pd0 - si.x;
            double xr = (double)(cx0 + c + 1) * g.xs + g.pd0 - si.x;
            double lo = INFINITY, hi = -INFINITY;
            if (P.rv[c]) { lo = fmin(lo, P.elo[c]); hi = fmax(hi, P.ehi[c]); }
            if (P.lv[c + 1]) { lo = fmin(lo, P.elo[c + 1]); hi = fmax(hi, P.ehi[c + 1]); }
            for (int k = 0; k < nv; k++) {
                double vx = P.X[k];
                if (vx > xl && vx < xr) { lo = fmin(lo, P.Y[k]); hi = fmax(hi, P.Y[k]); }
            }
            P.slo[c] = lo;
            P.shi[c] = hi;
        }
        __syncwarp();
        int rows = hy - ly;
        int npx = cw * rows;
        for (int p = lane; p < npx; p += 32) {
            int c = p % cw, r = p / cw;
            int ix = cx0 + c, iy = ly + r;
            // pixel box exactly as basic_function.cuh:806-809, relative to the site
            double x0 = (double)ix * g.xs + g.pd0 - si.x;
            double x1 = (double)(ix + 1) * g.xs + g.pd0 - si.x;
            double y0 = (double)iy * g.ys + g.pd2 - si.y;
            double y1 = (double)(iy + 1) * g.ys + g.pd2 - si.y;
            if (!(P.shi[c] > y0 && P.slo[c] < y1)) continue;
            double xc = 0.5 * (x0 + x1), yc = 0.5 * (y0 + y1);
            double hxp = 0.5 * (x1 - x0), hyp = 0.5 * (y1 - y0);
            Mom m = {0.0, 0.0, 0.0, 0.0};
            bool full = P.rv[c] && P.lv[c + 1] && P.elo[c] <= y0 && P.ehi[c] >= y1 && P.elo[c + 1] <= y0 &&
                        P.ehi[c + 1] >= y1;
            if (full) {
                m.A = 4.0 * hxp * hyp;
                m.I2 = m.A * (hxp * hxp + hyp * hyp) * (1.0 / 3.0);
            } else {
                for (int k = 0; k < nv; k++) {
                    int kn = (k + 1 == nv) ? 0 : k + 1;
                    double px = P.X[k], py = P.Y[k], qx = P.X[kn], qy = P.Y[kn];
                    if (px == qx && (px == x0 || px == x1)) continue;  // counted by the pixel side
                    if (fmax(px, qx) < x0 || fmin(px, qx) > x1 || fmax(py, qy) < y0 || fmin(py, qy) > y1) continue;
                    // Liang-Barsky against the pixel box (reciprocals precomputed)
                    double dx = qx - px, dy = qy - py, t0 = 0.0, t1 = 1.0;
                    if (dx != 0.0) {
                        double ta = (x0 - px) * P.EIX[k], tb = (x1 - px) * P.EIX[k];
                        t0 = fmax(t0, fmin(ta, tb));
                        t1 = fmin(t1, fmax(ta, tb));
                    } else if (px < x0 || px > x1) {
                        continue;
                    }
                    if (dy != 0.0) {
                        double ta = (y0 - py) * P.EIY[k], tb = (y1 - py) * P.EIY[k];
                        t0 = fmax(t0, fmin(ta, tb));
                        t1 = fmin(t1, fmax(ta, tb));
                    } else if (py < y0 || py > y1) {
                        continue;
                    }
                    if (!(t0 < t1)) continue;
                    double ax0 = (t0 == 0.0 ? px : px + t0 * dx) - xc;
                    double by0 = (t0 == 0.0 ? py : py + t0 * dy) - yc;
                    double ax1 = (t1 == 1.0 ? qx : px + t1 * dx) - xc;
                    double by1 = (t1 == 1.0 ? qy : py + t1 * dy) - yc;
                    seg_terms(ax0, by0, ax1, by1, m);
                }
                if (P.lv[c + 1]) {  // right side, upwards
                    double b0 = fmax(P.elo[c + 1], y0), b1 = fmin(P.ehi[c + 1], y1);
                    if (b1 > b0) vside_terms(x1 - xc, b0 - yc, b1 - yc, m);
                }
                if (P.rv[c]) {      // left side, downwards
                    double b0 = fmax(P.elo[c], y0), b1 = fmin(P.ehi[c], y1);
                    if (b1 > b0) vside_terms(x0 - xc, b1 - yc, b0 - yc, m);
                }
            }
            if (!(m.A > 0.0)) continue;
            if (g.splat != nullptr) atomicAdd(g.splat + ix + iy * g.nx, g.splat_w * m.A);
            double rho = g.rho[ix + iy * g.nx];
            mu += rho * m.A;
            S += rho * (m.A * (xc * xc + yc * yc) + 2.0 * (xc * m.Ia + yc * m.Ib) + m.I2);
            if (m.A > 1e-10) {  // compute_center skips tiny pieces (basic_function.cuh:1153)
                Mt += rho * m.A;
                Mx += rho * (m.A * xc + m.Ia);
                My += rho * (m.A * yc + m.Ib);
            }
        }
        __syncwarp();
    }
    acc.mu = warp_sum(mu);
    acc.S = warp_sum(S);
    acc.Mt = warp_sum(Mt);
    acc.Mx = warp_sum(Mx);
    acc.My = warp_sum(My);
    return acc;
}

// compute_solid_angle (basic_function.cuh:558-588): solid angle of the planar
// polygon (absolute vertices, plane z) seen from the light, as the sum over
// the fan from vertex 0 of 2 atan(num / den), triangles with |den| < 1e-6
// skipped, absolute value at the end.  One lane does the sum in ring order.
template <class SP>
__device__ double solid_angle_of(const SP &P, int nv, double2 si, double z, const double *L)
{
    auto unit = [](double v[3]) {
        double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] /= l;
        v[1] /= l;
        v[2] /= l;
    };
    double ang = 0.0;
    for (int k = 0; k < nv - 2; k++) {
        double v1[3] = {si.x + P.X[0] - L[0], si.y + P.Y[0] - L[1], z - L[2]};
        double v2[3] = {si.x + P.X[k + 1] - L[0], si.y + P.Y[k + 1] - L[1], z - L[2]};
        double v3[3] = {si.x + P.X[k + 2] - L[0], si.y + P.Y[k + 2] - L[1], z - L[2]};
        unit(v1);
        unit(v2);
        unit(v3);
        double cr[3] = {v2[1] * v3[2] - v2[2] * v3[1], v2[2] * v3[0] - v2[0] * v3[2], v2[0] * v3[1] - v2[1] * v3[0]};
        double num = v1[0] * cr[0] + v1[1] * cr[1] + v1[2] * cr[2];
        double d12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
        double d23 = v2[0] * v3[0] + v2[1] * v3[1] + v2[2] * v3[2];
        double d13 = v1[0] * v3[0] + v1[1] * v3[1] + v1[2] * v3[2];
        double den = 1.0 + d12 + d23 + d13;
        if (fabs(den) < 1e-6) continue;
        ang += 2.0 * atan(num / den);
    }
    return fabs(ang);
}

// Position of pixel line c (x0 + c s), one explicitly rounded form for every
// use: the crossings of an edge, the pixel that a piece lies in and the
// vertical lines of part (b) all see the same line in the same bits.
__device__ __forceinline__ double lpos(int c, double s, double x0) { return __fma_rn((double)c, s, x0); }

// Edge parameter t where the edge from p (inverse length component inv)
// meets the line at X.
__device__ __forceinline__ double line_t(double X, double p, double inv) { return __dmul_rn(__dsub_rn(X, p), inv); }

// Mass and second moment of the cell, regrouped by Green's theorem.
// For each pixel p, int over cell ∩ p of g equals the sum over the boundary
// of cell ∩ p of G dy (dG/dx = g).  Summed over the pixels with their
// densities this is: (a) the cell's edges, cut at the pixel lines they
// cross, each piece weighted by its own pixel's density; plus (b) the
// vertical pixel lines inside the cell, each segment weighted by the density
// of the pixel on its left minus the one on its right (horizontal pieces have
// dy = 0).  (b) also produces the fully covered pixels.  Coordinates are
// taken relative to the centre of the cell's box for accuracy and shifted
// to the site at the end.  Used when neither centroids (whose reference rule
// needs per-pixel areas) nor the render are wanted.
//
// Both parts run one piece per lane.  (a): edge k has 1 + (x lines it
// crosses) + (y lines it crosses) events (its start, then each crossing);
// a scan over the edges hands every lane one event, and the piece that
// starts there ends at the next crossing of either family (found in closed
// form) or at the edge's end.  The pieces are those of walking each edge
// from crossing to crossing, with the same parameters.  (b): every
// (vertical line, pixel row) segment inside the cell, likewise handed out
// by a scan over the lines.  One lane per edge: rings of up to LPC = 32
// vertices.
//
// SPLIT: one part of a cell shared by `nparts` warps (the cells with very
// large pixel boxes): part 0 takes the edge pieces, and part p the vertical
// lines lx + p + nparts q; the part's raw sums {A, Ia, Ib, I2} and the box
// origin go to raw[0..5] (every lane), and the caller adds the parts.
template <int LPC, class SP, bool SPLIT = false>
__device__ __forceinline__ CellAcc integrate_fast(SP &P, int nv, const PixGeo g, double2 si, int lane,
                                                  int part = 0, int nparts = 1, double *raw = nullptr)
{
    static_assert(LPC == 32, "one lane per edge of a ring of up to 32 vertices");
    const Seg<LPC> W;
    CellAcc acc = {0.0, 0.0, 0.0, 0.0, 0.0};
    const bool act = lane < nv;
    const int kn = (lane + 1 >= nv) ? 0 : lane + 1;
    double px = 0.0, py = 0.0, qx = 0.0, qy = 0.0;
    double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
    if (act) {
        px = P.X[lane]; py = P.Y[lane]; qx = P.X[kn]; qy = P.Y[kn];
        const double dx = qx - px, dy = qy - py;
        P.EIX[lane] = dx != 0.0 ? 1.0 / dx : 0.0;
        P.EIY[lane] = dy != 0.0 ? 1.0 / dy : 0.0;
        P.ESL[lane] = dx != 0.0 ? dy / dx : 0.0;
        mnx = px; mxx = px; mny = py; mxy = py;
    }
    mnx = W.min(mnx); mxx = W.max(mxx); mny = W.min(mny); mxy = W.max(mxy);
    W.sync();
    const double ox = 0.5 * (mnx + mxx), oy = 0.5 * (mny + mxy);  // local origin
    const double cx0 = g.pd0 - si.x, cy0 = g.pd2 - si.y;           // pixel line 0, site frame
    double sA = 0.0, sIa = 0.0, sIb = 0.0, sI2 = 0.0;

    // ---- (a) edge pieces --------------------------------------------------
    // edge `lane`: first x line beyond p and count of x lines strictly
    // between p and q (cf, nxc), the same for y (rf, nyc)
    int cf = 0, nxc = 0, rf = 0, nyc = 0, cnt = 0;
    if (!SPLIT || part == 0) {
        const double dx = qx - px, dy = qy - py;
        bool skip = !act || dy == 0.0;  // horizontal: no x-dy term
        if (!skip && dx == 0.0) {
            // a vertical edge on a pixel line is counted with the lines in (b)
            const int ci = (int)floor((px - cx0) * g.ixs + 0.5);
            if (lpos(ci, g.xs, cx0) == px) skip = true;
        }
        if (!skip) {
            if (dx != 0.0) {
                const bool up = dx > 0.0;
                int c = (int)floor((px - cx0) * g.ixs) + (up ? 0 : 1);
                for (int gd = 0; gd < 4; gd++) {
                    const double X = lpos(c, g.xs, cx0);
                    if (up ? X > px : X < px) break;
                    c += up ? 1 : -1;
                }
                int e = (int)floor((qx - cx0) * g.ixs) + (up ? 0 : 1);  // last line short of q
                for (int gd = 0; gd < 4; gd++) {
                    const double X = lpos(e, g.xs, cx0);
                    if (up ? X < qx : X > qx) break;
                    e += up ? -1 : 1;
                }
                for (int gd = 0; gd < 4; gd++) {
                    const double X = lpos(e + (up ? 1 : -1), g.xs, cx0);
                    if (!(up ? X < qx : X > qx)) break;
                    e += up ? 1 : -1;
                }
                cf = c;
                nxc = max(0, (up ? e - c : c - e) + 1);
            }
            {
                const bool up = dy > 0.0;
                int r = (int)floor((py - cy0) * g.iys) + (up ? 0 : 1);
                for (int gd = 0; gd < 4; gd++) {
                    const double Y = lpos(r, g.ys, cy0);
                    if (up ? Y > py : Y < py) break;
                    r += up ? 1 : -1;
                }
                int e = (int)floor((qy - cy0) * g.iys) + (up ? 0 : 1);
                for (int gd = 0; gd < 4; gd++) {
                    const double Y = lpos(e, g.ys, cy0);
                    if (up ? Y < qy : Y > qy) break;
                    e += up ? -1 : 1;
                }
                for (int gd = 0; gd < 4; gd++) {
                    const double Y = lpos(e + (up ? 1 : -1), g.ys, cy0);
                    if (!(up ? Y < qy : Y > qy)) break;
                    e += up ? 1 : -1;
                }
                rf = r;
                nyc = max(0, (up ? e - r : r - e) + 1);
            }
            cnt = 1 + nxc + nyc;
        }
    }
    {
        const int inc = W.incl_scan(cnt);
        const int tot = W.shfl(inc, LPC - 1);
        for (int base = 0; base < tot; base += LPC) {
            const int t = base + lane;
            int k = 0;  // edges whose events end at or before t
#pragma unroll
            for (int sft = LPC / 2; sft >= 1; sft >>= 1) {
                const int v = W.shfl(inc, k + sft - 1);
                if (v <= t) k += sft;
            }
            k &= LPC - 1;
            const int ik = W.shfl(inc, k), ck = W.shfl(cnt, k);
            const int kcf = W.shfl(cf, k), knx = W.shfl(nxc, k), krf = W.shfl(rf, k), kny = W.shfl(nyc, k);
            if (t >= tot) continue;
            const int m = t - (ik - ck);
            const int kk = (k + 1 >= nv) ? 0 : k + 1;
            const double ex = P.X[k], ey = P.Y[k], fx = P.X[kk], fy = P.Y[kk];
            const double dx = fx - ex, dy = fy - ey;
            const double idx = P.EIX[k], idy = P.EIY[k];
            const int cs = dx > 0.0 ? 1 : -1, rs = dy > 0.0 ? 1 : -1;
            // t of the j-th x / y crossing of the edge
            auto tx = [&](int j) -> double { return line_t(lpos(kcf + j * cs, g.xs, cx0), ex, idx); };
            auto ty = [&](int j) -> double { return line_t(lpos(krf + j * rs, g.ys, cy0), ey, idy); };
            double t0;
            int jx, jy;  // first x / y crossing after t0
            bool dup = false;
            if (m == 0) {
                t0 = 0.0;
                jx = 0;
                jy = 0;
            } else if (m <= knx) {
                jx = m;
                t0 = tx(m - 1);
                // first y crossing past t0: estimate from the position, then settle
                const double ym = __fma_rn(t0, dy, ey);
                int r = (int)floor((ym - cy0) * g.iys) + (rs > 0 ? 1 : 0);
                jy = min(max((r - krf) * rs, 0), kny);
                for (int gd = 0; gd < 4 && jy > 0 && ty(jy - 1) > t0; gd++) jy--;
                for (int gd = 0; gd < 4 && jy < kny && ty(jy) <= t0; gd++) jy++;
            } else {
                jy = m - knx;
                t0 = ty(jy - 1);
                const double xm = __fma_rn(t0, dx, ex);
                int c = (int)floor((xm - cx0) * g.ixs) + (cs > 0 ? 1 : 0);
                jx = knx > 0 ? min(max((c - kcf) * cs, 0), knx) : 0;
                for (int gd = 0; gd < 4 && jx > 0 && tx(jx - 1) > t0; gd++) jx--;
                for (int gd = 0; gd < 4 && jx < knx && tx(jx) <= t0; gd++) jx++;
                // an x crossing at the same t (a pixel corner) owns the piece
                dup = jx > 0 && tx(jx - 1) == t0;
            }
            const double t1 = fmin(fmin(jx < knx ? tx(jx) : 2.0, jy < kny ? ty(jy) : 2.0), 1.0);
            if (dup || !(t1 > t0)) continue;
            const double ax = t0 == 0.0 ? ex : __fma_rn(t0, dx, ex), ay = t0 == 0.0 ? ey : __fma_rn(t0, dy, ey);
            const double bx = t1 == 1.0 ? fx : __fma_rn(t1, dx, ex), by = t1 == 1.0 ? fy : __fma_rn(t1, dy, ey);
            const double tm = 0.5 * (t0 + t1);
            // pixel of the piece, settled against the line positions
            const double xm = __fma_rn(tm, dx, ex), ym = __fma_rn(tm, dy, ey);
            int ix = (int)floor((xm - cx0) * g.ixs);
            int iy = (int)floor((ym - cy0) * g.iys);
            if (lpos(ix, g.xs, cx0) > xm) ix--;
            else if (lpos(ix + 1, g.xs, cx0) <= xm) ix++;
            if (lpos(iy, g.ys, cy0) > ym) iy--;
            else if (lpos(iy + 1, g.ys, cy0) <= ym) iy++;
            // a piece outside the image (a rounding sliver along the domain
            // sides) carries no density
            if (ix < 0 || ix >= g.nx || iy < 0 || iy >= g.ny) continue;
            const double rho = g.rho[ix + iy * g.nx];
            Mom mm = {0.0, 0.0, 0.0, 0.0};
            seg_terms(ax - ox, ay - oy, bx - ox, by - oy, mm);
            sA += rho * mm.A;
            sIa += rho * mm.Ia;
            sIb += rho * mm.Ib;
            sI2 += rho * mm.I2;
        }
    }

    // ---- (b) vertical pixel lines inside the cell --------------------------
    // pixel columns [lx, hx) and rows [ly, hy) of the cell's box, one pixel
    // wider on each side; lines lx .. hx
    int lx = (int)floor((mnx - cx0) * g.ixs) - 1;
    int ly = (int)floor((mny - cy0) * g.iys) - 1;
    int hx = (int)floor((mxx - cx0) * g.ixs) + 2;
    int hy = (int)floor((mxy - cy0) * g.iys) + 2;
    lx = max(lx, 0);
    ly = max(ly, 0);
    hx = min(hx, g.nx);
    hy = min(hy, g.ny);
    const int lstep = SPLIT ? nparts : 1;
    for (int cxs = lx + (SPLIT ? part : 0); cxs <= hx; cxs += LPC * lstep) {
        const int l = cxs + lane * lstep;
        double lo = INFINITY, hi = -INFINITY, xl = 0.0;
        int r0 = 0, rc = 0;
        bool fl = false, fr = false;
        if (l <= hx) {
            xl = lpos(l, g.xs, cx0);
            fl = l - 1 >= lx && mnx < xl && xl <= mxx;  // right side of pixel l-1 (a left limit)
            fr = l < hx && mnx <= xl && xl < mxx;       // left side of pixel l (a right limit)
            if (fl || fr) {
                section_at(P, nv, xl, lo, hi);
                if (hi > lo) {
                    r0 = max((int)floor((lo - cy0) * g.iys) - 1, ly);
                    const int r1 = min((int)floor((hi - cy0) * g.iys) + 1, hy - 1);
                    rc = max(0, r1 - r0 + 1);
                }
            }
        }
        const int inc = W.incl_scan(rc);
        const int tot = W.shfl(inc, LPC - 1);
        for (int base = 0; base < tot; base += LPC) {
            const int t = base + lane;
            int k = 0;
#pragma unroll
            for (int sft = LPC / 2; sft >= 1; sft >>= 1) {
                const int v = W.shfl(inc, k + sft - 1);
                if (v <= t) k += sft;
            }
            k &= LPC - 1;
            const int ik = W.shfl(inc, k), ck = W.shfl(rc, k), kr0 = W.shfl(r0, k);
            const double klo = W.shfl(lo, k), khi = W.shfl(hi, k), kxl = W.shfl(xl, k);
            const bool kfl = W.shfl((int)fl, k) != 0, kfr = W.shfl((int)fr, k) != 0;
            if (t >= tot) continue;
            const int r = kr0 + (t - (ik - ck));
            const double b0 = fmax(klo, lpos(r, g.ys, cy0)), b1 = fmin(khi, lpos(r + 1, g.ys, cy0));
            if (!(b1 > b0)) continue;
            const int lk = cxs + k * lstep;
            const double wl = kfl ? g.rho[(lk - 1) + r * g.nx] : 0.0;
            const double wr = kfr ? g.rho[lk + r * g.nx] : 0.0;
            Mom mm = {0.0, 0.0, 0.0, 0.0};
            vside_terms(kxl - ox, b0 - oy, b1 - oy, mm);  // upwards: the left pixel's right side
            const double wd = wl - wr;
            sA += wd * mm.A;
            sIa += wd * mm.Ia;
            sIb += wd * mm.Ib;
            sI2 += wd * mm.I2;
        }
    }
    sA = W.sum(sA);
    sIa = W.sum(sIa);
    sIb = W.sum(sIb);
    sI2 = W.sum(sI2);
    if constexpr (SPLIT) {
        raw[0] = sA;
        raw[1] = sIa;
        raw[2] = sIb;
        raw[3] = sI2;
        raw[4] = ox;
        raw[5] = oy;
        return acc;
    }
    acc.mu = sA;
    // int |x - s_i|^2 = int |(x - o) + o|^2 in the site frame
    acc.S = sI2 + 2.0 * (ox * sIa + oy * sIb) + (ox * ox + oy * oy) * sA;
    return acc;
}

// Plain area centroid of the polygon (relative to the site).
template <class SP>
__device__ void poly_centroid(const SP &P, int nv, int lane, double &cx, double &cy)
{
    double a = 0.0, mx = 0.0, my = 0.0;
    for (int k = lane; k < nv; k += 32) {
        int kn = (k + 1 == nv) ? 0 : k + 1;
        double x0 = P.X[k], y0 = P.Y[k], x1 = P.X[kn], y1 = P.Y[kn];
        double cr = x0 * y1 - x1 * y0;
        a += cr;
        mx += (x0 + x1) * cr;
        my += (y0 + y1) * cr;
    }
    a = warp_sum(a);
    mx = warp_sum(mx);
    my = warp_sum(my);
    cx = a != 0.0 ? mx / (3.0 * a) : 0.0;
    cy = a != 0.0 ? my / (3.0 * a) : 0.0;
}

// ---------------------------------------------------------------------------
// fast path: the polygon lives in registers, one vertex per lane
// ---------------------------------------------------------------------------
struct FastScratch {
    double X[32], Y[32];              // polygon snapshot (tree tests, integration)
    double A[32], B[32], C[32];       // compaction scratch of the general clip
    int L[32];
    double EIX[32], EIY[32], ESL[32]; // per edge: 1/dx, 1/dy, dy/dx
    int fr[2][COT_FRMAX];
    double elo[33], ehi[33];
    double slo[32], shi[32];
    unsigned char lv[33], rv[33];
    int KL[32];                       // ring labels just before the ring emptied
    int kn, kill;                     // their count and the label that emptied it
};

// Lane k < nv holds vertex k and the line a x + b y <= c (generator l) of the
// edge from vertex k to vertex k+1; coordinates relative to the site.
struct RegPoly {
    double x, y, a, b, c;
    int l;
    int nv;
};

__device__ __forceinline__ unsigned lanes_below(int n) { return n >= 32 ? FULLMASK : ((1u << n) - 1u); }

// Clip by a x + b y <= c.  Returns false when the ring would exceed LPC
// vertices.  A convex ring crossed twice is a pure register permutation;
// any other pattern (rounding on nearly collinear vertices) is compacted
// through shared memory.
template <int LPC>
__device__ __forceinline__ bool rclip(RegPoly &P, double a, double b, double c, int lab, int lane, FastScratch &S)
{
    const Seg<LPC> W;
    const int nv = P.nv;
    const bool valid = lane < nv;
    const double d = side(a, b, c, P.x, P.y);
    const unsigned vm = W.below(nv);
    const unsigned outm = W.ballot(valid && d > 0.0);
    if (outm == 0u) return true;
    if (outm == vm) {
        // hidden cell: remember what hid it, to seed the next evaluation
        if (valid) S.KL[lane] = P.l;
        if (lane == 0) {
            S.kn = nv;
            S.kill = lab;
        }
        P.nv = 0;
        return true;
    }
    const int nx = (lane + 1 >= nv) ? 0 : lane + 1;
    const double xn = W.shfl(P.x, nx);
    const double yn = W.shfl(P.y, nx);
    const double dn = W.shfl(d, nx);
    const bool in = !((outm >> lane) & 1u);
    const bool inn = !((outm >> nx) & 1u);
    const bool cross = valid && (in != inn);
    double ix = 0.0, iy = 0.0;
    if (cross) {
        if (!line_meet(P.a, P.b, P.c, a, b, c, ix, iy)) {
            double t = d / (d - dn);
            ix = P.x + t * (xn - P.x);
            iy = P.y + t * (yn - P.y);
        }
    }
    const unsigned cm = W.ballot(cross);
    const int K = __popc(vm & ~outm);
    if (__popc(cm) == 2) {
        const unsigned em = W.ballot(cross && !in);  // edge entering the half-plane
        const int e = __ffs(em) - 1;
        const int l = __ffs(cm & ~em) - 1;                         // edge leaving it
        const int nn = K + 2;
        if (nn > LPC) return false;
        // new ring: I_e, v_{e+1} .. v_{e+K} (= v_l), I_l
        int src = e;
        if (lane >= 1 && lane <= K) {
            src = e + lane;
            if (src >= nv) src -= nv;
        } else if (lane == K + 1) {
            src = l;
        }
        const double gx = W.shfl(P.x, src);
        const double gy = W.shfl(P.y, src);
        const double ga = W.shfl(P.a, src);
        const double gb = W.shfl(P.b, src);
        const double gc = W.shfl(P.c, src);
        const int gl = W.shfl(P.l, src);
        const double iex = W.shfl(ix, e), iey = W.shfl(iy, e);
        const double ilx = W.shfl(ix, l), ily = W.shfl(iy, l);
        if (lane == 0) {
            P.x = iex; P.y = iey; P.a = ga; P.b = gb; P.c = gc; P.l = gl;
        } else if (lane <= K) {
            P.x = gx; P.y = gy; P.a = ga; P.b = gb; P.c = gc; P.l = gl;
        } else if (lane == K + 1) {
            P.x = ilx; P.y = ily; P.a = a; P.b = b; P.c = c; P.l = lab;
        }
        P.nv = nn;
        return true;
    }
    const int cnt = valid ? ((in ? 1 : 0) + (cross ? 1 : 0)) : 0;
    const int inc = W.incl_scan(cnt);
    const int tot = W.shfl(inc, LPC - 1);
    if (tot > LPC) return false;
    W.sync();
    if (valid) {
        int p = inc - cnt;
        if (in) {
            S.X[p] = P.x; S.Y[p] = P.y; S.A[p] = P.a; S.B[p] = P.b; S.C[p] = P.c; S.L[p] = P.l;
            p++;
        }
        if (cross) {
            S.X[p] = ix; S.Y[p] = iy;
            if (in) { S.A[p] = a; S.B[p] = b; S.C[p] = c; S.L[p] = lab; }
            else { S.A[p] = P.a; S.B[p] = P.b; S.C[p] = P.c; S.L[p] = P.l; }
        }
    }
    W.sync();
    if (lane < tot) {
        P.x = S.X[lane]; P.y = S.Y[lane]; P.a = S.A[lane]; P.b = S.B[lane]; P.c = S.C[lane]; P.l = S.L[lane];
    }
    W.sync();
    P.nv = tot;
    return true;
}

// Ascending bitonic sort of (key, idx) across the segment.
template <int LPC>
__device__ __forceinline__ void warp_sort(double &key, int &idx, int lane)
{
    const Seg<LPC> W;
#pragma unroll
    for (int k = 2; k <= LPC; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            double ok = W.shfl_xor(key, j);
            int oi = W.shfl_xor(idx, j);
            bool up = (lane & k) == 0;
            bool lower = (lane & j) == 0;
            bool less = ok < key || (ok == key && oi < idx);
            bool greater = ok > key || (ok == key && oi > idx);
            if (lower == up ? less : greater) { key = ok; idx = oi; }
        }
    }
}

// Apply the candidates of one chunk (lane t holds site jl, -1 = none).  Each
// lane first tests its own candidate against the whole ring (snapshot in
// shared memory); only candidates that cut are then applied one by one with a
// register clip (one that no longer cuts after an earlier clip is a no-op).
// `nearest` applies the cutting ones in order of distance from the site.
template <int LPC>
__device__ __forceinline__ RegPoly apply_chunk(RegPoly P, int jl, const double2 *__restrict__ sxy, double2 si, double wi,
                                            const double *__restrict__ wt, int lane, FastScratch &S, bool nearest)
{
    const Seg<LPC> W;
    if (W.ballot(jl >= 0) == 0u) return P;
    double al = 0.0, bl = 0.0, cl = 0.0, key = INFINITY;
    if (jl >= 0) site_line(sxy[jl], si, wt[jl], wi, al, bl, cl, key);
    const int nv = P.nv;
    if (lane < nv) { S.X[lane] = P.x; S.Y[lane] = P.y; S.L[lane] = P.l; }
    W.sync();
    bool cut = false;
    if (jl >= 0) {
        for (int k = 0; k < nv; k++) {
            if (S.L[k] == jl) { cut = false; break; }   // already bounds the ring
            if (side(al, bl, cl, S.X[k], S.Y[k]) > 0.0) cut = true;
        }
    }
    W.sync();
    unsigned have = W.ballot(cut);
#ifdef COT_PHASE_STATS
    const int ntested = __popc(W.ballot(jl >= 0));  // segment-wide, outside the lane-0 branch
    PSTAT_ADD(4, ntested);
#endif
    if (have == 0u) return P;
    int ord = lane;
    if (nearest && __popc(have) > 1) {
        double k2 = cut ? key : INFINITY;
        warp_sort<LPC>(k2, ord, lane);
        have = W.below(__popc(have));
    } else {
        nearest = false;
    }
    while (have != 0u && P.nv > 0) {
        const int t = __ffs(have) - 1;
        have &= have - 1u;
        const int src = nearest ? W.shfl(ord, t) : t;
        const int j = W.shfl(jl, src);
        const double a = W.shfl(al, src);
        const double b = W.shfl(bl, src);
        const double c = W.shfl(cl, src);
        const int before = P.nv;
        if (!rclip<LPC>(P, a, b, c, j, lane, S)) {
            P.nv = -1;
            return P;
        }
        if (P.nv != before) PSTAT_ADD(3, 1);
    }
    return P;
}

// Clip by the domain sides that the ring crosses (nv = -1: the ring grew past
// LPC vertices).  Rarely needed, so kept out of line.
template <int LPC>
__device__ __noinline__ RegPoly clip_sides(RegPoly P, double4 box, int lane, FastScratch &S)
{
    const Seg<LPC> W;
    for (int k = 0; k < 4 && P.nv > 0; k++) {
        double a, b, c;
        side_line(k, box, a, b, c);
        const bool out = lane < P.nv && side(a, b, c, P.x, P.y) > 0.0;
        if (W.any(out)) {
            if (!rclip<LPC>(P, a, b, c, -(k + 1), lane, S)) {
                P.nv = -1;
                return P;
            }
        }
    }
    return P;
}

// The ring of the last evaluation, rebuilt in one step: lane k < m holds the
// generator `lab` of edge k (a site, or -1..-4 for a domain side), vertex k
// is where the lines of edges k-1 and k meet.  Accepted only if every vertex
// lies inside every other line, every edge runs forward along its line and
// every corner turns left; the ring is then the intersection of those
// half-planes, with the vertices a sequence of clips would compute (same
// line pair, same symmetric meet).  Otherwise the result has nv = -2, and
// `backward` marks the lanes whose edge runs backward (a line that no longer
// reaches the ring, e.g. after an edge flip).
template <int LPC>
__device__ __forceinline__ RegPoly ring_try(int lab, int m, const double2 *__restrict__ sxy, double4 box, double2 si,
                                            double wi, const double *__restrict__ wt, int lane, unsigned &backward)
{
    const Seg<LPC> W;
    RegPoly P;
    const bool act = lane < m;
    double la = 0.0, lb = 0.0, lc = 0.0, key;
    if (act) {
        if (lab >= 0) site_line(sxy[lab], si, wt[lab], wi, la, lb, lc, key);
        else side_line(-lab - 1, box, la, lb, lc);
    }
    const int pv = act ? (lane == 0 ? m - 1 : lane - 1) : lane;
    const int nx = act ? (lane + 1 == m ? 0 : lane + 1) : lane;
    const double pa = W.shfl(la, pv), pb = W.shfl(lb, pv);
    const double pc = W.shfl(lc, pv);
    double vx = 0.0, vy = 0.0;
    bool ok = true;
    if (act) ok = line_meet(pa, pb, pc, la, lb, lc, vx, vy);
    for (int j = 0; j < m; j++) {
        const double ja = W.shfl(la, j), jb = W.shfl(lb, j);
        const double jc = W.shfl(lc, j);
        if (act && j != lane && j != pv && side(ja, jb, jc, vx, vy) > 0.0) ok = false;
    }
    const double nvx = W.shfl(vx, nx), nvy = W.shfl(vy, nx);
    const double na = W.shfl(la, nx), nb = W.shfl(lb, nx);
    bool back = false;
    if (act) {
        // edge k runs along (-b, a) from vertex k to vertex k+1
        const double len = __fma_rn(nvx - vx, -lb, __dmul_rn(nvy - vy, la));
        const double turn = __fma_rn(-lb, na, __dmul_rn(la, nb));
        back = !(len > 0.0);
        if (back || !(turn > 0.0)) ok = false;
    }
    backward = W.ballot(back);
    if (!W.all(ok)) {
        P.nv = -2;
        return P;
    }
    P.x = vx;
    P.y = vy;
    P.a = la;
    P.b = lb;
    P.c = lc;
    P.l = act ? lab : 0;
    P.nv = m;
    return P;
}

// A cached ring that failed its check: drop the generators whose edges run
// backward and try again (a few times).  Any subset of the cell's true
// half-planes bounds a superset of the cell, and the certificate walk adds
// the cuts that are missing, so the result is the same as clipping from the
// domain rectangle.  nv = -2 when this does not give a valid ring.
template <int LPC>
__device__ __noinline__ RegPoly ring_repair(int lab, int m, const double2 *__restrict__ sxy, double4 box, double2 si,
                                            double wi, const double *__restrict__ wt, int lane, FastScratch &S,
                                            unsigned backward)
{
    const Seg<LPC> W;
    RegPoly P;
    P.nv = -2;
    for (int attempt = 0; attempt < 3 && backward != 0u; attempt++) {
        const bool keep = lane < m && !((backward >> lane) & 1u);
        const unsigned km = W.ballot(keep);
        W.sync();
        if (keep) S.L[__popc(km & W.below(lane))] = lab;
        W.sync();
        m = __popc(km);
        lab = lane < m ? S.L[lane] : -1;
        W.sync();
        if (m < 3) break;
        P = ring_try<LPC>(lab, m, sxy, box, si, wi, wt, lane, backward);
        if (P.nv != -2) return P;
    }
    P.nv = -2;
    return P;
}

// The cached ring rebuilt in one step (ring_try), repaired when generators
// dropped out.  Cuts by sites outside the list are found by the certificate;
// cuts by domain sides outside it are applied here (nv = -1: the ring grew
// past LPC vertices).  nv = -2: the caller clips from the domain rectangle.
template <int LPC>
__device__ __forceinline__ RegPoly ring_from_cache(int lab, int m, const double2 *__restrict__ sxy, double4 box,
                                                double2 si, double wi, const double *__restrict__ wt, int lane,
                                                FastScratch &S)
{
    const Seg<LPC> W;
    unsigned backward = 0u;
    RegPoly P = ring_try<LPC>(lab, m, sxy, box, si, wi, wt, lane, backward);
    if (P.nv == -2) {
        if (backward == 0u) return P;
        P = ring_repair<LPC>(lab, m, sxy, box, si, wi, wt, lane, S, backward);
        if (P.nv == -2) return P;
    }
    // domain sides that the cell now reaches (rare: clipped out of line)
    bool out = false;
    if (lane < P.nv) out = P.x < box.x || P.x > box.y || P.y < box.z || P.y > box.w;
    if (W.any(out)) P = clip_sides<LPC>(P, box, lane, S);
    return P;
}

// Sites of `cnt[k]` consecutive ranges starting at `st[k]` (k = lane, up to
// LPC ranges), applied in chunks of LPC.  inc = inclusive scan of cnt.
template <int LPC>
__device__ __forceinline__ RegPoly apply_ranges(RegPoly P, int st, int cnt, int inc, int self, const double2 *__restrict__ sxy,
                                             double2 si, double wi, const double *__restrict__ wt, int lane,
                                             FastScratch &S, bool nearest)
{
    const Seg<LPC> W;
    const int tot = W.shfl(inc, LPC - 1);
    for (int base = 0; base < tot && P.nv > 0; base += LPC) {
        const int t = base + lane;
        // k = number of ranges that end at or before t
        int k = 0;
#pragma unroll
        for (int sft = LPC / 2; sft >= 1; sft >>= 1) {
            int v = W.shfl(inc, k + sft - 1);
            if (v <= t) k += sft;
        }
        const int ik = W.shfl(inc, k & (LPC - 1));
        const int sk = W.shfl(st, k & (LPC - 1));
        const int ck = W.shfl(cnt, k & (LPC - 1));
        int j = (t < tot) ? sk + (t - (ik - ck)) : -1;
        if (j == self) j = -1;
        P = apply_chunk<LPC>(P, j, sxy, si, wi, wt, lane, S, nearest);
        if (P.nv < 0) return P;
    }
    return P;
}

// Out-of-line copies for the paths a cell takes rarely once a solve runs warm
// (no usable cache, frontier overflow): the hot path keeps one inlined copy
// of the clip code, which keeps the kernel's working set of instructions
// small.
template <int LPC>
__device__ __noinline__ RegPoly apply_ranges_cold(RegPoly P, int st, int cnt, int inc, int self,
                                                  const double2 *__restrict__ sxy, double2 si, double wi,
                                                  const double *__restrict__ wt, int lane, FastScratch &S, bool nearest)
{
    return apply_ranges<LPC>(P, st, cnt, inc, self, sxy, si, wi, wt, lane, S, nearest);
}

template <int LPC>
__device__ __noinline__ RegPoly apply_chunk_cold(RegPoly P, int jl, const double2 *__restrict__ sxy, double2 si,
                                                 double wi, const double *__restrict__ wt, int lane, FastScratch &S,
                                                 bool nearest)
{
    return apply_chunk<LPC>(P, jl, sxy, si, wi, wt, lane, S, nearest);
}

// Upper bound of P_j(x) = x.s_j - phi_j over the sites of a tree node at the
// absolute point x: F(x + a) + B, the bound node_excluded tests (-inf for an
// empty node).
__device__ __forceinline__ double node_upper(const CotGeo &g, int node, double x, double y)
{
    const double4 st = g.tstat[node];
    if (st.z < 0.0) return -INFINITY;
    const double4 dy = g.tdyn[node];
    const double tx = x + dy.x, ty = y + dy.y;
    const double ex = fmax(fabs(tx - st.x) - st.z, 0.0);
    const double ey = fmax(fabs(ty - st.y) - st.w, 0.0);
    return 0.5 * (__fma_rn(tx, tx, ty * ty) - __fma_rn(ex, ex, ey * ey)) + dy.z;
}

// Shrinks a ring that is far larger than its cell, for a certificate walk
// whose frontier overflowed.  Each lane takes one vertex x of the ring and
// descends the bound tree greedily (at every level the node with the largest
// bound at x, at the leaf the site with the largest P_j(x)); a site that
// beats P_i at x cuts that vertex off.  The distinct sites found are applied
// like any other candidates, and the search repeats on the new ring, up to
// `rounds` times or until no vertex finds a site.  Every clip is by a site
// that cuts the ring, so the ring still contains the cell; the walk that
// follows certifies it, and the cell's result is the one any other clip
// order gives.
template <int LPC>
__device__ __noinline__ RegPoly refine_by_vertices(const CotGeo &g, const double *__restrict__ wt, int i, double2 si,
                                                   double wi, RegPoly P, FastScratch &S, int rounds)
{
    const Seg<LPC> SG;
    const int lane = SG.sl;
    int top = g.nlev - 1;
    while (top > 0 && g.lev_w[top - 1] * g.lev_h[top - 1] <= (LPC < 16 ? 16 : LPC)) top--;
    const int tw = g.lev_w[top], ntop = tw * g.lev_h[top], toff = g.lev_off[top];
    const double phi_i = 0.5 * (__fma_rn(si.x, si.x, si.y * si.y) - wi);
    for (int r = 0; r < rounds && P.nv > 0; r++) {
        int jl = -1;
        if (lane < P.nv) {
            const double x = si.x + P.x, y = si.y + P.y;
            const double pi = __fma_rn(x, si.x, y * si.y) - phi_i;
            int bu = -1, bv = -1;
            double best = -INFINITY;
            for (int q = 0; q < ntop; q++) {
                const double ub = node_upper(g, toff + q, x, y);
                if (ub > best) { best = ub; bu = q % tw; bv = q / tw; }
            }
            for (int L = top; L > 0 && bu >= 0; L--) {
                const int cw = g.lev_w[L - 1], ch = g.lev_h[L - 1], off = g.lev_off[L - 1];
                int nu = -1, nw = -1;
                best = -INFINITY;
                for (int bb = 0; bb < 2; bb++)
                    for (int aa = 0; aa < 2; aa++) {
                        const int cu = 2 * bu + aa, cv = 2 * bv + bb;
                        if (cu < cw && cv < ch) {
                            const double ub = node_upper(g, off + cu + cv * cw, x, y);
                            if (ub > best) { best = ub; nu = cu; nw = cv; }
                        }
                    }
                bu = nu;
                bv = nw;
            }
            if (bu >= 0) {
                const int b = bu + bv * g.lev_w[0];
                double bp = pi;
                for (int j = g.bstart[b], e = g.bstart[b + 1]; j < e; j++) {
                    if (j == i) continue;
                    const double2 sj = g.xy[j];
                    const double pj = __fma_rn(x, sj.x, y * sj.y) - 0.5 * (__fma_rn(sj.x, sj.x, sj.y * sj.y) - wt[j]);
                    if (pj > bp) { bp = pj; jl = j; }
                }
            }
        }
        // one copy of each site
        for (int t = 0; t < LPC; t++) {
            const int o = SG.shfl(jl, t);
            if (t < lane && o == jl) jl = -1;
        }
        if (SG.ballot(jl >= 0) == 0u) break;
        P = apply_chunk<LPC>(P, jl, g.xy, si, wi, wt, lane, S, false);
        if (P.nv < 0) break;
    }
    return P;
}

// Every bucket tested against the current ring, and the sites of those
// that can cut it applied (the buckets of the window around (bu, bv) are
// skipped: their sites were applied already).  The last resort of a
// certificate whose frontier overflows.
template <int LPC>
__device__ __noinline__ RegPoly scan_all_buckets(const CotGeo &g, const double *__restrict__ wt, int i, double2 si,
                                                 double wi, RegPoly P, FastScratch &S, int bu, int bv, int win)
{
    const Seg<LPC> SG;
    const int lane = SG.sl;
    const int nb = g.bx * g.by;
    for (int base = 0; base < nb && P.nv > 0; base += LPC) {
        if (lane < P.nv) { S.X[lane] = P.x; S.Y[lane] = P.y; }
        SG.sync();
        const int b = base + lane;
        bool keep = false;
        if (b < nb) {
            const int u = b % g.bx, v = b / g.bx;
            const bool inwin = abs(u - bu) <= win && abs(v - bv) <= win;
            keep = !inwin && !node_excluded(S, P.nv, g, b, si, wi);
        }
        SG.sync();
        int st = 0, cnt = 0;
        if (keep) {
            st = g.bstart[b];
            cnt = g.bstart[b + 1] - st;
        }
        const int inc = SG.incl_scan(cnt);
        P = apply_ranges<LPC>(P, st, cnt, inc, i, g.xy, si, wi, wt, lane, S, false);
    }
    return P;
}

// One cell, worked by one segment of LPC lanes (lane = index in the segment),
// in three phases: cell_first (the first candidates), cell_walk (the
// certificate over the bound tree) and cell_finish (integrals or the ring
// buffer, the next evaluation's cache, the per-cell outputs).  A ring that
// outgrows LPC vertices has nv = -1 from then on and goes to olist / ocount
// for the next pass.  EXACT = true: the per-pixel path that also yields
// centroids (with the reference's 1e-10 piece rule) and the render, a whole
// warp per cell; false: the solver's hot path (masses and objective only).
//
// Phase 1: the domain rectangle clipped by the last evaluation's ring (or
// neighbours), else by the 3x3 buckets around the site.  cached: the cell
// had a usable cache (the certificate then skips no window).
template <int LPC>
__device__ __forceinline__ RegPoly cell_first(const CotGeo &g, const CellsArgs &a, const int i, const double2 si,
                                              const double wi, FastScratch &S, bool &cached)
{
    const Seg<LPC> SG;
    const int lane = SG.sl;
    const double *__restrict__ wt = a.wt;
    PSTAT_CLOCK(t0);
    // domain rectangle, CCW, relative to the site
    RegPoly P;
    P.nv = 4;
    {
        const double x0 = g.pd[0] - si.x, x1 = g.pd[1] - si.x, y0 = g.pd[2] - si.y, y1 = g.pd[3] - si.y;
        P.x = (lane == 1 || lane == 2) ? x1 : x0;
        P.y = (lane >= 2) ? y1 : y0;
        P.a = lane == 1 ? 1.0 : (lane == 3 ? -1.0 : 0.0);
        P.b = lane == 0 ? -1.0 : (lane == 2 ? 1.0 : 0.0);
        P.c = lane == 0 ? -y0 : (lane == 1 ? x1 : (lane == 2 ? y1 : -x0));
        P.l = -(lane + 1);
    }
    if (lane == 0) S.kn = -1;
    SG.sync();
    const int bi = g.sbucket[i];
    const int bu = bi % g.bx, bv = bi / g.bx;
    // ---- 1. first candidates: last evaluation's ring or neighbours, else
    //         the 3x3 buckets around the site, nearest first ---------------
    // cache: +m = the ring's m generators in order (domain sides
    // included), -m = m sites in no order (long rings), hidden cells
    // -(COT_NB_HIDDEN + m)
    const int nraw = (a.nbn != nullptr) ? a.nbn[i] : 0;
    const bool hidden = nraw < -COT_NB_HIDDEN;
    const int ncache = min(nraw >= 0 ? nraw : (hidden ? -nraw - COT_NB_HIDDEN : -nraw), COT_NBC);
    cached = ncache > 0;
    if (cached) {
        const int lab = lane < ncache ? a.nbc[(size_t)i * COT_NBC + lane] : -1;
        bool direct = false;
        if (nraw >= 3 && ncache <= LPC) {
            const double4 box = make_double4(g.pd[0] - si.x, g.pd[1] - si.x, g.pd[2] - si.y, g.pd[3] - si.y);
            const RegPoly Q = ring_from_cache<LPC>(lab, ncache, g.xy, box, si, wi, wt, lane, S);
            if (Q.nv != -2) {
                P = Q;
                direct = true;
            }
        }
        PSTAT_ADD(12, direct ? 1 : 0);
        PSTAT_ADD(13, (!hidden && nraw < 0) ? 1 : 0);     // unordered cache (long ring)
        PSTAT_ADD(14, (nraw >= 3 && !direct) ? 1 : 0);    // ordered cache that failed its check
        PSTAT_ADD(15, hidden ? 1 : 0);
        if (!direct) {
            const int j = (lane < ncache && lab >= 0) ? lab : -1;
            P = apply_chunk_cold<LPC>(P, j, g.xy, si, wi, wt, lane, S, false);
            if constexpr (LPC < COT_NBC) {
                // the cached sites past the segment's lanes, a chunk at a time
                for (int c0 = LPC; c0 < ncache && P.nv > 0; c0 += LPC) {
                    const int lb = c0 + lane < ncache ? a.nbc[(size_t)i * COT_NBC + c0 + lane] : -1;
                    P = apply_chunk_cold<LPC>(P, lb >= 0 ? lb : -1, g.xy, si, wi, wt, lane, S, false);
                }
            }
        }
        // a hidden cell that reappears gets the window as well, so that
        // the certificate starts from a tight ring
#ifndef COT_HIDDEN_WINDOW
#define COT_HIDDEN_WINDOW 1
#endif
        if (COT_HIDDEN_WINDOW && hidden && P.nv > 0) cached = false;
    }
    // the 3x3 buckets around the site: one round of lanes for 16 or 32, two
    // for an 8-lane segment
    constexpr int WROUNDS = LPC >= 16 ? 1 : 2;
#pragma unroll
    for (int r = 0; r < WROUNDS; r++) {
        if (cached || P.nv <= 0) break;
        const int k = r * LPC + lane;
        int bcnt = 0, bst = 0;
        if (k < 9) {
            const int du = (k == 1 || k == 5 || k == 7) ? 1 : (k == 2 || k == 6 || k == 8) ? -1 : 0;
            const int dv = (k == 3 || k == 5 || k == 6) ? 1 : (k == 4 || k == 7 || k == 8) ? -1 : 0;
            const int u = bu + du, v = bv + dv;
            if (u >= 0 && u < g.bx && v >= 0 && v < g.by) {
                const int b = u + v * g.bx;
                bst = g.bstart[b];
                bcnt = g.bstart[b + 1] - bst;
            }
        }
        const int inc = SG.incl_scan(bcnt);
        P = apply_ranges_cold<LPC>(P, bst, bcnt, inc, i, g.xy, si, wi, wt, lane, S, true);
    }
    PSTAT_CLOCK(t1);
    PSTAT_ADD(0, t1 - t0);
    PSTAT_ADD(10, cached ? 1 : 0);
    return P;
}

// Phase 2: every bucket whose sites could cut the ring is found through the
// bound tree and its sites are applied.
template <int LPC>
__device__ __forceinline__ RegPoly cell_walk(const CotGeo &g, const CellsArgs &a, const int i, const double2 si,
                                             const double wi, RegPoly P, const bool cached, FastScratch &S)
{
    const Seg<LPC> SG;
    const int lane = SG.sl;
    const double *__restrict__ wt = a.wt;
    PSTAT_CLOCK(t1);
    bool ok = P.nv >= 0;
    const int bi = g.sbucket[i];
    const int bu = bi % g.bx, bv = bi / g.bx;
    const int win = cached ? -1 : COT_WIN;
    // ---- 2. certificate over the bound tree --------------------------------
    // A walk whose frontier overflows means a ring far larger than its cell:
    // the ring is shrunk by point location at its vertices and walked again
    // (COT_REFINE_PASSES times at most) before every bucket is tested.
    bool brute = false;
    for (int pass = 0;; pass++) {
    if (ok && P.nv > 0 && g.nlev > 0) {
        if (lane < P.nv) { S.X[lane] = P.x; S.Y[lane] = P.y; }
        SG.sync();
        const int nv0 = P.nv;
        // start at the deepest level that still fits one round of lanes:
        // every node there is tested, a superset of what the levels above
        // would keep, without their rounds
        // (at least the first level of at most 16 nodes: the levels above it
        // are not built; an 8-lane segment takes it in two rounds)
        int top = g.nlev - 1;
        while (top > 0 && g.lev_w[top - 1] * g.lev_h[top - 1] <= (LPC < 16 ? 16 : LPC)) top--;
        int ncur = g.lev_w[top] * g.lev_h[top];
        if (ncur > COT_FRMAX) brute = true;
        int cur = 0;
        bool have = false;  // the surviving leaves are in S.fr[cur][0, ncur)
        if constexpr (LPC == 32) {
            // the leaf buckets k_bucket_walk listed for the cell's bucket: one
            // round of leaf tests against this ring, in the walk's order
            if (!brute && a.bcnt != nullptr) {
                const int bc = a.bcnt[bi];
                if (bc >= 0) {
                    int nl = 0;
                    for (int base = 0; base < bc; base += LPC) {
                        const int e = base + lane < bc ? a.blist[(size_t)bi * COT_BLEAF + base + lane] : -1;
                        bool keep = false;
                        if (e >= 0) {
                            const int u = e % g.bx, v = e / g.bx;
                            const bool inwin = abs(u - bu) <= win && abs(v - bv) <= win;
                            keep = !inwin && !node_excluded(S, nv0, g, e, si, wi);
                        }
                        const unsigned m = SG.ballot(keep);
                        if (keep) S.fr[1][nl + __popc(m & ((1u << lane) - 1u))] = e;
                        nl += __popc(m);
                    }
                    SG.sync();
                    ncur = nl;
                    cur = 1;
                    have = true;
                }
            }
        }
        if (!brute && !have) {
            // frontier entries are packed node coordinates u | v << 16
            const int tw = g.lev_w[top];
            for (int q = lane; q < ncur; q += LPC) S.fr[0][q] = (q % tw) | ((q / tw) << 16);
            SG.sync();
        }
        for (int L = top; L >= 0 && !brute && !have; L--) {
            int nnext = 0;
            const int off = g.lev_off[L], W = g.lev_w[L];
            PSTAT_ADD(7, ncur);
            for (int base = 0; base < ncur; base += LPC) {
                const int q = (base + lane < ncur) ? S.fr[cur][base + lane] : -1;
                bool keep = false;
                int u = 0, v = 0;
                if (q >= 0) {
                    u = q & 0xffff;
                    v = q >> 16;
                    const bool inwin = L == 0 && abs(u - bu) <= win && abs(v - bv) <= win;
                    keep = !inwin && !node_excluded(S, nv0, g, off + u + v * W, si, wi);
                }
                if (L == 0) {
                    const unsigned m = SG.ballot(keep);
                    const int cnt = __popc(m);
                    if (nnext + cnt > COT_FRMAX) { brute = true; break; }
                    if (keep) S.fr[1 - cur][nnext + __popc(m & ((1u << lane) - 1u))] = u + v * W;
                    nnext += cnt;
                } else {
                    const int cw = g.lev_w[L - 1], ch = g.lev_h[L - 1];
                    int chc = 0;
                    if (keep) {
                        chc = (2 * u + 1 < cw ? 2 : 1) * (2 * v + 1 < ch ? 2 : 1);
                    }
                    const int inc = SG.incl_scan(chc);
                    const int cnt = SG.shfl(inc, LPC - 1);
                    if (nnext + cnt > COT_FRMAX) { brute = true; break; }
                    int pos = nnext + inc - chc;
                    if (keep) {
                        for (int bb = 0; bb < 2; bb++)
                            for (int aa = 0; aa < 2; aa++)
                                if (2 * u + aa < cw && 2 * v + bb < ch) S.fr[1 - cur][pos++] = (2 * u + aa) | ((2 * v + bb) << 16);
                    }
                    nnext += cnt;
                }
            }
            SG.sync();
            if (brute) break;
            cur = 1 - cur;
            ncur = nnext;
        }
        if constexpr (LPC == 32) {
            // many surviving leaves: applied in bucket order, their sites
            // would cost a real clip nearly each; k_cells_heavy tests them
            // with a block and clips the deepest first
            if (!brute && ncur > COT_DEFER_LEAVES && a.wlist != nullptr) {
                if (lane < P.nv) {
                    a.rbuf[(size_t)i * COT_RCAP + lane] = make_double2(P.x, P.y);
                    a.lbuf[(size_t)i * COT_RCAP + lane] = P.l;
                }
                if (lane == 0) {
                    a.cstate[i] = P.nv;
                    a.wlist[atomicAdd(a.ovf_count + 11, 1)] = i;
                }
                P.nv = COT_DEFERRED;
                return P;
            }
        }
        if (!brute && ncur > 0) {
            // sites of every surviving leaf, LPC leaves at a time
            PSTAT_ADD(5, ncur);
            for (int lb = 0; lb < ncur && ok && P.nv > 0; lb += LPC) {
                int st = 0, cnt = 0;
                if (lb + lane < ncur) {
                    const int b = S.fr[cur][lb + lane];
                    st = g.bstart[b];
                    cnt = g.bstart[b + 1] - st;
                }
                const int inc = SG.incl_scan(cnt);
                P = apply_ranges<LPC>(P, st, cnt, inc, i, g.xy, si, wi, wt, lane, S, false);
                ok = P.nv >= 0;
            }
        }
    }
    if (!brute || !ok || P.nv <= 0) break;
    if (pass == COT_DEFER_PASS || pass == COT_REFINE_PASSES) {
        if constexpr (LPC == 32) {
            // on the two-kernel path the refined ring goes to the ring
            // buffer and k_cells_heavy finishes the cell with a block
            if (a.wlist != nullptr) {
                if (lane < P.nv) {
                    a.rbuf[(size_t)i * COT_RCAP + lane] = make_double2(P.x, P.y);
                    a.lbuf[(size_t)i * COT_RCAP + lane] = P.l;
                }
                if (lane == 0) {
                    a.cstate[i] = P.nv;
                    a.wlist[atomicAdd(a.ovf_count + 11, 1)] = i;
                }
                P.nv = COT_DEFERRED;
                return P;
            }
        }
        if (pass == COT_REFINE_PASSES) break;
    }
    P = refine_by_vertices<LPC>(g, wt, i, si, wi, P, S, COT_REFINE_ROUNDS);
    ok = P.nv >= 0;
    brute = false;
    SG.sync();
    }
    PSTAT_ADD(9, brute ? 1 : 0);
    if (ok && brute && P.nv > 0) P = scan_all_buckets<LPC>(g, wt, i, si, wi, P, S, bu, bv, win);
    PSTAT_CLOCK(t2);
    PSTAT_ADD(1, t2 - t1);
    return P;
}

// Phase 3: overflow hand-off, or the ring's integrals (EXACT) / the ring
// buffer (solve path), the next evaluation's cache and the per-cell outputs.
template <bool EXACT, int LPC, bool KEEP = false>
__device__ __forceinline__ void cell_finish(const CotGeo &g, const CellsArgs &a, const int i, const double2 si,
                                            const double wi, RegPoly P, FastScratch &S, int *olist, int *ocount)
{
    const Seg<LPC> SG;
    const int lane = SG.sl;
    if (P.nv < 0) {
        // ring above LPC vertices: hand the cell to the next pass
        if (lane == 0) {
            const int slot = atomicAdd(ocount, 1);
            olist[slot] = i;
            a.nv[i] = LPC + 1;
        }
        SG.sync();
        return;
    }
    // ---- 3. integrate the density over the cell --------------------------
    PSTAT_CLOCK(t2);
    const int nv = P.nv;
    if (nv >= 3) {
        // canonical ring start (smallest edge generator) so the integration
        // sums in the same order whatever order the clips came in
        const int key = lane < nv ? P.l : 0x7fffffff;
        const int mn = SG.imin(key);
        const int r = __ffs(SG.ballot(key == mn)) - 1;
        int src = lane + r;
        if (src >= nv) src -= nv;
        P.x = SG.shfl(P.x, src);
        P.y = SG.shfl(P.y, src);
        P.a = SG.shfl(P.a, src);
        P.b = SG.shfl(P.b, src);
        P.c = SG.shfl(P.c, src);
        P.l = SG.shfl(P.l, src);
    }
    if (lane < nv) { S.X[lane] = P.x; S.Y[lane] = P.y; }
    SG.sync();
    CellAcc acc = {0.0, 0.0, 0.0, 0.0, 0.0};
    // the solve's path only builds the ring here: k_integrate sums over it
    // from the ring buffer (two kernels with smaller instruction footprints
    // than one fused kernel)
    constexpr bool split = !EXACT;
    if (nv >= 3) {
        if constexpr (EXACT)
            acc = integrate_cell(S, nv, splat_geo(g, a, S, nv, i, lane), si, lane);
        else if (lane < nv)
            a.rbuf[(size_t)i * COT_RCAP + lane] = make_double2(P.x, P.y);
        if constexpr (!EXACT && LPC == 32) {
            // a cell whose pixel box is large goes on the heavy list: the
            // integration kernel starts those cells first, so that they run
            // beside the many small ones instead of after them
            if (a.hlist != nullptr) {
                const double ox = si.x - g.pd[0], oy = si.y - g.pd[2];
                const int cx = lane < nv ? (int)floor((ox + P.x) * g.ixs) : INT_MAX;
                const int cy = lane < nv ? (int)floor((oy + P.y) * g.iys) : INT_MAX;
                const int c0 = __reduce_min_sync(FULLMASK, cx), r0 = __reduce_min_sync(FULLMASK, cy);
                const int c1 = __reduce_max_sync(FULLMASK, lane < nv ? cx : INT_MIN);
                const int r1 = __reduce_max_sync(FULLMASK, lane < nv ? cy : INT_MIN);
                const double box = (double)(c1 - c0 + 1) * (double)(r1 - r0 + 1);
                if (box > (double)COT_HEAVY_PIX && lane == 0) {
                    // the largest boxes are shared by COT_SPLIT warps (while
                    // the split list has room), the others start first whole
                    int slot = a.hsplit_cap;
                    if (box > (double)COT_SPLIT_PIX && a.hsplit != nullptr) slot = atomicAdd(a.ovf_count + 13, 1);
                    if (slot < a.hsplit_cap) a.hsplit[slot] = i;
                    else a.hlist[atomicAdd(a.ovf_count + 10, 1)] = i;
                    a.cstate[i] = CST_HEAVY;
                }
            }
        }
        // the Newton solve's Jacobian reads the final ring's generators
        if constexpr (KEEP) {
            if (lane < nv) a.lbuf[(size_t)i * COT_RCAP + lane] = P.l;
        }
    }
    PSTAT_CLOCK(t3);
    PSTAT_ADD(2, t3 - t2);
    PSTAT_ADD(8, 1);
    PSTAT_ADD(11, nv);
    double pcx = 0.0, pcy = 0.0;
    if constexpr (EXACT) {
        if (a.cen != nullptr && nv >= 3 && (!a.weighted || acc.Mt == 0.0)) poly_centroid(S, nv, lane, pcx, pcy);
    }
    if (a.ring_xy != nullptr && lane < nv && lane < a.ring_cap) {
        a.ring_xy[2 * ((size_t)i * a.ring_cap + lane)] = si.x + P.x;
        a.ring_xy[2 * ((size_t)i * a.ring_cap + lane) + 1] = si.y + P.y;
        a.ring_lab[(size_t)i * a.ring_cap + lane] = P.l;
    }
    if constexpr (EXACT) {
        if (a.solid != nullptr && lane == 0) a.solid[i] = nv >= 3 ? solid_angle_of(S, nv, si, a.solid_z, a.solid_light) : 0.0;
    }
    if (a.nbn != nullptr) {
        // this evaluation seeds the next: a ring of up to COT_NBC edges
        // in order (domain sides included); else its sites, or for a
        // hidden cell the site that emptied its ring and that ring's sites
        if (nv >= 3 && nv <= COT_NBC) {
            if (lane < nv) a.nbc[(size_t)i * COT_NBC + lane] = P.l;
            if (lane == 0) a.nbn[i] = nv;
        } else {
            int lab = lane < nv ? P.l : -1;
            if (nv == 0) {
                SG.sync();
                const int kn = S.kn;
                lab = -1;
                if (kn >= 0) lab = lane == 0 ? S.kill : (lane - 1 < kn ? S.KL[lane - 1] : -1);
            }
            const bool isn = lab >= 0;
            const unsigned m = SG.ballot(isn);
            const int pos = __popc(m & ((1u << lane) - 1u));
            if (isn && pos < COT_NBC) a.nbc[(size_t)i * COT_NBC + pos] = lab;
            const int cnt = min(__popc(m), COT_NBC);
            if (lane == 0) a.nbn[i] = cnt == 0 ? 0 : (nv == 0 ? -(COT_NB_HIDDEN + cnt) : -cnt);
        }
    }
    if (lane == 0) {
        if (!split) {
            a.mu[i] = acc.mu;
            // f_i = -w_i nu_i - sum_pix rho (int |x-s_i|^2 - w_i area)   (basic_function.cuh:875-941);
            // stored without its -w_i nu_i term, which the reduction adds, so
            // that nu may change after the cells are built
            a.fc[i] = -(acc.S - wi * acc.mu);
        }
        a.nv[i] = nv;
        if (a.cen != nullptr) {
            const bool ex = nv >= 3;
            a.exist[i] = ex ? 1 : 0;
            double cx = si.x, cy = si.y;
            if (ex) {
                if (a.weighted && acc.Mt != 0.0) {
                    cx = si.x + acc.Mx / acc.Mt;
                    cy = si.y + acc.My / acc.Mt;
                } else {
                    cx = si.x + pcx;
                    cy = si.y + pcy;
                }
            }
            a.cen[2 * i] = cx;
            a.cen[2 * i + 1] = cy;
        }
    }
}

template <bool EXACT, int LPC>
__device__ __forceinline__ void fast_cell(const CotGeo &g, const CellsArgs &a, const int i, FastScratch &S,
                                          int *olist, int *ocount)
{
    const double2 si = g.xy[i];
    const double wi = a.wt[i];
    bool cached = false;
    RegPoly P = cell_first<LPC>(g, a, i, si, wi, S, cached);
    P = cell_walk<LPC>(g, a, i, si, wi, P, cached, S);
    cell_finish<EXACT, LPC>(g, a, i, si, wi, P, S, olist, ocount);
}

// The persistent cell kernel: each warp fetches 32 / LPC cells at a time
// (one per segment) from a counter, so that large cells leave no tail and the
// segments of a warp run the same phases together.  pass 0: every cell,
// rings above LPC vertices into ovf_list; pass 1: the cells of ovf_list,
// rings above LPC into ovf_list2.
template <int MINB, bool EXACT, int LPC>
__global__ void __launch_bounds__(128, MINB) k_cells_fast(const __grid_constant__ CotGeo g, CellsArgs a, int pass)
{
    static_assert(!EXACT || LPC == 32, "the exact path works a whole warp per cell");
    constexpr int CPW = 32 / LPC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastScratch &S = reinterpret_cast<FastScratch *>(smem_raw)[threadIdx.x / LPC];
    PSTAT_INIT();
    const int total = pass == 0 ? g.n : a.ovf_count[0];
    int *fetch = a.ovf_count + (pass == 0 ? 1 : 4);
    int *olist = pass == 0 ? a.ovf_list : a.ovf_list2;
    int *ocount = a.ovf_count + (pass == 0 ? 0 : 3);
    while (true) {
        int base = 0;
        if ((threadIdx.x & 31) == 0) base = atomicAdd(fetch, CPW);
        base = __shfl_sync(FULLMASK, base, 0);
        if (base >= total) break;
        const int slot = base + (int)(threadIdx.x & 31) / LPC;
        if (slot < total) fast_cell<EXACT, LPC>(g, a, pass == 0 ? slot : a.ovf_list[slot], S, olist, ocount);
        __syncwarp();
    }
    PSTAT_FLUSH();
}

// The solve's path in two launches with smaller instruction footprints than
// k_cells_fast<.., false, 32>, and the same results: k_cells_first runs
// phase 1 for every cell and leaves each ring (vertices, edge generators) in
// the ring buffers; k_cells_walk takes the rings back, rebuilds their edge
// lines from the generators (the same explicitly rounded site_line /
// side_line as the clips used, so the same bits) and runs phases 2 and 3.
// Cells that phase 1 empties or overflows are finished by k_cells_first
// (cstate < 0); otherwise cstate = nv, plus CST_CACHED for a cached cell.
#define CST_CACHED 0x100
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_cells_first(CotGeo g, CellsArgs a)
{
    constexpr int LPC = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastScratch &S = reinterpret_cast<FastScratch *>(smem_raw)[threadIdx.x >> 5];
    PSTAT_INIT();
    const int lane = threadIdx.x & 31;
    int *fetch = a.ovf_count + 1;
    while (true) {
        int i = 0;
        if (lane == 0) i = atomicAdd(fetch, 1);
        i = __shfl_sync(FULLMASK, i, 0);
        if (i >= g.n) break;
        const double2 si = g.xy[i];
        const double wi = a.wt[i];
        bool cached = false;
        const RegPoly P = cell_first<LPC>(g, a, i, si, wi, S, cached);
        if (P.nv <= 0) {
            // emptied (hidden cell) or outgrew 32 vertices: finished here
            cell_finish<false, LPC>(g, a, i, si, wi, P, S, a.ovf_list, a.ovf_count);
            if (lane == 0) a.cstate[i] = -1;
        } else {
            if (lane < P.nv) {
                a.rbuf[(size_t)i * COT_RCAP + lane] = make_double2(P.x, P.y);
                a.lbuf[(size_t)i * COT_RCAP + lane] = P.l;
            }
            if (lane == 0) a.cstate[i] = P.nv | (cached ? CST_CACHED : 0);
        }
        __syncwarp();
    }
    PSTAT_FLUSH();
}

// One warp per bucket, between k_cells_first and k_cells_walk: the leaf
// buckets whose sites could cut the ring of any cell of the bucket.  The
// rings phase 1 left lie in a box; with i0 the bucket's first site and
// Delta = max over the rings' vertices of P_i0 - P_i (P_i0 - P_i is affine on
// a ring, so its vertices bound it), P_i0 - Delta <= P_i on ring i.  A node
// whose bound stays below P_i0 - Delta - margin at the box's four corners
// (node_excluded with w_i0 - 2 Delta) therefore cuts no ring of the bucket.
// The surviving leaves are listed in walk order (COT_BLEAF at most; -1 when
// more), so that k_cells_walk tests only them, in one or two rounds a cell.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_bucket_walk(CotGeo g, CellsArgs a)
{
    constexpr int LPC = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastScratch &S = reinterpret_cast<FastScratch *>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int nb = g.bx * g.by;
    int *fetch = a.ovf_count + 9;
    int top = g.nlev - 1;
    while (top > 0 && g.lev_w[top - 1] * g.lev_h[top - 1] <= 32) top--;
    const int ntop = g.lev_w[top] * g.lev_h[top];
    while (true) {
        int b = 0;
        if (lane == 0) b = atomicAdd(fetch, 1);
        b = __shfl_sync(FULLMASK, b, 0);
        if (b >= nb) break;
        const int s0 = g.bstart[b], s1 = g.bstart[b + 1];
        const double2 so = s1 > s0 ? g.xy[s0] : make_double2(0.0, 0.0);
        const double wo = s1 > s0 ? a.wt[s0] : 0.0;
        double lx = INFINITY, hx = -INFINITY, ly = INFINITY, hy = -INFINITY, dl = 0.0;
        for (int i = s0 + lane; i < s1; i += 32) {
            const int st = a.cstate[i];
            if (st < 0) continue;
            const int nv = st & 0xff;
            const double2 si = g.xy[i];
            const double ex = si.x - so.x, ey = si.y - so.y;
            // P_i0 - P_i at s_i + v: (w_i0 - w_i)/2 - |e|^2/2 - v.e, e = s_i - s_i0
            const double k0 = 0.5 * (wo - a.wt[i]) - 0.5 * __fma_rn(ex, ex, ey * ey);
            for (int k = 0; k < nv; k++) {
                const double2 v = a.rbuf[(size_t)i * COT_RCAP + k];
                const double X = v.x + ex, Y = v.y + ey;
                lx = fmin(lx, X);
                hx = fmax(hx, X);
                ly = fmin(ly, Y);
                hy = fmax(hy, Y);
                dl = fmax(dl, k0 - __fma_rn(v.x, ex, v.y * ey));
            }
        }
        lx = warp_min(lx);
        hx = warp_max(hx);
        ly = warp_min(ly);
        hy = warp_max(hy);
        dl = warp_max(dl);
        if (!(lx <= hx)) {
            // no ring of the bucket is walked
            if (lane == 0) a.bcnt[b] = 0;
            continue;
        }
        if (lane < 4) {
            S.X[lane] = (lane == 1 || lane == 2) ? hx : lx;
            S.Y[lane] = lane >= 2 ? hy : ly;
        }
        for (int q = lane; q < ntop; q += 32) S.fr[0][q] = (q % g.lev_w[top]) | ((q / g.lev_w[top]) << 16);
        __syncwarp();
        const double wq = wo - 2.0 * dl;
        int cur = 0, ncur = ntop;
        bool over = ntop > COT_FRMAX;
        for (int L = top; L >= 0 && !over; L--) {
            int nnext = 0;
            const int off = g.lev_off[L], W = g.lev_w[L];
            for (int base = 0; base < ncur; base += 32) {
                const int q = (base + lane < ncur) ? S.fr[cur][base + lane] : -1;
                bool keep = false;
                int u = 0, v = 0;
                if (q >= 0) {
                    u = q & 0xffff;
                    v = q >> 16;
                    keep = !node_excluded(S, 4, g, off + u + v * W, so, wq);
                }
                if (L == 0) {
                    const unsigned m = __ballot_sync(FULLMASK, keep);
                    const int cnt = __popc(m);
                    if (nnext + cnt > COT_BLEAF) { over = true; break; }
                    if (keep) S.fr[1 - cur][nnext + __popc(m & ((1u << lane) - 1u))] = u + v * W;
                    nnext += cnt;
                } else {
                    const int cw = g.lev_w[L - 1], ch = g.lev_h[L - 1];
                    const int chc = keep ? (2 * u + 1 < cw ? 2 : 1) * (2 * v + 1 < ch ? 2 : 1) : 0;
                    const int inc = warp_incl_scan(chc, lane);
                    const int cnt = __shfl_sync(FULLMASK, inc, 31);
                    if (nnext + cnt > COT_FRMAX) { over = true; break; }
                    int pos = nnext + inc - chc;
                    if (keep) {
                        for (int bb = 0; bb < 2; bb++)
                            for (int aa = 0; aa < 2; aa++)
                                if (2 * u + aa < cw && 2 * v + bb < ch) S.fr[1 - cur][pos++] = (2 * u + aa) | ((2 * v + bb) << 16);
                    }
                    nnext += cnt;
                }
            }
            __syncwarp();
            if (over) break;
            cur = 1 - cur;
            ncur = nnext;
        }
        if (!over)
            for (int k = lane; k < ncur; k += 32) a.blist[(size_t)b * COT_BLEAF + k] = S.fr[cur][k];
        if (lane == 0) a.bcnt[b] = over ? -1 : ncur;
        __syncwarp();
    }
}

// KEEP: leave the final ring's generators in lbuf (the Newton solve's
// Jacobian reads them); a separate instance keeps the solve's path as it is.
template <int MINB, bool KEEP>
__global__ void __launch_bounds__(128, MINB) k_cells_walk(const __grid_constant__ CotGeo g, CellsArgs a)
{
    constexpr int LPC = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastScratch &S = reinterpret_cast<FastScratch *>(smem_raw)[threadIdx.x >> 5];
    PSTAT_INIT();
    const int lane = threadIdx.x & 31;
    int *fetch = a.ovf_count + 8;
    while (true) {
        int i = 0;
        if (lane == 0) i = atomicAdd(fetch, 1);
        i = __shfl_sync(FULLMASK, i, 0);
        if (i >= g.n) break;
        const int st = a.cstate[i];
        if (st < 0) continue;
        const double2 si = g.xy[i];
        const double wi = a.wt[i];
        RegPoly P;
        P.nv = st & 0xff;
        P.x = P.y = P.a = P.b = P.c = 0.0;
        P.l = 0;
        if (lane < P.nv) {
            const double2 v = a.rbuf[(size_t)i * COT_RCAP + lane];
            P.x = v.x;
            P.y = v.y;
            P.l = a.lbuf[(size_t)i * COT_RCAP + lane];
            if (P.l >= 0) {
                double key;
                site_line(g.xy[P.l], si, a.wt[P.l], wi, P.a, P.b, P.c, key);
            } else {
                const double4 box = make_double4(g.pd[0] - si.x, g.pd[1] - si.x, g.pd[2] - si.y, g.pd[3] - si.y);
                side_line(-P.l - 1, box, P.a, P.b, P.c);
            }
        }
        if (lane == 0) S.kn = -1;
        __syncwarp();
        P = cell_walk<LPC>(g, a, i, si, wi, P, (st & CST_CACHED) != 0, S);
        if (P.nv != COT_DEFERRED) cell_finish<false, LPC, KEEP>(g, a, i, si, wi, P, S, a.ovf_list, a.ovf_count);
        __syncwarp();
    }
    PSTAT_FLUSH();
}

// The cells whose certificate walk still overflowed its frontier after the
// ring refinements (listed by k_cells_walk, the refined ring in the ring
// buffer), one block of HEAVY_WARPS warps a cell.  Every warp tests its share
// of the buckets against the ring, then the sites of the buckets that can cut
// it, lanes over sites, and lists the sites that cut with their depth (how
// far the ring reaches past the site's line).  Then, round by round, warp 0
// applies the 32 deepest listed sites, deepest first, and the warps drop the
// listed sites that no longer cut the smaller ring.  A site that cuts the
// final ring cuts every ring that contains it, so none is missed, and the
// cell is the one any other clip order gives; the order is fixed (depth, then
// index), so a run repeats bit for bit.  Lists that outgrow their room are
// cut short: the rounds run on what was found, and the search starts again
// (HEAVY_RETRY times, then warp 0 scans every bucket).
#define HEAVY_WARPS 8
#define HEAVY_KCAP 256  // buckets that can cut, per warp
#define HEAVY_CCAP 512  // sites that cut, per warp
#define HEAVY_RETRY 4
struct HeavyShared {
    int kept[HEAVY_WARPS][HEAVY_KCAP];
    int cut[HEAVY_WARPS][HEAVY_CCAP];
    float dep[HEAVY_WARPS][HEAVY_CCAP];
    float tdep[HEAVY_WARPS][32];
    int tj[HEAVY_WARPS][32];
    int ncut[HEAVY_WARPS], over[HEAVY_WARPS];
    int cell, nv;
};
static_assert(sizeof(FastScratch) + sizeof(HeavyShared) <= 48 * 1024, "k_cells_heavy fits the default shared memory");

// Depth of site j's cut into the ring snapshot (S.X, S.Y, S.L, nv vertices):
// the largest distance of a vertex past the site's line, or -1 when the site
// does not cut (apply_chunk's test).
__device__ __forceinline__ float site_depth(const CotGeo &g, const double *__restrict__ wt, int j, double2 si,
                                            double wi, const FastScratch &S, int nv)
{
    double al, bl, cl, key;
    site_line(g.xy[j], si, wt[j], wi, al, bl, cl, key);
    double dm = 0.0;
    for (int q = 0; q < nv; q++) {
        if (S.L[q] == j) return -1.0f;
        dm = fmax(dm, side(al, bl, cl, S.X[q], S.Y[q]));
    }
    if (!(dm > 0.0)) return -1.0f;
    return (float)(dm / sqrt(key));
}

// (depth, index) order: deeper first, then the lower index.
__device__ __forceinline__ bool deeper(float d1, int j1, float d2, int j2)
{
    return d1 > d2 || (d1 == d2 && j1 < j2);
}

// Bitonic step helpers over a warp holding one (depth, index) pair a lane.
__device__ __forceinline__ void cmpx(float &d, int &j, int mask, bool keep_deeper)
{
    const float od = __shfl_xor_sync(FULLMASK, d, mask);
    const int oj = __shfl_xor_sync(FULLMASK, j, mask);
    const bool od_first = deeper(od, oj, d, j);
    if (od_first == keep_deeper) { d = od; j = oj; }
}

// Sorts the warp's pairs, deepest at lane 0.
__device__ __forceinline__ void warp_sort_deep(float &d, int &j, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int m = k >> 1; m > 0; m >>= 1) {
            const bool lower = (lane & m) == 0;
            const bool asc = (lane & k) == 0;  // this run sorts deepest first
            cmpx(d, j, m, lower == asc);
        }
}

// top (sorted, deepest at lane 0) := the 32 deepest of top and the sorted c.
__device__ __forceinline__ void warp_merge_top(float &td, int &tj, float cd, int cj, int lane)
{
    // c reversed against top is a bitonic sequence; the lane-wise deeper half
    // holds the 32 deepest, sorted again by a bitonic clean-up
    const float rd = __shfl_sync(FULLMASK, cd, 31 - lane);
    const int rj = __shfl_sync(FULLMASK, cj, 31 - lane);
    if (deeper(rd, rj, td, tj)) { td = rd; tj = rj; }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) cmpx(td, tj, m, (lane & m) == 0);
}

template <bool KEEP>
__global__ void __launch_bounds__(32 * HEAVY_WARPS, 2) k_cells_heavy(const __grid_constant__ CotGeo g, CellsArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastScratch &S = *reinterpret_cast<FastScratch *>(smem_raw);
    HeavyShared &H = *reinterpret_cast<HeavyShared *>(smem_raw + sizeof(FastScratch));
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int total = a.ovf_count[11];
    const int nb = g.bx * g.by;
    while (true) {
        if (threadIdx.x == 0) H.cell = atomicAdd(a.ovf_count + 12, 1);
        __syncthreads();
        const int f = H.cell;
        if (f >= total) break;
        const int i = a.wlist[f];
        const double2 si = g.xy[i];
        const double wi = a.wt[i];
        RegPoly P;
        if (wp == 0) {
            P.nv = a.cstate[i] & 0xff;
            P.x = P.y = P.a = P.b = P.c = 0.0;
            P.l = 0;
            if (lane < P.nv) {
                const double2 v = a.rbuf[(size_t)i * COT_RCAP + lane];
                P.x = v.x;
                P.y = v.y;
                P.l = a.lbuf[(size_t)i * COT_RCAP + lane];
                if (P.l >= 0) {
                    double key;
                    site_line(g.xy[P.l], si, a.wt[P.l], wi, P.a, P.b, P.c, key);
                } else {
                    const double4 box = make_double4(g.pd[0] - si.x, g.pd[1] - si.x, g.pd[2] - si.y, g.pd[3] - si.y);
                    side_line(-P.l - 1, box, P.a, P.b, P.c);
                }
                S.X[lane] = P.x;
                S.Y[lane] = P.y;
                S.L[lane] = P.l;
            }
            if (lane == 0) {
                S.kn = -1;
                H.nv = P.nv;
            }
        }
        __syncthreads();
        bool over = false;
        for (int attempt = 0;; attempt++) {
            // the sites that cut the ring, per warp in a fixed order, with the
            // warp's 32 deepest
            int nv = H.nv;
            if (nv > 0) {
                int nk = 0, nc = 0;
                bool ov = false;
                for (int base = wp * 32; base < nb; base += 32 * HEAVY_WARPS) {
                    const int b = base + lane;
                    const bool keep = b < nb && !node_excluded(S, nv, g, b, si, wi);
                    const unsigned m = __ballot_sync(FULLMASK, keep);
                    if (nk + __popc(m) > HEAVY_KCAP) { ov = true; break; }
                    if (keep) H.kept[wp][nk + __popc(m & lt)] = b;
                    nk += __popc(m);
                }
                __syncwarp();
                float td = -1.0f;
                int tj = INT_MAX;
                for (int k = 0; k < nk; k++) {
                    const int b = H.kept[wp][k];
                    const int s1 = g.bstart[b + 1];
                    bool full = false;
                    for (int j0 = g.bstart[b]; j0 < s1; j0 += 32) {
                        const int j = j0 + lane;
                        const float dj = (j < s1 && j != i) ? site_depth(g, a.wt, j, si, wi, S, nv) : -1.0f;
                        const bool cut = dj > 0.0f;
                        const unsigned m = __ballot_sync(FULLMASK, cut);
                        if (nc + __popc(m) > HEAVY_CCAP) { full = true; break; }
                        if (cut) {
                            H.cut[wp][nc + __popc(m & lt)] = j;
                            H.dep[wp][nc + __popc(m & lt)] = dj;
                        }
                        nc += __popc(m);
                        if (m != 0u) {
                            float cd = cut ? dj : -1.0f;
                            int cj = cut ? j : INT_MAX;
                            warp_sort_deep(cd, cj, lane);
                            warp_merge_top(td, tj, cd, cj, lane);
                        }
                    }
                    if (full) { ov = true; break; }
                }
                H.tdep[wp][lane] = td;
                H.tj[wp][lane] = tj;
                if (lane == 0) {
                    H.ncut[wp] = nc;
                    H.over[wp] = ov ? 1 : 0;
                }
            }
            __syncthreads();
            over = false;
            for (int q = 0; q < HEAVY_WARPS; q++) over = over || (nv > 0 && H.over[q] != 0);
            // rounds: the 32 deepest first; then drop what no longer cuts
            while (nv > 0) {
                if (wp == 0) {
                    float td = H.tdep[0][lane];
                    int tj = H.tj[0][lane];
                    for (int q = 1; q < HEAVY_WARPS; q++) warp_merge_top(td, tj, H.tdep[q][lane], H.tj[q][lane], lane);
                    const int jl = td > 0.0f ? tj : -1;
                    if (__ballot_sync(FULLMASK, jl >= 0) != 0u) {
                        P = apply_chunk<32>(P, jl, g.xy, si, wi, a.wt, lane, S, false);
                        if (lane < P.nv) { S.X[lane] = P.x; S.Y[lane] = P.y; S.L[lane] = P.l; }
                        if (lane == 0) H.nv = P.nv;
                    } else if (lane == 0) {
                        H.nv = -100 - P.nv;  // nothing left to apply (decoded below)
                    }
                }
                __syncthreads();
                nv = H.nv;
                if (nv <= -100) {
                    nv = -100 - nv;
                    __syncthreads();
                    if (threadIdx.x == 0) H.nv = nv;
                    __syncthreads();
                    break;
                }
                if (nv <= 0) break;
                const int n0 = H.ncut[wp];
                int nk = 0;
                float td = -1.0f;
                int tj = INT_MAX;
                for (int base = 0; base < n0; base += 32) {
                    const int k = base + lane;
                    const int j = k < n0 ? H.cut[wp][k] : -1;
                    const float dj = j >= 0 ? site_depth(g, a.wt, j, si, wi, S, nv) : -1.0f;
                    const bool cut = dj > 0.0f;
                    const unsigned m = __ballot_sync(FULLMASK, cut);
                    if (cut) {
                        H.cut[wp][nk + __popc(m & lt)] = j;
                        H.dep[wp][nk + __popc(m & lt)] = dj;
                    }
                    nk += __popc(m);
                    if (m != 0u) {
                        float cd = cut ? dj : -1.0f;
                        int cj = cut ? j : INT_MAX;
                        warp_sort_deep(cd, cj, lane);
                        warp_merge_top(td, tj, cd, cj, lane);
                    }
                    __syncwarp();
                }
                H.tdep[wp][lane] = td;
                H.tj[wp][lane] = tj;
                if (lane == 0) H.ncut[wp] = nk;
                __syncthreads();
            }
            if (nv <= 0 || !over || attempt == HEAVY_RETRY) break;
        }
        if (H.nv > 0 && over && wp == 0) P = scan_all_buckets<32>(g, a.wt, i, si, wi, P, S, 0, 0, -1);
        if (wp == 0) cell_finish<false, 32, KEEP>(g, a, i, si, wi, P, S, a.ovf_list, a.ovf_count);
        __syncthreads();
    }
}

// One part of a split cell's integration, out of line so that the rare path
// leaves the integration kernel's registers to the common one.
__device__ __noinline__ void integrate_part(FastScratch &S, int nv, const PixGeo pg, double2 si, int lane, int part,
                                            double *raw)
{
    integrate_fast<32, FastScratch, true>(S, nv, pg, si, lane, part, COT_SPLIT, raw);
}

// The masses and objective terms of the cells whose rings k_cells_fast left
// in the ring buffer: one warp per cell, fetched from a counter, the same
// edge-walk integration as the fused path (so the same sums).  Cells above
// COT_RCAP vertices are integrated by the large-ring pass instead.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_integrate(CotGeo g, CellsArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastScratch &S = reinterpret_cast<FastScratch *>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    int *fetch = a.ovf_count + 6;
    // the parts of the split cells first, then the heavy list, then every
    // other cell in order
    const int nh = a.hlist != nullptr ? a.ovf_count[10] : 0;
    const int np = a.hsplit != nullptr ? min(a.ovf_count[13], a.hsplit_cap) * COT_SPLIT : 0;
    while (true) {
        int f = 0;
        if (lane == 0) f = atomicAdd(fetch, 1);
        f = __shfl_sync(FULLMASK, f, 0);
        if (f >= g.n + nh + np) break;
        if (f < np) {
            // one part of a split cell: its raw sums to the slot, and the
            // part that finishes last adds the parts in order
            const int slot = f / COT_SPLIT, part = f % COT_SPLIT;
            const int i = a.hsplit[slot];
            const int nv = a.nv[i];
            if (lane < nv) {
                const double2 v = a.rbuf[(size_t)i * COT_RCAP + lane];
                S.X[lane] = v.x;
                S.Y[lane] = v.y;
            }
            __syncwarp();
            double raw[6];
            integrate_part(S, nv, pix_geo(g), g.xy[i], lane, part, raw);
            if (lane == 0) {
                double *pp = a.hpart + ((size_t)slot * COT_SPLIT + part) * 4;
                pp[0] = raw[0];
                pp[1] = raw[1];
                pp[2] = raw[2];
                pp[3] = raw[3];
                __threadfence();
                if (atomicAdd(a.hticket + slot, 1u) == COT_SPLIT - 1) {
                    __threadfence();
                    const volatile double *q = a.hpart + (size_t)slot * COT_SPLIT * 4;
                    double sA = q[0], sIa = q[1], sIb = q[2], sI2 = q[3];
                    for (int k = 1; k < COT_SPLIT; k++) {
                        sA += q[4 * k];
                        sIa += q[4 * k + 1];
                        sIb += q[4 * k + 2];
                        sI2 += q[4 * k + 3];
                    }
                    const double ox = raw[4], oy = raw[5];
                    const double Sv = sI2 + 2.0 * (ox * sIa + oy * sIb) + (ox * ox + oy * oy) * sA;
                    a.mu[i] = sA;
                    a.fc[i] = -(Sv - a.wt[i] * sA);
                    a.hticket[slot] = 0u;
                }
            }
            __syncwarp();
            continue;
        }
        f -= np;
        int i;
        if (f < nh) {
            i = a.hlist[f];
        } else {
            i = f - nh;
            if ((nh > 0 || np > 0) && a.cstate[i] == CST_HEAVY) continue;
        }
        const int nv = a.nv[i];
        if (nv > COT_RCAP) continue;
        double mu = 0.0, fcv = 0.0;
        if (nv >= 3) {
            if (lane < nv) {
                const double2 v = a.rbuf[(size_t)i * COT_RCAP + lane];
                S.X[lane] = v.x;
                S.Y[lane] = v.y;
            }
            __syncwarp();
            const CellAcc acc = integrate_fast<32>(S, nv, pix_geo(g), g.xy[i], lane);
            mu = acc.mu;
            fcv = -(acc.S - a.wt[i] * acc.mu);
        }
        if (lane == 0) {
            a.mu[i] = mu;
            a.fc[i] = fcv;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// the cell kernel
// ---------------------------------------------------------------------------
// mode 0: every cell; mode 1: the cells listed in ovf_list; mode 2: those in
// ovf_list2.  Warps fetch cells dynamically from a counter so that large cells
// do not leave a tail.
template <int MAXV, int MINB>
__global__ void __launch_bounds__(128, MINB) k_cells(CotGeo g, CellsArgs a, int mode)
{
    PSTAT_LPC32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    WarpPoly<MAXV> &P = reinterpret_cast<WarpPoly<MAXV> *>(smem_raw)[wib];
    const double *__restrict__ wt = a.wt;
    PSTAT_INIT();

    // counters: [0] ovf_list size, [1] pass-0 fetch, [2] mode-1 fetch,
    // [3] ovf_list2 size, [4] second-pass fetch, [5] mode-2 fetch
    const int total = (mode == 0) ? g.n : a.ovf_count[mode == 1 ? 0 : 3];
    int *fetch = a.ovf_count + (mode == 0 ? 1 : (mode == 1 ? 2 : 5));
    const int *list = mode == 1 ? a.ovf_list : a.ovf_list2;
    while (true) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(fetch, 1);
        idx = __shfl_sync(FULLMASK, idx, 0);
        if (idx >= total) break;
        const int i = (mode == 0) ? idx : list[idx];
        const double2 si = g.xy[i];
        const double wi = wt[i];
        int status = 0;
        // domain rectangle, CCW, relative to the site
        int nv = 4;
        if (lane == 0) {
            double x0 = g.pd[0] - si.x, x1 = g.pd[1] - si.x, y0 = g.pd[2] - si.y, y1 = g.pd[3] - si.y;
            P.X[0] = x0; P.Y[0] = y0; P.A[0] = 0.0;  P.B[0] = -1.0; P.C[0] = -y0; P.L[0] = -1;
            P.X[1] = x1; P.Y[1] = y0; P.A[1] = 1.0;  P.B[1] = 0.0;  P.C[1] = x1;  P.L[1] = -2;
            P.X[2] = x1; P.Y[2] = y1; P.A[2] = 0.0;  P.B[2] = 1.0;  P.C[2] = y1;  P.L[2] = -3;
            P.X[3] = x0; P.Y[3] = y1; P.A[3] = -1.0; P.B[3] = 0.0;  P.C[3] = -x0; P.L[3] = -4;
        }
        __syncwarp();
        PSTAT_CLOCK(t0);
        const int bi = g.sbucket[i];
        const int bu = bi % g.bx, bv = bi / g.bx;
        // ---- 1. first candidates: the cell's neighbours at the previous
        //         evaluation, or the 3x3 buckets around the site ---------------
        // cache entries: +m ordered ring (domain sides -1..-4 skipped here),
        // -m unordered sites, -(COT_NB_HIDDEN + m) the sites that hid the cell
        const int nraw = (a.nbn != nullptr) ? a.nbn[i] : 0;
        const int ncache = min(nraw >= 0 ? nraw : (nraw < -COT_NB_HIDDEN ? -nraw - COT_NB_HIDDEN : -nraw), COT_NBC);
        const bool cached = ncache > 0;
        if (cached) {
            int j = lane < ncache ? a.nbc[(size_t)i * COT_NBC + lane] : -1;
            if (j < 0) j = -1;
            nv = clip_chunk<MAXV>(P, nv, j, g, si, wi, wt, lane, status, false);
        } else {
            int bcnt = 0, bst = 0;
            if (lane < 9) {
                // own bucket, then the 4 edge neighbours, then the corners
                const int du = (lane == 1 || lane == 5 || lane == 7) ? 1 : (lane == 2 || lane == 6 || lane == 8) ? -1 : 0;
                const int dv = (lane == 3 || lane == 5 || lane == 6) ? 1 : (lane == 4 || lane == 7 || lane == 8) ? -1 : 0;
                int u = bu + du, v = bv + dv;
                if (u >= 0 && u < g.bx && v >= 0 && v < g.by) {
                    int b = u + v * g.bx;
                    bst = g.bstart[b];
                    bcnt = g.bstart[b + 1] - bst;
                }
            }
            int inc = warp_incl_scan(bcnt, lane);
            int tot = __shfl_sync(FULLMASK, inc, 31);
            for (int base = 0; base < tot && nv > 0 && status == 0; base += 32) {
                int t = base + lane, j = -1;
#pragma unroll
                for (int k = 0; k < 9; k++) {
                    int ik = __shfl_sync(FULLMASK, inc, k);
                    int sk = __shfl_sync(FULLMASK, bst, k);
                    int ck = __shfl_sync(FULLMASK, bcnt, k);
                    if (j < 0 && t < tot && t < ik) j = sk + (t - (ik - ck));
                }
                if (j == i) j = -1;
                nv = clip_chunk<MAXV>(P, nv, j, g, si, wi, wt, lane, status, false);
            }
        }
        // leaves already processed in full (the window path only)
        const int win = cached ? -1 : COT_WIN;
        PSTAT_CLOCK(t1);
        PSTAT_ADD(0, t1 - t0);
        PSTAT_ADD(10, cached ? 1 : 0);
        // ---- 2. certificate over the bound tree --------------------------------
            bool brute = false;
        if (nv > 0 && status == 0 && g.nlev > 0) {
            int top = g.nlev - 1;
            while (top > 0 && g.lev_w[top - 1] * g.lev_h[top - 1] <= 32) top--;
            int ncur = g.lev_w[top] * g.lev_h[top];
            if (ncur > COT_FRMAX) brute = true;
            int cur = 0;
            if (!brute) {
                for (int q = lane; q < ncur; q += 32) P.fr[0][q] = q;
                __syncwarp();
            }
            for (int L = top; L >= 0 && !brute && nv > 0 && status == 0; L--) {
                int nnext = 0;
                const int off = g.lev_off[L], W = g.lev_w[L];
                PSTAT_ADD(7, ncur);
                for (int base = 0; base < ncur; base += 32) {
                    int q = (base + lane < ncur) ? P.fr[cur][base + lane] : -1;
                    bool keep = false;
                    if (q >= 0) {
                        if (L == 0) {
                            int u = q % W, v = q / W;
                            bool inwin = abs(u - bu) <= win && abs(v - bv) <= win;
                            keep = !inwin && !node_excluded(P, nv, g, off + q, si, wi);
                        } else {
                            keep = !node_excluded(P, nv, g, off + q, si, wi);
                        }
                    }
                    if (L == 0) {
                        unsigned m = __ballot_sync(FULLMASK, keep);
                        int pos = nnext + __popc(m & ((1u << lane) - 1u));
                        int cnt = __popc(m);
                        if (nnext + cnt > COT_FRMAX) { brute = true; break; }
                        if (keep) P.fr[1 - cur][pos] = q;
                        nnext += cnt;
                    } else {
                        int chc = 0;
                        int u = 0, v = 0, cw = g.lev_w[L - 1], ch = g.lev_h[L - 1];
                        if (keep) {
                            u = q % W; v = q / W;
                            for (int bb = 0; bb < 2; bb++)
                                for (int aa = 0; aa < 2; aa++)
                                    if (2 * u + aa < cw && 2 * v + bb < ch) chc++;
                        }
                        int inc = warp_incl_scan(chc, lane);
                        int cnt = __shfl_sync(FULLMASK, inc, 31);
                        if (nnext + cnt > COT_FRMAX) { brute = true; break; }
                        int pos = nnext + inc - chc;
                        if (keep) {
                            for (int bb = 0; bb < 2; bb++)
                                for (int aa = 0; aa < 2; aa++)
                                    if (2 * u + aa < cw && 2 * v + bb < ch) P.fr[1 - cur][pos++] = (2 * u + aa) + (2 * v + bb) * cw;
                        }
                        nnext += cnt;
                    }
                }
                __syncwarp();
                cur = 1 - cur;
                ncur = nnext;
                if (brute) break;
                if (L == 0) {
                    // clip by the sites of every leaf that survived
                    PSTAT_ADD(5, ncur);
                    for (int li = 0; li < ncur && nv > 0 && status == 0; li++) {
                        int b = P.fr[cur][li];
                        int s0 = g.bstart[b], s1 = g.bstart[b + 1];
                        for (int base = s0; base < s1 && nv > 0 && status == 0; base += 32) {
                            int j = base + lane < s1 ? base + lane : -1;
                            if (j == i) j = -1;
                            nv = clip_chunk<MAXV>(P, nv, j, g, si, wi, wt, lane, status, cached);
                        }
                    }
                }
            }
        }
        PSTAT_ADD(9, brute ? 1 : 0);
        if (brute && nv > 0 && status == 0) {
            // frontier overflow: test every bucket against the current polygon
            const int nb = g.bx * g.by;
            for (int base = 0; base < nb && nv > 0 && status == 0; base += 32) {
                int b = base + lane;
                bool keep = false;
                if (b < nb) {
                    int u = b % g.bx, v = b / g.bx;
                    bool inwin = abs(u - bu) <= win && abs(v - bv) <= win;
                    keep = !inwin && !node_excluded(P, nv, g, b, si, wi);
                }
                unsigned m = __ballot_sync(FULLMASK, keep);
                while (m != 0u && nv > 0 && status == 0) {
                    int l = __ffs(m) - 1;
                    m &= m - 1u;
                    int bb = base + l;
                    int s0 = g.bstart[bb], s1 = g.bstart[bb + 1];
                    for (int sb = s0; sb < s1 && nv > 0 && status == 0; sb += 32) {
                        int j = sb + lane < s1 ? sb + lane : -1;
                        if (j == i) j = -1;
                        nv = clip_chunk<MAXV>(P, nv, j, g, si, wi, wt, lane, status, cached);
                    }
                }
            }
        }
        if (status != 0) {
            // ring above MAXV: hand the cell to the large-capacity pass
            if (mode == 0 && lane == 0) {
                int slot = atomicAdd(a.ovf_count, 1);
                a.ovf_list[slot] = i;
                a.nv[i] = MAXV + 1;
            } else if (lane == 0) {
                a.nv[i] = MAXV + 1;
                a.mu[i] = 0.0;
                a.fc[i] = 0.0;
            }
            __syncwarp();
            continue;
        }
        // ---- 3. integrate the density over the cell --------------------------
        PSTAT_CLOCK(t2);
        PSTAT_ADD(1, t2 - t1);
        CellAcc acc = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (nv >= 3) acc = integrate_cell(P, nv, splat_geo(g, a, P, nv, i, lane), si, lane);
        PSTAT_CLOCK(t3);
        PSTAT_ADD(2, t3 - t2);
        PSTAT_ADD(8, 1);
        PSTAT_ADD(11, nv);
        double pcx = 0.0, pcy = 0.0;
        if (a.cen != nullptr && nv >= 3 && (!a.weighted || acc.Mt == 0.0)) poly_centroid(P, nv, lane, pcx, pcy);
        if (a.ring_xy != nullptr) {
            for (int k = lane; k < nv && k < a.ring_cap; k += 32) {
                a.ring_xy[2 * ((size_t)i * a.ring_cap + k)] = si.x + P.X[k];
                a.ring_xy[2 * ((size_t)i * a.ring_cap + k) + 1] = si.y + P.Y[k];
                a.ring_lab[(size_t)i * a.ring_cap + k] = P.L[k];
            }
        }
        if (a.solid != nullptr && lane == 0) a.solid[i] = nv >= 3 ? solid_angle_of(P, nv, si, a.solid_z, a.solid_light) : 0.0;
        if (a.keep_labels && nv >= 3) {
            // the Newton solve's Jacobian: a ring that ended at most COT_RCAP
            // vertices goes to the ring buffer like the fast path's rings, a
            // longer one has its row built here
            if (nv <= COT_RCAP) {
                if (lane < nv) {
                    a.rbuf[(size_t)i * COT_RCAP + lane] = make_double2(P.X[lane], P.Y[lane]);
                    a.lbuf[(size_t)i * COT_RCAP + lane] = P.L[lane];
                }
            } else if (a.hbig_val != nullptr) {
                int slot = 0;
                if (lane == 0) slot = atomicAdd(a.ovf_count + 7, 1);
                slot = __shfl_sync(FULLMASK, slot, 0);
                if (slot >= a.hbig_cap) {
                    if (lane == 0) atomicExch(a.herr, 1);
                } else {
                    const size_t base = (size_t)slot * COT_HBIG_W;
                    int cnt = 0;
                    double dsum = 0.0;
                    for (int k0 = 0; k0 < nv; k0 += 32) {
                        const int k = k0 + lane;
                        double av = 0.0;
                        int j = -1;
                        if (k < nv) {
                            j = P.L[k];
                            if (j >= 0) {
                                const int k1 = k + 1 == nv ? 0 : k + 1;
                                const double2 sj = g.xy[j];
                                const double ex = sj.x - si.x, ey = sj.y - si.y;
                                av = edge_rho_integral(g, si.x + P.X[k], si.y + P.Y[k], si.x + P.X[k1], si.y + P.Y[k1]) /
                                     (2.0 * sqrt(ex * ex + ey * ey));
                            }
                        }
                        const unsigned site = __ballot_sync(FULLMASK, j >= 0);
                        if (j >= 0) {
                            const int pos = cnt + __popc(site & ((1u << lane) - 1u));
                            a.hbig_val[base + pos] = av;
                            a.hbig_col[base + pos] = j;
                        }
                        cnt += __popc(site);
                        dsum += warp_sum(av);
                    }
                    if (lane == 0) {
                        if (cnt < COT_HBIG_W) a.hbig_col[base + cnt] = -1;
                        a.hcnt[i] = -(slot + 1);
                        a.hdiag[i] = dsum;
                    }
                }
            }
        }
        if (a.nbn != nullptr) {
            // neighbours of this evaluation seed the next one
            int lab = -1;
            if (lane < nv) lab = P.L[lane];
            bool isn = lab >= 0;
            unsigned m = __ballot_sync(FULLMASK, isn);
            int pos = __popc(m & ((1u << lane) - 1u));
            if (isn && pos < COT_NBC) a.nbc[(size_t)i * COT_NBC + pos] = lab;
            if (lane == 0) a.nbn[i] = -min(__popc(m), COT_NBC);
        }
        if (lane == 0) {
            a.mu[i] = acc.mu;
            // f_i = -w_i nu_i - sum_pix rho (int |x-s_i|^2 - w_i area)   (basic_function.cuh:875-941);
            // stored without its -w_i nu_i term, which the reduction adds, so
            // that nu may change after the cells are built
            a.fc[i] = -(acc.S - wi * acc.mu);
            a.nv[i] = nv;
            if (a.cen != nullptr) {
                bool ex = nv >= 3;
                a.exist[i] = ex ? 1 : 0;
                double cx = si.x, cy = si.y;
                if (ex) {
                    if (a.weighted && acc.Mt != 0.0) {
                        cx = si.x + acc.Mx / acc.Mt;
                        cy = si.y + acc.My / acc.Mt;
                    } else {
                        cx = si.x + pcx;
                        cy = si.y + pcy;
                    }
                }
                a.cen[2 * i] = cx;
                a.cen[2 * i + 1] = cy;
            }
        }
        __syncwarp();
    }
    PSTAT_FLUSH();
}

static size_t cells_smem(int maxv, int warps)
{
    switch (maxv) {
    case 32: return sizeof(WarpPoly<32>) * (size_t)warps;
    default: return sizeof(WarpPoly<256>) * (size_t)warps;
    }
}

#define CELLS_WPB 4
#define CELLS_MINB 6
#ifndef FIRST_MINB
#define FIRST_MINB 6  // k_cells_first: blocks per SM its registers are sized for
#endif
#ifndef WALK_MINB
#define WALK_MINB 8   // k_cells_walk (64 registers; 6 blocks measured 2 % slower)
#endif
static int g_blocks_per_sm32 = 0, g_blocks_per_sm16 = 0, g_blocks_per_sm8 = 0, g_blocks_per_smi = 0;
static int g_blocks_per_smf = 0, g_blocks_per_smw = 0, g_blocks_per_smb = 0;

template <bool EXACT, int LPC>
static void launch_fast(const CotGeo &g, const CellsArgs &a, int pass, int blocks, cudaStream_t s)
{
    const size_t sm = sizeof(FastScratch) * CELLS_WPB * (32 / LPC);
    k_cells_fast<CELLS_MINB, EXACT, LPC><<<blocks, 32 * CELLS_WPB, sm, s>>>(g, a, pass);
}

// One evaluation: bucket and tree bounds, then the cells.  cells_per_warp 2
// (4) runs the hot path on 16-lane (8-lane) segments, two (four) cells per
// warp, with a 32-lane second pass for rings above 16 (8) vertices; every
// path ends with the 256-vertex pass for rings above 32.
void launch_eval(const CotGeo &g, const CellsArgs &args, int cells_per_warp, int num_sms, CotCtx &c)
{
    cudaStream_t s = c.s;
    CellsArgs a = args;
    const int nb = g.bx * g.by;
    // tree levels up to the first one of at most 16 nodes: the highest level
    // any certificate walk starts from (one round of a 16- or 32-lane segment)
    int lmax = 0;
    while (lmax < g.nlev - 1 && g.lev_w[lmax] * g.lev_h[lmax] > 16) lmax++;
    // ovf_count[0..5]: overflow list sizes and fetch counters, [6]: the
    // integration kernel's fetch counter, [8]: k_cells_walk's fetch counter,
    // [9]: k_bucket_walk's, [10]: the heavy integration list's size, [11]:
    // the overflowed walks' list size, [12]: k_cells_heavy's fetch counter,
    // [13]: the split integration list's size
    const int segs = (nb * BSEG + 127) / 128;
    k_bucket_phi<<<segs, 128, 0, s>>>(g, a.w, a.d, a.tptr, a.wt, a.wbar, a.ovf_count, 14);
    k_tree_build<<<(nb * BSEG + TREE_THREADS - 1) / TREE_THREADS, TREE_THREADS, 0, s>>>(g, a.wt, a.wbar);
    c.launches += 2;
    int upper = 0;  // nodes of levels 1..lmax
    for (int L = 1; L <= lmax; L++) upper += g.lev_w[L] * g.lev_h[L];
    if (upper > 0) {
        k_tree_levels<<<upper, TREE_THREADS, 0, s>>>(g, a.wt);
        c.launches++;
    }
    const int sms = num_sms > 0 ? num_sms : 148;
    const bool exact = a.cen != nullptr || a.splat != nullptr || a.solid != nullptr;
    const int lpc = (exact || cells_per_warp < 2) ? 32 : (cells_per_warp == 2 ? 16 : 8);
    // the bucket walk's lists exist only on the path that runs it: every
    // other path walks in full
    if (exact || lpc != 32) a.blist = a.bcnt = nullptr;
    // the heavy integration list (ovf_list2, which only the 16- and 8-lane
    // paths use otherwise) on the two-kernel path
    a.hlist = (exact || lpc != 32) ? nullptr : a.ovf_list2;
    if (exact || lpc != 32) {
        a.wlist = nullptr;
        a.hsplit = nullptr;
    }
    const int per_sm32 = g_blocks_per_sm32 > 0 ? g_blocks_per_sm32 : CELLS_MINB;
    const int per_sm16 = g_blocks_per_sm16 > 0 ? g_blocks_per_sm16 : CELLS_MINB;
    const int per_sm8 = g_blocks_per_sm8 > 0 ? g_blocks_per_sm8 : 1;
    const int cells_per_block = CELLS_WPB * (32 / lpc);
    const int want = (g.n + cells_per_block - 1) / cells_per_block;
    const int blocks = std::min(want, sms * (lpc == 32 ? per_sm32 : (lpc == 16 ? per_sm16 : per_sm8)));
    bool timed = c.profile && c.ev != nullptr && c.ev_used + 2 <= c.ev_cap;
    if (timed) cudaEventRecord(c.ev[c.ev_used], s);
    if (exact) {
        launch_fast<true, 32>(g, a, 0, blocks, s);
    } else if (lpc == 32) {
        const int bw = std::min(g.n, sms * (g_blocks_per_smw > 0 ? g_blocks_per_smw : WALK_MINB) * CELLS_WPB);
        const int bf = std::min(g.n, sms * (g_blocks_per_smf > 0 ? g_blocks_per_smf : FIRST_MINB) * CELLS_WPB);
        const size_t sm = sizeof(FastScratch) * CELLS_WPB;
        k_cells_first<FIRST_MINB><<<(bf + CELLS_WPB - 1) / CELLS_WPB, 32 * CELLS_WPB, sm, s>>>(g, a);
        if (a.bcnt != nullptr) {
            const int bb = std::min(nb, sms * (g_blocks_per_smb > 0 ? g_blocks_per_smb : WALK_MINB) * CELLS_WPB);
            k_bucket_walk<WALK_MINB><<<(bb + CELLS_WPB - 1) / CELLS_WPB, 32 * CELLS_WPB, sm, s>>>(g, a);
            c.launches++;
        }
        if (a.keep_labels)
            k_cells_walk<WALK_MINB, true><<<(bw + CELLS_WPB - 1) / CELLS_WPB, 32 * CELLS_WPB, sm, s>>>(g, a);
        else
            k_cells_walk<WALK_MINB, false><<<(bw + CELLS_WPB - 1) / CELLS_WPB, 32 * CELLS_WPB, sm, s>>>(g, a);
        c.launches++;
        // the cells whose walk overflowed, a block each (an empty list
        // returns at once)
        const size_t hsm = sizeof(FastScratch) + sizeof(HeavyShared);
        if (a.keep_labels)
            k_cells_heavy<true><<<2 * sms, 32 * HEAVY_WARPS, hsm, s>>>(g, a);
        else
            k_cells_heavy<false><<<2 * sms, 32 * HEAVY_WARPS, hsm, s>>>(g, a);
        c.launches++;
    } else if (lpc == 16) {
        launch_fast<false, 16>(g, a, 0, blocks, s);
        launch_fast<false, 32>(g, a, 1, sms, s);
        c.launches++;
    } else {
        launch_fast<false, 8>(g, a, 0, blocks, s);
        launch_fast<false, 32>(g, a, 1, sms, s);
        c.launches++;
    }
    if (!exact) {
        const int per_smi = g_blocks_per_smi > 0 ? g_blocks_per_smi : 8;
        const int bi = std::min((g.n + CELLS_WPB - 1) / CELLS_WPB, sms * per_smi);
        k_integrate<8><<<bi, 32 * CELLS_WPB, sizeof(FastScratch) * CELLS_WPB, s>>>(g, a);
        c.launches++;
    }
    if (timed) {
        cudaEventRecord(c.ev[c.ev_used + 1], s);
        c.ev_used += 2;
    }
    // cells above 32 vertices (rare): one warp per block, 256-vertex rings
    k_cells<256, 1><<<sms, 32, cells_smem(256, 1), s>>>(g, a, lpc == 32 ? 1 : 2);
    c.launches += 2;
    c.cell_launches += 1;
    c.evaluations += 1;
}

#ifdef COT_PHASE_STATS
extern "C" __attribute__((visibility("default"))) int cot_debug_phase_stats(unsigned long long *out, int reset)
{
    cudaDeviceSynchronize();
    cudaMemcpyFromSymbol(out, cot_phase_stats, sizeof(unsigned long long) * 16);
    if (reset) {
        unsigned long long z[16] = {0};
        cudaMemcpyToSymbol(cot_phase_stats, z, sizeof z);
    }
    return 0;
}
#endif

void configure_cells_kernels()
{
    const int sm32 = (int)(sizeof(FastScratch) * CELLS_WPB), sm16 = 2 * sm32, sm8 = 4 * sm32;
    cudaFuncSetAttribute(k_cells_fast<CELLS_MINB, false, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    cudaFuncSetAttribute(k_cells_fast<CELLS_MINB, true, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    cudaFuncSetAttribute(k_cells_fast<CELLS_MINB, false, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm16);
    cudaFuncSetAttribute(k_cells_fast<CELLS_MINB, false, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm8);
    cudaFuncSetAttribute(k_cells<256, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cells_smem(256, 1));
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_cells_fast<CELLS_MINB, false, 32>, 32 * CELLS_WPB,
                                                      sm32) == cudaSuccess && nb > 0)
        g_blocks_per_sm32 = nb;
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_cells_fast<CELLS_MINB, false, 16>, 32 * CELLS_WPB,
                                                      sm16) == cudaSuccess && nb > 0)
        g_blocks_per_sm16 = nb;
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_cells_fast<CELLS_MINB, false, 8>, 32 * CELLS_WPB,
                                                      sm8) == cudaSuccess && nb > 0)
        g_blocks_per_sm8 = nb;
    cudaFuncSetAttribute(k_integrate<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    cudaFuncSetAttribute(k_cells_first<FIRST_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    cudaFuncSetAttribute(k_cells_walk<WALK_MINB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    cudaFuncSetAttribute(k_cells_walk<WALK_MINB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    cudaFuncSetAttribute(k_bucket_walk<WALK_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm32);
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_cells_first<FIRST_MINB>, 32 * CELLS_WPB, sm32) ==
            cudaSuccess &&
        nb > 0)
        g_blocks_per_smf = nb;
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_cells_walk<WALK_MINB, false>, 32 * CELLS_WPB, sm32) ==
            cudaSuccess &&
        nb > 0)
        g_blocks_per_smw = nb;
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bucket_walk<WALK_MINB>, 32 * CELLS_WPB, sm32) ==
            cudaSuccess &&
        nb > 0)
        g_blocks_per_smb = nb;
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_integrate<8>, 32 * CELLS_WPB, sm32) == cudaSuccess &&
        nb > 0)
        g_blocks_per_smi = nb;
}

}  // namespace cot
