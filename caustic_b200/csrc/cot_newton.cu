// Kernels of the damped Newton solve (cot_solve_newton; no counterpart in the
// reference, whose solvers are L-BFGS and Anderson acceleration).
//
//  - k_hessian: the mass Jacobian dmu/dw at the rings the last evaluation
//    left in the ring buffer: one warp per cell, one lane per edge, each
//    edge's density line integral (cot_edge.cuh) over 2|s_i - s_j|.  Rows go
//    to an ELL layout, entry k of cell i at [k * n + i], so that a thread per
//    row reads coalesced in the solver's matrix products; rings above 32
//    vertices have their rows built by the large-ring pass of the cell kernel.
//  - k_newton_stats: |g|^2, min mu, max relative error, empty cells and the
//    largest ring at a trial point, in fixed order (last block sums).
//  - k_pcg: the Jacobi-preconditioned conjugate gradient for dmu/dw d = nu -
//    mu as ONE cooperative persistent launch: a thread owns rows, blocks meet
//    at bounded grid barriers (two per iteration: the new search direction is
//    formed on the fly from z and the previous direction inside the matrix
//    product), and every block sums the per-block partials in block order, so
//    that all blocks take the same decisions and the result repeats bit for
//    bit.  A barrier that waits longer than its limit sets an error flag; every
//    block then leaves at its next barrier and the host falls back.
#include "cot_common.cuh"
#include "cot_edge.cuh"

#include <algorithm>

namespace cot {

#define HESS_THREADS 128
#define PCG_THREADS 512
#define PCG_SPIN_LIMIT (1u << 22)  // polls of __nanosleep(64): well under a few seconds

__device__ __forceinline__ double hsum32(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(HESS_THREADS) k_hessian(CotGeo g, const double2 *__restrict__ rbuf,
                                                         const int *__restrict__ lbuf, const int *__restrict__ nv,
                                                         double *__restrict__ hval, int *__restrict__ hcol,
                                                         int *__restrict__ hcnt, double *__restrict__ hdiag)
{
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (HESS_THREADS / 32) + (threadIdx.x >> 5);
    if (i >= g.n) return;
    const int m = nv[i];
    if (m > 32) return;  // a big row, built by the large-ring pass
    if (m < 3) {
        if (lane == 0) {
            hcnt[i] = 0;
            hdiag[i] = 0.0;
        }
        return;
    }
    const double2 si = g.xy[i];
    double a = 0.0;
    int j = -1;
    if (lane < m) {
        j = lbuf[(size_t)i * 32 + lane];
        if (j >= 0) {
            const double2 p = rbuf[(size_t)i * 32 + lane];
            const double2 q = rbuf[(size_t)i * 32 + (lane + 1 == m ? 0 : lane + 1)];
            const double2 sj = g.xy[j];
            const double ex = sj.x - si.x, ey = sj.y - si.y;
            a = edge_rho_integral(g, si.x + p.x, si.y + p.y, si.x + q.x, si.y + q.y) / (2.0 * sqrt(ex * ex + ey * ey));
        }
    }
    const unsigned site = __ballot_sync(0xffffffffu, j >= 0);
    const int pos = __popc(site & ((1u << lane) - 1u));
    if (j >= 0) {
        hval[(size_t)pos * g.n + i] = a;
        hcol[(size_t)pos * g.n + i] = j;
    }
    const double d = hsum32(a);
    if (lane == 0) {
        hcnt[i] = __popc(site);
        hdiag[i] = d;
    }
}

void launch_hessian(const CotGeo &g, const double2 *rbuf, const int *lbuf, const int *nv, double *hval, int *hcol,
                    int *hcnt, double *hdiag, CotCtx &c)
{
    const int per = HESS_THREADS / 32;
    k_hessian<<<(g.n + per - 1) / per, HESS_THREADS, 0, c.s>>>(g, rbuf, lbuf, nv, hval, hcol, hcnt, hdiag);
    c.launches++;
}

// ---------------------------------------------------------------------------
// statistics of a trial point
// ---------------------------------------------------------------------------
#define NST_THREADS 256
#define NST_VALS 5

__device__ __forceinline__ double nmax_keep_nan(double a, double b) { return (a != a || b != b) ? INFINITY : fmax(a, b); }

__global__ void __launch_bounds__(NST_THREADS) k_newton_stats(int n, const double *__restrict__ mu,
                                                             const double *__restrict__ nu, const int *__restrict__ nv,
                                                             double *partials, unsigned int *ticket,
                                                             NewtonEvalStats *out)
{
    __shared__ double sh[NST_VALS][NST_THREADS / 32];
    __shared__ bool last;
    double g2 = 0.0, mn = INFINITY, mx = 0.0, emp = 0.0, mnv = 0.0;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double m = mu[i], g = m - nu[i];
        g2 += g * g;
        mn = fmin(mn, m);
        const double rel = nu[i] > 0.0 ? fabs(g) / nu[i] : (g != 0.0 ? INFINITY : 0.0);
        mx = (rel == rel) ? fmax(mx, rel) : INFINITY;
        emp += m == 0.0 ? 1.0 : 0.0;
        mnv = fmax(mnv, (double)nv[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        g2 += __shfl_xor_sync(0xffffffffu, g2, o);
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = nmax_keep_nan(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        emp += __shfl_xor_sync(0xffffffffu, emp, o);
        mnv = fmax(mnv, __shfl_xor_sync(0xffffffffu, mnv, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = g2;
        sh[1][wid] = mn;
        sh[2][wid] = mx;
        sh[3][wid] = emp;
        sh[4][wid] = mnv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[NST_VALS] = {0.0, INFINITY, 0.0, 0.0, 0.0};
        for (int k = 0; k < NST_THREADS / 32; k++) {
            r[0] += sh[0][k];
            r[1] = fmin(r[1], sh[1][k]);
            r[2] = nmax_keep_nan(r[2], sh[2][k]);
            r[3] += sh[3][k];
            r[4] = fmax(r[4], sh[4][k]);
        }
        for (int k = 0; k < NST_VALS; k++) partials[(size_t)blockIdx.x * NST_VALS + k] = r[k];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double r[NST_VALS] = {0.0, INFINITY, 0.0, 0.0, 0.0};
    for (unsigned b = 0; b < gridDim.x; b++) {
        const double *p = partials + (size_t)b * NST_VALS;
        r[0] += __ldcg(p + 0);
        r[1] = fmin(r[1], __ldcg(p + 1));
        r[2] = nmax_keep_nan(r[2], __ldcg(p + 2));
        r[3] += __ldcg(p + 3);
        r[4] = fmax(r[4], __ldcg(p + 4));
    }
    NewtonEvalStats o;
    o.gnorm2 = r[0];
    o.minmu = r[1];
    o.maxrel = r[2];
    o.empty = (int)r[3];
    o.maxnv = (int)r[4];
    *out = o;
    *ticket = 0u;
}

void launch_newton_stats(int n, const double *mu, const double *nu, const int *nv, double *partials,
                         unsigned int *ticket, NewtonEvalStats *out, CotCtx &c)
{
    const int blocks = std::min(reduce_blocks(n), 256);
    k_newton_stats<<<blocks, NST_THREADS, 0, c.s>>>(n, mu, nu, nv, partials, ticket, out);
    c.launches++;
}

// ---------------------------------------------------------------------------
// conjugate gradient, one cooperative launch
// ---------------------------------------------------------------------------
// Grid barrier with a bounded wait.  Returns false (and raises st->error)
// when a block waited longer than PCG_SPIN_LIMIT polls or saw the flag set.
__device__ bool pcg_barrier(PcgState *st)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned int *gen = &st->bar_gen;
        const unsigned int g0 = *gen;
        __threadfence();
        if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
            st->bar_count = 0u;
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        } else {
            unsigned int spins = 0;
            while (*gen == g0) {
                if (++spins > PCG_SPIN_LIMIT || *(volatile int *)&st->error != 0) {
                    atomicExch(&st->error, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile int *)&st->error != 0) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// Block sum of two values into partials[2 * blockIdx.x + k].
__device__ __forceinline__ void pcg_block_partials(double v0, double v1, double *partials)
{
    __shared__ double sh[2][PCG_THREADS / 32];
    v0 = hsum32(v0);
    v1 = hsum32(v1);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        sh[0][wid] = v0;
        sh[1][wid] = v1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < PCG_THREADS / 32; k++) {
            a += sh[0][k];
            b += sh[1][k];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// Every block sums the partials of all blocks in one fixed order (the same
// result in every block).
__device__ __forceinline__ double2 pcg_grid_sums(const double *partials)
{
    __shared__ double2 res;
    __shared__ double la[32], lb[32];
    if (threadIdx.x < 32) {
        double a = 0.0, b = 0.0;
        // lane l sums blocks l, l + 32, ... then the lanes are summed in order
        for (unsigned k = threadIdx.x; k < gridDim.x; k += 32) {
            a += __ldcg(partials + 2 * k);
            b += __ldcg(partials + 2 * k + 1);
        }
        la[threadIdx.x] = a;
        lb[threadIdx.x] = b;
        __syncwarp();
        if (threadIdx.x == 0) {
            double sa = 0.0, sb = 0.0;
            for (int l = 0; l < 32; l++) {
                sa += la[l];
                sb += lb[l];
            }
            res = make_double2(sa, sb);
        }
    }
    __syncthreads();
    return res;
}

// Row i of (dmu/dw) applied to the direction p = z + beta * pold (formed on
// the fly from the two vectors, which are final at this point).
__device__ __forceinline__ double pcg_row(int n, int i, const double *__restrict__ hval, const int *__restrict__ hcol,
                                          const int *__restrict__ hcnt, const double *__restrict__ hbig_val,
                                          const int *__restrict__ hbig_col, double diag, const double *z,
                                          const double *pold, double beta, double pi)
{
    double acc = diag * pi;
    const int c = hcnt[i];
    if (c >= 0) {
        for (int k = 0; k < c; k++) {
            const int j = hcol[(size_t)k * n + i];
            acc -= hval[(size_t)k * n + i] * (__ldcg(z + j) + beta * __ldcg(pold + j));
        }
    } else {
        const size_t base = (size_t)(-c - 1) * COT_HBIG_W;
        for (int k = 0; k < COT_HBIG_W; k++) {
            const int j = hbig_col[base + k];
            if (j < 0) break;
            acc -= hbig_val[base + k] * (__ldcg(z + j) + beta * __ldcg(pold + j));
        }
    }
    return acc;
}

__global__ void __launch_bounds__(PCG_THREADS) k_pcg(int n, const double *__restrict__ hval,
                                                     const int *__restrict__ hcol, const int *__restrict__ hcnt,
                                                     const double *__restrict__ hbig_val,
                                                     const int *__restrict__ hbig_col, const double *__restrict__ hdiag,
                                                     const double *__restrict__ b, double *x, double *r, double *z,
                                                     double *pa, double *pb, double *q, double *partials,
                                                     PcgState *st, double rtol, int max_it)
{
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double *P0 = partials, *P1 = partials + 2 * gridDim.x;
    // mean of the right-hand side (the Jacobian's range is mean-free)
    double sb = 0.0;
    for (int i = t0; i < n; i += stride) sb += b[i];
    pcg_block_partials(sb, 0.0, P0);
    if (!pcg_barrier(st)) return;
    const double mean = pcg_grid_sums(P0).x / (double)n;
    // Jacobi weights; an empty cell's row is zero and keeps a unit diagonal
    double rz_l = 0.0, rr_l = 0.0;
    for (int i = t0; i < n; i += stride) {
        const double ri = b[i] - mean;
        const double di = hdiag[i] > 0.0 ? hdiag[i] : 1.0;
        const double zi = ri / di;
        r[i] = ri;
        z[i] = zi;
        x[i] = 0.0;
        pa[i] = 0.0;
        rz_l += ri * zi;
        rr_l += ri * ri;
    }
    pcg_block_partials(rz_l, rr_l, P1);
    if (!pcg_barrier(st)) return;
    double2 s2 = pcg_grid_sums(P1);
    double rz = s2.x;
    const double rr0 = s2.y;
    double rr = rr0;
    double beta = 0.0;
    int it = 0;
    double *pold = pa, *pnew = pb;
    const double stop = rtol * rtol * rr0;
    // P0 is read by every block between the two barriers of an iteration and
    // written again only after the second; P1 likewise across iterations
    while (it < max_it && rr > stop && rz > 0.0) {
        // p = z + beta pold; q = J p; partial p.q
        double pq_l = 0.0;
        for (int i = t0; i < n; i += stride) {
            const double di = hdiag[i] > 0.0 ? hdiag[i] : 1.0;
            const double pi = z[i] + beta * pold[i];
            pnew[i] = pi;
            const double qi = pcg_row(n, i, hval, hcol, hcnt, hbig_val, hbig_col, di, z, pold, beta, pi);
            q[i] = qi;
            pq_l += pi * qi;
        }
        pcg_block_partials(pq_l, 0.0, P0);
        if (!pcg_barrier(st)) return;
        const double pq = pcg_grid_sums(P0).x;
        if (!(pq > 0.0)) break;
        const double alpha = rz / pq;
        double rz2_l = 0.0, rr2_l = 0.0;
        for (int i = t0; i < n; i += stride) {
            const double di = hdiag[i] > 0.0 ? hdiag[i] : 1.0;
            x[i] += alpha * pnew[i];
            const double ri = r[i] - alpha * q[i];
            const double zi = ri / di;
            r[i] = ri;
            z[i] = zi;
            rz2_l += ri * zi;
            rr2_l += ri * ri;
        }
        pcg_block_partials(rz2_l, rr2_l, P1);
        if (!pcg_barrier(st)) return;
        s2 = pcg_grid_sums(P1);
        beta = s2.x / rz;
        rz = s2.x;
        rr = s2.y;
        double *tp = pold;
        pold = pnew;
        pnew = tp;
        it++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->iterations = it;
        st->rr0 = rr0;
        st->rr = rr;
    }
}

int pcg_max_blocks(int n, int num_sms)
{
    // one block of PCG_THREADS per SM at most (the kernel's registers allow
    // one), so that every block of the cooperative launch is resident
    const int want = (n + PCG_THREADS - 1) / PCG_THREADS;
    return std::max(1, std::min(want, num_sms));
}

cudaError_t launch_pcg(int n, const double *hval, const int *hcol, const int *hcnt, const double *hbig_val,
                       const int *hbig_col, const double *hdiag, const double *b, double *x, double *r, double *z,
                       double *pa, double *pb, double *q, double *partials, PcgState *st, double rtol, int max_it,
                       int blocks, CotCtx &c)
{
    void *args[] = {&n, &hval, &hcol, &hcnt, &hbig_val, &hbig_col, &hdiag, &b, &x, &r, &z, &pa, &pb, &q,
                    &partials, &st, &rtol, &max_it};
    c.launches++;
    return cudaLaunchCooperativeKernel((const void *)k_pcg, dim3(blocks), dim3(PCG_THREADS), args, 0, c.s);
}

}  // namespace cot
