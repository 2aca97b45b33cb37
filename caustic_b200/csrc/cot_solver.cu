// Device-resident L-BFGS for the dual weights.
//
// Replaces the solver loop of direct_ot (ot_op.cuh:289-537).  The reference
// runs the two-loop recursion with one kernel per vector operation and moves
// every dot product to the host (2m+1 device->host copies of N doubles per
// iteration, ot_op.cuh:298-337).  Here the two-loop runs on the Gram matrix of
// the basis {s_0..s_{m-1}, y_0..y_{m-1}, g} (the vector-free form of the
// recursion): after each accepted step one pass over N computes the 5m+1 new
// dot products, one device thread runs the recursion on the (2m+1)^2 matrix,
// and one pass forms d = sum_j delta_j b_j.  Every reduction is a fixed-order
// tree (per-block partials summed in block order by the last block), so a
// solve is bit-reproducible run to run.  Line-search decisions are taken by
// one device thread as well; the host only reads a flag.
#include "cot_common.cuh"
#include "../../include/causticot.h"
#include <math.h>

namespace cot {

#define FULLMASK 0xffffffffu
#define RED_THREADS 256
#define RED_VALS 8

int reduce_blocks(int n)
{
    int b = (n + RED_THREADS * 4 - 1) / (RED_THREADS * 4);
    if (b < 1) b = 1;
    if (b > 1024) b = 1024;
    return b;
}

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
    return v;
}
__device__ __forceinline__ double wmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULLMASK, v, o));
    return v;
}

// Sum (or max) of stride-separated partials in block order, with the loads
// issued ahead in groups (L2 reads: partials of other blocks are never taken
// from a stale L1 line).
template <bool MAX>
__device__ __forceinline__ double sum_partials(const double *p, unsigned nblocks, size_t stride)
{
    double r = 0.0;
    unsigned b = 0;
    for (; b + 8 <= nblocks; b += 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) v[q] = __ldcg(p + (size_t)(b + q) * stride);
#pragma unroll
        for (int q = 0; q < 8; q++) r = MAX ? fmax(r, v[q]) : r + v[q];
    }
    for (; b < nblocks; b++) {
        const double v = __ldcg(p + (size_t)b * stride);
        r = MAX ? fmax(r, v) : r + v;
    }
    return r;
}

// Fixed-order block reduction of one value (sum or max).  All threads call it.
template <bool MAX>
__device__ double block_reduce(double v, double *sh)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = MAX ? wmax(v) : wsum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = MAX ? -INFINITY : 0.0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < nw; k++) r = MAX ? fmax(r, sh[k]) : r + sh[k];
        sh[32] = r;
    }
    __syncthreads();
    return sh[32];
}

#define COT_F_NOISE 1e-12  // relative noise of the objective the line search tolerates

// Line-search decision for the trial just reduced (one thread).
__device__ void ls_decide(CotSolver *S, const CotEvalOut &o)
{
    S->evals++;
    S->last = o;
    S->accepted = 0;
    if (S->mode == COT_SOLVE_REFERENCE) {
        // ot_op.cuh:360-426
        if (o.overflow > 0) {
            S->ring_rejects++;
            S->t *= 0.5;
        } else if (o.f < S->f) {
            S->accepted = 1;
            S->ls_active = 0;
            return;
        } else {
            S->t *= 0.5;
        }
        if (S->t <= 1e-4 * S->t0) S->ls_active = 0;  // restart
        return;
    }
    // a solve that only has to give every cell mass takes the first trial
    // point where none is empty
    if (S->stop_nonempty && o.empty == 0 && o.overflow == 0) {
        S->accepted = 1;
        S->ls_active = 0;
        return;
    }
    // strong Wolfe: bracket by doubling, zoom by bisection
    if (S->final_eval) {
        S->accepted = 1;
        S->ls_active = 0;
        return;
    }
    double t = S->t;
    bool bad = o.overflow > 0;
    if (bad) S->ring_rejects++;
    // approximate Wolfe (Hager and Zhang): near convergence the objective's
    // evaluation noise (rounding in every cell's terms, about 1e-16 of |f|
    // per cell) exceeds the decrease a step can still make, and comparisons
    // of f stop telling steps apart.  A change of f within COT_F_NOISE |f|
    // is then not held against the step, provided the slope at the trial
    // point g(t).d <= (2 c1 - 1) g.d: the directional derivative decides.
    const bool approx = o.f <= S->f + COT_F_NOISE * fabs(S->f) && o.gtd <= (2.0 * S->c1 - 1.0) * S->gd;
    if (bad || (!approx && (!(o.f <= S->f + S->c1 * t * S->gd) || o.f >= S->f_lo))) {
        S->hi = t;
    } else if (fabs(o.gtd) <= S->c2 * fabs(S->gd)) {
        S->accepted = 1;
        S->ls_active = 0;
        return;
    } else if (o.gtd > 0.0) {
        S->hi = t;
    } else {
        // a step taken on the approximate conditions may sit a rounding
        // above f_lo: it moves the bracket's low end but never raises f_lo
        S->lo = t;
        S->f_lo = fmin(S->f_lo, o.f);
    }
    S->trials++;
    if (S->trials >= S->max_ls) {
        if (S->lo > 0.0) {
            S->t = S->lo;
            S->final_eval = 1;
        } else {
            S->ls_active = 0;  // failed
        }
        return;
    }
    S->t = isinf(S->hi) ? 2.0 * t : 0.5 * (S->lo + S->hi);
}

// One pass over the cells: objective, gradient statistics, directional
// derivative; the last block finishes the sums and (in a solve) decides.
__global__ void __launch_bounds__(RED_THREADS) k_reduce_eval(int n, const double *__restrict__ mu,
                                                            const double *__restrict__ fc, const int *__restrict__ nv,
                                                            const double *__restrict__ wt,
                                                            const double *__restrict__ nu, const double *__restrict__ d,
                                                            int max_ring, double *partials, unsigned int *ticket,
                                                            CotEvalOut *out, CotSolver *S)
{
    __shared__ double sh[33];
    __shared__ bool last;
    if (S != nullptr && (S->done || !S->ls_active)) return;
    double f = 0.0, gtd = 0.0, mx = 0.0, gn = 0.0, emp = 0.0, ovf = 0.0, mnv = 0.0;
    int per = (n + gridDim.x - 1) / gridDim.x;
    int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        double g = mu[i] - nu[i];
        f += fc[i] - wt[i] * nu[i];
        if (d != nullptr) gtd += g * d[i];
        double rel = nu[i] > 0.0 ? fabs(g) / nu[i] : (g != 0.0 ? INFINITY : 0.0);
        mx = (rel == rel) ? fmax(mx, rel) : INFINITY;  // a NaN mass counts as unconverged
        gn += g * g;
        emp += (mu[i] == 0.0) ? 1.0 : 0.0;
        ovf += (nv[i] > max_ring) ? 1.0 : 0.0;
        mnv = fmax(mnv, (double)nv[i]);
    }
    double v[RED_VALS];
    v[0] = block_reduce<false>(f, sh);
    v[1] = block_reduce<false>(gtd, sh);
    v[2] = block_reduce<true>(mx, sh);
    v[3] = block_reduce<false>(gn, sh);
    v[4] = block_reduce<false>(emp, sh);
    v[5] = block_reduce<false>(ovf, sh);
    v[6] = block_reduce<true>(mnv, sh);
    v[7] = 0.0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < RED_VALS; k++) partials[blockIdx.x * RED_VALS + k] = v[k];
        __threadfence();
        unsigned int tk = atomicAdd(ticket, 1u);
        last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // one thread per value, each summing the blocks in order
    if (threadIdx.x < 7) {
        const int k = threadIdx.x;
        sh[k] = (k == 2 || k == 6) ? sum_partials<true>(partials + k, gridDim.x, RED_VALS)
                                   : sum_partials<false>(partials + k, gridDim.x, RED_VALS);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double *r = sh;
        CotEvalOut o;
        o.f = r[0];
        o.gtd = r[1];
        o.maxrel = r[2];
        o.gnorm2 = r[3];
        o.empty = (int)r[4];
        o.overflow = (int)r[5];
        o.maxnv = (int)r[6];
        o.pad = 0;
        *out = o;
        *ticket = 0u;
        if (S != nullptr) ls_decide(S, o);
    }
}

void launch_reduce(const CotGeo &g, const double *mu, const double *fc, const int *nv, const double *wt,
                   const double *d, int max_ring, double *partials, unsigned int *ticket, CotEvalOut *out,
                   CotSolver *solver, CotCtx &c)
{
    int nb = reduce_blocks(g.n);
    k_reduce_eval<<<nb, RED_THREADS, 0, c.s>>>(g.n, mu, fc, nv, wt, g.nu, d, max_ring, partials, ticket, out, solver);
    c.launches++;
}

// ---------------------------------------------------------------------------
// iteration control (single thread)
// ---------------------------------------------------------------------------
// Two-loop recursion on the Gram matrix (ot_op.cuh:291-351): delta gives
// d = sum_j delta_j basis_j; then the descent safeguard.  One warp: the
// (2m+1)^2 matrix is staged in shared memory and every row product is a
// warp-wide dot product.
__global__ void __launch_bounds__(32) k_begin_iteration(CotSolver *S)
{
    __shared__ double G[COT_BASIS * COT_BASIS];
    __shared__ double dl[COT_BASIS];
    __shared__ double rh[COT_MAX_HIST], alpha[COT_MAX_HIST];
    const int lane = threadIdx.x;
    // only at an iteration boundary: inside a device-driven loop this kernel
    // also runs before every further trial of a line search
    if (S->done || !S->need_begin) return;
    const int m = S->m, B = 2 * m + 1, gi = 2 * m;
    const int k = S->k;
    // the control block's arrays once into shared memory: the recursion
    // below is a chain of 2m dependent steps
    for (int q = lane; q < B * B; q += 32) G[q] = S->G[(q / B) * COT_BASIS + q % B];
    for (int c = lane; c < B; c += 32) dl[c] = (c == gi) ? -1.0 : 0.0;
    for (int c = lane; c < m; c += 32) rh[c] = S->rho[c];
    __syncwarp();
    auto gdot = [&](int row) -> double {
        double r = 0.0;
        for (int c = lane; c < B; c += 32) r += G[row * B + c] * dl[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(FULLMASK, r, o);
        return r;
    };
    const int cnt = k < m ? k : m;
    const bool skip = (S->mode == COT_SOLVE_REFERENCE) && S->restart;
    const double H0 = S->H0;
    if (!skip) {
        for (int i = 1; i <= cnt; i++) {
            const int idx = ((k - i) % m + m) % m;
            const double a = gdot(idx) * rh[idx];
            __syncwarp();
            if (lane == 0) {
                alpha[i - 1] = a;
                dl[m + idx] -= a;
            }
            __syncwarp();
        }
        for (int c = lane; c < B; c += 32) dl[c] *= H0;
        __syncwarp();
        for (int i = cnt; i > 0; i--) {
            const int idx = ((k - i) % m + m) % m;
            const double beta = rh[idx] * gdot(m + idx);
            __syncwarp();
            if (lane == 0) dl[idx] += alpha[i - 1] - beta;
            __syncwarp();
        }
    }
    double gd = gdot(gi);
    __syncwarp();
    const bool reset = !(gd < 0.0);  // not a descent direction: steepest descent
    if (reset) {
        for (int c = lane; c < B; c += 32) dl[c] = (c == gi) ? -1.0 : 0.0;
        gd = -G[gi * B + gi];
    }
    __syncwarp();
    for (int c = lane; c < COT_BASIS; c += 32) S->delta[c] = c < B ? dl[c] : 0.0;
    if (lane != 0) return;
    if (!skip)
        for (int i = 1; i <= cnt; i++) S->alpha[((k - i) % m + m) % m] = alpha[i - 1];
    if (reset) {
        S->k = 0;
        S->H0 = 1.0;
    }
    S->need_begin = 0;
    S->eval_mark = S->evals;
    S->gnorm_stale = sqrt(S->gnorm2);
    S->empty_stale = S->empty;
    S->gd = gd;
    S->t = S->t0;
    S->lo = 0.0;
    S->hi = INFINITY;
    S->f_lo = S->f;
    S->trials = 0;
    S->ls_active = 1;
    S->accepted = 0;
    S->final_eval = 0;
}

void launch_begin_iteration(CotSolver *S, CotCtx &c)
{
    k_begin_iteration<<<1, 32, 0, c.s>>>(S);
    c.launches++;
}

// d = sum_j delta_j basis_j
__global__ void k_direction(int n, const CotSolver *__restrict__ S, const double *__restrict__ Sv,
                            const double *__restrict__ Yv, const double *__restrict__ mu,
                            const double *__restrict__ nu, double *__restrict__ d)
{
    // only right after k_begin_iteration (no trial evaluated since)
    if (S->done || S->evals != S->eval_mark || !S->ls_active) return;
    __shared__ double dl[COT_BASIS];
    const int m = S->m;
    for (int c = threadIdx.x; c < 2 * m + 1; c += blockDim.x) dl[c] = S->delta[c];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double r = dl[2 * m] * (mu[i] - nu[i]);
        for (int j = 0; j < m; j++) {
            double a = dl[j], b = dl[m + j];
            if (a != 0.0) r += a * Sv[(size_t)j * n + i];
            if (b != 0.0) r += b * Yv[(size_t)j * n + i];
        }
        d[i] = r;
    }
}

void launch_direction(const CotGeo &g, const CotSolver *S, const double *Sv, const double *Yv, const double *mu,
                      double *d, CotCtx &c)
{
    int blocks = (g.n + 255) / 256;
    if (blocks > 4 * 148) blocks = 4 * 148;
    k_direction<<<blocks, 256, 0, c.s>>>(g.n, S, Sv, Yv, mu, g.nu, d);
    c.launches++;
}

// Accept the trial: s_h = t d, y_h = mu_t - mu, w = w_t, mu = mu_t, then the
// new Gram entries s_h.y_j, y_h.s_j, y_h.y_j, g.s_j, g.y_j, g.g; the last
// block updates the matrix, the history scalars (ot_op.cuh:434-466) and the
// stop test (ot_op.cuh:468-476, 510).
#define ACC_PER 4
__global__ void __launch_bounds__(RED_THREADS) k_accept(int n, CotSolver *S, double *Sv, double *Yv, double *w,
                                                       const double *__restrict__ wt, double *mu,
                                                       const double *__restrict__ mut, const double *__restrict__ nu,
                                                       const double *__restrict__ d, double *partials,
                                                       unsigned int *ticket, int initial)
{
    constexpr int NW = RED_THREADS / 32;
    __shared__ double red[(5 * COT_MAX_HIST + 1) * NW];
    __shared__ double tot[5 * COT_MAX_HIST + 1];
    __shared__ bool last;
    if (S->done) return;
    if (!initial && !S->accepted) return;
    const int m = S->m;
    const int h = S->k % m;
    const double t = S->t;
    const int nvals = 5 * m + 1;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int per = (n + gridDim.x - 1) / gridDim.x;
    int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    // new vectors (each thread later reads back only what it wrote)
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        double mt = mut[i];
        if (!initial) {
            Sv[(size_t)h * n + i] = __dmul_rn(t, d[i]);
            Yv[(size_t)h * n + i] = mt - mu[i];
            w[i] = wt[i];
        }
        mu[i] = mt;
    }
    int cnt = initial ? 0 : (S->k + 1 < m ? S->k + 1 : m);  // slots that hold pairs after this update
    // the new pair and the gradient of this thread's first ACC_REG elements
    // stay in registers across the m passes below (same sums, same order)
    constexpr int ACC_REG = 4;
    double csn[ACC_REG], cyn[ACC_REG], cg[ACC_REG];
#pragma unroll
    for (int q = 0; q < ACC_REG; q++) {
        const int i = b0 + threadIdx.x + q * blockDim.x;
        csn[q] = cyn[q] = cg[q] = 0.0;
        if (i < b1) {
            csn[q] = Sv[(size_t)h * n + i];
            cyn[q] = Yv[(size_t)h * n + i];
            cg[q] = mu[i] - nu[i];
        }
    }
    const int brest = b0 + threadIdx.x + ACC_REG * blockDim.x;
    // all 5m+1 sums in one sweep: per-warp partials in shared memory, summed
    // in warp order, then block partials summed in block order by the last
    // block (the order of a per-value block reduction, in one barrier)
    for (int j = 0; j < m; j++) {
        double sy = 0.0, ys = 0.0, yy = 0.0, gs = 0.0, gy = 0.0;
        const int age = ((h - j) % m + m) % m;
        if (cnt > 0 && age < cnt) {
#pragma unroll
            for (int q = 0; q < ACC_REG; q++) {
                const int i = b0 + threadIdx.x + q * blockDim.x;
                if (i < b1) {
                    const double sj = Sv[(size_t)j * n + i], yj = Yv[(size_t)j * n + i];
                    sy += csn[q] * yj;
                    ys += cyn[q] * sj;
                    yy += cyn[q] * yj;
                    gs += cg[q] * sj;
                    gy += cg[q] * yj;
                }
            }
            for (int i = brest; i < b1; i += blockDim.x) {
                double sj = Sv[(size_t)j * n + i], yj = Yv[(size_t)j * n + i];
                double sn = Sv[(size_t)h * n + i], yn = Yv[(size_t)h * n + i];
                double g = mu[i] - nu[i];
                sy += sn * yj;
                ys += yn * sj;
                yy += yn * yj;
                gs += g * sj;
                gy += g * yj;
            }
            sy = wsum(sy);
            ys = wsum(ys);
            yy = wsum(yy);
            gs = wsum(gs);
            gy = wsum(gy);
        }
        if (lane == 0) {
            red[(5 * j + 0) * NW + wid] = sy;
            red[(5 * j + 1) * NW + wid] = ys;
            red[(5 * j + 2) * NW + wid] = yy;
            red[(5 * j + 3) * NW + wid] = gs;
            red[(5 * j + 4) * NW + wid] = gy;
        }
    }
    double gg = 0.0;
#pragma unroll
    for (int q = 0; q < ACC_REG; q++)
        if (b0 + threadIdx.x + q * blockDim.x < b1) gg += cg[q] * cg[q];
    for (int i = brest; i < b1; i += blockDim.x) {
        double g = mu[i] - nu[i];
        gg += g * g;
    }
    gg = wsum(gg);
    if (lane == 0) red[5 * m * NW + wid] = gg;
    __syncthreads();
    for (int v = threadIdx.x; v < nvals; v += blockDim.x) {
        double r = 0.0;
        for (int k = 0; k < NW; k++) r += red[v * NW + k];
        partials[(size_t)blockIdx.x * nvals + v] = r;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int tk = atomicAdd(ticket, 1u);
        last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int v = threadIdx.x; v < nvals; v += blockDim.x) tot[v] = sum_partials<false>(partials + v, gridDim.x, nvals);
    __syncthreads();
    if (threadIdx.x != 0) return;
    *ticket = 0u;
    const int gi = 2 * m;
    double *G = S->G;
    for (int j = 0; j < m; j++) {
        int age = ((h - j) % m + m) % m;
        bool valid = cnt > 0 && age < cnt;
        if (!valid) continue;
        if (!initial) {
            G[h * COT_BASIS + (m + j)] = G[(m + j) * COT_BASIS + h] = tot[5 * j + 0];
            G[(m + h) * COT_BASIS + j] = G[j * COT_BASIS + (m + h)] = tot[5 * j + 1];
            G[(m + h) * COT_BASIS + (m + j)] = G[(m + j) * COT_BASIS + (m + h)] = tot[5 * j + 2];
        }
        G[gi * COT_BASIS + j] = G[j * COT_BASIS + gi] = tot[5 * j + 3];
        G[gi * COT_BASIS + (m + j)] = G[(m + j) * COT_BASIS + gi] = tot[5 * j + 4];
    }
    G[gi * COT_BASIS + gi] = tot[5 * m];
    // current point
    S->f = S->last.f;
    S->maxrel = S->last.maxrel;
    S->gnorm2 = S->last.gnorm2;
    S->empty = S->last.empty;
    if (initial) {
        // a Wolfe-mode solve whose start already meets the tolerance stops at
        // its first evaluation (as the oracle's restatement does); the
        // reference mode always takes an iteration, as direct_ot does
        if (S->mode == COT_SOLVE_WOLFE && S->maxrel <= S->tol) {
            S->converged = 1;
            S->done = 1;
        }
        if (S->stop_nonempty && S->empty == 0) S->done = 1;
        return;
    }
    double ys = G[(m + h) * COT_BASIS + h];
    double yy = G[(m + h) * COT_BASIS + (m + h)];
    if (S->mode == COT_SOLVE_REFERENCE) {
        S->rho[h] = 1.0 / ys;
        S->H0 = (yy > 1e-5) ? ys / yy : 1.0;
        S->k++;
        S->restart = 0;
    } else if (ys > 0.0) {
        S->rho[h] = 1.0 / ys;
        S->H0 = ys / yy;
        S->k++;
    }
    S->iter++;
    S->need_begin = 1;
    if (S->mode == COT_SOLVE_REFERENCE) {
        if (S->gnorm_stale < S->tol && S->empty_stale == 0) { S->converged = 1; S->done = 1; }
    } else {
        if (S->maxrel <= S->tol) { S->converged = 1; S->done = 1; }
    }
    if (S->stop_nonempty && S->empty == 0) S->done = 1;
    if (S->iter >= S->max_iter) S->done = 1;
}

void launch_accept(const CotGeo &g, CotSolver *S, double *Sv, double *Yv, double *w, const double *wt, double *mu,
                   const double *mut, const double *d, double *partials, unsigned int *ticket, int initial,
                   CotCtx &c)
{
    int nb = reduce_blocks(g.n);
    k_accept<<<nb, RED_THREADS, 0, c.s>>>(g.n, S, Sv, Yv, w, wt, mu, mut, g.nu, d, partials, ticket, initial);
    c.launches++;
}

// Line search gave up (ot_op.cuh:413-425): keep the point, drop the history.
__device__ __forceinline__ void reject(CotSolver *S)
{
    if (S->done || S->accepted || S->ls_active) return;
    S->need_begin = 1;
    if (S->mode == COT_SOLVE_REFERENCE) {
        S->restart = 1;
    } else if (S->k == 0) {
        S->failed = 1;
        S->done = 1;
        return;
    }
    S->k = 0;
    S->H0 = 1.0;
    S->restarts++;
    S->iter++;
    if (S->iter >= S->max_iter) S->done = 1;
}

__global__ void k_reject(CotSolver *S) { reject(S); }

void launch_reject(CotSolver *S, CotCtx &c)
{
    k_reject<<<1, 1, 0, c.s>>>(S);
    c.launches++;
}

// Condition of the device-driven trial loop (a WHILE node of a CUDA graph):
// go on until the solve is done or reaches the iteration where the host
// wants to look (a progress report).
__global__ void k_loop_cond(cudaGraphConditionalHandle hc, const CotSolver *S)
{
    cudaGraphSetConditional(hc, (!S->done && S->iter < S->pause_iter) ? 1u : 0u);
}

void launch_loop_cond(cudaGraphConditionalHandle hc, const CotSolver *S, CotCtx &c)
{
    k_loop_cond<<<1, 1, 0, c.s>>>(hc, S);
    c.launches++;
}

// The end of a pass of the device-driven trial loop: reject (if the line
// search just gave up) and the loop condition, in one launch.
__global__ void k_reject_cond(cudaGraphConditionalHandle hc, CotSolver *S)
{
    reject(S);
    cudaGraphSetConditional(hc, (!S->done && S->iter < S->pause_iter) ? 1u : 0u);
}

void launch_reject_cond(cudaGraphConditionalHandle hc, CotSolver *S, CotCtx &c)
{
    k_reject_cond<<<1, 1, 0, c.s>>>(hc, S);
    c.launches++;
}

// The first evaluation becomes the current point without a line search.
__global__ void k_init_from_eval(CotSolver *S, const CotEvalOut *out)
{
    S->last = *out;
    S->evals++;
}

void launch_init_from_eval(CotSolver *S, const CotEvalOut *out, CotCtx &c)
{
    k_init_from_eval<<<1, 1, 0, c.s>>>(S, out);
    c.launches++;
}

// ---------------------------------------------------------------------------
// helpers of cot_eval and of the Fresnel-reweighted Anderson solve
// ---------------------------------------------------------------------------

// f_i with its -w_i nu_i term (the cell kernels store it without)
__global__ void k_fcell_full(int n, const double *__restrict__ fc, const double *__restrict__ wt,
                             const double *__restrict__ nu, double *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = fc[i] - wt[i] * nu[i];
}

void launch_fcell_full(int n, const double *fc, const double *wt, const double *nu, double *out, CotCtx &c)
{
    k_fcell_full<<<(n + 255) / 256, 256, 0, c.s>>>(n, fc, wt, nu, out);
    c.launches++;
}

// fresnel_T_unpolarized (basic_function.cuh:407-435)
__device__ double fresnel_t(const double wi[3], const double wt[3], const double nrm[3], double eta_i, double eta_t)
{
    const double eps = 1e-12;
    double ci = fabs(wi[0] * nrm[0] + wi[1] * nrm[1] + wi[2] * nrm[2]);
    double ct = fabs(wt[0] * nrm[0] + wt[1] * nrm[1] + wt[2] * nrm[2]);
    ci = fmin(1.0, fmax(0.0, ci));
    ct = fmin(1.0, fmax(0.0, ct));
    double ds = eta_i * ci + eta_t * ct;
    double dp = eta_i * ct + eta_t * ci;
    if (fabs(ds) < eps) ds = eps;
    if (fabs(dp) < eps) dp = eps;
    double rs = (eta_i * ci - eta_t * ct) / ds;
    double rp = (eta_i * ct - eta_t * ci) / dp;
    rs *= rs;
    rp *= rp;
    return 1.0 - 0.5 * (rs + rp);
}

__device__ void normalize3(double v[3])
{
    double nn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (nn < 1e-12) {
        v[0] = v[1] = v[2] = 0.0;
        return;
    }
    v[0] /= nn;
    v[1] /= nn;
    v[2] /= nn;
}

// compute_energy_remain_rate (basic_function.cuh:437-494) times the source
// mass: energy_i = lambda_i * T1_i * T2_i, from the cell centroids.
__global__ void k_fresnel_energy(int n, const double *__restrict__ cen, const double *__restrict__ src,
                                 const double *__restrict__ inl, const double *__restrict__ insl,
                                 const double *__restrict__ hgt, const double *__restrict__ lam, double zl,
                                 double zr, double eta, double *__restrict__ energy)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double p[3] = {src[2 * i], src[2 * i + 1], zl};
    double wi[3] = {inl[3 * i], inl[3 * i + 1], inl[3 * i + 2]};
    double ins[3] = {insl[3 * i], insl[3 * i + 1], insl[3 * i + 2]};
    double op[3] = {p[0] + hgt[i] * ins[0], p[1] + hgt[i] * ins[1], p[2] + hgt[i] * ins[2]};
    double wo[3] = {cen[2 * i] - op[0], cen[2 * i + 1] - op[1], zr - op[2]};
    normalize3(wo);
    double n2[3] = {eta * ins[0] - wo[0], eta * ins[1] - wo[1], eta * ins[2] - wo[2]};
    normalize3(n2);
    const double n1[3] = {0.0, 0.0, 1.0};
    double t1 = fresnel_t(wi, ins, n1, 1.0, eta);
    double t2 = fresnel_t(ins, wo, n2, eta, 1.0);
    energy[i] = lam[i] * (t1 * t2);
}

// Fixed-order sum of x: block partials in block order; every block of the
// scale kernel re-reduces the partials identically.
__global__ void __launch_bounds__(RED_THREADS) k_sum_partials(int n, const double *__restrict__ x, double *partials)
{
    __shared__ double sh[33];
    int per = (n + gridDim.x - 1) / gridDim.x;
    int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    double v = 0.0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) v += x[i];
    v = block_reduce<false>(v, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

// nu_i = energy_i / sum(energy) * total
__global__ void k_scale_to_total(int n, const double *__restrict__ energy, const double *__restrict__ partials,
                                 int nparts, double total, double *__restrict__ nu)
{
    double s = 0.0;
    for (int k = 0; k < nparts; k++) s += partials[k];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) nu[i] = energy[i] / s * total;
}

void launch_fresnel_nu(int n, const double *cen, const double *src, const double *inl, const double *insl,
                       const double *hgt, const double *lam, double zl, double zr, double eta, double total,
                       double *energy, double *partials, double *nu, CotCtx &c)
{
    k_fresnel_energy<<<(n + 255) / 256, 256, 0, c.s>>>(n, cen, src, inl, insl, hgt, lam, zl, zr, eta, energy);
    int nb = reduce_blocks(n);
    k_sum_partials<<<nb, RED_THREADS, 0, c.s>>>(n, energy, partials);
    k_scale_to_total<<<(n + 255) / 256, 256, 0, c.s>>>(n, energy, partials, nb, total, nu);
    c.launches += 3;
}

// Anderson history slot h: G_h = mu - nu, F_h = w + alpha G_h
// (storage + compute_fixed_function, ot_op.cuh:1139-1142)
__global__ void k_aa_store(int n, const double *__restrict__ w, const double *__restrict__ mu,
                           const double *__restrict__ nu, double alpha, double *__restrict__ gh,
                           double *__restrict__ fh)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double g = mu[i] - nu[i];
    gh[i] = g;
    fh[i] = w[i] + alpha * g;
}

// row[j] = G_h . G_j for j < cnt (fixed order: block partials, last block sums)
__global__ void __launch_bounds__(RED_THREADS) k_aa_gram_row(int n, const double *__restrict__ G, int h, int cnt,
                                                            double *partials, unsigned int *ticket, double *row)
{
    __shared__ double sh[33];
    __shared__ bool last;
    int per = (n + gridDim.x - 1) / gridDim.x;
    int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    const double *gh = G + (size_t)h * n;
    for (int j = 0; j < cnt; j++) {
        const double *gj = G + (size_t)j * n;
        double v = 0.0;
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) v += gh[i] * gj[i];
        v = block_reduce<false>(v, sh);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * COT_MAX_HIST + j] = v;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        volatile double *p = partials;
        for (int j = 0; j < cnt; j++) {
            double r = 0.0;
            for (unsigned b = 0; b < gridDim.x; b++) r += p[(size_t)b * COT_MAX_HIST + j];
            row[j] = r;
        }
        *ticket = 0u;
    }
}

void launch_aa_store_gram(int n, const double *w, const double *mu, const double *nu, double alpha, double *G,
                          double *F, int h, int cnt, double *partials, unsigned int *ticket, double *row, CotCtx &c)
{
    k_aa_store<<<(n + 255) / 256, 256, 0, c.s>>>(n, w, mu, nu, alpha, G + (size_t)h * n, F + (size_t)h * n);
    k_aa_gram_row<<<reduce_blocks(n), RED_THREADS, 0, c.s>>>(n, G, h, cnt, partials, ticket, row);
    c.launches += 2;
}

// d = sum_j coef_j F_j - w   (compute_weighted_sum + compute_subtract, ot_op.cuh:1172-1173)
__global__ void k_aa_combine(int n, const double *__restrict__ F, const double *__restrict__ coef, int cnt,
                             const double *__restrict__ w, double *__restrict__ d)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int j = 0; j < cnt; j++) s += coef[j] * F[(size_t)j * n + i];
    d[i] = s - w[i];
}

void launch_aa_combine(int n, const double *F, const double *coef, int cnt, const double *w, double *d, CotCtx &c)
{
    k_aa_combine<<<(n + 255) / 256, 256, 0, c.s>>>(n, F, coef, cnt, w, d);
    c.launches++;
}

}  // namespace cot
